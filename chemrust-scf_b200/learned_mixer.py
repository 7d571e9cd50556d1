"""Training and evaluation of the learned density mixer.

The mixer is an MLP (512 -> 256 -> 256 -> 128, GELU, BF16 weights, FP32
accumulation) that maps the |G|-shell-binned history of density residuals to
a per-shell update (a_s, b_s); see include/chfsi.h.  This module generates
SCF trajectories with the library itself on seeded random cells, turns them
into (features, targets) with the library's shell reductions, trains the
network with the library's own forward/backward/Adam kernels, and compares
SCF iteration counts and wall time against Pulay.

    python chemrust-scf_b200/learned_mixer.py train --cells 300 --out mixer.npz
    python chemrust-scf_b200/learned_mixer.py evaluate --weights mixer.npz --cells 8

The reference crate has no mixer implementation (src/mixing.rs:24 is a
todo!()); Pulay (alpha 0.3, history 6) is its planned method and the
baseline here.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import chfsi  # noqa: E402

WEIGHTS = os.path.join(HERE, "mixer_weights.npz")

# (lattice: 0 diamond, 1 simple cubic, 2 bcc; n_rep; atoms per conventional
# cell): 8, 16, 27 and 64 atoms
CELL_KINDS = [(0, 1, 8), (2, 2, 2), (1, 3, 1), (0, 2, 8)]
VOLUME_PER_ATOM = 10.26 ** 3 / 8.0  # the 8-atom diamond cell's density


def cell_params(seed, kinds=(0, 1, 2, 3), weights=(0.4, 0.3, 0.2, 0.1), jitter=0.3, ecut=15.0):
    """Seeded random cell: 8-64 atoms, Z in {1..6}, fixed atomic density."""
    rng = np.random.default_rng(seed)
    k = kinds[rng.choice(len(kinds), p=np.asarray(weights) / np.sum(weights))]
    lattice, n_rep, per_conv = CELL_KINDS[k]
    p = chfsi.SynthParams()
    chfsi._check(chfsi.lib().chfsi_synth_defaults(0, chfsi.C.byref(p)))
    p.lattice, p.n_rep = lattice, n_rep
    p.a_conv = (per_conv * VOLUME_PER_ATOM) ** (1.0 / 3.0)
    p.jitter = jitter
    p.z_val = float(rng.integers(1, 7))
    p.ecut = ecut
    for i in range(3):
        p.ngrid[i] = 0
    p.n_bands = 0
    p.seed = int(seed)
    return p


def trajectories(seed, ndeg=12, max_iter=60, tol=1e-8):
    """Two trajectories of one cell: Pulay with a random alpha (also gives the
    converged density rho*) and linear mixing with a random alpha."""
    rng = np.random.default_rng(seed + 1_000_003)
    s = chfsi.SyntheticSystem(cell_params(seed))
    ctx = chfsi.Context(s)
    r = ctx.run_scf(ndeg, tol_per_atom=tol, max_iter=max_iter, kT=0.01,
                    alpha=float(rng.uniform(0.1, 0.5)), trace=True)
    if not r["converged"]:
        return s, ctx, []
    star = r["trace_out"][-1]
    out = [(r["trace_in"], r["trace_out"])]
    ctx2 = chfsi.Context(s)
    r2 = ctx2.run_scf(ndeg, tol_per_atom=tol, max_iter=30, kT=0.01, max_hist=1,
                      alpha=float(rng.uniform(0.05, 0.4)), trace=True)
    out.append((r2["trace_in"], r2["trace_out"]))
    return s, ctx, [(a, b, star) for a, b in out]


def dataset(seeds, log=print):
    X, T = [], []
    t0 = time.time()
    for i, sd in enumerate(seeds):
        s, ctx, trs = trajectories(sd)
        for rin, rout, star in trs:
            x, t = ctx.mixer_samples(rin, rout, star)
            X.append(x)
            T.append(t)
        if (i + 1) % 25 == 0:
            log("  %d/%d cells, %d samples, %.1f s" % (i + 1, len(seeds), sum(len(a) for a in X),
                                                       time.time() - t0))
    return np.concatenate(X), np.concatenate(T)


def save(mixer, path, meta=None):
    np.savez_compressed(path, params=mixer.get_params(), meta=json.dumps(meta or {}))


def load(path=WEIGHTS, device=0):
    z = np.load(path)
    return chfsi.Mixer(device=device, params=z["params"])


def train(n_cells=300, epochs=150, batch=256, lr=1e-3, seed=0, out=WEIGHTS, log=print):
    seeds = list(range(10_000 + seed, 10_000 + seed + n_cells))
    log("generating trajectories on %d cells" % n_cells)
    X, T = dataset(seeds, log)
    log("%d samples; training" % len(X))
    m = chfsi.Mixer(seed=seed)
    t0 = time.time()
    losses = m.train(X, T, epochs=epochs, batch=batch, lr=lr, seed=seed)
    log("loss %.4f -> %.4f in %.1f s" % (losses[0], losses[-1], time.time() - t0))
    meta = {"cells": n_cells, "samples": int(len(X)), "epochs": epochs, "batch": batch, "lr": lr,
            "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
            "train_seconds": time.time() - t0}
    save(m, out, meta)
    return m, meta


def evaluate(mixer, seeds, ndeg=12, max_iter=80, tol=1e-6, kinds=(0, 1, 2, 3), log=print):
    """Iterations and device seconds to |dE| < tol per atom: Pulay vs learned."""
    rows = []
    for sd in seeds:
        s = chfsi.SyntheticSystem(cell_params(sd, kinds=kinds, weights=[1] * len(kinds)))
        row = {"seed": sd, "atoms": s.n_atoms, "z": s.params.z_val}
        for name, mode in [("pulay", chfsi.MIXER_PULAY), ("learned", chfsi.MIXER_LEARNED),
                           ("learned_pulay", chfsi.MIXER_LEARNED_PULAY)]:
            ctx = chfsi.Context(s)
            if mode != chfsi.MIXER_PULAY:
                ctx.set_mixer(mixer)
            r = ctx.run_scf(ndeg, tol_per_atom=tol, max_iter=max_iter, kT=0.01, mixer=mode)
            row[name] = {"iterations": r["n_iter"], "seconds": r["seconds"],
                         "converged": r["converged"], "e_total": r["e_total"],
                         "fell_back": r["fell_back"], "learned_steps": r["n_iter_learned"]}
        log(json.dumps(row))
        rows.append(row)
    return rows


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("train")
    a.add_argument("--cells", type=int, default=300)
    a.add_argument("--epochs", type=int, default=150)
    a.add_argument("--batch", type=int, default=256)
    a.add_argument("--lr", type=float, default=1e-3)
    a.add_argument("--seed", type=int, default=0)
    a.add_argument("--out", default=WEIGHTS)
    b = sub.add_parser("evaluate")
    b.add_argument("--weights", default=WEIGHTS)
    b.add_argument("--cells", type=int, default=8)
    b.add_argument("--first-seed", type=int, default=90_000)
    b.add_argument("--out", default=None)
    args = ap.parse_args()
    if args.cmd == "train":
        train(args.cells, args.epochs, args.batch, args.lr, args.seed, args.out)
    else:
        m = load(args.weights)
        rows = evaluate(m, list(range(args.first_seed, args.first_seed + args.cells)))
        summary = {}
        for k in ("pulay", "learned", "learned_pulay"):
            it = [r[k]["iterations"] for r in rows]
            sec = [r[k]["seconds"] for r in rows]
            conv = sum(r[k]["converged"] for r in rows)
            summary[k] = {"mean_iterations": float(np.mean(it)), "total_seconds": float(np.sum(sec)),
                          "converged": conv}
        print(json.dumps(summary))
        if args.out:
            with open(args.out, "w") as f:
                json.dump({"rows": rows, "summary": summary}, f, indent=1)


if __name__ == "__main__":
    main()
