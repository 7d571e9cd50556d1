"""Training and evaluation of the learned density mixer.

The mixer is an MLP (512 -> 256 -> 256 -> 128, GELU, BF16 weights, FP32
accumulation) that maps the |G|-shell-binned history of density residuals to
a per-shell update (a_s, b_s); see include/chfsi.h.  This module generates
SCF trajectories with the library itself on seeded random cells, turns them
into (features, targets) with the library's shell reductions, trains the
network with the library's own forward/backward/Adam kernels, and compares
SCF iteration counts and wall time against Pulay.

    python chemrust-scf_b200/learned_mixer.py train --cells 300 --dagger-cells 150 --out mixer.npz
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
# cell): 8, 16, 27 and 64 atoms for training; 216 atoms (the size of the
# 216-atom diamond supercell) for evaluation only
CELL_KINDS = [(0, 1, 8), (2, 2, 2), (1, 3, 1), (0, 2, 8), (0, 3, 8)]
VOLUME_PER_ATOM = 10.26 ** 3 / 8.0  # the 8-atom diamond cell's density


# dilute cells: 64 atoms at 1.5-3.375x the volume per atom (edges of 23.5 to
# 30.78 bohr, the 216-atom cell's), so that the lowest |G| shells of the large
# cells (shells 8 and 9) occur in training
DILUTE_RANGE = (1.5, 3.375)
DILUTE_KIND = 3


def cell_params(seed, kinds=(0, 1, 2, 3), weights=(0.4, 0.3, 0.2, 0.1), jitter=0.3, ecut=15.0,
                dilute_frac=0.0):
    """Seeded random cell: 8-64 atoms, Z in {1..6}, the 8-atom diamond cell's
    atomic density, or with probability dilute_frac a 64-atom cell with a
    volume per atom DILUTE_RANGE times larger."""
    rng = np.random.default_rng(seed)
    k = kinds[rng.choice(len(kinds), p=np.asarray(weights) / np.sum(weights))]
    vol = VOLUME_PER_ATOM
    if dilute_frac > 0.0 and rng.uniform() < dilute_frac:
        k = DILUTE_KIND
        vol *= rng.uniform(*DILUTE_RANGE)
    lattice, n_rep, per_conv = CELL_KINDS[k]
    p = chfsi.SynthParams()
    chfsi._check(chfsi.lib().chfsi_synth_defaults(0, chfsi.C.byref(p)))
    p.lattice, p.n_rep = lattice, n_rep
    p.a_conv = (per_conv * vol) ** (1.0 / 3.0)
    p.jitter = jitter
    p.z_val = float(rng.integers(1, 7))
    p.ecut = ecut
    for i in range(3):
        p.ngrid[i] = 0
    p.n_bands = 0
    p.seed = int(seed)
    return p


def trajectories(seed, ndeg=12, max_iter=60, tol=1e-8, dilute_frac=0.0):
    """Two trajectories of one cell: Pulay with a random alpha (also gives the
    converged density rho*) and linear mixing with a random alpha."""
    rng = np.random.default_rng(seed + 1_000_003)
    s = chfsi.SyntheticSystem(cell_params(seed, dilute_frac=dilute_frac))
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


def on_policy_samples(mixer, seed, ndeg=12, max_iter=60, tol=1e-8, dilute_frac=0.0):
    """Samples from the network's own trajectories (learned-preconditioned
    Pulay and pure learned mixing), so that training sees the states the
    network itself produces."""
    s = chfsi.SyntheticSystem(cell_params(seed, dilute_frac=dilute_frac))
    out = []
    for mode in (chfsi.MIXER_LEARNED_PULAY, chfsi.MIXER_LEARNED):
        ctx = chfsi.Context(s)
        ctx.set_mixer(mixer)
        r = ctx.run_scf(ndeg, tol_per_atom=tol, max_iter=max_iter, kT=0.01, mixer=mode, trace=True)
        if r["converged"]:
            out.append(ctx.mixer_samples(r["trace_in"], r["trace_out"], r["trace_out"][-1]))
    return out


def dataset(seeds, log=print, dilute_frac=0.0):
    X, T = [], []
    t0 = time.time()
    for i, sd in enumerate(seeds):
        s, ctx, trs = trajectories(sd, dilute_frac=dilute_frac)
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


def train(n_cells=300, epochs=150, batch=256, lr=1e-3, seed=0, out=WEIGHTS, dagger_cells=0,
          log=print, dilute_frac=0.0):
    """Off-policy data (Pulay and linear-mixing trajectories), Adam at lr then
    lr/10; optionally one on-policy round on dagger_cells further cells."""
    seeds = list(range(10_000 + seed, 10_000 + seed + n_cells))
    log("generating trajectories on %d cells" % n_cells)
    t0 = time.time()
    X, T = dataset(seeds, log, dilute_frac)
    gen_s = time.time() - t0
    log("%d samples; training" % len(X))
    m = chfsi.Mixer(seed=seed)
    t0 = time.time()
    l1 = m.train(X, T, epochs=epochs, batch=batch, lr=lr, seed=seed)
    l2 = m.train(X, T, epochs=max(1, epochs // 2), batch=batch, lr=lr * 0.1, seed=seed + 1)
    train_s = time.time() - t0
    log("loss %.4f -> %.4f -> %.4f in %.1f s" % (l1[0], l1[-1], l2[-1], train_s))
    meta = {"cells": n_cells, "dilute_frac": dilute_frac, "samples": int(len(X)), "epochs": epochs,
            "batch": batch, "lr": lr,
            "loss_first": float(l1[0]), "loss_last": float(l2[-1]),
            "generate_seconds": gen_s, "train_seconds": train_s}
    if dagger_cells:
        t0 = time.time()
        Xd, Td = [], []
        for sd in range(50_000 + seed, 50_000 + seed + dagger_cells):
            for x, t in on_policy_samples(m, sd, dilute_frac=dilute_frac):
                Xd.append(x)
                Td.append(t)
        X = np.concatenate([X] + Xd)
        T = np.concatenate([T] + Td)
        gen2 = time.time() - t0
        t0 = time.time()
        l3 = m.train(X, T, epochs=max(1, epochs // 2), batch=batch, lr=lr * 0.3, seed=seed + 2)
        l4 = m.train(X, T, epochs=max(1, epochs // 2), batch=batch, lr=lr * 0.03, seed=seed + 3)
        log("on-policy round: %d cells, %d samples in all; loss %.4f -> %.4f" %
            (dagger_cells, len(X), l3[0], l4[-1]))
        meta.update({"on_policy_cells": dagger_cells, "samples_total": int(len(X)),
                     "loss_last": float(l4[-1]), "generate_seconds_on_policy": gen2,
                     "train_seconds_on_policy": time.time() - t0})
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
    a.add_argument("--dagger-cells", type=int, default=0)
    a.add_argument("--dilute-frac", type=float, default=0.0,
                   help="share of training cells with a larger volume per atom")
    b = sub.add_parser("evaluate")
    b.add_argument("--weights", default=WEIGHTS)
    b.add_argument("--cells", type=int, default=8)
    b.add_argument("--first-seed", type=int, default=90_000)
    b.add_argument("--out", default=None)
    b.add_argument("--kinds", default="0,1,2,3", help="cell kinds (4 = 216 atoms)")
    args = ap.parse_args()
    if args.cmd == "train":
        train(args.cells, args.epochs, args.batch, args.lr, args.seed, args.out, args.dagger_cells,
              dilute_frac=args.dilute_frac)
    else:
        m = load(args.weights)
        kinds = tuple(int(k) for k in args.kinds.split(","))
        rows = evaluate(m, list(range(args.first_seed, args.first_seed + args.cells)), kinds=kinds)
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
