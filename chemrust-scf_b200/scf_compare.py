"""Time-to-SCF of the plain FP64 path against the mixed-precision path with
Pulay and with the learned mixer, on one of the synthetic configurations.

    python chemrust-scf_b200/scf_compare.py --config 2 --max-iter 90

Arms: FP64 filter + Pulay (alpha 0.3, history 6); FP32 filter (BF16x3
tcgen05 projector GEMMs) / FP64 Rayleigh-Ritz with Pulay; the same with the learned
per-shell preconditioner inside Pulay.  The mixed runs switch to FP64 only
for the confirming iterations (|dE| < tol) and only declare convergence on
an FP64 iteration.  Times are device seconds of the SCF loop (CUDA events),
set-up excluded; one JSON line per arm and a summary line.
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
import learned_mixer  # noqa: E402

NDEG = {0: 12, 1: 16, 2: 16}


def run_arm(s, name, prec, mode, ndeg, max_iter, tol, mixer=None, verbose=False):
    t = time.time()
    ctx = chfsi.Context(s, precision=prec)
    setup = time.time() - t
    if mixer is not None:
        ctx.set_mixer(mixer)
    r = ctx.run_scf(ndeg, max_iter=max_iter, tol_per_atom=tol, kT=0.01, mixer=mode,
                    fp64_switch_per_atom=tol, verbose=verbose)
    ctx.close()
    out = {"arm": name, "converged": r["converged"], "iterations": r["n_iter"],
           "iterations_in_mixed_precision": r["n_iter_mixed"], "seconds": r["seconds"],
           "setup_seconds": setup, "e_total": r["e_total"], "fp64_retries": r["n_fp64_retries"],
           "learned_steps": r["n_iter_learned"], "fell_back": r["fell_back"],
           "eigenvalues": r["eigenvalues"]}
    print(json.dumps({k: v for k, v in out.items() if k != "eigenvalues"}), flush=True)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--max-iter", type=int, default=90)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--arms", default="fp64,mixed,mixed_learned")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    s = chfsi.SyntheticSystem(config_index=args.config)
    ndeg = NDEG.get(args.config, 16)
    net = learned_mixer.load()
    arms = {"fp64": (chfsi.PREC_FP64, chfsi.MIXER_PULAY, None),
            "mixed": (chfsi.PREC_MIXED, chfsi.MIXER_PULAY, None),
            "mixed_learned": (chfsi.PREC_MIXED, chfsi.MIXER_LEARNED_PULAY, net),
            "fp64_learned": (chfsi.PREC_FP64, chfsi.MIXER_LEARNED_PULAY, net)}
    res = {}
    for name in args.arms.split(","):
        prec, mode, mixer = arms[name]
        res[name] = run_arm(s, name, prec, mode, ndeg, args.max_iter, args.tol, mixer, args.verbose)
    summary = {"config": args.config, "atoms": s.n_atoms, "n_pw": s.n_pw, "n_bands": s.n_bands,
               "n_proj": s.n_proj, "grid": list(s.ngrid), "density_grid": list(s.ngrid_density)}
    if "fp64" in res:
        f = res["fp64"]
        n_occ = int(round(s.n_elec / 2))
        for name, r in res.items():
            if name == "fp64":
                continue
            summary[name] = {
                "speedup_vs_fp64": f["seconds"] / r["seconds"] if r["seconds"] > 0 else None,
                "energy_diff_per_atom_Ha": abs(r["e_total"] - f["e_total"]) / s.n_atoms,
                "max_occupied_eigenvalue_diff_Ha":
                    float(np.abs(np.asarray(r["eigenvalues"][:n_occ]) - f["eigenvalues"][:n_occ]).max())}
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
