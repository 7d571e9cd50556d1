"""Writes the golden fixtures of this directory.

reference_known_answers.json — the known-answer cases of the reference
crate's own unit tests for this path, transcribed as data (inputs and
expected outputs) with the file:line of each case in chemrust-scf:
  * src/eigensolver/subspace_diag.rs:535-590  4x4 generalised RR, H = diag(1,2,3,4),
    S = diag(2,1.5,1,0.8) -> [0.5, 4/3, 3, 5] (1e-12)
  * src/device/solver.rs:113-163  ZHEGVD A = diag(1,2,3,4), B = I -> [1,2,3,4] (1e-8)
  * src/device/fft.rs:239-281  8^3 Z2Z forward then inverse = N^3 x input (1e-10),
    input[i] = (i, 2i) for i < 10, else 0
  * src/device/blas.rs:258-310  2x2 ZGEMM A = [[1+i,0],[0,1-i]], B = [[1,2],[3,4]]
    -> [[1+i, 2+2i], [3-3i, 4-4i]]
  * src/eigensolver/subspace_diag.rs:434-447  deterministic LCG
    state <- state * 25214903917 + 11 mod 2^48, x = state / 2^48 (seed 42)

cfg0_oracle.json — outputs of the CPU oracle on the 8-atom, 40^3 benchmark
cell (seed 0): eigenvalues after one and after three ChFSI iterations on
V_eff = V_loc (degree 12, reference spectral bounds), and the first three SCF
energies (Fermi-Dirac kT = 0.01 Ha, Pulay alpha 0.3 / history 6).

  * src/eigensolver/line_search.rs:217-394  closed-form line search: parabola
    (1, 1, 3, 0) -> step 1/3, E 2/3; rational (0, -0.5, 1, 1) -> step sqrt2 - 1;
    clamp (0, -5, 0.01, 0.001) -> 15 (status 1); no minimum (0, 0, -0.1, 0) -> status -1

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "chemrust-scf_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def lcg_sequence(seed, n):
    s, out = seed, []
    for _ in range(n):
        s = (s * 25214903917 + 11) & 0xFFFFFFFFFFFF
        out.append(s / 281474976710656.0)
    return out


def known_answers():
    return {
        "rr_4x4": {"source": "src/eigensolver/subspace_diag.rs:535-590",
                   "h_diag": [1.0, 2.0, 3.0, 4.0], "s_diag": [2.0, 1.5, 1.0, 0.8],
                   "expected": [0.5, 4.0 / 3.0, 3.0, 5.0], "tol": 1e-12},
        "zhegvd_4x4": {"source": "src/device/solver.rs:113-163",
                       "a_diag": [1.0, 2.0, 3.0, 4.0], "expected": [1.0, 2.0, 3.0, 4.0],
                       "tol": 1e-8},
        "fft_8cubed_identity": {"source": "src/device/fft.rs:239-281", "n": [8, 8, 8],
                                "nonzero": 10, "tol": 1e-10},
        "zgemm_2x2": {"source": "src/device/blas.rs:258-310",
                      "a": [[[1, 1], [0, 0]], [[0, 0], [1, -1]]],
                      "b": [[[1, 0], [2, 0]], [[3, 0], [4, 0]]],
                      "expected": [[[1, 1], [2, 2]], [[3, -3], [4, -4]]], "tol": 1e-10},
        "lcg_seed42": {"source": "src/eigensolver/subspace_diag.rs:434-447",
                       "first8": lcg_sequence(42, 8)},
        "line_search_parabola": {"source": "src/eigensolver/line_search.rs:219-234",
                                 "args": [1.0, 1.0, 3.0, 0.0], "step": 1.0 / 3.0,
                                 "eigenvalue": 2.0 / 3.0, "norm": 1.0, "status": 0, "tol": 1e-12},
        "line_search_rational": {"source": "src/eigensolver/line_search.rs:250-280",
                                 "args": [0.0, -0.5, 1.0, 1.0], "step": 2.0 ** 0.5 - 1.0,
                                 "eigenvalue": ((1 - 2 ** 0.5) + (1 - 2 ** 0.5) ** 2) / (1 + (1 - 2 ** 0.5) ** 2),
                                 "tol": 1e-12},
        "line_search_clamp": {"source": "src/eigensolver/line_search.rs:318-333",
                              "args": [0.0, -5.0, 0.01, 0.001], "step": 15.0, "status": 1,
                              "tol": 1e-12},
        "line_search_no_minimum": {"source": "src/eigensolver/line_search.rs:335-345",
                                   "args": [0.0, 0.0, -0.1, 0.0], "step": 0.0, "status": -1},
    }


def cfg0_oracle():
    import chfsi
    import oracle
    s = chfsi.SyntheticSystem(config_index=0)
    o = oracle.Oracle.from_system(s)
    o.set_veff(o.vloc_r())
    w1 = o.diagonalize(12)
    b1 = o.bounds()
    w = w1
    for _ in range(2):
        w = o.diagonalize(12, w)
    o2 = oracle.Oracle.from_system(s)
    r = o2.run_scf(12, max_iter=3, kT=0.01)
    return {"system": "8-atom diamond cell a=10.26, Ecut 15, 40^3, 20 bands, seed 0",
            "ndeg": 12, "eig_iter1": w1.tolist(), "bounds_iter1": b1.tolist(),
            "eig_iter3": w.tolist(), "scf_energies_3": r["energies"].tolist()}


def main():
    with open(os.path.join(HERE, "reference_known_answers.json"), "w") as f:
        json.dump(known_answers(), f, indent=1)
    if "--known-answers-only" not in sys.argv:
        with open(os.path.join(HERE, "cfg0_oracle.json"), "w") as f:
            json.dump(cfg0_oracle(), f, indent=1)


if __name__ == "__main__":
    main()
