"""Residual-based ChFSI (R-ChFSI, reference_paper/2025 main.tex Algorithm 3)
restated in the oracle: with the exact S^-1 and FP64 matrix-vector products
it is algebraically the sigma-scaled Chebyshev filter, so one R-ChFSI pass
from a set of Ritz pairs gives the same Rayleigh-Ritz eigenvalues as one
ChFSI pass (chebyshev.rs:626-816 + rayleigh_ritz.rs:48-245) from the same
pairs, for the standard and the generalised (ultrasoft) problem."""
import numpy as np
import pytest

import synth


def _pair(oracle, s, qmat=False):
    a = oracle.Oracle.from_system(s)
    b = oracle.Oracle.from_system(s)
    if qmat:
        a.set_qmat(s.qmat())
        b.set_qmat(s.qmat())
    v = a.vloc_r()
    a.set_veff(v)
    b.set_veff(v)
    return a, b


@pytest.mark.parametrize("kind", ["local", "kb", "uspp"])
def test_rchfsi_pass_equals_chfsi_pass(oracle, kind):
    if kind == "local":
        s = synth.System(config_index=0)
    elif kind == "kb":
        s = synth.System(config_index=0, n_shell=1, lmax=1, rc_proj=[1.2, 0, 0, 0], d_min=0.5,
                         d_max=2.0)
    else:
        s = synth.System(config_index=2, n_rep=1, ecut=8.0, ngrid=[0, 0, 0], n_bands=24)
    a, b = _pair(oracle, s, qmat=kind == "uspp")
    w = None
    for _ in range(2):  # Ritz pairs to start from
        w = a.diagonalize(10, w)
    b.set_psi(a.get_psi())
    wc = a.diagonalize(10, w)
    wr = b.rchfsi_diagonalize(10, w)
    np.testing.assert_allclose(wr, wc, atol=1e-10, rtol=0)
    np.testing.assert_allclose(b.bounds(), a.bounds(), rtol=1e-14)
