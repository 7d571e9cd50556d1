"""Residual-based ChFSI (R-ChFSI, reference_paper/2025 main.tex Algorithm 3)
on the device against the oracle's restatement, and its point: in the
mixed-precision mode the FP32/BF16x3 residual recurrence reaches the FP64
eigenvalues where the plain FP32 filter stalls at its rounding level."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _systems(chfsi):
    return {
        "local": chfsi.SyntheticSystem(config_index=0),
        "kb": chfsi.SyntheticSystem(config_index=1, n_bands=132),
        "uspp": chfsi.SyntheticSystem(config_index=2, n_rep=1, ecut=8.0, ngrid=[0, 0, 0],
                                      n_bands=24),
    }


@pytest.mark.parametrize("kind", ["local", "kb", "uspp"])
def test_rchfsi_fp64_matches_oracle(chfsi, oracle, kind):
    s = _systems(chfsi)[kind]
    ndeg = 12
    ctx = chfsi.Context(s, filter_form=chfsi.FILTER_RESIDUAL)
    o = oracle.Oracle.from_system(s)
    if s.uspp:
        ctx.set_qmat(s.qmat())
        o.set_qmat(s.qmat())
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    wg = ctx.diagonalize(ndeg)           # no Ritz values yet: Chebyshev filter
    wc = o.diagonalize(ndeg)
    np.testing.assert_allclose(wg, wc, atol=1e-10, rtol=0)
    for _ in range(2 if kind != "kb" else 1):  # residual filter from the Ritz pairs
        wg_next = ctx.diagonalize(ndeg, wg)
        wc_next = o.rchfsi_diagonalize(ndeg, wc)
        err = np.abs(wg_next - wc_next).max()
        print("%s R-ChFSI pass: device vs oracle %.3e Ha" % (kind, err))
        np.testing.assert_allclose(wg_next, wc_next, atol=1e-10, rtol=0)
        np.testing.assert_allclose(ctx.bounds(), o.bounds(), rtol=1e-12)
        wg, wc = wg_next, wc_next


@pytest.mark.parametrize("kind", ["kb", "uspp"])
def test_mixed_rchfsi_reaches_fp64_eigenvalues(chfsi, kind):
    s = _systems(chfsi)[kind]
    ndeg = 12
    ctxs = {"fp64": chfsi.Context(s),
            "mixed": chfsi.Context(s, precision=chfsi.PREC_MIXED),
            "mixed_rchfsi": chfsi.Context(s, precision=chfsi.PREC_MIXED,
                                          filter_form=chfsi.FILTER_RESIDUAL)}
    v = ctxs["fp64"].get_vloc()
    for c in ctxs.values():
        if s.uspp:
            c.set_qmat(s.qmat())
        c.set_veff(v)
    ref = ctxs["fp64"].diagonalize(ndeg)
    for _ in range(40):
        ref = ctxs["fp64"].diagonalize(ndeg, ref)
    n_occ = s.n_occ
    err = {}
    for name in ("mixed", "mixed_rchfsi"):
        c = ctxs[name]
        w = c.diagonalize(ndeg)
        hist = []
        for _ in range(40):
            w = c.diagonalize(ndeg, w)
            hist.append(np.abs(w[:n_occ] - ref[:n_occ]).max())
        err[name] = min(hist[-5:])
        print("%s %s: occupied-eigenvalue error vs converged FP64 over passes %s"
              % (kind, name, " ".join("%.1e" % h for h in hist[::5])))
    assert err["mixed_rchfsi"] < 1e-9
    assert err["mixed_rchfsi"] < err["mixed"]
