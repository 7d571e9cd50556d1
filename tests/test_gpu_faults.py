"""Error paths driven by host-side fault injection (no GPU fault is made).

* A tensor-core GEMM whose producer issues no loads: the MMA warp's bounded
  wait runs out (20 ms), the kernel retires what it issued, frees its TMEM and
  returns; the call reports CHFSI_ERR_TIMEOUT and the context stays usable
  (the next pass matches a fresh context's).
* A device allocation that fails inside chfsi_create: CHFSI_ERR_OUT_OF_MEMORY,
  nothing leaks into the next context.
* A learned mixer whose output is not finite: the SCF falls back to Pulay and
  converges (the fallback rule of the learned mixers).
Error variants follow src/types.rs:226-248 (Cuda / OutOfMemory) plus the
TIMEOUT status of the drop-in boundary.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def sys_kb(chfsi):
    # 8-atom cell with Kleinman-Bylander projectors (l = 0, 1): the mixed
    # filter's projector products run on the tensor cores
    return chfsi.SyntheticSystem(config_index=0, n_shell=1, lmax=1, rc_proj=[1.2, 0, 0, 0],
                                 d_min=0.5, d_max=2.0)


@pytest.fixture(autouse=True)
def _clear(chfsi):
    yield
    chfsi.inject_fault(chfsi.INJECT_NONE)


def test_tensor_core_wait_timeout_is_reported_and_recoverable(chfsi, sys_kb):
    assert sys_kb.n_proj > 0
    ctx = chfsi.Context(sys_kb, precision=chfsi.PREC_MIXED)
    ref = chfsi.Context(sys_kb, precision=chfsi.PREC_MIXED)
    v = ref.get_vloc()
    ctx.set_veff(v)
    ref.set_veff(v)
    # the first pass (no Ritz values yet) is FP64; the second is mixed and
    # runs the projector products on the tensor cores
    w = ctx.diagonalize(8)
    wr = ref.diagonalize(8)
    psi1 = ctx.get_psi()
    chfsi.inject_fault(chfsi.INJECT_TC_NO_LOADS, 1)
    with pytest.raises(chfsi.Timeout, match="timed out"):
        ctx.diagonalize(8, w)
    chfsi.inject_fault(chfsi.INJECT_NONE)
    # the context is usable: the same mixed pass from the same start as the
    # context that saw no fault
    ctx.set_psi(psi1)
    w1 = ctx.diagonalize(8, w)
    w2 = ref.diagonalize(8, wr)
    np.testing.assert_allclose(w1, w2, atol=1e-12, rtol=0)


def test_bf16x3_entry_point_timeout(chfsi):
    rng = np.random.default_rng(3)
    m, n, k = 64, 96, 4000
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    B = rng.standard_normal((n, k)) + 1j * rng.standard_normal((n, k))
    a = torch.from_numpy(A).cuda()
    b = torch.from_numpy(B).cuda()
    c = torch.zeros((m, n), dtype=torch.complex128, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    chfsi.inject_fault(chfsi.INJECT_TC_NO_LOADS, 1)
    with pytest.raises(chfsi.Timeout):
        chfsi.zgemm_cn_bf16x3(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(), st)
    chfsi.zgemm_cn_bf16x3(a.data_ptr(), k, b.data_ptr(), k, m, n, k, c.data_ptr(), st)
    ref = A.conj() @ B.T
    err = np.abs(c.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 1e-6


@pytest.mark.parametrize("nth", [0, 5, 20])
def test_allocation_failure_in_create(chfsi, sys_kb, nth):
    chfsi.inject_fault(chfsi.INJECT_ALLOC_FAIL, nth)
    with pytest.raises(chfsi.OutOfMemory):
        chfsi.Context(sys_kb)
    chfsi.inject_fault(chfsi.INJECT_NONE)
    ctx = chfsi.Context(sys_kb)
    ctx.set_veff(ctx.get_vloc())
    w = ctx.diagonalize(8)
    assert np.all(np.isfinite(w))


def test_non_finite_learned_mixer_falls_back_to_pulay(chfsi):
    s = chfsi.SyntheticSystem(config_index=0)
    m = chfsi.Mixer(device=0, seed=1)
    p = m.get_params()
    p[:] = np.nan
    m.set_params(p)
    ctx = chfsi.Context(s)
    ctx.set_mixer(m)
    r = ctx.run_scf(12, tol_per_atom=1e-6, max_iter=40, kT=0.01,
                    mixer=chfsi.MIXER_LEARNED_PULAY)
    assert r["fell_back"]
    assert r["converged"]
    assert np.isfinite(r["e_total"])
    plain = chfsi.Context(s).run_scf(12, tol_per_atom=1e-6, max_iter=40, kT=0.01)
    # after the first (fallen-back) step the run is plain Pulay
    assert abs(r["e_total"] - plain["e_total"]) / s.n_atoms < 1e-6


def test_stalled_learned_mixer_hands_over_to_pulay(chfsi):
    # a network with all weights zero outputs a_s = b_s = 0: the learned
    # steps leave the density where it is, the residual stops falling, and
    # the stall rule (or the rise rule) hands the run to Pulay
    s = chfsi.SyntheticSystem(config_index=0)
    m = chfsi.Mixer(device=0, seed=1)
    p = m.get_params()
    p[:] = 0.0
    m.set_params(p)
    ctx = chfsi.Context(s)
    ctx.set_mixer(m)
    r = ctx.run_scf(12, tol_per_atom=1e-6, max_iter=60, kT=0.01,
                    mixer=chfsi.MIXER_LEARNED_PULAY)
    assert r["fell_back"]
    assert r["converged"]
    assert r["n_iter_learned"] <= 12
    plain = chfsi.Context(s).run_scf(12, tol_per_atom=1e-6, max_iter=60, kT=0.01)
    assert abs(r["e_total"] - plain["e_total"]) / s.n_atoms < 1e-6
