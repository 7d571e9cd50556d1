"""Parity of the CUDA path (through the C ABI) against the CPU oracle.

FP64 tolerances: H|psi> 1e-12 relative; filtered psi 1e-10 relative;
eigenvalues and energies 1e-10 Ha (the bar for the plain FP64 method).
"""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def sys0(chfsi):
    return chfsi.SyntheticSystem(config_index=0)


@pytest.fixture(scope="module")
def sys1s(chfsi):
    # config-1 physics (64 atoms, KB projectors) with fewer bands: fast parity case
    return chfsi.SyntheticSystem(config_index=1, n_bands=132)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def gpu_apply(chfsi, ctx, psi):
    x = torch.from_numpy(np.ascontiguousarray(psi)).cuda()
    y = torch.empty_like(x)
    ctx.apply_h(x.data_ptr(), y.data_ptr(), psi.shape[0])
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.mark.parametrize("which", ["sys0", "sys1s"])
def test_apply_h_parity(chfsi, oracle, which, request):
    s = request.getfixturevalue(which)
    ctx = chfsi.Context(s)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r() + 0.05 * np.sin(np.arange(s.ng) * 1e-3)
    ctx.set_veff(v)
    o.set_veff(v)
    psi = s.psi0()[:8]
    h_gpu = gpu_apply(chfsi, ctx, psi)
    h_cpu = o.apply_h(psi)
    assert rel(h_gpu, h_cpu) < 1e-12


@pytest.mark.parametrize("which", ["sys0", "sys1s"])
def test_plane_kernel_variants_match_oracle(chfsi, oracle, which, request):
    """xy-plane pass with compile-time radices (launch configurations 0-8)
    and the generic plane kernel (9-17): both against the oracle, and
    against each other to rounding."""
    s = request.getfixturevalue(which)
    ctx = chfsi.Context(s)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r() + 0.05 * np.sin(np.arange(s.ng) * 1e-3)
    ctx.set_veff(v)
    o.set_veff(v)
    psi = s.psi0()[:8]
    h_cpu = o.apply_h(psi)
    out = {}
    for c in (1, 4, 7, 10, 13, 16):
        ctx.set_launch_config(c)
        out[c] = gpu_apply(chfsi, ctx, psi)
        assert rel(out[c], h_cpu) < 1e-12, c
    for c in (1, 4, 7):
        assert rel(out[c], out[c + 9]) < 1e-14


def test_plane_kernel_variants_agree_108(chfsi):
    """The 108^3 grid of the 216-atom cell (radices 12 x 9): compile-time and
    generic plane kernels give the same local H|psi> in FP64."""
    s = chfsi.SyntheticSystem(config_index=2)
    ctx = chfsi.Context(s)  # V_eff = V_loc after creation
    x = torch.from_numpy(np.ascontiguousarray(s.psi0()[:8])).cuda()
    ys = []
    for c in (1, 10):
        ctx.set_launch_config(c)
        y = torch.empty_like(x)
        ctx.apply_h_local(x.data_ptr(), y.data_ptr(), 8)
        torch.cuda.synchronize()
        ys.append(y.cpu().numpy())
    assert np.abs(ys[0]).max() > 0
    assert rel(ys[0], ys[1]) < 1e-14


def test_vloc_parity(chfsi, oracle, sys0):
    ctx = chfsi.Context(sys0)
    o = oracle.Oracle.from_system(sys0)
    np.testing.assert_allclose(ctx.get_vloc(), o.vloc_r(), atol=1e-12)


def test_filter_parity(chfsi, oracle, sys0):
    ctx = chfsi.Context(sys0)
    o = oracle.Oracle.from_system(sys0)
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    ctx.chebyshev_filter(12)
    st, _ = o.chebyshev_filter(12)
    assert st == 0
    np.testing.assert_allclose(ctx.bounds(), o.bounds(), rtol=1e-13)
    np.testing.assert_allclose(ctx.filter_norms(12), o.norms(), rtol=1e-11)
    assert rel(ctx.get_psi(), o.get_psi()) < 1e-10


@pytest.mark.parametrize("which,ndeg,passes", [("sys0", 12, 3), ("sys1s", 16, 2)])
def test_diagonalize_eigenvalue_parity(chfsi, oracle, which, ndeg, passes, request):
    s = request.getfixturevalue(which)
    ctx = chfsi.Context(s)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    wg = wc = None
    for _ in range(passes):
        wg = ctx.diagonalize(ndeg, wg)
        wc = o.diagonalize(ndeg, wc)
        np.testing.assert_allclose(wg, wc, atol=1e-10, rtol=0)


def test_golden_cfg0_first_iteration(chfsi, sys0):
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "cfg0_oracle.json")))
    ctx = chfsi.Context(sys0)
    ctx.set_veff(ctx.get_vloc())
    w = ctx.diagonalize(12)
    np.testing.assert_allclose(w, g["eig_iter1"], atol=1e-10, rtol=0)
    for _ in range(2):
        w = ctx.diagonalize(12, w)
    np.testing.assert_allclose(w, g["eig_iter3"], atol=1e-10, rtol=0)


def test_density_and_veff_parity(chfsi, oracle, sys0):
    ctx = chfsi.Context(sys0)
    o = oracle.Oracle.from_system(sys0)
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    w = ctx.diagonalize(12)
    o.diagonalize(12)
    ctx.set_occupations(sys0.occupations())
    rg = ctx.construct_density()
    rc = o.density()
    assert rel(rg, rc) < 1e-11
    assert abs(rg.sum() * sys0.omega / sys0.ng - 32.0) < 1e-9
    ctx.build_v_eff(rc)
    o.build_veff(rc)
    np.testing.assert_allclose(ctx.get_veff(), o.get_veff(), atol=1e-11)


def test_scf_energy_parity(chfsi, oracle, sys0):
    """Energies of six SCF iterations and the final eigenvalues at 1e-10 Ha,
    the plain method's bar (phase0_gate1 single-step tolerance)."""
    ctx = chfsi.Context(sys0)
    o = oracle.Oracle.from_system(sys0)
    rg = ctx.run_scf(12, max_iter=6, kT=0.01)
    rc = o.run_scf(12, max_iter=6, kT=0.01)
    de = np.abs(rg["energies"] - rc["energies"]).max()
    dw = np.abs(rg["eigenvalues"] - rc["eigenvalues"]).max()
    print("SCF parity: energies %.3e Ha, eigenvalues %.3e Ha" % (de, dw))
    np.testing.assert_allclose(rg["energies"], rc["energies"], atol=1e-10, rtol=0)
    np.testing.assert_allclose(rg["eigenvalues"], rc["eigenvalues"], atol=1e-10, rtol=0)


def test_diagonalize_parity_cfg1_all_bands(chfsi, oracle):
    """The 64-atom configuration at its full 160 bands: one degree-16 ChFSI
    iteration (filter + Rayleigh-Ritz) from the seeded start, 1e-10 Ha."""
    s = chfsi.SyntheticSystem(config_index=1)
    assert s.n_bands == 160
    ctx = chfsi.Context(s)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    wg = ctx.diagonalize(16)
    wc = o.diagonalize(16)
    print("160-band parity: %.3e Ha" % np.abs(wg - wc).max())
    np.testing.assert_allclose(wg, wc, atol=1e-10, rtol=0)


@pytest.mark.parametrize("kpt", [(0.125, 0.125, 0.375), (-0.375, 0.125, -0.125)])
def test_kpoint_member_parity(chfsi, oracle, kpt):
    """A k != 0 member of the 4x4x4 Monkhorst-Pack set of the 8-atom cell
    (|G+k|^2 kinetic, k-phased projectors) against the oracle: H|psi> and
    two ChFSI iterations."""
    s = chfsi.SyntheticSystem(config_index=0, kpt=kpt, n_shell=1, lmax=1,
                              rc_proj=[1.2, 0, 0, 0], d_min=0.5, d_max=2.0)
    assert s.n_proj > 0
    ctx = chfsi.Context(s)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    psi = s.psi0()[:8]
    assert rel(gpu_apply(chfsi, ctx, psi), o.apply_h(psi)) < 1e-12
    wg = wc = None
    for _ in range(2):
        wg = ctx.diagonalize(12, wg)
        wc = o.diagonalize(12, wc)
        np.testing.assert_allclose(wg, wc, atol=1e-10, rtol=0)


def test_scf_converges_cfg0(chfsi, oracle, sys0):
    g = json.load(open(os.path.join(ROOT, "tests", "golden", "cfg0_oracle.json")))
    ctx = chfsi.Context(sys0)
    r = ctx.run_scf(12, max_iter=40, kT=0.01)
    assert r["converged"]
    np.testing.assert_allclose(r["energies"][:3], g["scf_energies_3"], atol=1e-9)


def test_lanczos_bound_parity(chfsi, oracle, sys1s):
    ctx = chfsi.Context(sys1s, bound_mode=chfsi.BOUND_LANCZOS, lanczos_steps=10)
    o = oracle.Oracle.from_system(sys1s)
    o.set_bound_mode(1, 10)
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    ctx.chebyshev_filter(4)
    o.chebyshev_filter(4)
    np.testing.assert_allclose(ctx.bounds(), o.bounds(), rtol=1e-10)


def test_shuffled_plane_wave_order(chfsi, oracle, sys0):
    """The boundary accepts any plane-wave order (pw_coords_to_fft_indices)."""
    rng = np.random.default_rng(5)
    perm = rng.permutation(sys0.n_pw)
    mil = sys0.miller()[perm]
    kin = sys0.kinetic()[perm]
    psi = sys0.psi0()[:, perm]
    ctx = chfsi.Context(dims={"ngrid": sys0.ngrid, "n_pw": sys0.n_pw, "n_bands": sys0.n_bands})
    ctx.set_basis(mil, kin, sys0.gmax)
    ref = chfsi.Context(sys0)
    v = ref.get_vloc()
    ctx.set_veff(v)
    ref.set_veff(v)
    ctx.set_psi(psi)
    np.testing.assert_array_equal(ctx.get_psi(), psi)
    w1 = ctx.diagonalize(12)
    w2 = ref.diagonalize(12)
    np.testing.assert_allclose(w1, w2, atol=1e-10)


def test_rr_failure_is_reported(chfsi, sys0):
    ctx = chfsi.Context(sys0)
    ctx.set_veff(ctx.get_vloc())
    psi = sys0.psi0()
    psi[1] = psi[0]  # rank-deficient subspace -> S_sub not positive definite
    ctx.set_psi(psi)
    with pytest.raises(chfsi.RayleighRitzFailed):
        ctx.diagonalize(0)


def test_norm_guard_reports_divergence(chfsi, sys0):
    """chebyshev.rs:552-563: growth > 10x between degrees is ChebyshevDiverged.

    Previous eigenvalues far above the spectrum push the cut to 0.95 lambda_max
    (chebyshev.rs:243-249), so the whole occupied spectrum sits far below the
    filter interval and |psi_k| grows by ~2|sigma| per degree.
    """
    ctx = chfsi.Context(sys0)
    ctx.set_veff(ctx.get_vloc())
    with pytest.raises(chfsi.ChebyshevDiverged):
        ctx.chebyshev_filter(6, eigenvalues=np.linspace(0.0, 1e4, sys0.n_bands))


@pytest.mark.parametrize("n_bands,z_val", [(1, 0.25), (21, 4.0), (261, 4.0)])
def test_diagonalize_band_count_edges(chfsi, oracle, n_bands, z_val):
    """Band counts that exercise the eigensolver's edge paths: one band, an
    odd count (the round-robin Jacobi pads with a phantom index) and a count
    above 256 (the grid-wide Jacobi instead of the cluster one), against the
    oracle on the 8-atom cell."""
    s = chfsi.SyntheticSystem(config_index=0, n_bands=n_bands, z_val=z_val)
    assert s.n_bands == n_bands
    ctx = chfsi.Context(s)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r()
    ctx.set_veff(v)
    o.set_veff(v)
    wg = wc = None
    for _ in range(1 if n_bands > 256 else 2):  # the oracle's 261-band pass takes ~20 s
        wg = ctx.diagonalize(12, wg)
        wc = o.diagonalize(12, wc)
    print("%d bands: %.3e Ha" % (n_bands, np.abs(wg - wc).max()))
    np.testing.assert_allclose(wg, wc, atol=1e-10, rtol=0)


def test_fused_lanczos_bound_parity(chfsi, oracle, sys1s):
    """Lanczos bound carried as one extra column of the filter's own H
    applies (Zhou 2010; notes/pr-reviews/phase-2/deferred.md:131-161): the
    bound a filter leaves for the next one equals the oracle's separate
    k-step Lanczos bound on the same V_eff, and the filter that carries it
    launches no H|psi> pass beyond the heuristic-bound filter's (only the
    3k + 1 vector kernels of the Lanczos recurrence)."""
    k = 10
    fused = chfsi.Context(sys1s, bound_mode=chfsi.BOUND_LANCZOS_FUSED, lanczos_steps=k)
    plain = chfsi.Context(sys1s)
    o = oracle.Oracle.from_system(sys1s)
    o.set_bound_mode(1, k)
    v = o.vloc_r()
    for c in (fused, plain):
        c.set_veff(v)
    o.set_veff(v)
    fused.chebyshev_filter(16)   # first filter: separate Lanczos, carries the next one
    plain.chebyshev_filter(16)
    l0 = chfsi.launch_count()
    fused.chebyshev_filter(16)   # bound from the carried column
    l1 = chfsi.launch_count()
    plain.chebyshev_filter(16)
    l2 = chfsi.launch_count()
    o.chebyshev_filter(16)
    np.testing.assert_allclose(fused.bounds(), o.bounds(), rtol=1e-10)
    assert (l1 - l0) - (l2 - l1) == 3 * k + 1
