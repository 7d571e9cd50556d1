"""Pins the CPU oracle to the reference's known-answer tests and to independent
numpy / scipy restatements (no GPU needed)."""
import json
import os

import numpy as np
import pytest

from conftest import ROOT

GOLD = os.path.join(ROOT, "tests", "golden")


def ka():
    return json.load(open(os.path.join(GOLD, "reference_known_answers.json")))


def test_rr_4x4_known_eigenvalues(oracle):
    # subspace_diag.rs:535-590 (generalised RR via Cholesky reduction)
    c = ka()["rr_4x4"]
    w, v = oracle.hegv(np.diag(c["h_diag"]).astype(complex), np.diag(c["s_diag"]).astype(complex))
    np.testing.assert_allclose(w, c["expected"], atol=c["tol"], rtol=0)
    # eigenvectors are S-orthonormal
    S = np.diag(c["s_diag"])
    np.testing.assert_allclose(v.conj().T @ S @ v, np.eye(4), atol=1e-12)


def test_zhegvd_known_eigenvalues(oracle):
    # solver.rs:113-163
    c = ka()["zhegvd_4x4"]
    w, _ = oracle.hegv(np.diag(c["a_diag"]).astype(complex), np.eye(4, dtype=complex))
    np.testing.assert_allclose(w, c["expected"], atol=c["tol"], rtol=0)


def test_fft_forward_inverse_identity(oracle):
    # fft.rs:239-281: 8^3, input[i] = (i, 2i) for i < 10, forward then inverse = N^3 x
    c = ka()["fft_8cubed_identity"]
    n = c["n"]
    x = np.zeros(n[0] * n[1] * n[2], complex)
    for i in range(c["nonzero"]):
        x[i] = i + 2j * i
    g = x.reshape(n[2], n[1], n[0])
    y = oracle.fft3d(oracle.fft3d(g, -1), +1).ravel() / np.prod(n)
    assert np.abs(y - x).max() < c["tol"]


@pytest.mark.parametrize("shape", [(8, 8, 8), (40, 40, 40), (12, 10, 15), (9, 6, 5)])
def test_fft_matches_numpy(oracle, shape):
    rng = np.random.default_rng(3)
    g = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    np.testing.assert_allclose(oracle.fft3d(g, -1), np.fft.fftn(g), atol=1e-9 * np.sqrt(g.size))
    np.testing.assert_allclose(oracle.fft3d(g, +1), np.fft.ifftn(g) * g.size,
                               atol=1e-9 * np.sqrt(g.size))


def test_lcg_matches_reference_sequence():
    c = ka()["lcg_seed42"]
    s, out = 42, []
    for _ in range(8):
        s = (s * 25214903917 + 11) & 0xFFFFFFFFFFFF
        out.append(s / 281474976710656.0)
    np.testing.assert_array_equal(out, c["first8"])


def lcg_matrix(seed, rows, cols):
    s = seed
    out = np.zeros((rows, cols), complex)
    for i in range(rows):
        for j in range(cols):
            s = (s * 25214903917 + 11) & 0xFFFFFFFFFFFF
            re = s / 281474976710656.0 - 0.5
            s = (s * 25214903917 + 11) & 0xFFFFFFFFFFFF
            im = s / 281474976710656.0 - 0.5
            out[i, j] = re + 1j * im
    return out


def test_hegv_matches_scipy(oracle):
    scipy_linalg = pytest.importorskip("scipy.linalg")
    psi = lcg_matrix(42, 12, 40)
    hp = lcg_matrix(7, 40, 40)
    hp = hp + hp.conj().T
    H = psi.conj() @ hp @ psi.T
    S = psi.conj() @ psi.T
    w, v = oracle.hegv(H, S)
    ws = scipy_linalg.eigh(H, S, eigvals_only=True)
    np.testing.assert_allclose(w, ws, atol=1e-10 * np.abs(ws).max())
    # S-orthonormality after rotation (subspace_diag.rs:681-865, < 1e-10)
    np.testing.assert_allclose(v.conj().T @ S @ v, np.eye(12), atol=1e-10)
    np.testing.assert_allclose(v.conj().T @ H @ v, np.diag(w), atol=1e-9)


def test_hegv_rejects_indefinite_overlap(oracle):
    with pytest.raises(RuntimeError):
        oracle.hegv(np.eye(3, dtype=complex), np.diag([1.0, -1.0, 1.0]).astype(complex))


def numpy_apply_h(s, o, psi, veff):
    """Independent H|psi> with numpy FFTs (chebyshev.rs:279-365, 416-500)."""
    nx, ny, nz = s.ngrid
    mil = s.miller()
    kin = s.kinetic()
    out = np.empty_like(psi)
    V = veff.reshape(nz, ny, nx)
    for b in range(psi.shape[0]):
        g = np.zeros((nz, ny, nx), complex)
        g[mil[:, 2] % nz, mil[:, 1] % ny, mil[:, 0] % nx] = psi[b]
        r = np.fft.ifftn(g) * g.size
        back = np.fft.fftn(r * V)
        out[b] = kin * psi[b] + back[mil[:, 2] % nz, mil[:, 1] % ny, mil[:, 0] % nx] / g.size
    if s.n_proj:
        beta = s.beta()
        off = s.proj_offsets()
        dm = s.dmat()
        D = np.zeros((s.n_proj, s.n_proj), complex)
        pos = 0
        for i in range(len(off) - 1):
            ne = off[i + 1] - off[i]
            D[off[i]:off[i + 1], off[i]:off[i + 1]] = dm[pos:pos + ne * ne].reshape(ne, ne)
            pos += ne * ne
        out += (beta.T @ (D @ (beta.conj() @ psi.T))).T
    return out


def small_system(chfsi, cfg=1):
    return chfsi.SyntheticSystem(config_index=cfg, n_rep=1, ecut=5.0, ngrid=[0, 0, 0], n_bands=20)


@pytest.mark.parametrize("cfg", [0, 1])
def test_oracle_apply_h_matches_numpy(chfsi, oracle, cfg):
    s = small_system(chfsi, cfg)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r() + 0.1 * np.cos(np.arange(s.ng) * 0.001)
    o.set_veff(v)
    psi = s.psi0()
    np.testing.assert_allclose(o.apply_h(psi), numpy_apply_h(s, o, psi, v), atol=1e-11)


def test_vloc_r_is_inverse_fft_of_vloc_g(chfsi, oracle, cfg0):
    o = oracle.Oracle.from_system(cfg0)
    nx, ny, nz = cfg0.ngrid
    ref = (np.fft.ifftn(cfg0.vloc_g().reshape(nz, ny, nx)) * cfg0.ng).real.ravel()
    np.testing.assert_allclose(o.vloc_r(), ref, atol=1e-12)


def test_filter_matches_numpy_recurrence(chfsi, oracle):
    s = small_system(chfsi, 1)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r()
    o.set_veff(v)
    psi = s.psi0()
    st, _ = o.chebyshev_filter(6)
    assert st == 0
    lm, cut, c, e = o.bounds()
    kin_max = 0.5 * s.gmax ** 2
    assert lm == pytest.approx(kin_max + v.max() - v.min(), rel=1e-14)
    assert cut == pytest.approx(lm / 3, rel=1e-14)
    a = psi
    h = numpy_apply_h(s, o, a, v)
    b = h / e - c / e * a
    for _ in range(2, 7):
        h = numpy_apply_h(s, o, b, v)
        a, b = b, 2 * (h / e - c / e * b) - a
    scale = np.abs(b).max()
    np.testing.assert_allclose(o.get_psi(), b, atol=1e-11 * scale)
    np.testing.assert_allclose(o.get_hpsi(), numpy_apply_h(s, o, b, v), atol=1e-10 * scale)


def test_rr_eigenvalues_match_dense_diagonalisation(chfsi, oracle):
    """After enough filter passes the Ritz values equal the lowest eigenvalues of H."""
    scipy_linalg = pytest.importorskip("scipy.linalg")
    s = small_system(chfsi, 1)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r()
    o.set_veff(v)
    w = o.diagonalize(10)
    for _ in range(25):
        w = o.diagonalize(10, w)
    Hd = numpy_apply_h(s, o, np.eye(s.n_pw, dtype=complex), v)  # rows = H e_g
    Hd = Hd.T
    ev = scipy_linalg.eigh(0.5 * (Hd + Hd.conj().T), eigvals_only=True)[: s.n_bands]
    np.testing.assert_allclose(w[:16], ev[:16], atol=1e-8)


def test_lanczos_bound_is_an_upper_bound(chfsi, oracle):
    scipy_linalg = pytest.importorskip("scipy.linalg")
    s = small_system(chfsi, 1)
    o = oracle.Oracle.from_system(s)
    v = o.vloc_r()
    o.set_veff(v)
    o.set_bound_mode(1, 10)
    o.chebyshev_filter(2)
    lm = o.bounds()[0]
    Hd = numpy_apply_h(s, o, np.eye(s.n_pw, dtype=complex), v).T
    emax = scipy_linalg.eigh(0.5 * (Hd + Hd.conj().T), eigvals_only=True)[-1]
    assert emax <= lm <= emax * 1.5


def test_fermi_occupations(oracle):
    e = np.linspace(-1, 1, 21)
    f, ts = oracle.fermi(e, 16.0, 0.01)
    assert abs(f.sum() - 16.0) < 1e-10 and np.all(np.diff(f) <= 0)
    assert ts <= 0
    f0, ts0 = oracle.fermi(e, 16.0, 0.0)
    assert np.all(f0[:8] == 2) and np.all(f0[8:] == 0) and ts0 == 0


def test_cfg0_golden_regression(chfsi, oracle, cfg0):
    g = json.load(open(os.path.join(GOLD, "cfg0_oracle.json")))
    o = oracle.Oracle.from_system(cfg0)
    o.set_veff(o.vloc_r())
    w = o.diagonalize(12)
    np.testing.assert_allclose(w, g["eig_iter1"], atol=1e-10)
    np.testing.assert_allclose(o.bounds(), g["bounds_iter1"], rtol=1e-13)


def uspp_small(chfsi):
    # ultrasoft physics of the 216-atom configuration on one conventional cell
    return chfsi.SyntheticSystem(config_index=2, n_rep=1, ecut=4.0, ngrid=[0, 0, 0], n_bands=20)


def dense_s(s):
    beta = s.beta()
    off = s.proj_offsets()
    qm = s.qmat()
    Q = np.zeros((s.n_proj, s.n_proj), complex)
    pos = 0
    for i in range(len(off) - 1):
        ne = off[i + 1] - off[i]
        Q[off[i]:off[i + 1], off[i]:off[i + 1]] = qm[pos:pos + ne * ne].reshape(ne, ne)
        pos += ne * ne
    return np.eye(s.n_pw) + beta.T @ Q @ beta.conj()


def test_uspp_overlap_and_woodbury_inverse(chfsi, oracle):
    s = uspp_small(chfsi)
    o = oracle.Oracle.from_system(s)
    o.set_qmat(s.qmat())
    x = s.psi0()[:4]
    Sd = dense_s(s)
    np.testing.assert_allclose(o.apply_s(x), (Sd @ x.T).T, atol=1e-12)
    np.testing.assert_allclose(o.apply_sinv(o.apply_s(x)), x, atol=1e-11)
    ev = np.linalg.eigvalsh(0.5 * (Sd + Sd.conj().T))
    assert ev.min() > 0 and o.s_min() <= ev.min() + 1e-12


def test_uspp_generalised_ritz_values(chfsi, oracle):
    """Filtered subspace iteration on S^-1 H converges to the lowest
    generalised eigenvalues of (H, S) (the H psi = e S psi problem)."""
    scipy_linalg = pytest.importorskip("scipy.linalg")
    s = uspp_small(chfsi)
    o = oracle.Oracle.from_system(s)
    o.set_qmat(s.qmat())
    v = o.vloc_r()
    o.set_veff(v)
    w = o.diagonalize(10)
    for _ in range(30):
        w = o.diagonalize(10, w)
    Hd = numpy_apply_h(s, o, np.eye(s.n_pw, dtype=complex), v).T
    Sd = dense_s(s)
    ev = scipy_linalg.eigh(0.5 * (Hd + Hd.conj().T), 0.5 * (Sd + Sd.conj().T), eigvals_only=True)
    np.testing.assert_allclose(w[:16], ev[:16], atol=1e-8)
    # the rotated bands are S-orthonormal
    psi = o.get_psi()
    np.testing.assert_allclose(psi.conj() @ o.apply_s(psi).T, np.eye(s.n_bands), atol=1e-10)


@pytest.mark.parametrize("case", ["line_search_parabola", "line_search_rational", "line_search_clamp",
                                  "line_search_no_minimum"])
def test_line_search_known_answers(oracle, case):
    # line_search.rs:217-394
    c = ka()[case]
    step, eig, norm, status = oracle.line_search(*c["args"])
    assert abs(step - c["step"]) < c.get("tol", 1e-12)
    if "eigenvalue" in c:
        assert abs(eig - c["eigenvalue"]) < c["tol"]
    if "status" in c:
        assert status == c["status"]
    if "norm" in c:
        assert abs(norm - c["norm"]) < 1e-12


@pytest.mark.parametrize("args", [(-0.4, -0.15, 1.2, 0.8), (-0.38, -0.2, 1.5, 0.7)])
def test_line_search_energy_decreases(oracle, args):
    # line_search.rs energy_decrease / energy_monotonicity
    step, eig, norm, status = oracle.line_search(*args)
    assert eig <= args[0] + 1e-14 and norm > 0 and step > 0 and status in (0, -1)


def test_tpa_diag_properties(oracle):
    # uspp_preconditioner.rs: T(0) = 1, monotone decreasing, floor > 0
    k = np.linspace(0.0, 40.0, 200)
    t = oracle.tpa_diag(k)
    assert abs(t[0] - 1.0) < 1e-15 and np.all(np.diff(t) <= 0) and t[-1] > 0


def test_band_cg_refines_towards_eigenpairs(chfsi, oracle):
    """band_cg.rs semantics: after a coarse filter, a few CG steps per band lower
    the band energies towards the exact generalised eigenvalues and keep the
    refined bands S-orthonormal (cg_helpers.rs S-orthogonalisation)."""
    scipy_linalg = pytest.importorskip("scipy.linalg")
    s = uspp_small(chfsi)
    o = oracle.Oracle.from_system(s)
    o.set_qmat(s.qmat())
    v = o.vloc_r()
    o.set_veff(v)
    w = o.diagonalize(8)
    w = o.diagonalize(8, w)
    e, steps, nconv = o.band_cg(6, 1e-10)
    Hd = numpy_apply_h(s, o, np.eye(s.n_pw, dtype=complex), v).T
    Sd = dense_s(s)
    ev = scipy_linalg.eigh(0.5 * (Hd + Hd.conj().T), 0.5 * (Sd + Sd.conj().T), eigvals_only=True)
    # Ky Fan: the band energies of an S-orthonormal set sum to at least the sum
    # of the lowest exact eigenvalues; CG lowers that sum from the Ritz values
    k = 12
    assert e[:k].sum() >= ev[:k].sum() - 1e-10
    assert e[:k].sum() <= w[:k].sum() + 1e-10
    assert np.all(steps >= 1)
    # each refined band is S-normalised (cg_helpers.rs s_normalize)
    psi = o.get_psi()
    np.testing.assert_allclose(np.einsum("bg,bg->b", psi.conj(), o.apply_s(psi)).real, 1.0, atol=1e-10)
