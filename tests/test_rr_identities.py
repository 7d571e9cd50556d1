"""CPU checks, on the oracle, of the identities behind the mixed-precision
Rayleigh-Ritz.  Its FP32 filter hands over only the local part H_loc psi of
the last filter step; the subspace matrices are then assembled in FP64 as

    H_sub = psi^H (H_loc psi) + C^H D C,    S_sub = psi^H psi + C^H q C,

with C = beta^H psi (one projection shared by both).  On the oracle these must
equal the reference's psi^H (H psi) with the full operator
(src/eigensolver/chebyshev.rs:371-403, rayleigh_ritz.rs:48-245) and psi^H S psi
of the ultrasoft overlap (tests/phase0_gate2_convergence.rs:279-322)."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def uspp8(chfsi):
    # the 216-atom ultrasoft model on its 8-atom cell (per-ion D and q blocks)
    return chfsi.SyntheticSystem(config_index=2, n_rep=1, ecut=10.0, ngrid=(0, 0, 0), n_bands=0,
                                 ngrid_density=(32, 32, 32))


def _blocks_apply(blocks, off, c):
    """Per-ion ne x ne blocks (row-major, concatenated) applied to C (n_proj x nb)."""
    out = np.zeros_like(c)
    pos = 0
    for i in range(len(off) - 1):
        p0, ne = off[i], off[i + 1] - off[i]
        b = blocks[pos:pos + ne * ne].reshape(ne, ne)
        out[p0:p0 + ne] = b @ c[p0:p0 + ne]
        pos += ne * ne
    return out


def test_subspace_matrices_from_local_part_and_projections(uspp8, oracle):
    s = uspp8
    o = oracle.Oracle.from_system(s)
    rng = np.random.default_rng(3)
    v = o.vloc_r() + 0.05 * rng.standard_normal(s.ng)
    o.set_veff(v)
    psi = s.psi0()[:6]
    dmat, qmat = s.dmat(), s.qmat()
    off = s.proj_offsets()
    assert np.abs(qmat).max() > 0 and np.abs(dmat).max() > 0

    h_full = o.apply_h(psi)
    o.set_dmat(np.zeros_like(dmat))
    h_loc = o.apply_h(psi)
    o.set_dmat(dmat)

    assert np.abs(h_full - h_loc).max() > 1e-3 * np.abs(h_full).max()  # non-local part matters
    c = s.beta().conj() @ psi.T  # C = beta^H psi, n_proj x nb
    h_ref = psi.conj() @ h_full.T
    h_sub = psi.conj() @ h_loc.T + c.conj().T @ _blocks_apply(dmat, off, c)
    assert np.abs(h_sub - h_ref).max() <= 1e-12 * np.abs(h_ref).max()

    o.set_qmat(qmat)
    s_ref = psi.conj() @ o.apply_s(psi).T
    assert np.abs(s_ref - psi.conj() @ psi.T).max() > 1e-5 * np.abs(s_ref).max()  # q part matters
    s_sub = psi.conj() @ psi.T + c.conj().T @ _blocks_apply(qmat, off, c)
    assert np.abs(s_sub - s_ref).max() <= 1e-12 * np.abs(s_ref).max()
    o.close()


def test_ultrasoft_filter_step_from_local_part_and_propagated_projection(uspp8, oracle):
    """The S^-1 H step of the ultrasoft filter needs only two n_pw-long
    projector products: with B = beta^H beta and M = q (1 + B q)^-1,
    S^-1 H x = H_loc x + beta X with X = D C - M (P + B D C), C = beta^H x,
    P = beta^H H_loc x, and beta^H of the next recurrence vector follows from
    beta^H S^-1 H x = P + B X without a projection.  Checked against the
    oracle's S^-1 H (cg_helpers.rs:86-92 Woodbury form) over eight steps of
    the Chebyshev recurrence in FP64."""
    s = uspp8
    full = oracle.Oracle.from_system(s)
    loc = oracle.Oracle.from_system(s)
    v = full.vloc_r()
    full.set_veff(v)
    loc.set_veff(v)
    qmat, dmat, off = s.qmat(), s.dmat(), s.proj_offsets()
    full.set_qmat(qmat)
    loc.set_dmat(np.zeros_like(dmat))
    beta = s.beta()
    n_proj = beta.shape[0]
    q = np.zeros((n_proj, n_proj), complex)
    pos = 0
    for i in range(len(off) - 1):
        p0, ne = off[i], off[i + 1] - off[i]
        q[p0:p0 + ne, p0:p0 + ne] = qmat[pos:pos + ne * ne].reshape(ne, ne)
        pos += ne * ne
    b = beta.conj() @ beta.T
    m = q @ np.linalg.inv(np.eye(n_proj) + b @ q)

    def step(x, cx):
        hx = loc.apply_h(x)
        p = beta.conj() @ hx.T
        dc = _blocks_apply(dmat, off, cx)
        xx = dc - m @ (p + b @ dc)
        return hx + (beta.T @ xx).T, p + b @ xx

    def sinv_h(x):
        return full.apply_sinv(full.apply_h(x))

    c, e = 20.5, 19.5
    x0 = s.psi0()[:6]
    y0, by0 = step(x0, beta.conj() @ x0.T)
    assert np.abs(y0 - sinv_h(x0)).max() <= 1e-13 * np.abs(y0).max()
    # recurrence psi_{k+1} = 2 (S^-1 H - c) psi_k / e - psi_{k-1}, both ways
    r_prev, r = x0, (sinv_h(x0) - c * x0) / e
    t_prev, t = x0, (y0 - c * x0) / e
    ct_prev, ct = beta.conj() @ x0.T, (by0 - c * (beta.conj() @ x0.T)) / e
    for _ in range(2, 9):
        y, by = step(t, ct)
        t_prev, t = t, 2 * (y - c * t) / e - t_prev
        ct_prev, ct = ct, 2 * (by - c * ct) / e - ct_prev
        r_prev, r = r, 2 * (sinv_h(r) - c * r) / e - r_prev
        assert np.abs(t - r).max() <= 1e-13 * np.abs(r).max()
        direct = beta.conj() @ t.T
        assert np.abs(ct - direct).max() <= 1e-13 * np.abs(direct).max()
    full.close()
    loc.close()
