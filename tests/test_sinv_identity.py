"""Algebra of the ultrasoft filter operator as the device applies it.

With projector columns P (n_pw x n_proj), S = 1 + P q P^H and H = H_loc + P D P^H,
the Woodbury inverse is S^-1 = 1 - P M P^H with M = q (1 + B q)^-1, B = P^H P, and

    S^-1 H x = H_loc x - P F,   F = M (E + B G) - G,   G = D P^H x,   E = P^H (H_loc x),

two projections (P^H x, P^H H_loc x) and one expansion (P F) per application
(the form of sinv_h_parts / sinv_h_parts32 in the CUDA library)."""
import numpy as np


def _blocks(rng, n_ions, ne, scale):
    n = n_ions * ne
    out = np.zeros((n, n), dtype=complex)
    for i in range(n_ions):
        a = rng.standard_normal((ne, ne)) + 1j * rng.standard_normal((ne, ne))
        out[i * ne:(i + 1) * ne, i * ne:(i + 1) * ne] = scale * (a + a.conj().T) / 2
    return out


def test_woodbury_inverse_and_merged_form():
    rng = np.random.default_rng(11)
    npw, n_ions, ne, nb = 160, 3, 4, 7
    nproj = n_ions * ne
    P = 0.1 * (rng.standard_normal((npw, nproj)) + 1j * rng.standard_normal((npw, nproj)))
    q = _blocks(rng, n_ions, ne, 0.2)
    D = _blocks(rng, n_ions, ne, 1.0)
    a = rng.standard_normal((npw, npw)) + 1j * rng.standard_normal((npw, npw))
    h_loc = (a + a.conj().T) / 2
    x = rng.standard_normal((npw, nb)) + 1j * rng.standard_normal((npw, nb))

    S = np.eye(npw) + P @ q @ P.conj().T
    H = h_loc + P @ D @ P.conj().T
    B = P.conj().T @ P
    M = q @ np.linalg.inv(np.eye(nproj) + B @ q)
    s_inv = np.eye(npw) - P @ M @ P.conj().T
    np.testing.assert_allclose(s_inv @ S, np.eye(npw), atol=1e-12)

    G = D @ (P.conj().T @ x)
    E = P.conj().T @ (h_loc @ x)
    F = M @ (E + B @ G) - G
    merged = h_loc @ x - P @ F
    direct = np.linalg.solve(S, H @ x)
    np.testing.assert_allclose(merged, direct, atol=1e-11 * np.abs(direct).max())


def test_merged_form_with_singular_q():
    # M = q (1 + B q)^-1 needs no inverse of q (projector pairs without
    # augmentation give zero blocks)
    rng = np.random.default_rng(12)
    npw, nproj, nb = 90, 8, 3
    P = 0.2 * (rng.standard_normal((npw, nproj)) + 1j * rng.standard_normal((npw, nproj)))
    q = np.zeros((nproj, nproj), dtype=complex)
    q[:4, :4] = _blocks(rng, 1, 4, 0.3)
    D = _blocks(rng, 2, 4, 1.0)
    h_loc = np.diag(rng.uniform(0.0, 5.0, npw)).astype(complex)
    x = rng.standard_normal((npw, nb)) + 1j * rng.standard_normal((npw, nb))
    S = np.eye(npw) + P @ q @ P.conj().T
    B = P.conj().T @ P
    M = q @ np.linalg.inv(np.eye(nproj) + B @ q)
    G = D @ (P.conj().T @ x)
    F = M @ (P.conj().T @ (h_loc @ x) + B @ G) - G
    direct = np.linalg.solve(S, (h_loc + P @ D @ P.conj().T) @ x)
    np.testing.assert_allclose(h_loc @ x - P @ F, direct, atol=1e-11 * np.abs(direct).max())
