"""Band-parallel ChFSI on the device (chemrust-scf_b200/band_parallel.py) at
world size 1: the block filter plus the band-split Rayleigh-Ritz on the
library's GEMMs and eigensolver (chfsi_zgemm_cn, chfsi_zgemm_tn,
chfsi_hegv_dev) against the context's own diagonalisation, 1e-10 Ha."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "chemrust-scf_b200"))


def test_band_parallel_world1_matches_context(chfsi):
    import band_parallel as bp
    s = chfsi.SyntheticSystem(config_index=1, n_bands=132)
    ref = chfsi.Context(s)
    v = ref.get_vloc()
    ref.set_veff(v)
    par = bp.BandParallelChfsi(s)
    par.set_veff(v)
    wr = wp = None
    for _ in range(2):
        wr = ref.diagonalize(16, wr)
        wp = par.diagonalize(16, wp)
        print("band-parallel vs context: %.3e Ha" % np.abs(wp - wr).max())
        np.testing.assert_allclose(wp, wr, atol=1e-10, rtol=0)


def test_hegv_dev_known_answer(chfsi):
    """solver.rs:113-163: diag(1, 2, 3, 4) with B = I gives 1, 2, 3, 4; and the
    4 x 4 pair of subspace_diag.rs:535-590 against the oracle's eigensolver."""
    import torch
    import oracle
    h = torch.diag(torch.tensor([1.0, 2.0, 3.0, 4.0], dtype=torch.complex128)).cuda()
    s = torch.eye(4, dtype=torch.complex128).cuda()
    v = torch.empty_like(h)
    w = chfsi.hegv_dev(h.data_ptr(), s.data_ptr(), 4, v.data_ptr())
    np.testing.assert_allclose(w, [1, 2, 3, 4], atol=1e-12)
    rng = np.random.default_rng(4)
    a = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    b = rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))
    H = a + a.conj().T
    S = b @ b.conj().T + 6 * np.eye(6)
    wo, _ = oracle.hegv(H, S)
    ht, st = torch.from_numpy(H).cuda(), torch.from_numpy(S).cuda()
    v = torch.empty_like(ht)
    w = chfsi.hegv_dev(ht.data_ptr(), st.data_ptr(), 6, v.data_ptr())
    np.testing.assert_allclose(w, wo, atol=1e-12)
    V = v.cpu().numpy()
    np.testing.assert_allclose(V.conj().T @ S @ V, np.eye(6), atol=1e-12)
    np.testing.assert_allclose(H @ V, S @ V @ np.diag(w), atol=1e-11)
