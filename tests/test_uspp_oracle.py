"""CPU checks of the ultrasoft SCF oracle with augmentation charges on a
finer density grid (oracle/uspp_oracle.py): charge conservation through the
augmentation (int rho = N_e for S-orthonormal wavefunctions) and the grid
transfers between the wavefunction and density grids."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))


@pytest.fixture(scope="module")
def small_uspp(chfsi):
    # the 216-atom ultrasoft model on its 8-atom cell: 2 shells x (l = 0, 1),
    # q_ij Gaussians of width 0.8, density grid finer than the FFT grid
    return chfsi.SyntheticSystem(config_index=2, n_rep=1, ecut=10.0, ngrid=(0, 0, 0), n_bands=0,
                                 ngrid_density=(32, 32, 32))


def test_grid_transfer_round_trip(small_uspp):
    import uspp_oracle as uo
    u = uo.UsppScf(small_uspp)
    rng = np.random.default_rng(0)
    nx, ny, nz = u.nw
    w = rng.standard_normal(nx * ny * nz)
    # a wave-grid field without Nyquist content survives up -> down exactly
    cw = np.fft.fftn(w.reshape(nz, ny, nx)) / w.size
    for ax, n in zip((2, 1, 0), (nz, ny, nx)):
        if n % 2 == 0:
            idx = [slice(None)] * 3
            idx[ax] = n // 2
            cw[tuple(idx)] = 0
    w0 = (np.fft.ifftn(cw) * cw.size).real.ravel()
    up = u.up_coeffs(cw).real.ravel()
    np.testing.assert_allclose(u.down(up), w0, atol=1e-12)
    # the mean is kept by the interpolation
    assert abs(up.mean() - w0.mean()) < 1e-12


def test_uspp_scf_conserves_charge(small_uspp):
    import uspp_oracle as uo
    u = uo.UsppScf(small_uspp)
    r = u.run_scf(12, max_iter=3)
    q = r["rho"].sum() * small_uspp.omega / r["rho"].size
    assert abs(q - small_uspp.n_elec) < 1e-8
    assert np.isfinite(r["energies"]).all()
    # the augmentation carries a share of the charge
    occ, _ = __import__("oracle").fermi(r["eigenvalues"], small_uspp.n_elec, 0.01)
    rho_aug, c = u.density(occ)
    assert np.abs(c).max() > 1e-4
