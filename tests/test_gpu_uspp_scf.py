"""Ultrasoft SCF with augmentation charges on the device against the oracle
(oracle/uspp_oracle.py): density-grid interpolation, augmentation density,
screened D and energies per iteration, on the 8-atom cell of the 216-atom
ultrasoft model (density grid finer than the wavefunction grid) and with the
density grid equal to the wavefunction grid."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))


def _system(chfsi, dens):
    return chfsi.SyntheticSystem(config_index=2, n_rep=1, ecut=10.0, ngrid=(0, 0, 0), n_bands=0,
                                 ngrid_density=dens)


@pytest.mark.parametrize("dens", [(32, 32, 32), (0, 0, 0)])
def test_uspp_scf_energies_match_oracle(chfsi, dens):
    import uspp_oracle as uo
    s = _system(chfsi, dens)
    ref = uo.UsppScf(s).run_scf(12, max_iter=4)
    ctx = chfsi.Context(s)
    assert ctx.ngrid_density == s.ngrid_density
    r = ctx.run_scf(12, max_iter=4, kT=0.01)
    print("density grid %s: device %s oracle %s" % (s.ngrid_density, r["energies"], ref["energies"]))
    print("max energy difference %.3e Ha" % np.abs(r["energies"] - ref["energies"]).max())
    np.testing.assert_allclose(r["energies"], ref["energies"], rtol=0, atol=1e-10)
    rho = ctx.get_density()
    assert abs(rho.sum() * s.omega / rho.size - s.n_elec) < 1e-8
    np.testing.assert_allclose(rho, ref["rho"], rtol=0, atol=1e-8 * np.abs(ref["rho"]).max())


def test_uspp_scf_converges_to_oracle(chfsi):
    import uspp_oracle as uo
    s = _system(chfsi, (32, 32, 32))
    ref = uo.UsppScf(s).run_scf(12, max_iter=40)
    r = chfsi.Context(s).run_scf(12, max_iter=40, kT=0.01)
    print("converged: device %d iterations E %.10f, oracle %d iterations E %.10f"
          % (r["n_iter"], r["e_total"], ref["n_iter"], ref["energies"][-1]))
    assert r["converged"] and ref["converged"]
    assert abs(r["e_total"] - ref["energies"][-1]) / s.n_atoms < 1e-8
    np.testing.assert_allclose(r["eigenvalues"], ref["eigenvalues"], atol=1e-8)


def test_mixed_precision_uspp_scf_matches_fp64(chfsi):
    """FP32 filter of S^-1 H with tcgen05 projections, FP64 Rayleigh-Ritz with
    the ultrasoft overlap, final FP64 passes: same converged energy and
    occupied eigenvalues (within 1e-6 Ha) as the FP64 run, both converged to
    1e-9 Ha/atom so that the comparison measures precision, not the SCF stop."""
    s = _system(chfsi, (32, 32, 32))
    rf = chfsi.Context(s).run_scf(12, max_iter=80, kT=0.01, tol_per_atom=1e-9)
    rm = chfsi.Context(s, precision=chfsi.PREC_MIXED).run_scf(12, max_iter=80, kT=0.01,
                                                              tol_per_atom=1e-9,
                                                              fp64_switch_per_atom=1e-6)
    n_occ = int(round(s.n_elec / 2))
    de = abs(rm["e_total"] - rf["e_total"]) / s.n_atoms
    docc = np.abs(rm["eigenvalues"][:n_occ] - rf["eigenvalues"][:n_occ]).max()
    print("mixed ultrasoft SCF: %d iterations (%d mixed) vs %d; dE/atom %.2e, occupied eig %.2e"
          % (rm["n_iter"], rm["n_iter_mixed"], rf["n_iter"], de, docc))
    assert rf["converged"] and rm["converged"] and rm["n_iter_mixed"] >= 1
    assert de < 1e-8
    assert docc < 1e-6
