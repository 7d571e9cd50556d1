"""The oracle's PBE and Ewald-force restatements (oracle/gga_oracle.py):
PBE reduces to LDA exchange at zero gradient and its correction vanishes
there; V_xc is the functional derivative of E_xc (central differences of
E_xc along a smooth perturbation); the Ewald forces are minus the
derivative of the generator's Ewald energy (displaced atoms)."""
import numpy as np

import gga_oracle as go
import synth


def test_pbe_zero_gradient_limits():
    rho = np.array([1e-3, 1e-2, 0.1, 1.0])
    e = go.pbe_e(rho, np.zeros_like(rho))
    ex_lda = -0.75 * (3.0 / np.pi) ** (1.0 / 3.0) * rho ** (4.0 / 3.0)
    rs = (3.0 / (4.0 * np.pi * rho)) ** (1.0 / 3.0)
    b1, b2, b3, b4 = go.PW_B
    den = 2 * go.PW_A * (b1 * np.sqrt(rs) + b2 * rs + b3 * rs ** 1.5 + b4 * rs ** 2)
    ec = -2 * go.PW_A * (1 + go.PW_A1 * rs) * np.log(1 + 1 / den)
    np.testing.assert_allclose(e, ex_lda + rho * ec, rtol=1e-14)
    # large reduced gradient: F_x -> 1 + kappa
    big = go.pbe_e(np.array([0.1]), np.array([1e12]))
    assert np.all(np.isfinite(big))


def test_pbe_potential_is_the_functional_derivative():
    s = synth.System(config_index=0, ecut=6.0, ngrid=[0, 0, 0])
    n = s.ngrid
    z, y, x = np.meshgrid(*[np.arange(k) / k for k in n[::-1]], indexing="ij")
    rho = 0.05 * (1.0 + 0.4 * np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y) + 0.2 * np.cos(4 * np.pi * z))
    d = np.cos(2 * np.pi * (x + 2 * y)) * np.exp(np.sin(2 * np.pi * z))
    rho, d = rho.ravel(), d.ravel()
    lat = s.lattice
    _, v = go.pbe_exc_vxc(rho, n, lat)
    eps = 1e-5
    ep, _ = go.pbe_exc_vxc(rho + eps * d, n, lat)
    em, _ = go.pbe_exc_vxc(rho - eps * d, n, lat)
    dv = s.omega / rho.size
    fd = (ep - em) / (2 * eps)
    an = float(np.sum(v * d) * dv)
    assert abs(fd - an) < 1e-8 * max(1.0, abs(an))


def test_ewald_forces_are_minus_the_energy_gradient():
    s = synth.System(config_index=0)
    pos = s.positions()
    z = np.full(s.n_atoms, s.params.z_val)
    f = go.ewald_forces(s.lattice, pos, z)
    h = 1e-4
    for atom, ax in ((0, 0), (5, 2)):
        e = []
        for sg in (1, -1):
            p = pos.copy()
            p[atom, ax] += sg * h
            e.append(synth.System(config_index=0, positions=p).e_ewald)
        fd = -(e[0] - e[1]) / (2 * h)
        assert abs(fd - f[atom, ax]) < 1e-6, (atom, ax, fd, f[atom, ax])
    assert np.abs(f.sum(0)).max() < 1e-9
