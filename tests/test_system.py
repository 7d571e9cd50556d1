"""Synthetic-system generator (host set-up code) against direct numpy formulas."""
import math

import numpy as np
import pytest


def test_sphere_matches_brute_force(cfg0):
    s = cfg0
    a = s.lattice[0, 0]
    b = 2 * np.pi / a
    m = 12
    r = np.arange(-m, m + 1)
    h, k, l = np.meshgrid(r, r, r, indexing="ij")
    g2 = b * b * (h * h + k * k + l * l)
    assert s.n_pw == int(np.count_nonzero(0.5 * g2 <= s.params.ecut))
    mil = s.miller()
    assert len({tuple(x) for x in mil}) == s.n_pw
    kin = s.kinetic()
    np.testing.assert_allclose(kin, 0.5 * b * b * (mil ** 2).sum(1), rtol=1e-14)
    assert kin.max() <= s.params.ecut + 1e-12
    assert abs(0.5 * s.gmax ** 2 - kin.max()) < 1e-12


def test_plane_waves_sorted_by_column(cfg0):
    s = cfg0
    nx, ny, nz = s.ngrid
    mil = s.miller()
    col = (mil[:, 1] % ny) * nx + (mil[:, 0] % nx)
    assert np.all(np.diff(col) >= 0)
    same = np.diff(col) == 0
    assert np.all(np.diff(mil[:, 2])[same] == 1)  # contiguous l runs
    assert s.info.n_columns == len(np.unique(col))


def test_vloc_g_formula(cfg0):
    s = cfg0
    nx, ny, nz = s.ngrid
    v = s.vloc_g().reshape(nz, ny, nx)
    pos = s.positions()
    a = s.lattice[0, 0]
    b = 2 * np.pi / a
    rng = np.random.default_rng(1)
    for _ in range(50):
        iz, iy, ix = rng.integers(0, nz), rng.integers(0, ny), rng.integers(0, nx)
        h = ix if ix < (nx + 1) // 2 else ix - nx
        k = iy if iy < (ny + 1) // 2 else iy - ny
        l = iz if iz < (nz + 1) // 2 else iz - nz
        G = b * np.array([h, k, l], float)
        g2 = G @ G
        if g2 == 0 or 2 * abs(h) == nx or 2 * abs(k) == ny or 2 * abs(l) == nz:
            assert v[iz, iy, ix] == 0
            continue
        vg = -4 * np.pi * s.params.z_val / (s.omega * g2) * math.exp(-g2 * s.params.rc_loc ** 2 / 4)
        sf = np.exp(-1j * pos @ G).sum()
        assert abs(v[iz, iy, ix] - vg * sf) < 1e-12 * max(1.0, abs(vg * sf))


def test_beta_formula(chfsi):
    s = chfsi.SyntheticSystem(config_index=1, n_rep=1, ecut=6.0, ngrid=[0, 0, 0], n_bands=20)
    beta = s.beta()
    mil = s.miller()
    pos = s.positions()
    a = s.lattice[0, 0]
    q = 2 * np.pi / a * mil
    q2 = (q * q).sum(1)
    rc = s.params.rc_proj[0]
    pref = 4 * np.pi / math.sqrt(s.omega)
    e = np.exp(-q2 * rc * rc / 4)
    for ia in (0, 3):
        ph = np.exp(-1j * q @ pos[ia])
        b0 = pref / math.sqrt(4 * np.pi) * math.sqrt(np.pi) / 4 * rc ** 3 * e * ph
        np.testing.assert_allclose(beta[4 * ia], b0, atol=1e-14)
        for m in range(3):
            b1 = -1j * pref * math.sqrt(3 / (4 * np.pi)) * math.sqrt(np.pi) / 8 * rc ** 5 * q[:, m] * e * ph
            np.testing.assert_allclose(beta[4 * ia + 1 + m], b1, atol=1e-14)
    d = s.dmat().reshape(s.n_atoms, 4, 4)
    for ia in range(s.n_atoms):
        dd = np.diag(d[ia]).real
        assert np.all((dd >= 0.5) & (dd <= 2.0))
        assert dd[1] == dd[2] == dd[3]  # one D per (atom, l)
        assert np.count_nonzero(d[ia] - np.diag(np.diag(d[ia]))) == 0


def test_determinism_and_seed(chfsi):
    a = chfsi.SyntheticSystem(config_index=0)
    b = chfsi.SyntheticSystem(config_index=0)
    c = chfsi.SyntheticSystem(config_index=0, seed=7)
    np.testing.assert_array_equal(a.psi0(), b.psi0())
    np.testing.assert_array_equal(a.positions(), b.positions())
    assert not np.array_equal(a.psi0(), c.psi0())
    p = a.positions()
    assert p.shape == (8, 3)
    ideal = 10.26 * np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]] +
                             [[.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    assert np.abs(p - ideal).max() <= 0.05 + 1e-12
    psi = a.psi0()
    assert abs(psi.real.mean()) < 0.05 and abs(psi.real.std() - 1) < 0.05


def test_occupations_and_bands(chfsi):
    for cfg, nb, nocc in ((0, 20, 16), (1, 160, 128)):
        p = chfsi.SynthParams()
        chfsi.lib().chfsi_synth_defaults(cfg, p)
        assert p.n_bands == nb
    s = chfsi.SyntheticSystem(config_index=0)
    occ = s.occupations()
    assert s.n_elec == 32 and s.n_occ == 16
    assert occ.sum() == 32 and np.all(occ[:16] == 2) and np.all(occ[16:] == 0)


def ewald_numpy(pos, z, a, eta):
    omega = a ** 3
    n = len(z)
    e = 0.0
    rng = range(-3, 4)
    for L in np.array(np.meshgrid(rng, rng, rng, indexing="ij")).reshape(3, -1).T:
        d = pos[:, None, :] - pos[None, :, :] + a * L
        r = np.linalg.norm(d, axis=2)
        mask = r > 1e-12
        e += 0.5 * (np.outer(z, z)[mask] * np.array([math.erfc(eta * x) for x in r[mask]]) / r[mask]).sum()
    b = 2 * np.pi / a
    gm = 14
    g = np.arange(-gm, gm + 1)
    H = np.array(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1).T
    H = H[np.any(H != 0, axis=1)]
    G = b * H
    g2 = (G * G).sum(1)
    S = (z[None, :] * np.exp(1j * G @ pos.T)).sum(1)
    e += (2 * np.pi / omega * np.abs(S) ** 2 * np.exp(-g2 / (4 * eta * eta)) / g2).sum()
    e += -eta / math.sqrt(math.pi) * (z * z).sum() - math.pi * z.sum() ** 2 / (2 * omega * eta * eta)
    return e


def test_ewald_is_independent_of_splitting(cfg0):
    s = cfg0
    z = np.full(s.n_atoms, s.params.z_val)
    a = s.lattice[0, 0]
    ref = ewald_numpy(s.positions(), z, a, 4.0 / a)
    assert abs(ref - s.e_ewald) < 1e-9
