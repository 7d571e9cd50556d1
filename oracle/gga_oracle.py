"""ORACLE — test infrastructure only.

numpy restatement of the PBE exchange-correlation functional (Perdew, Burke,
Ernzerhof, PRL 77, 3865 (1996); PW92 correlation, Perdew & Wang, PRB 45,
13244 (1992)), spin-unpolarised, on a periodic grid [nz][ny][nx]:

    E_xc = sum_r e(rho, |grad rho|^2) dV,   V_xc = de/drho - div(2 de/dsigma grad rho)

with spectral gradients (Nyquist planes dropped) and the partial derivatives
of e by the complex-step method (Im e(x + i h) / h, exact to rounding for this
analytic e), independent of the library's dual-number evaluation.
"""
import numpy as np

KAPPA = 0.804
BETA = 0.06672455060314922
MU = BETA * np.pi ** 2 / 3.0
GAMMA = (1.0 - np.log(2.0)) / np.pi ** 2
PW_A, PW_A1, PW_B = 0.031091, 0.21370, (7.5957, 3.5876, 1.6382, 0.49294)
RHO_FLOOR = 1e-12


def pbe_e(rho, sigma):
    """PBE energy density per volume (works on complex arguments)."""
    kf = (3.0 * np.pi ** 2 * rho) ** (1.0 / 3.0)
    s2 = sigma / (4.0 * kf ** 2 * rho ** 2)
    fx = 1.0 + KAPPA - KAPPA / (1.0 + MU * s2 / KAPPA)
    ex = -3.0 * kf / (4.0 * np.pi) * rho * fx
    rs = (3.0 / (4.0 * np.pi * rho)) ** (1.0 / 3.0)
    b1, b2, b3, b4 = PW_B
    den = 2.0 * PW_A * (b1 * np.sqrt(rs) + b2 * rs + b3 * rs ** 1.5 + b4 * rs ** 2)
    ec = -2.0 * PW_A * (1.0 + PW_A1 * rs) * np.log(1.0 + 1.0 / den)
    ks = np.sqrt(4.0 * kf / np.pi)
    t2 = sigma / (4.0 * ks ** 2 * rho ** 2)
    A = (BETA / GAMMA) / (np.exp(-ec / GAMMA) - 1.0)
    frac = t2 * (1.0 + A * t2) / (1.0 + A * t2 + A ** 2 * t2 ** 2)
    H = GAMMA * np.log(1.0 + BETA / GAMMA * frac)
    return ex + rho * (ec + H)


def pbe_partials(rho, sigma):
    """e, de/drho, de/dsigma by complex steps."""
    h = 1e-20
    e = pbe_e(rho, sigma)
    er = np.imag(pbe_e(rho + 1j * h * rho, sigma + 0j)) / (h * rho)
    es = np.imag(pbe_e(rho + 0j, sigma + 1j * h * np.maximum(sigma, 1e-300))) / (
        h * np.maximum(sigma, 1e-300))
    return e, er, es


def gvectors(ngrid, lattice):
    """Cartesian G per grid point [nz][ny][nx] and the Nyquist mask."""
    nx, ny, nz = ngrid
    rec = 2.0 * np.pi * np.linalg.inv(np.asarray(lattice, dtype=float).reshape(3, 3)).T
    f = [np.fft.fftfreq(n, 1.0 / n) for n in (nx, ny, nz)]
    L, K, H = np.meshgrid(f[2], f[1], f[0], indexing="ij")
    G = H[..., None] * rec[0] + K[..., None] * rec[1] + L[..., None] * rec[2]
    nyq = np.zeros(L.shape, bool)
    for arr, n in ((H, nx), (K, ny), (L, nz)):
        if n % 2 == 0:
            nyq |= arr == -n // 2
    return G, nyq


def pbe_exc_vxc(rho, ngrid, lattice):
    """(E_xc, V_xc) of a real density on the grid (flattened, grid order)."""
    nx, ny, nz = ngrid
    omega = abs(np.linalg.det(np.asarray(lattice, dtype=float).reshape(3, 3)))
    r = np.asarray(rho, dtype=float).reshape(nz, ny, nx)
    dv = omega / r.size
    G, nyq = gvectors(ngrid, lattice)
    rg = np.fft.fftn(r) / r.size
    rg[nyq] = 0.0
    grad = [np.real(np.fft.ifftn(1j * G[..., a] * rg) * r.size) for a in range(3)]
    sigma = grad[0] ** 2 + grad[1] ** 2 + grad[2] ** 2
    ok = r >= RHO_FLOOR
    e = np.zeros_like(r)
    v1 = np.zeros_like(r)
    v2 = np.zeros_like(r)
    e[ok], v1[ok], v2[ok] = pbe_partials(r[ok], sigma[ok])
    div = np.zeros(r.shape, dtype=complex)
    for a in range(3):
        hg = np.fft.fftn(2.0 * v2 * grad[a]) / r.size
        hg[nyq] = 0.0
        div += 1j * G[..., a] * hg
    div = np.real(np.fft.ifftn(div) * r.size)
    return float(e.sum() * dv), (v1 - div).ravel()


def hartree(rho, ngrid, lattice):
    """(E_H, V_H) of a real density, G = 0 dropped."""
    nx, ny, nz = ngrid
    omega = abs(np.linalg.det(np.asarray(lattice, dtype=float).reshape(3, 3)))
    r = np.asarray(rho, dtype=float).reshape(nz, ny, nx)
    G, _ = gvectors(ngrid, lattice)
    g2 = (G * G).sum(-1)
    rg = np.fft.fftn(r) / r.size
    g2s = g2.copy()
    g2s[0, 0, 0] = 1.0
    vg = 4.0 * np.pi * rg / g2s
    vg[0, 0, 0] = 0.0
    eh = 0.5 * omega * np.sum((4.0 * np.pi * np.abs(rg) ** 2 / g2s)[g2 > 0])
    return float(eh), np.real(np.fft.ifftn(vg) * r.size).ravel()


def ewald_forces(lattice, pos, z):
    """Point-charge Ewald forces (eta = 5 / Omega^(1/3); images |n| <= 2,
    reciprocal |m| <= 10), restated from the Ewald energy's derivative."""
    from math import erfc
    A = np.asarray(lattice, dtype=float).reshape(3, 3)
    omega = abs(np.linalg.det(A))
    rec = 2.0 * np.pi * np.linalg.inv(A).T
    eta = 5.0 / omega ** (1.0 / 3.0)
    pos = np.asarray(pos, dtype=float).reshape(-1, 3)
    n = len(pos)
    f = np.zeros((n, 3))
    rng = range(-2, 3)
    L = np.array([[a, b, c] for a in rng for b in rng for c in rng], dtype=float) @ A
    for i in range(n):
        for j in range(n):
            d = pos[i] - pos[j] + L
            r = np.linalg.norm(d, axis=1)
            m = r > 1e-12
            d, r = d[m], r[m]
            g = np.array([erfc(eta * x) for x in r]) / r ** 2 + \
                2.0 * eta / np.sqrt(np.pi) * np.exp(-eta ** 2 * r ** 2) / r
            f[i] += z[i] * z[j] * np.sum((g / r)[:, None] * d, axis=0)
    m = np.arange(-10, 11)
    M = np.array(np.meshgrid(m, m, m, indexing="ij")).reshape(3, -1).T
    M = M[np.any(M != 0, axis=1)]
    G = M @ rec
    g2 = (G * G).sum(1)
    w = 4.0 * np.pi / omega * np.exp(-g2 / (4.0 * eta ** 2)) / g2
    ph = G @ pos.T
    S = (np.asarray(z)[None, :] * np.exp(1j * ph)).sum(1)
    for i in range(n):
        im = np.imag(np.conj(S) * np.exp(1j * ph[:, i]))
        f[i] += z[i] * np.sum((w * im)[:, None] * G, axis=0)
    return f
