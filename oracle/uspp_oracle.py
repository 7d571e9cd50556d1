"""ORACLE — test infrastructure only: CPU restatement of the ultrasoft SCF
with augmentation charges on a separate density grid.

Only tests/ import this module.  It drives the C++ oracle (oracle.cpp) for
the filter, Rayleigh-Ritz and the smooth density, and states the density-grid
steps in numpy:

  * Q_ij(r) = q_ij g(|r - R_I|), g(r) = exp(-r^2/w^2) / (pi^{3/2} w^3),
    g^(G) = exp(-G^2 w^2 / 4); the overlap S = 1 + beta q beta^H is the one
    of the phase-0 gate (tests/phase0_gate2_convergence.rs:279-322 in the
    reference crate);
  * rho(G) = rho_smooth(G) + (1/Omega) g^(G) sum_I c_I e^{-iG.R_I},
    c_I = sum_n f_n C_n^H q_I C_n with C = beta^H psi; the smooth part is
    interpolated from the wavefunction grid by zero padding (Nyquist planes
    of even axes dropped);
  * D_I = D0_I + q_I v_I, v_I = sum_G V_G g^(G) e^{+iG.R_I};
  * V_eff = V_loc + V_H + V_xc (PZ81 LDA) on the density grid, brought to
    the wavefunction grid by truncation in G (downsample_array_to_wave_grid,
    src/scf.rs:413-454);
  * E = sum f eps - int (V_H + V_xc)[in] rho_out + E_H[out] + E_xc[out]
    + E_ewald - kT S, Pulay over (rho_in, rho_out - rho_in) as oracle.cpp's
    oracle_pulay.
"""
import numpy as np

import oracle as orc


def lda_pz(rho):
    r = np.maximum(rho, 0.0)
    exc = np.zeros_like(r)
    vxc = np.zeros_like(r)
    m = r >= 1e-30
    rs = np.cbrt(3.0 / (4.0 * np.pi * r[m]))
    ex = -0.4581652932831429 / rs
    vx = 4.0 / 3.0 * ex
    ec = np.empty_like(rs)
    vc = np.empty_like(rs)
    hi = rs >= 1.0
    g, b1, b2 = -0.1423, 1.0529, 0.3334
    sr = np.sqrt(rs[hi])
    den = 1.0 + b1 * sr + b2 * rs[hi]
    ec[hi] = g / den
    vc[hi] = ec[hi] * (1.0 + 7.0 / 6.0 * b1 * sr + 4.0 / 3.0 * b2 * rs[hi]) / den
    lo = ~hi
    A, B, Cc, D = 0.0311, -0.048, 0.0020, -0.0116
    lr = np.log(rs[lo])
    ec[lo] = A * lr + B + Cc * rs[lo] * lr + D * rs[lo]
    vc[lo] = A * lr + (B - A / 3.0) + 2.0 / 3.0 * Cc * rs[lo] * lr + (2.0 * D - Cc) / 3.0 * rs[lo]
    exc[m] = ex + ec
    vxc[m] = vx + vc
    return exc, vxc


def pulay(hist_in, hist_res, alpha):
    m = len(hist_in)
    if m == 1:
        c = np.ones(1)
    else:
        A = np.zeros((m + 1, m + 1))
        for i in range(m):
            for j in range(m):
                A[i, j] = hist_res[i] @ hist_res[j]
        A[:m, m] = A[m, :m] = 1.0
        rhs = np.zeros(m + 1)
        rhs[m] = 1.0
        c = np.linalg.solve(A, rhs)[:m]
    return sum(ci * (a + alpha * r) for ci, a, r in zip(c, hist_in, hist_res))


class UsppScf:
    """Density-grid pieces of the ultrasoft SCF for one synthetic system."""

    def __init__(self, s):
        self.s = s
        beta = s.beta()  # one host copy shared by the oracle and the augmentation sums
        self.o = orc.Oracle(s.ngrid, s.miller(), s.kinetic(), beta, s.proj_offsets(), s.dmat(),
                            s.psi0(), s.occupations(), s.vloc_g(), s.omega, s.gmax, s.e_ewald,
                            s.n_atoms)
        self._beta_all = beta
        self._qmat_set = False
        self.nw = tuple(s.ngrid)
        self.nf = tuple(s.ngrid_density)
        self.omega = s.omega
        self.width = s.q_width
        self.pos = s.positions().reshape(-1, 3)
        self.beta = beta.reshape(s.n_proj, s.n_pw)
        self.poff = s.proj_offsets()
        self.d0 = s.dmat()
        self.q = s.qmat()
        self.recip = 2 * np.pi * np.linalg.inv(s.lattice).T
        nx, ny, nz = self.nf
        fx, fy, fz = (np.fft.fftfreq(n, 1.0 / n) for n in (nx, ny, nz))
        L, K, H = np.meshgrid(fz, fy, fx, indexing="ij")
        G = H[..., None] * self.recip[0] + K[..., None] * self.recip[1] + L[..., None] * self.recip[2]
        self.G = G
        self.g2 = (G * G).sum(-1)
        self.ghat = np.exp(-0.25 * self.g2 * self.width ** 2)
        # phases e^{-i G.R_I} are formed one ion at a time (a table over all
        # ions of the 216-atom cell on its 144^3 grid would take 10 GB)
        # blocks of q and D0 per ion
        self.blocks = []
        off = 0
        for i in range(len(self.poff) - 1):
            ne = self.poff[i + 1] - self.poff[i]
            self.blocks.append((self.poff[i], ne, off))
            off += ne * ne
        self.vloc = self.up_coeffs(self.wave_coeffs_vloc()).real.ravel()

    def _phase(self, i):
        return np.exp(-1j * (self.G @ self.pos[i]))

    def _phase_sum(self, c):
        """sum_I c_I e^{-i G.R_I} on the density grid."""
        out = np.zeros(self.g2.shape, dtype=complex)
        for i, ci in enumerate(c):
            out += ci * self._phase(i)
        return out

    # --- grids
    def _wave_idx(self):
        out = []
        for n, f in zip(self.nw, self.nf):
            h = np.arange(n)
            hs = np.where(h >= (n + 1) // 2, h - n, h)
            keep = ~((n % 2 == 0) & (h == n // 2)) if f != n else np.ones(n, bool)
            out.append((h[keep], (hs[keep] + f) % f))
        return out

    def wave_coeffs_vloc(self):
        nx, ny, nz = self.nw
        return self.s.vloc_g().reshape(nz, ny, nx)  # coefficients of e^{iGr}

    def up_coeffs(self, cw):
        """Fine-grid real-space field with the given wave-grid coefficients."""
        (hx, fx), (hy, fy), (hz, fz) = self._wave_idx()
        F = np.zeros(self.nf[::-1], dtype=complex)
        F[np.ix_(fz, fy, fx)] = cw[np.ix_(hz, hy, hx)]
        return np.fft.ifftn(F) * F.size

    def down(self, vf):
        """Wave-grid field from a fine-grid one by G truncation."""
        nx, ny, nz = self.nf
        Vg = np.fft.fftn(vf.reshape(nz, ny, nx)) / vf.size
        (hx, fx), (hy, fy), (hz, fz) = self._wave_idx()
        W = np.zeros(self.nw[::-1], dtype=complex)
        W[np.ix_(hz, hy, hx)] = Vg[np.ix_(fz, fy, fx)]
        return (np.fft.ifftn(W) * W.size).real.ravel()

    # --- physics
    def hartree_xc(self, rho):
        nx, ny, nz = self.nf
        rg = np.fft.fftn(rho.reshape(nz, ny, nx)) / rho.size
        g2 = self.g2.copy()
        g2[0, 0, 0] = 1.0
        vg = 4 * np.pi * rg / g2
        vg[0, 0, 0] = 0.0
        eh = 0.5 * self.omega * np.sum((4 * np.pi * np.abs(rg) ** 2 / g2)[self.g2 > 0])
        vh = (np.fft.ifftn(vg) * rho.size).real.ravel()
        exc, vxc = lda_pz(rho)
        e_xc = np.sum(rho * exc) * self.omega / rho.size
        return vh, vxc, eh, e_xc

    def screened_d(self, vf):
        nx, ny, nz = self.nf
        Vg = np.fft.fftn(vf.reshape(nz, ny, nx)) / vf.size
        vq = Vg * self.ghat
        v = np.array([np.sum(vq * np.conj(self._phase(I))).real for I in range(len(self.pos))])
        d = self.d0.copy()
        for I, (p0, ne, off) in enumerate(self.blocks):
            d[off:off + ne * ne] += v[I] * self.q[off:off + ne * ne]
        return d, v

    def density(self, occ):
        """Smooth density (oracle, wave grid) interpolated + augmentation."""
        nx, ny, nz = self.nw
        self.o.set_occ(occ)
        rw = self.o.density()
        cw = np.fft.fftn(rw.reshape(nz, ny, nx)) / rw.size
        psi = self.o.get_psi().reshape(self.s.n_bands, self.s.n_pw)
        Cm = np.conj(self.beta) @ psi.T  # n_proj x n_bands
        c = np.zeros(len(self.pos))
        for I, (p0, ne, off) in enumerate(self.blocks):
            qI = self.q[off:off + ne * ne].reshape(ne, ne)
            CI = Cm[p0:p0 + ne]
            c[I] = np.sum(occ * np.einsum("in,in->n", np.conj(CI), qI @ CI).real)
        (hx, fx), (hy, fy), (hz, fz) = self._wave_idx()
        F = np.zeros(self.nf[::-1], dtype=complex)
        F[np.ix_(fz, fy, fx)] = cw[np.ix_(hz, hy, hx)]
        F += self.ghat / self.omega * self._phase_sum(c)
        return (np.fft.ifftn(F) * F.size).real.ravel(), c

    def run_scf(self, ndeg, max_iter=30, tol_per_atom=1e-6, alpha=0.3, max_hist=6,
                first_passes=4, kT=0.01):
        s = self.s
        if not self._qmat_set:
            # the generalised eigenproblem of the SCF needs S
            self.o.set_qmat(s.qmat(), beta=self._beta_all)
            self._qmat_set = True
        ngf = int(np.prod(self.nf))
        dv = self.omega / ngf
        n_elec = s.n_elec
        rin = np.full(ngf, n_elec / self.omega)
        hin, hres = [], []
        eig = None
        energies = []
        e_prev = None
        rout = None
        for it in range(1, max_iter + 1):
            vh, vx, _, _ = self.hartree_xc(rin)
            vf = self.vloc + vh + vx
            d, _ = self.screened_d(vf)
            self.o.set_veff(self.down(vf))
            self.o.set_dmat(d)
            for _ in range(max(1, first_passes) if it == 1 else 1):
                eig = self.o.diagonalize(ndeg, eig)
            occ, e_ts = orc.fermi(eig, n_elec, kT)
            rout, _ = self.density(occ)
            _, _, eh, exc = self.hartree_xc(rout)
            dc = np.sum((vh + vx) * rout) * dv
            etot = np.sum(occ * eig) - dc + eh + exc + s.e_ewald + e_ts
            energies.append(etot)
            if e_prev is not None and abs(etot - e_prev) / s.n_atoms < tol_per_atom:
                return {"converged": True, "energies": np.array(energies), "eigenvalues": eig,
                        "rho": rout, "n_iter": it}
            e_prev = etot
            hin.append(rin.copy())
            hres.append(rout - rin)
            hin, hres = hin[-max_hist:], hres[-max_hist:]
            rin = pulay(hin, hres, alpha)
        return {"converged": False, "energies": np.array(energies), "eigenvalues": eig,
                "rho": rout, "n_iter": max_iter}

