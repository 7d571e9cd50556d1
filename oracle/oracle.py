"""ORACLE — test infrastructure only (ctypes binding of oracle/liboracle.so).

CPU restatement of the chemrust-scf ChFSI path (see oracle.cpp).  Only
tests/, __graft_entry__.smoke() and bench.py's CPU baseline import this
module; the product library never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        import build_oracle  # noqa: F401  (same directory)
        build_oracle.build()
    L = C.CDLL(LIB_PATH)
    vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
    i32p = C.POINTER(C.c_int32)
    L.oracle_create.argtypes = [C.c_int] * 7 + [C.c_double] * 3 + [C.c_int, i32p, dp, vp, i32p,
                                                                    vp, vp, dp, vp]
    L.oracle_create.restype = vp
    L.oracle_destroy.argtypes = [vp]
    L.oracle_destroy.restype = None
    protos = {
        "oracle_num_threads": ([], C.c_int),
        "oracle_set_num_threads": ([C.c_int], None),
        "oracle_set_veff": ([vp, dp], None),
        "oracle_set_dmat": ([vp, vp], None),
        "oracle_set_occ": ([vp, dp], None),
        "oracle_get_veff": ([vp, dp], None),
        "oracle_get_vloc_r": ([vp, dp], None),
        "oracle_set_psi": ([vp, vp], None),
        "oracle_get_psi": ([vp, vp], None),
        "oracle_get_hpsi": ([vp, vp], None),
        "oracle_set_bound_mode": ([vp, C.c_int, C.c_int], None),
        "oracle_get_bounds": ([vp, dp], None),
        "oracle_get_norms": ([vp, dp, C.c_int], C.c_int),
        "oracle_fft3d": ([C.c_int, C.c_int, C.c_int, vp, C.c_int], None),
        "oracle_apply_h": ([vp, vp, vp, C.c_int], None),
        "oracle_spectral_bounds": ([vp, dp, C.c_int, dp], None),
        "oracle_chebyshev_filter": ([vp, C.c_int, dp, C.c_int, ip], C.c_int),
        "oracle_rchfsi_filter": ([vp, C.c_int, dp, C.c_int], C.c_int),
        "oracle_rayleigh_ritz": ([vp, dp, ip], C.c_int),
        "oracle_diagonalize": ([vp, C.c_int, dp, C.c_int, dp], C.c_int),
        "oracle_hegv": ([C.c_int, vp, vp, dp, vp], C.c_int),
        "oracle_density": ([vp, dp], None),
        "oracle_build_veff": ([vp, dp, dp, dp], None),
        "oracle_pulay": ([vp, dp, dp, C.c_double, C.c_int, dp], None),
        "oracle_energy": ([vp, dp, dp, dp, dp], None),
        "oracle_scf_run": ([vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                            C.c_double, dp, ip, dp, dp], C.c_int),
        "oracle_fermi": ([dp, C.c_int, C.c_double, C.c_double, dp], C.c_double),
        "oracle_set_qmat": ([vp, vp], C.c_int),
        "oracle_set_qmat_b": ([vp, vp, vp], C.c_int),
        "oracle_line_search": ([C.c_double, C.c_double, C.c_double, C.c_double, dp], None),
        "oracle_tpa_diag": ([dp, C.c_int, dp], None),
        "oracle_band_cg": ([vp, C.c_int, C.c_double, dp, ip], C.c_int),
        "oracle_apply_s": ([vp, vp, vp, C.c_int], None),
        "oracle_apply_sinv": ([vp, vp, vp, C.c_int], None),
        "oracle_s_min": ([vp], C.c_double),
    }
    for name, (args, res) in protos.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def _p(a, t=None):
    return a.ctypes.data_as(C.c_void_p if t is None else C.POINTER(t))


def fft3d(grid, sign):
    """Unnormalised 3D DFT of a [nz, ny, nx] complex grid (sign +1: G->r)."""
    g = np.ascontiguousarray(grid, dtype=np.complex128).copy()
    nz, ny, nx = g.shape
    lib().oracle_fft3d(nx, ny, nz, _p(g), sign)
    return g


def fermi(eig, n_elec, kT):
    """Fermi-Dirac occupations and the entropy term -kT S."""
    e = np.ascontiguousarray(eig, dtype=np.float64)
    f = np.zeros_like(e)
    ts = lib().oracle_fermi(_p(e, C.c_double), len(e), n_elec, kT, _p(f, C.c_double))
    return f, ts


def line_search(a, hpsi_dir, hdir_dir, sdir_dir):
    """Closed-form 2x2 Rayleigh-quotient line search -> (step, eigenvalue, norm, status)."""
    out = np.zeros(4)
    lib().oracle_line_search(a, hpsi_dir, hdir_dir, sdir_dir, _p(out, C.c_double))
    return out[0], out[1], out[2], int(out[3])


def tpa_diag(kin):
    k = np.ascontiguousarray(kin, dtype=np.float64)
    out = np.zeros_like(k)
    lib().oracle_tpa_diag(_p(k, C.c_double), len(k), _p(out, C.c_double))
    return out


def hegv(h, s):
    """Generalised Hermitian eigenproblem H x = e S x (eigenvalues ascending)."""
    n = h.shape[0]
    H = np.ascontiguousarray(h, dtype=np.complex128)
    S = np.ascontiguousarray(s, dtype=np.complex128)
    w = np.zeros(n)
    v = np.zeros((n, n), dtype=np.complex128)
    st = lib().oracle_hegv(n, _p(H), _p(S), _p(w, C.c_double), _p(v))
    if st != 0:
        raise RuntimeError("oracle_hegv failed: %d" % st)
    return w, v


class Oracle:
    """CPU oracle context built from the same arrays the device context gets."""

    def __init__(self, ngrid, miller, kinetic, beta, proj_offsets, dmat, psi, occ, vloc_g,
                 omega, gmax, e_ewald, n_atoms):
        L = lib()
        nx, ny, nz = ngrid
        self.ngrid = tuple(ngrid)
        self.ng = nx * ny * nz
        self._keep = [np.ascontiguousarray(miller, dtype=np.int32),
                      np.ascontiguousarray(kinetic, dtype=np.float64),
                      np.ascontiguousarray(beta, dtype=np.complex128),
                      np.ascontiguousarray(proj_offsets, dtype=np.int32),
                      np.ascontiguousarray(dmat, dtype=np.complex128),
                      np.ascontiguousarray(psi, dtype=np.complex128),
                      np.ascontiguousarray(occ, dtype=np.float64),
                      None if vloc_g is None else np.ascontiguousarray(vloc_g, dtype=np.complex128)]
        m, k, b, o, d, p, f, v = self._keep
        self.n_pw = k.shape[0]
        self.n_bands = p.shape[0]
        n_proj = b.shape[0] if b.ndim == 2 else 0
        n_ions = max(0, o.shape[0] - 1)
        self.h = L.oracle_create(nx, ny, nz, self.n_pw, self.n_bands, n_proj, n_ions, omega, gmax,
                                 e_ewald, n_atoms, _p(m, C.c_int32), _p(k, C.c_double), _p(b),
                                 _p(o, C.c_int32), _p(d), _p(p), _p(f, C.c_double),
                                 None if v is None else _p(v))

    @classmethod
    def from_system(cls, s):
        return cls(s.ngrid, s.miller(), s.kinetic(), s.beta(), s.proj_offsets(), s.dmat(),
                   s.psi0(), s.occupations(), s.vloc_g(), s.omega, s.gmax, s.e_ewald, s.n_atoms)

    def close(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.oracle_destroy(self.h)
            self.h = None

    __del__ = close

    def set_veff(self, v):
        v = np.ascontiguousarray(v, dtype=np.float64).ravel()
        lib().oracle_set_veff(self.h, _p(v, C.c_double))

    def get_veff(self):
        v = np.zeros(self.ng)
        lib().oracle_get_veff(self.h, _p(v, C.c_double))
        return v

    def vloc_r(self):
        v = np.zeros(self.ng)
        lib().oracle_get_vloc_r(self.h, _p(v, C.c_double))
        return v

    def set_psi(self, psi):
        p = np.ascontiguousarray(psi, dtype=np.complex128)
        lib().oracle_set_psi(self.h, _p(p))

    def get_psi(self):
        p = np.zeros((self.n_bands, self.n_pw), dtype=np.complex128)
        lib().oracle_get_psi(self.h, _p(p))
        return p

    def get_hpsi(self):
        p = np.zeros((self.n_bands, self.n_pw), dtype=np.complex128)
        lib().oracle_get_hpsi(self.h, _p(p))
        return p

    def set_qmat(self, qmat, beta=None):
        """Ultrasoft overlap S = 1 + beta q beta^H (per-ion q blocks).  With the
        projector array given, B = beta^H beta is formed by numpy's BLAS
        (the same product, faster than the oracle's loop at 1,728 projectors)."""
        self._q = np.ascontiguousarray(qmat, dtype=np.complex128)
        if beta is not None:
            b = np.asarray(beta).reshape(-1, self.n_pw)
            bm = np.ascontiguousarray(np.conj(b) @ b.T)
            st = lib().oracle_set_qmat_b(self.h, _p(self._q), _p(bm))
        else:
            st = lib().oracle_set_qmat(self.h, _p(self._q))
        if st != 0:
            raise RuntimeError("oracle_set_qmat failed")

    def apply_s(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros_like(x)
        lib().oracle_apply_s(self.h, _p(x), _p(y), x.shape[0])
        return y

    def apply_sinv(self, x):
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros_like(x)
        lib().oracle_apply_sinv(self.h, _p(x), _p(y), x.shape[0])
        return y

    def s_min(self):
        return lib().oracle_s_min(self.h)

    def band_cg(self, max_steps, tol):
        """Sequential band-by-band preconditioned CG refinement of the current psi."""
        e = np.zeros(self.n_bands)
        steps = np.zeros(self.n_bands, dtype=np.int32)
        nconv = lib().oracle_band_cg(self.h, max_steps, tol, _p(e, C.c_double),
                                     steps.ctypes.data_as(C.POINTER(C.c_int)))
        return e, steps, nconv

    def set_bound_mode(self, mode, k=10):
        lib().oracle_set_bound_mode(self.h, mode, k)

    def bounds(self):
        b = np.zeros(4)
        lib().oracle_get_bounds(self.h, _p(b, C.c_double))
        return b

    def norms(self):
        n = np.zeros(256)
        m = lib().oracle_get_norms(self.h, _p(n, C.c_double), 256)
        return n[:m].copy()

    def apply_h(self, psi):
        p = np.ascontiguousarray(psi, dtype=np.complex128)
        out = np.zeros_like(p)
        lib().oracle_apply_h(self.h, _p(p), _p(out), p.shape[0])
        return out

    def chebyshev_filter(self, ndeg, eigenvalues=None):
        fk = C.c_int(0)
        if eigenvalues is None:
            st = lib().oracle_chebyshev_filter(self.h, ndeg, None, 0, C.byref(fk))
        else:
            e = np.ascontiguousarray(eigenvalues, dtype=np.float64)
            st = lib().oracle_chebyshev_filter(self.h, ndeg, _p(e, C.c_double), len(e), C.byref(fk))
        return st, fk.value

    def rchfsi_filter(self, ndeg, eigenvalues):
        """Residual-based Chebyshev filter (R-ChFSI) of the current Ritz pairs."""
        e = np.ascontiguousarray(eigenvalues, dtype=np.float64)
        st = lib().oracle_rchfsi_filter(self.h, ndeg, _p(e, C.c_double), len(e))
        if st != 0:
            raise RuntimeError("oracle R-ChFSI filter failed: %d" % st)

    def rchfsi_diagonalize(self, ndeg, eigenvalues):
        """R-ChFSI filter + Rayleigh-Ritz."""
        self.rchfsi_filter(ndeg, eigenvalues)
        st, w = self.rayleigh_ritz()
        if st != 0:
            raise RuntimeError("oracle Rayleigh-Ritz failed: %d" % st)
        return w

    def rayleigh_ritz(self):
        w = np.zeros(self.n_bands)
        info = C.c_int(0)
        st = lib().oracle_rayleigh_ritz(self.h, _p(w, C.c_double), C.byref(info))
        return st, w

    def diagonalize(self, ndeg, eigenvalues=None):
        w = np.zeros(self.n_bands)
        if eigenvalues is None:
            st = lib().oracle_diagonalize(self.h, ndeg, None, 0, _p(w, C.c_double))
        else:
            e = np.ascontiguousarray(eigenvalues, dtype=np.float64)
            st = lib().oracle_diagonalize(self.h, ndeg, _p(e, C.c_double), len(e), _p(w, C.c_double))
        if st != 0:
            raise RuntimeError("oracle diagonalize failed: %d" % st)
        return w

    def density(self):
        r = np.zeros(self.ng)
        lib().oracle_density(self.h, _p(r, C.c_double))
        return r

    def set_dmat(self, dmat):
        d = np.ascontiguousarray(dmat, dtype=np.complex128)
        lib().oracle_set_dmat(self.h, _p(d))

    def set_occ(self, occ):
        o = np.ascontiguousarray(occ, dtype=np.float64)
        lib().oracle_set_occ(self.h, _p(o, C.c_double))

    def build_veff(self, rho):
        r = np.ascontiguousarray(rho, dtype=np.float64).ravel()
        vh, vx = np.zeros(self.ng), np.zeros(self.ng)
        lib().oracle_build_veff(self.h, _p(r, C.c_double), _p(vh, C.c_double), _p(vx, C.c_double))
        return vh, vx

    def energy(self, rho_in, rho_out, eig):
        a = np.ascontiguousarray(rho_in, dtype=np.float64).ravel()
        b = np.ascontiguousarray(rho_out, dtype=np.float64).ravel()
        e = np.ascontiguousarray(eig, dtype=np.float64)
        out = np.zeros(5)
        lib().oracle_energy(self.h, _p(a, C.c_double), _p(b, C.c_double), _p(e, C.c_double),
                            _p(out, C.c_double))
        return out

    def run_scf(self, ndeg, tol_per_atom=1e-6, max_iter=30, alpha=0.3, max_hist=6,
                first_passes=4, kT=0.01):
        e = np.zeros(max_iter)
        it = C.c_int(0)
        eig = np.zeros(self.n_bands)
        rho = np.zeros(self.ng)
        st = lib().oracle_scf_run(self.h, ndeg, max_iter, tol_per_atom, alpha, max_hist,
                                  first_passes, kT, _p(e, C.c_double), C.byref(it),
                                  _p(eig, C.c_double), _p(rho, C.c_double))
        return {"status": st, "converged": st == 0, "n_iter": it.value,
                "energies": e[:it.value].copy(), "eigenvalues": eig, "rho": rho}
