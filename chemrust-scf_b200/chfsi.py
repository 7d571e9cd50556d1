"""ctypes binding of libchfsi_b200.so (include/chfsi.h).

Python-side mirror of the chemrust-scf ChFSI interface (paths relative to
that project):

    Context.chebyshev_filter   src/eigensolver/chebyshev.rs:626   chebyshev_filter()
    Context.rayleigh_ritz      src/eigensolver/rayleigh_ritz.rs:48 rayleigh_ritz()
    Context.diagonalize        src/scf.rs:169 ScfIteration::diagonalize()
    Context.apply_h            src/eigensolver/chebyshev.rs:371 apply_full_hamiltonian()
    Context.construct_density  src/scf.rs:275 construct_density()
    Context.build_v_eff        src/scf.rs:157 build_v_eff()
    Context.run_scf            src/scf.rs:358 run_scf()

Errors are raised as ChfsiError subclasses named after the crate's Error
variants (src/types.rs:226-248).  There is no CPU fallback: every compute
call goes to the CUDA library, and creating a context without a GPU raises
NoDevice.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchfsi_b200.so")

OK, NOT_CONVERGED, NOT_IMPLEMENTED, CHEB_DIVERGED, RR_FAILED, CUDA_ERROR, BAD_INPUT, \
    NO_DEVICE, OUT_OF_MEMORY, NUMERIC, TIMEOUT = 0, -1, -2, -3, -4, -5, -6, -7, -8, -9, -10
INJECT_NONE, INJECT_TC_NO_LOADS, INJECT_ALLOC_FAIL = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
BOUND_HEURISTIC, BOUND_LANCZOS, BOUND_LANCZOS_FUSED = 0, 1, 2
FILTER_CHEBYSHEV, FILTER_RESIDUAL = 0, 1
XC_LDA_PZ, XC_PBE = 0, 1
MIXER_PULAY, MIXER_LEARNED, MIXER_LEARNED_PULAY = 0, 1, 2
MIXER_FEATURES, MIXER_OUTPUTS, MIXER_TARGETS, MIXER_SHELLS = 512, 128, 320, 64


class ChfsiError(RuntimeError):
    status = None


class NotConverged(ChfsiError):
    status = NOT_CONVERGED


class NotImplementedErr(ChfsiError):
    status = NOT_IMPLEMENTED


class ChebyshevDiverged(ChfsiError):
    status = CHEB_DIVERGED


class RayleighRitzFailed(ChfsiError):
    status = RR_FAILED


class CudaError(ChfsiError):
    status = CUDA_ERROR


class BadInput(ChfsiError):
    status = BAD_INPUT


class NoDevice(ChfsiError):
    status = NO_DEVICE


class OutOfMemory(ChfsiError):
    status = OUT_OF_MEMORY


class NumericError(ChfsiError):
    status = NUMERIC


class Timeout(ChfsiError):
    """A bounded device-side wait ran out; the kernel retired what it had
    issued and returned, so the context stays usable."""
    status = TIMEOUT


_ERRORS = {c.status: c for c in (NotConverged, NotImplementedErr, ChebyshevDiverged,
                                  RayleighRitzFailed, CudaError, BadInput, NoDevice, OutOfMemory,
                                  NumericError, Timeout)}


class SynthParams(C.Structure):
    _fields_ = [("lattice", C.c_int), ("n_rep", C.c_int), ("a_conv", C.c_double),
                ("jitter", C.c_double), ("z_val", C.c_double), ("rc_loc", C.c_double),
                ("ecut", C.c_double), ("ngrid", C.c_int * 3), ("n_bands", C.c_int),
                ("n_shell", C.c_int), ("rc_proj", C.c_double * 4), ("lmax", C.c_int),
                ("d_min", C.c_double), ("d_max", C.c_double), ("uspp", C.c_int),
                ("q_width", C.c_double), ("q_amp", C.c_double), ("kpt", C.c_double * 3),
                ("seed", C.c_uint64), ("ngrid_density", C.c_int * 3)]


class SystemInfo(C.Structure):
    _fields_ = [("ngrid", C.c_int * 3), ("n_pw", C.c_int), ("n_bands", C.c_int),
                ("n_occ", C.c_int), ("n_atoms", C.c_int), ("n_proj", C.c_int),
                ("n_ions_with_proj", C.c_int), ("n_columns", C.c_int), ("omega", C.c_double),
                ("n_elec", C.c_double), ("gmax", C.c_double), ("e_ewald", C.c_double),
                ("lattice", C.c_double * 9), ("ngrid_density", C.c_int * 3),
                ("q_width", C.c_double), ("uspp", C.c_int)]


class Dims(C.Structure):
    _fields_ = [("ngrid", C.c_int * 3), ("n_pw", C.c_int), ("n_bands", C.c_int),
                ("n_proj", C.c_int), ("n_ions", C.c_int)]


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("bound_mode", C.c_int),
                ("lanczos_steps", C.c_int), ("check_norms", C.c_int), ("filter_form", C.c_int),
                ("reserved", C.c_int * 2)]


class ScfParams(C.Structure):
    _fields_ = [("ndeg", C.c_int), ("max_iter", C.c_int), ("tol_per_atom", C.c_double),
                ("alpha", C.c_double), ("max_hist", C.c_int), ("first_passes", C.c_int),
                ("kT", C.c_double), ("fp64_switch_per_atom", C.c_double),
                ("mixer", C.c_int), ("cg_steps", C.c_int), ("trace", C.POINTER(C.c_double)),
                ("verbose", C.c_int), ("restart", C.c_int), ("tol_eig", C.c_double),
                ("fp64_switch_eig", C.c_double)]


class ScfResult(C.Structure):
    _fields_ = [("status", C.c_int), ("n_iter", C.c_int), ("n_iter_mixed", C.c_int),
                ("e_total", C.c_double),
                ("e_band", C.c_double), ("e_hartree", C.c_double), ("e_xc", C.c_double),
                ("e_dc", C.c_double), ("e_entropy", C.c_double), ("mu", C.c_double),
                ("seconds", C.c_double),
                ("energies", C.POINTER(C.c_double)), ("eigenvalues", C.POINTER(C.c_double)),
                ("n_iter_learned", C.c_int), ("fell_back", C.c_int),
                ("residuals", C.POINTER(C.c_double)), ("n_fp64_retries", C.c_int)]


_lib = None


def lib():
    """Load libchfsi_b200.so (raises if the extension has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libchfsi_b200.so is missing: run chemrust-scf_b200/build.py")
    L = C.CDLL(LIB_PATH)
    vp, i32p, dp = C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    sig = {
        "chfsi_synth_defaults": [C.c_int, C.POINTER(SynthParams)],
        "chfsi_system_generate": [C.POINTER(SynthParams), C.POINTER(vp)],
        "chfsi_system_get_info": [vp, C.POINTER(SystemInfo)],
        "chfsi_system_get_miller": [vp, i32p],
        "chfsi_system_get_kinetic": [vp, dp],
        "chfsi_system_get_vloc_g": [vp, vp],
        "chfsi_system_get_beta": [vp, vp],
        "chfsi_system_get_proj_offsets": [vp, i32p],
        "chfsi_system_get_dmat": [vp, vp],
        "chfsi_system_get_qmat": [vp, vp],
        "chfsi_system_get_psi0": [vp, vp],
        "chfsi_system_get_occupations": [vp, dp],
        "chfsi_system_get_positions": [vp, dp],
        "chfsi_default_config": [C.POINTER(Config)],
        "chfsi_create": [C.POINTER(Dims), C.POINTER(Config), C.POINTER(vp)],
        "chfsi_create_from_system": [vp, C.POINTER(Config), C.POINTER(vp)],
        "chfsi_set_basis": [vp, i32p, dp, C.c_double],
        "chfsi_set_projectors": [vp, vp, i32p, vp],
        "chfsi_set_veff": [vp, dp],
        "chfsi_set_qmat": [vp, vp],
        "chfsi_get_s_min": [vp, dp],
        "chfsi_set_psi": [vp, vp],
        "chfsi_get_psi": [vp, vp],
        "chfsi_apply_h": [vp, vp, vp, C.c_int],
        "chfsi_apply_h_local": [vp, vp, vp, C.c_int],
        "chfsi_apply_sinv_h": [vp, vp, vp, C.c_int],
        "chfsi_get_stream": [vp, C.POINTER(vp)],
        "chfsi_zgemm_cn": [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp],
        "chfsi_zgemm_cn_bf16x3": [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp],
        "chfsi_zgemm_cn_bf16x3_shape": [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp,
                                        vp, C.c_int],
        "chfsi_get_tc_shapes": [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)],
        "chfsi_set_tc_shapes": [vp, C.c_int, C.c_int],
        "chfsi_zgemm_cn_noalloc": [vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp],
        "chfsi_chebyshev_filter": [vp, C.c_int, dp, C.c_int],
        "chfsi_rayleigh_ritz": [vp, dp],
        "chfsi_diagonalize": [vp, C.c_int, dp, C.c_int, dp],
        "chfsi_get_bounds": [vp, dp],
        "chfsi_get_filter_norms": [vp, dp, C.c_int],
        "chfsi_psi_device_ptr": [vp, C.POINTER(vp)],
        "chfsi_set_vloc_g": [vp, vp],
        "chfsi_get_vloc": [vp, dp],
        "chfsi_get_veff": [vp, dp],
        "chfsi_set_cell": [vp, dp, C.c_double, C.c_int],
        "chfsi_set_occupations": [vp, dp],
        "chfsi_construct_density": [vp, dp],
        "chfsi_build_veff": [vp, dp, dp],
        "chfsi_get_density": [vp, dp],
        "chfsi_scf_run": [vp, C.POINTER(ScfParams), C.POINTER(ScfResult)],
        "chfsi_mixer_create": [C.c_int, C.c_uint64, C.POINTER(vp)],
        "chfsi_mixer_get_params": [vp, fp],
        "chfsi_mixer_set_params": [vp, fp],
        "chfsi_mixer_forward": [vp, fp, C.c_int, fp],
        "chfsi_mixer_gradient": [vp, fp, fp, C.c_int, fp, fp],
        "chfsi_mixer_train": [vp, fp, fp, C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64, fp],
        "chfsi_set_mixer": [vp, vp],
        "chfsi_mixer_samples": [vp, dp, dp, C.c_int, dp, fp, fp],
        "chfsi_set_density_grid": [vp, C.POINTER(C.c_int)],
        "chfsi_get_rr_sweeps": [vp, C.POINTER(C.c_int)],
        "chfsi_get_density_grid": [vp, C.POINTER(C.c_int)],
        "chfsi_set_augmentation": [vp, dp, C.c_double],
        "chfsi_band_cg": [vp, C.c_int, C.c_double, dp, i32p, i32p],
        "chfsi_batch_create": [C.POINTER(vp), C.c_int, C.POINTER(vp)],
        "chfsi_batch_capture": [vp, C.c_int],
        "chfsi_batch_run": [vp, dp, i32p],
        "chfsi_batch_graph_nodes": [vp, C.POINTER(C.c_size_t)],
        "chfsi_autotune": [vp, C.POINTER(C.c_int), fp],
        "chfsi_set_launch_config": [vp, C.c_int],
        "chfsi_test_inject": [C.c_int, C.c_longlong],
        "chfsi_set_xc": [vp, C.c_int],
        "chfsi_set_ions": [vp, C.c_int, dp, dp, dp, dp],
        "chfsi_forces": [vp, dp],
        "chfsi_system_generate_at": [C.POINTER(SynthParams), dp, C.POINTER(vp)],
        "chfsi_zgemm_tn": [vp, C.c_int, vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, C.c_int,
                           C.c_double, C.c_double, vp],
        "chfsi_hegv_dev": [vp, vp, C.c_int, dp, vp, vp],
        "chfsi_hpsi_device_ptr": [vp, C.POINTER(vp)],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    L.chfsi_system_destroy.argtypes = [vp]
    L.chfsi_system_destroy.restype = None
    L.chfsi_destroy.argtypes = [vp]
    L.chfsi_destroy.restype = None
    L.chfsi_batch_destroy.argtypes = [vp]
    L.chfsi_batch_destroy.restype = None
    L.chfsi_mixer_destroy.argtypes = [vp]
    L.chfsi_mixer_destroy.restype = None
    L.chfsi_mixer_num_params.argtypes = []
    L.chfsi_mixer_num_params.restype = C.c_size_t
    L.chfsi_launch_count.argtypes = []
    L.chfsi_launch_count.restype = C.c_longlong
    L.chfsi_last_error.argtypes = [vp]
    L.chfsi_last_error.restype = C.c_char_p
    _lib = L
    return L


class Batch:
    """Mixed-precision diagonalisation passes of many contexts replayed as one
    CUDA graph (members on their own streams)."""

    def __init__(self, contexts):
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.handle.value for c in self.contexts])
        h = C.c_void_p()
        _check(lib().chfsi_batch_create(arr, len(self.contexts), C.byref(h)))
        self.handle = h
        self.n_bands = [c.n_bands for c in self.contexts]

    def close(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.chfsi_batch_destroy(self.handle)
            self.handle = None

    __del__ = close

    def capture(self, ndeg):
        _check(lib().chfsi_batch_capture(self.handle, ndeg))
        n = C.c_size_t()
        _check(lib().chfsi_batch_graph_nodes(self.handle, C.byref(n)))
        return n.value

    def run(self):
        """Replay; returns the list of per-member eigenvalue arrays."""
        e = np.zeros(sum(self.n_bands))
        st = np.zeros(len(self.contexts), dtype=np.int32)
        code = lib().chfsi_batch_run(self.handle, _ptr(e, C.c_double), _ptr(st, C.c_int32))
        if code != OK:
            _check(code)
        return np.split(e, np.cumsum(self.n_bands)[:-1])


class Mixer:
    """Learned density mixer: MLP 512 -> 256 -> 256 -> 128 (GELU), BF16 weights,
    FP32 accumulation; forward, backward and Adam run as the library's kernels."""

    def __init__(self, device=0, seed=0, params=None):
        h = C.c_void_p()
        _check(lib().chfsi_mixer_create(device, seed, C.byref(h)))
        self.handle = h
        self.num_params = int(lib().chfsi_mixer_num_params())
        if params is not None:
            self.set_params(params)

    def close(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.chfsi_mixer_destroy(self.handle)
            self.handle = None

    __del__ = close

    def get_params(self):
        w = np.zeros(self.num_params, dtype=np.float32)
        _check(lib().chfsi_mixer_get_params(self.handle, _ptr(w, C.c_float)))
        return w

    def set_params(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32).ravel()
        if w.size != self.num_params:
            raise ValueError("expected %d parameters" % self.num_params)
        _check(lib().chfsi_mixer_set_params(self.handle, _ptr(w, C.c_float)))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MIXER_FEATURES)
        y = np.zeros((x.shape[0], MIXER_OUTPUTS), dtype=np.float32)
        _check(lib().chfsi_mixer_forward(self.handle, _ptr(x, C.c_float), x.shape[0],
                                         _ptr(y, C.c_float)))
        return y

    def gradient(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MIXER_FEATURES)
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, MIXER_TARGETS)
        g = np.zeros(self.num_params, dtype=np.float32)
        loss = C.c_float()
        _check(lib().chfsi_mixer_gradient(self.handle, _ptr(x, C.c_float), _ptr(t, C.c_float),
                                          x.shape[0], _ptr(g, C.c_float), C.byref(loss)))
        return g, loss.value

    def train(self, x, t, epochs=50, batch=256, lr=1e-3, seed=0):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, MIXER_FEATURES)
        t = np.ascontiguousarray(t, dtype=np.float32).reshape(-1, MIXER_TARGETS)
        losses = np.zeros(epochs, dtype=np.float32)
        _check(lib().chfsi_mixer_train(self.handle, _ptr(x, C.c_float), _ptr(t, C.c_float),
                                       x.shape[0], epochs, batch, lr, seed,
                                       _ptr(losses, C.c_float)))
        return losses


def zgemm_cn(a_dev, lda, b_dev, ldb, m, n, k, c_dev, stream=0):
    """C[m][n] = sum_k conj(A[m][k]) B[n][k] on device pointers (blocks until done)."""
    _check(lib().chfsi_zgemm_cn(C.c_void_p(a_dev), lda, C.c_void_p(b_dev), ldb, m, n, k,
                                C.c_void_p(c_dev), C.c_void_p(stream)))


def zgemm_cn_noalloc(a_dev, lda, b_dev, ldb, m, n, k, c_dev, stream=0):
    """zgemm_cn without device allocation (static 4 MiB scratch; m * n <= 262144)."""
    _check(lib().chfsi_zgemm_cn_noalloc(C.c_void_p(a_dev), lda, C.c_void_p(b_dev), ldb, m, n, k,
                                        C.c_void_p(c_dev), C.c_void_p(stream)))


def zgemm_tn(w_dev, ldw, x_dev, ldx, o_dev, ldo, m, n, k, alpha=1.0, beta=0.0, stream=0):
    """O[m][n] = alpha sum_k W[k][m] X[k][n] + beta O[m][n] (device pointers)."""
    _check(lib().chfsi_zgemm_tn(C.c_void_p(w_dev), ldw, C.c_void_p(x_dev), ldx, C.c_void_p(o_dev),
                                ldo, m, n, k, alpha, beta, C.c_void_p(stream)))


def hegv_dev(h_dev, s_dev, n, v_dev, stream=0):
    """H x = e S x on device n x n matrices; returns the eigenvalues (host),
    eigenvectors as the columns of v_dev."""
    w = np.zeros(n)
    _check(lib().chfsi_hegv_dev(C.c_void_p(h_dev), C.c_void_p(s_dev), n, _ptr(w, C.c_double),
                                C.c_void_p(v_dev), C.c_void_p(stream)))
    return w


TC_SHAPES = 3


def zgemm_cn_bf16x3(a_dev, lda, b_dev, ldb, m, n, k, c_dev, stream=0, shape=None):
    """Same product on tcgen05 tensor cores, BF16 3-way split, FP32 accumulation;
    shape (0..TC_SHAPES-1) picks the kernel's launch shape."""
    if shape is None:
        _check(lib().chfsi_zgemm_cn_bf16x3(C.c_void_p(a_dev), lda, C.c_void_p(b_dev), ldb, m, n,
                                           k, C.c_void_p(c_dev), C.c_void_p(stream)))
    else:
        _check(lib().chfsi_zgemm_cn_bf16x3_shape(C.c_void_p(a_dev), lda, C.c_void_p(b_dev), ldb,
                                                 m, n, k, C.c_void_p(c_dev), C.c_void_p(stream),
                                                 shape))


def inject_fault(what, arg=0):
    """Host-side fault injection for error-path tests (INJECT_TC_NO_LOADS:
    the next `arg` tensor-core GEMM launches issue no loads and time out;
    INJECT_ALLOC_FAIL: the arg-th device allocation fails; INJECT_NONE clears)."""
    _check(lib().chfsi_test_inject(what, arg))


def launch_count():
    """Kernels launched by the library since it was loaded."""
    return int(lib().chfsi_launch_count())


def _check(st, ctx=None):
    if st == OK:
        return
    msg = lib().chfsi_last_error(ctx)
    msg = msg.decode() if msg else ""
    raise _ERRORS.get(st, ChfsiError)("chfsi status %d: %s" % (st, msg))


def _ptr(a, ctype=None):
    if ctype is None:
        return a.ctypes.data_as(C.c_void_p)
    return a.ctypes.data_as(C.POINTER(ctype))


# ---------------------------------------------------------------------------
# Synthetic systems
# ---------------------------------------------------------------------------
class SyntheticSystem:
    """Seeded synthetic plane-wave system (lattice, G-sphere, V_loc, projectors, psi0)."""

    @staticmethod
    def _L():
        """The library whose generator builds the system."""
        return lib()

    @staticmethod
    def _chk(st):
        _check(st)

    def __init__(self, params=None, config_index=None, positions=None, **overrides):
        """positions: Cartesian atom positions (n_atoms x 3, bohr) in place of
        the seeded jittered lattice."""
        L = self._L()
        if params is None:
            params = SynthParams()
            self._chk(L.chfsi_synth_defaults(0 if config_index is None else config_index,
                                             C.byref(params)))
        for k, v in overrides.items():
            if k in ("ngrid", "rc_proj", "kpt", "ngrid_density"):
                arr = getattr(params, k)
                for i, x in enumerate(v):
                    arr[i] = x
            else:
                setattr(params, k, v)
        self.params = params
        h = C.c_void_p()
        if positions is None:
            self._chk(L.chfsi_system_generate(C.byref(params), C.byref(h)))
        else:
            pos = np.ascontiguousarray(positions, dtype=np.float64).ravel()
            self._chk(L.chfsi_system_generate_at(C.byref(params), _ptr(pos, C.c_double),
                                                 C.byref(h)))
        self.handle = h
        info = SystemInfo()
        self._chk(L.chfsi_system_get_info(h, C.byref(info)))
        self.info = info
        self.ngrid = tuple(info.ngrid)
        self.n_pw, self.n_bands, self.n_occ = info.n_pw, info.n_bands, info.n_occ
        self.n_atoms, self.n_proj, self.n_ions = info.n_atoms, info.n_proj, info.n_ions_with_proj
        self.omega, self.n_elec, self.gmax, self.e_ewald = info.omega, info.n_elec, info.gmax, info.e_ewald
        self.lattice = np.array(info.lattice[:]).reshape(3, 3)
        self.ngrid_density = tuple(info.ngrid_density)
        self.ng_density = int(np.prod(self.ngrid_density))
        self.uspp, self.q_width = bool(info.uspp), info.q_width

    def __del__(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.chfsi_system_destroy(self.handle)
            self.handle = None

    def _get(self, fn, shape, dtype, ctype=None):
        a = np.zeros(shape, dtype=dtype)
        self._chk(getattr(self._L(), fn)(self.handle, _ptr(a, ctype)))
        return a

    @property
    def ng(self):
        return int(np.prod(self.ngrid))

    def miller(self):
        return self._get("chfsi_system_get_miller", (self.n_pw, 3), np.int32, C.c_int32)

    def kinetic(self):
        return self._get("chfsi_system_get_kinetic", self.n_pw, np.float64, C.c_double)

    def vloc_g(self):
        return self._get("chfsi_system_get_vloc_g", self.ng, np.complex128)

    def beta(self):
        return self._get("chfsi_system_get_beta", (self.n_proj, self.n_pw), np.complex128)

    def proj_offsets(self):
        n = self.n_ions + 1 if self.n_ions else 0
        return self._get("chfsi_system_get_proj_offsets", n, np.int32, C.c_int32)

    def _blocks_len(self):
        off = self.proj_offsets()
        return int(sum((off[i + 1] - off[i]) ** 2 for i in range(len(off) - 1)))

    def dmat(self):
        return self._get("chfsi_system_get_dmat", self._blocks_len(), np.complex128)

    def qmat(self):
        return self._get("chfsi_system_get_qmat", self._blocks_len(), np.complex128)

    def psi0(self):
        return self._get("chfsi_system_get_psi0", (self.n_bands, self.n_pw), np.complex128)

    def occupations(self):
        return self._get("chfsi_system_get_occupations", self.n_bands, np.float64, C.c_double)

    def positions(self):
        return self._get("chfsi_system_get_positions", (self.n_atoms, 3), np.float64, C.c_double)


# ---------------------------------------------------------------------------
# Device context
# ---------------------------------------------------------------------------
class Context:
    """Device-resident ChFSI state (one CUDA stream, all buffers on the GPU)."""

    def __init__(self, system=None, dims=None, precision=PREC_FP64, bound_mode=BOUND_HEURISTIC,
                 lanczos_steps=10, device=0, filter_form=FILTER_CHEBYSHEV):
        L = lib()
        cfg = Config()
        _check(L.chfsi_default_config(C.byref(cfg)))
        cfg.device, cfg.precision, cfg.bound_mode, cfg.lanczos_steps = \
            device, precision, bound_mode, lanczos_steps
        cfg.filter_form = filter_form
        h = C.c_void_p()
        if system is not None:
            _check(L.chfsi_create_from_system(system.handle, C.byref(cfg), C.byref(h)))
            self.ngrid, self.n_pw, self.n_bands = system.ngrid, system.n_pw, system.n_bands
        else:
            d = Dims()
            for i in range(3):
                d.ngrid[i] = dims["ngrid"][i]
            d.n_pw, d.n_bands = dims["n_pw"], dims["n_bands"]
            d.n_proj, d.n_ions = dims.get("n_proj", 0), dims.get("n_ions", 0)
            _check(L.chfsi_create(C.byref(d), C.byref(cfg), C.byref(h)))
            self.ngrid, self.n_pw, self.n_bands = tuple(dims["ngrid"]), d.n_pw, d.n_bands
        self.handle = h
        self.ng = int(np.prod(self.ngrid))
        if system is not None:
            self._n_atoms = system.n_atoms
        self._refresh_density_grid()

    def _refresh_density_grid(self):
        n3 = (C.c_int * 3)()
        _check(lib().chfsi_get_density_grid(self.handle, n3))
        self.ngrid_density = tuple(n3)
        self.ng_density = int(np.prod(self.ngrid_density))

    def rr_sweeps(self):
        v = C.c_int()
        self._c(lib().chfsi_get_rr_sweeps(self.handle, C.byref(v)))
        return v.value

    def set_density_grid(self, ngrid):
        n3 = (C.c_int * 3)(*ngrid)
        self._c(lib().chfsi_set_density_grid(self.handle, n3))
        self._refresh_density_grid()

    def set_augmentation(self, positions, width):
        p = np.ascontiguousarray(positions, dtype=np.float64).ravel()
        self._c(lib().chfsi_set_augmentation(self.handle, _ptr(p, C.c_double), width))

    def close(self):
        if getattr(self, "handle", None) and _lib is not None:
            _lib.chfsi_destroy(self.handle)
            self.handle = None

    __del__ = close

    def _c(self, st):
        _check(st, self.handle)

    # --- set-up -----------------------------------------------------------
    def set_basis(self, miller, kinetic, gmax):
        m = np.ascontiguousarray(miller, dtype=np.int32)
        k = np.ascontiguousarray(kinetic, dtype=np.float64)
        self._c(lib().chfsi_set_basis(self.handle, _ptr(m, C.c_int32), _ptr(k, C.c_double), gmax))

    def set_projectors(self, beta, proj_offsets, dmat):
        b = np.ascontiguousarray(beta, dtype=np.complex128)
        o = np.ascontiguousarray(proj_offsets, dtype=np.int32)
        d = np.ascontiguousarray(dmat, dtype=np.complex128)
        self._c(lib().chfsi_set_projectors(self.handle, _ptr(b), _ptr(o, C.c_int32), _ptr(d)))

    def set_qmat(self, qmat):
        """Ultrasoft overlap S = 1 + beta q beta^H (generalised problem)."""
        q = np.ascontiguousarray(qmat, dtype=np.complex128)
        self._c(lib().chfsi_set_qmat(self.handle, _ptr(q)))

    def s_min(self):
        v = C.c_double()
        self._c(lib().chfsi_get_s_min(self.handle, C.byref(v)))
        return v.value

    def set_veff(self, veff):
        v = np.ascontiguousarray(veff, dtype=np.float64).ravel()
        self._c(lib().chfsi_set_veff(self.handle, _ptr(v, C.c_double)))

    def set_psi(self, psi):
        p = np.ascontiguousarray(psi, dtype=np.complex128)
        self._c(lib().chfsi_set_psi(self.handle, _ptr(p)))

    def get_psi(self):
        p = np.zeros((self.n_bands, self.n_pw), dtype=np.complex128)
        self._c(lib().chfsi_get_psi(self.handle, _ptr(p)))
        return p

    def set_vloc_g(self, vloc_g):
        v = np.ascontiguousarray(vloc_g, dtype=np.complex128)
        self._c(lib().chfsi_set_vloc_g(self.handle, _ptr(v)))

    def set_cell(self, lattice, e_ewald, n_atoms):
        a = np.ascontiguousarray(lattice, dtype=np.float64).ravel()
        self._c(lib().chfsi_set_cell(self.handle, _ptr(a, C.c_double), e_ewald, n_atoms))

    def set_occupations(self, occ):
        o = np.ascontiguousarray(occ, dtype=np.float64)
        self._c(lib().chfsi_set_occupations(self.handle, _ptr(o, C.c_double)))

    def get_vloc(self):
        """V_loc on the density grid."""
        v = np.zeros(self.ng_density)
        self._c(lib().chfsi_get_vloc(self.handle, _ptr(v, C.c_double)))
        return v

    def get_veff(self):
        v = np.zeros(self.ng)
        self._c(lib().chfsi_get_veff(self.handle, _ptr(v, C.c_double)))
        return v

    def hpsi_device_ptr(self):
        p = C.c_void_p()
        self._c(lib().chfsi_hpsi_device_ptr(self.handle, C.byref(p)))
        return p.value

    def psi_device_ptr(self):
        p = C.c_void_p()
        self._c(lib().chfsi_psi_device_ptr(self.handle, C.byref(p)))
        return p.value

    # --- hot path -----------------------------------------------------------
    def apply_h(self, psi_dev_ptr, hpsi_dev_ptr, nb):
        """H|psi> on device pointers (e.g. torch CUDA tensors' data_ptr())."""
        self._c(lib().chfsi_apply_h(self.handle, C.c_void_p(psi_dev_ptr),
                                    C.c_void_p(hpsi_dev_ptr), nb))

    def apply_sinv_h(self, psi_dev_ptr, out_dev_ptr, nb):
        """S^-1 H|psi> (ultrasoft; H|psi> without q) on device pointers."""
        self._c(lib().chfsi_apply_sinv_h(self.handle, C.c_void_p(psi_dev_ptr),
                                         C.c_void_p(out_dev_ptr), nb))

    def apply_h_local(self, psi_dev_ptr, hpsi_dev_ptr, nb):
        """T + V_loc only, on device pointers."""
        self._c(lib().chfsi_apply_h_local(self.handle, C.c_void_p(psi_dev_ptr),
                                          C.c_void_p(hpsi_dev_ptr), nb))

    def stream(self):
        """The context's cudaStream_t as an integer handle."""
        p = C.c_void_p()
        self._c(lib().chfsi_get_stream(self.handle, C.byref(p)))
        return p.value or 0

    def chebyshev_filter(self, ndeg, eigenvalues=None):
        if eigenvalues is None:
            self._c(lib().chfsi_chebyshev_filter(self.handle, ndeg, None, 0))
        else:
            e = np.ascontiguousarray(eigenvalues, dtype=np.float64)
            self._c(lib().chfsi_chebyshev_filter(self.handle, ndeg, _ptr(e, C.c_double), len(e)))

    def rayleigh_ritz(self):
        w = np.zeros(self.n_bands)
        self._c(lib().chfsi_rayleigh_ritz(self.handle, _ptr(w, C.c_double)))
        return w

    def diagonalize(self, ndeg, eigenvalues=None):
        w = np.zeros(self.n_bands)
        if eigenvalues is None:
            self._c(lib().chfsi_diagonalize(self.handle, ndeg, None, 0, _ptr(w, C.c_double)))
        else:
            e = np.ascontiguousarray(eigenvalues, dtype=np.float64)
            self._c(lib().chfsi_diagonalize(self.handle, ndeg, _ptr(e, C.c_double), len(e),
                                            _ptr(w, C.c_double)))
        return w

    def bounds(self):
        b = np.zeros(4)
        self._c(lib().chfsi_get_bounds(self.handle, _ptr(b, C.c_double)))
        return b

    def filter_norms(self, ndeg):
        n = np.zeros(ndeg + 1)
        self._c(lib().chfsi_get_filter_norms(self.handle, _ptr(n, C.c_double), ndeg + 1))
        return n

    # --- SCF ---------------------------------------------------------------
    def construct_density(self):
        """rho on the density grid (with augmentation when set)."""
        r = np.zeros(self.ng_density)
        self._c(lib().chfsi_construct_density(self.handle, _ptr(r, C.c_double)))
        return r

    def build_v_eff(self, rho):
        r = np.ascontiguousarray(rho, dtype=np.float64).ravel()
        e2 = np.zeros(2)
        self._c(lib().chfsi_build_veff(self.handle, _ptr(r, C.c_double), _ptr(e2, C.c_double)))
        return e2

    def set_xc(self, functional):
        """XC_LDA_PZ (default) or XC_PBE for build_v_eff and run_scf."""
        self._c(lib().chfsi_set_xc(self.handle, functional))

    def set_ions(self, positions, zion, rc_loc, kpt=(0.0, 0.0, 0.0)):
        pos = np.ascontiguousarray(positions, dtype=np.float64).ravel()
        z = np.ascontiguousarray(zion, dtype=np.float64)
        rc = np.ascontiguousarray(rc_loc, dtype=np.float64)
        k = np.ascontiguousarray(kpt, dtype=np.float64)
        self._c(lib().chfsi_set_ions(self.handle, len(z), _ptr(pos, C.c_double), _ptr(z, C.c_double),
                                     _ptr(rc, C.c_double), _ptr(k, C.c_double)))
        self._n_atoms = len(z)

    def forces(self):
        """Hellmann-Feynman forces (n_atoms x 3, Ha/bohr) of the current state."""
        n = getattr(self, "_n_atoms", None)
        if n is None:
            raise BadInput("ions not set")
        f = np.zeros((n, 3))
        self._c(lib().chfsi_forces(self.handle, _ptr(f, C.c_double)))
        return f

    def get_density(self):
        r = np.zeros(self.ng_density)
        self._c(lib().chfsi_get_density(self.handle, _ptr(r, C.c_double)))
        return r

    def run_scf(self, ndeg, tol_per_atom=1e-6, max_iter=30, alpha=0.3, max_hist=6,
                first_passes=4, kT=0.01, fp64_switch_per_atom=1e-4, raise_not_converged=False,
                mixer=MIXER_PULAY, trace=False, cg_steps=0, verbose=False, tol_eig=0.0,
                restart=False, fp64_switch_eig=0.0):
        """Full SCF; mixer is MIXER_PULAY or, after set_mixer(), MIXER_LEARNED /
        MIXER_LEARNED_PULAY.  tol_eig > 0 adds the occupied-eigenvalue change test
        (mixed runs switch to FP64 below max(2 tol_eig, fp64_switch_eig));
        restart=True continues from this context's last state.  trace=True also
        returns rho_in and rho_out of every iteration (n_iter x N^3 each) as
        'trace_in' / 'trace_out'."""
        p = ScfParams(ndeg, max_iter, tol_per_atom, alpha, max_hist, first_passes, kT,
                      fp64_switch_per_atom, mixer, cg_steps, None, int(verbose), int(restart),
                      tol_eig, fp64_switch_eig)
        tr = None
        if trace:
            tr = np.zeros((max_iter, 2, self.ng_density))
            p.trace = _ptr(tr, C.c_double)
        energies = np.zeros(max_iter)
        residuals = np.zeros(max_iter)
        eigs = np.zeros(self.n_bands)
        r = ScfResult()
        r.energies = _ptr(energies, C.c_double)
        r.eigenvalues = _ptr(eigs, C.c_double)
        r.residuals = _ptr(residuals, C.c_double)
        st = lib().chfsi_scf_run(self.handle, C.byref(p), C.byref(r))
        if st not in (OK, NOT_CONVERGED) or (st == NOT_CONVERGED and raise_not_converged):
            _check(st, self.handle)
        out = {"converged": st == OK, "n_iter": r.n_iter, "n_iter_mixed": r.n_iter_mixed,
               "e_total": r.e_total,
               "e_band": r.e_band, "e_hartree": r.e_hartree, "e_xc": r.e_xc, "e_dc": r.e_dc,
               "e_entropy": r.e_entropy, "mu": r.mu,
               "seconds": r.seconds, "energies": energies[:r.n_iter].copy(), "eigenvalues": eigs,
               "residuals": residuals[:r.n_iter].copy(), "n_iter_learned": r.n_iter_learned,
               "fell_back": bool(r.fell_back), "n_fp64_retries": r.n_fp64_retries}
        if trace:
            out["trace_in"] = tr[:r.n_iter, 0].copy()
            out["trace_out"] = tr[:r.n_iter, 1].copy()
        return out

    def autotune(self):
        """Time the local H|psi> launch configurations; returns (choice, 18 timings)."""
        ch = C.c_int()
        t = np.zeros(18, dtype=np.float32)
        self._c(lib().chfsi_autotune(self.handle, C.byref(ch), _ptr(t, C.c_float)))
        return ch.value, t

    def set_launch_config(self, choice):
        self._c(lib().chfsi_set_launch_config(self.handle, choice))

    def tc_shapes(self):
        """Launch shapes of the projection and expansion tcgen05 GEMMs (-1: not tuned yet)."""
        a, b = C.c_int(), C.c_int()
        self._c(lib().chfsi_get_tc_shapes(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_tc_shapes(self, projection, expansion):
        self._c(lib().chfsi_set_tc_shapes(self.handle, projection, expansion))

    def band_cg(self, max_steps, tol=1e-10):
        """Band-by-band CG refinement; returns (band energies, steps, n_converged)."""
        e = np.zeros(self.n_bands)
        st = np.zeros(self.n_bands, dtype=np.int32)
        nc = C.c_int32()
        self._c(lib().chfsi_band_cg(self.handle, max_steps, tol, _ptr(e, C.c_double),
                                    _ptr(st, C.c_int32), C.byref(nc)))
        return e, st, nc.value

    # --- learned density mixer ------------------------------------------------
    def set_mixer(self, mixer):
        self._mixer = mixer  # keep the handle alive while attached
        self._c(lib().chfsi_set_mixer(self.handle, mixer.handle if mixer is not None else None))

    def mixer_samples(self, rho_in, rho_out, rho_star):
        """Features (T x 512) and targets (T x 320) of one trajectory on this grid."""
        a = np.ascontiguousarray(rho_in, dtype=np.float64).reshape(-1, self.ng_density)
        b = np.ascontiguousarray(rho_out, dtype=np.float64).reshape(-1, self.ng_density)
        st = np.ascontiguousarray(rho_star, dtype=np.float64).ravel()
        T = a.shape[0]
        x = np.zeros((T, MIXER_FEATURES), dtype=np.float32)
        t = np.zeros((T, MIXER_TARGETS), dtype=np.float32)
        self._c(lib().chfsi_mixer_samples(self.handle, _ptr(a, C.c_double), _ptr(b, C.c_double), T,
                                          _ptr(st, C.c_double), _ptr(x, C.c_float),
                                          _ptr(t, C.c_float)))
        return x, t
