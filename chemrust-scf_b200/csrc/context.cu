// chfsi_ctx: device-resident state of one ChFSI problem and the host-side
// drivers of the filter, Rayleigh-Ritz and SCF steps (C ABI in chfsi.h).
//
// Reference correspondence (paths relative to the chemrust-scf project):
//   chfsi_chebyshev_filter   src/eigensolver/chebyshev.rs:626-816
//   chfsi_rayleigh_ritz      src/eigensolver/rayleigh_ritz.rs:48-245 with the
//                            Cholesky-reduction math of subspace_diag.rs:229-391
//   chfsi_diagonalize        src/scf.rs:169-265
//   chfsi_scf_run            src/scf.rs:358-376 (+ intended bodies of the
//                            todo!() transitions, plans/phase-2/PHASE_PLAN.md)
// Every step runs on the device; the only host<->device traffic inside a
// diagonalize is the eigenvalue / status read-back at its end (the
// PcieAccount contract of src/scf.rs:238-251).
#include "chfsi.h"
#include "dense.hpp"
#include "gemm.hpp"
#include "gemm_tc.hpp"
#include "fft_plan.hpp"
#include "kernels.hpp"
#include "launch_count.hpp"
#include "mixer.hpp"
#include "system.hpp"

#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

namespace chfsi {

std::atomic<long long> g_launch_count{0};

chfsi_status cuda_fail(cudaError_t e, const char* expr, const char* file, int line);
bool invert_complex(std::vector<std::complex<double>>& a, int n);

namespace {

thread_local std::string g_last_error;

// ---------------------------------------------------------------- kernels
__global__ void k_gather_rows(const double2* __restrict__ src, int ld_src,
                              const int* __restrict__ perm, double2* __restrict__ dst, int n,
                              int rows) {
    const size_t tot = (size_t)rows * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < tot;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t b = t / n, i = t % n;
        dst[t] = src[b * ld_src + perm[i]];
    }
}
__global__ void k_scatter_rows(const double2* __restrict__ src, const int* __restrict__ perm,
                               double2* __restrict__ dst, int ld_dst, int n, int rows) {
    const size_t tot = (size_t)rows * n;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < tot;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t b = t / n, i = t % n;
        dst[b * ld_dst + perm[i]] = src[t];
    }
}
// cd[p][b] = sum_{j in ion(p)} D_ion[p - p0][j - p0] cp[j][b]
__global__ void k_apply_dmat(const double2* __restrict__ cp, double2* __restrict__ cd, int np,
                             int nb, const int* __restrict__ proj_ion, const int* __restrict__ poff,
                             const int* __restrict__ doff, const double2* __restrict__ dmat) {
    const size_t tot = (size_t)np * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < tot;
         t += (size_t)gridDim.x * blockDim.x) {
        const int p = (int)(t / nb), b = (int)(t % nb);
        const int ion = proj_ion[p];
        const int p0 = poff[ion], ne = poff[ion + 1] - p0;
        const double2* D = dmat + doff[ion] + (size_t)(p - p0) * ne;
        double2 s = make_double2(0.0, 0.0);
        for (int j = 0; j < ne; ++j) {
            const double2 d = D[j], c = cp[(size_t)(p0 + j) * nb + b];
            s.x += d.x * c.x - d.y * c.y;
            s.y += d.x * c.y + d.y * c.x;
        }
        cd[t] = s;
    }
}
__global__ void k_fill(double* x, size_t n, double v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        x[i] = v;
}

__global__ void k_f64_to_f32(const double2* __restrict__ a, float2* __restrict__ b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
__global__ void k_f32_to_f64(const float2* __restrict__ a, double2* __restrict__ b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        b[i] = make_double2((double)a[i].x, (double)a[i].y);
}

__global__ void __launch_bounds__(256) k_sumsq32(const float2* __restrict__ x, size_t n, double* acc) {
    __shared__ double red[8];
    double s = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        s += (double)x[i].x * x[i].x + (double)x[i].y * x[i].y;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        atomicAdd(acc, t);
    }
}

__global__ void k_conj(const double2* __restrict__ a, double2* __restrict__ b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        b[i] = make_double2(a[i].x, -a[i].y);
}

// Chebyshev step of the generalised problem: y = S^-1 H x = hx - corr, then
// the recurrence epilogue of the local pass (first degree / later degrees).
// C = double2 (FP64 filter) or float2 (FP32 filter; norms still summed in FP64).
// mode 3: residual step of R-ChFSI, out = a S^-1 H x + b x + c out + a lam[band] y
// with {a, b, c} = rc[0..2] (bands of npw elements).
template <typename C>
__global__ void __launch_bounds__(256)
k_cheb_combine(const C* __restrict__ hx, const C* __restrict__ corr, const C* __restrict__ x,
               C* out, size_t n, const double* coef, int mode, double* norm_acc,
               const C* __restrict__ yres = nullptr, const double* __restrict__ lam = nullptr,
               const double* __restrict__ rc = nullptr, int npw = 1) {
    using R = decltype(C{}.x);
    __shared__ double red[8];
    const R ie = (R)coef[4], nc = (R)coef[5];
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const R hr = hx[i].x - corr[i].x, hi = hx[i].y - corr[i].y;
        const C p = x[i];
        const R sr = hr * ie + nc * p.x, si = hi * ie + nc * p.y;
        R orr, oi;
        if (mode == 0) { orr = hr; oi = hi; }  // plain S^-1 H x
        else if (mode == 3) {
            const R a = (R)rc[0], b = (R)rc[1], c = (R)rc[2];
            const R ly = (R)(rc[0] * lam[i / (size_t)npw]);
            const C prev = out[i];
            const C y = yres[i];
            orr = a * hr + b * p.x + c * prev.x + ly * y.x;
            oi = a * hi + b * p.y + c * prev.y + ly * y.y;
        }
        else if (mode == 1) { orr = sr; oi = si; }
        else {
            const C prev = out[i];
            orr = (R)2 * sr - prev.x;
            oi = (R)2 * si - prev.y;
        }
        out[i].x = orr;
        out[i].y = oi;
        acc += (double)orr * orr + (double)oi * oi;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0 && norm_acc) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        atomicAdd(norm_acc, t);
    }
}

// ---- R-ChFSI (reference_paper/2025 main.tex Algorithm 3) coefficient tables:
// sigma-scaled Chebyshev steps {a_k, b_k, c_k} (k = 2..p) and the filtered
// Ritz values L_k(lambda_b) (k = 0..p) of every band; rc[0] = sigma_1 / e.
// coef: [lambda_max, cut, c, e, ..]; lambda_min = eig[0].
__global__ void k_rc_tables(const double* __restrict__ coef, const double* __restrict__ eig,
                            int nb, int p, double* __restrict__ rc, double* __restrict__ lam) {
    __shared__ double s_rc[3 * 65];
    const double c = coef[2], e = coef[3];
    if (threadIdx.x == 0) {
        double sigma = e / (eig[0] - c);
        const double sigma1 = sigma, gamma = 2.0 / sigma1;
        s_rc[0] = sigma1 / e;
        s_rc[1] = s_rc[2] = 0.0;
        for (int k = 2; k <= p; ++k) {
            const double s2 = 1.0 / (gamma - sigma);
            const double a = 2.0 * s2 / e;
            s_rc[3 * k] = a;
            s_rc[3 * k + 1] = -a * c;
            s_rc[3 * k + 2] = -sigma * s2;
            sigma = s2;
        }
        s_rc[3] = s_rc[4] = s_rc[5] = 0.0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 3 * (p + 1); i += blockDim.x) rc[i] = s_rc[i];
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const double l = eig[b];
        double l0 = 1.0, l1 = s_rc[0] * (l - c);
        lam[b] = l0;
        if (p >= 1) lam[nb + b] = l1;
        for (int k = 2; k <= p; ++k) {
            const double l2 = s_rc[3 * k] * l1 * l + s_rc[3 * k + 1] * l1 + s_rc[3 * k + 2] * l0;
            lam[(size_t)k * nb + b] = l2;
            l0 = l1;
            l1 = l2;
        }
    }
}

// t = hx - (x + sx_extra) lam[band]   (residual H X - S X Lam; sx_extra = S X - X or null)
__global__ void k_rc_resid(const double2* __restrict__ hx, const double2* __restrict__ x,
                           const double2* __restrict__ sx_extra, const double* __restrict__ lam,
                           int npw, size_t n, double2* __restrict__ t) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double l = lam[i / (size_t)npw];
        double2 v = x[i];
        if (sx_extra) { v.x += sx_extra[i].x; v.y += sx_extra[i].y; }
        t[i] = make_double2(hx[i].x - v.x * l, hx[i].y - v.y * l);
    }
}

// out = s y (precision of out)
template <typename C>
__global__ void k_rc_scale(const double2* __restrict__ y, const double* __restrict__ s, size_t n,
                           C* __restrict__ out, C* __restrict__ ycopy) {
    using R = decltype(C{}.x);
    const double f = *s;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        out[i].x = (R)(f * y[i].x);
        out[i].y = (R)(f * y[i].y);
        if (ycopy) { ycopy[i].x = (R)y[i].x; ycopy[i].y = (R)y[i].y; }
    }
}

// X_new = R + X lam[band], HX_new = HR + HX lam[band]  (FP64 out)
template <typename C>
__global__ void k_rc_final(const C* __restrict__ r, const C* __restrict__ hr,
                           const double2* __restrict__ x, const double2* __restrict__ hx,
                           const double* __restrict__ lam, int npw, size_t n,
                           double2* __restrict__ xo, double2* __restrict__ hxo) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double l = lam[i / (size_t)npw];
        xo[i] = make_double2((double)r[i].x + x[i].x * l, (double)r[i].y + x[i].y * l);
        hxo[i] = make_double2((double)hr[i].x + hx[i].x * l, (double)hr[i].y + hx[i].y * l);
    }
}

// ---- band-CG vector kernels
__global__ void k_tpa(const double* __restrict__ kin, double inv_mean, double* __restrict__ t,
                      size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double x = kin[i] * inv_mean;
        const double den = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x));
        t[i] = 1.0 / (1.0 + 16.0 * x * x * x * x / den);
    }
}

// out = diag(t) (x + u), u optional
__global__ void k_diag_apply(const double* __restrict__ t, const double2* __restrict__ x,
                             const double2* __restrict__ u, double2* __restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double2 v = x[i];
        if (u) { v.x += u[i].x; v.y += u[i].y; }
        out[i] = make_double2(t[i] * v.x, t[i] * v.y);
    }
}

// y = a y + b x (complex a, b)
__global__ void k_lincomb(double2* __restrict__ y, double2 a, const double2* __restrict__ x,
                          double2 b, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double2 yv = y[i];
        double2 r = make_double2(a.x * yv.x - a.y * yv.y, a.x * yv.y + a.y * yv.x);
        if (x) {
            const double2 xv = x[i];
            r.x += b.x * xv.x - b.y * xv.y;
            r.y += b.x * xv.y + b.y * xv.x;
        }
        y[i] = r;
    }
}

// Modified Gram-Schmidt overlaps from the classical ones: ov_j = v_j -
// sum_{i<j} G[j][i] ov_i with G[j][i] = <psi_j|S psi_i> (one warp, j in order).
__global__ void k_mgs_overlaps(const double2* __restrict__ v, const double2* __restrict__ G, int ld,
                               int k, double2* __restrict__ ov) {
    const int lane = threadIdx.x;
    for (int j = 0; j < k; ++j) {
        double sr = 0.0, si = 0.0;
        const double2* g = G + (size_t)j * ld;
        for (int i = lane; i < j; i += 32) {
            const double2 a = g[i], b = ov[i];
            sr += a.x * b.x - a.y * b.y;
            si += a.x * b.y + a.y * b.x;
        }
        for (int o = 16; o > 0; o >>= 1) {
            sr += __shfl_xor_sync(0xffffffffu, sr, o);
            si += __shfl_xor_sync(0xffffffffu, si, o);
        }
        if (lane == 0) ov[j] = make_double2(v[j].x - sr, v[j].y - si);
        __syncwarp();
    }
}

struct DotSet {
    const double2* a[6];
    const double2* b[6];
};
// out[2i], out[2i + 1] += Re, Im <a_i | b_i>
__global__ void __launch_bounds__(256)
k_multi_dot(DotSet ds, int k, size_t n, double* __restrict__ out) {
    __shared__ double red[6][2][8];
    double acc[6][2];
    for (int j = 0; j < 6; ++j) acc[j][0] = acc[j][1] = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            if (j >= k) break;
            const double2 x = ds.a[j][i], y = ds.b[j][i];
            acc[j][0] += x.x * y.x + x.y * y.y;
            acc[j][1] += x.x * y.y - x.y * y.x;
        }
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = 0; j < k; ++j)
        for (int c = 0; c < 2; ++c) {
            double v = acc[j][c];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) red[j][c][w] = v;
        }
    __syncthreads();
    if (threadIdx.x < 2 * k) {
        const int j = threadIdx.x >> 1, c = threadIdx.x & 1;
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[j][c][q];
        atomicAdd(out + threadIdx.x, t);
    }
}

int grid_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 148 * 8 ? b : 148 * 8);
}

// Position of frequency k after the in-place DIF (mixed-radix digit reversal).
void digit_reversal(const AxisPlan& P, std::vector<int>& pos) {
    const int n = P.n;
    pos.assign(n, 0);
    for (int k = 0; k < n; ++k) {
        int p = 0, span = n, kk = k;
        for (int t = 0; t < P.nst; ++t) {
            const int r = P.r[t];
            span /= r;
            p += (kk % r) * span;
            kk /= r;
        }
        pos[k] = p;
    }
}

// Test hook (chfsi_test_inject): device allocations left before one fails
// with cudaErrorMemoryAllocation; negative = no failure planned.
std::atomic<long long> g_alloc_fail_in{-1};

template <typename T> cudaError_t dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) return cudaSuccess;
    if (g_alloc_fail_in.load() >= 0 && g_alloc_fail_in.fetch_sub(1) == 0)
        return cudaErrorMemoryAllocation;
    return cudaMalloc((void**)p, n * sizeof(T));
}

// The context stream is non-blocking, so a legacy-stream cudaMemcpy or
// cudaMemset is not ordered with its kernels (a pageable host-to-device
// cudaMemcpy may even return before its DMA lands).  Every set-up copy and
// fill therefore goes through the context stream; copies wait for it so
// that pageable host buffers can be released or read right after.
cudaError_t copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind,
                      cudaStream_t st) {
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, st);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(st);
}

}  // namespace

void set_last_error(const char* msg) { g_last_error = msg; }

chfsi_status cuda_fail(cudaError_t e, const char* expr, const char* file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "CUDA error %s (%s) at %s:%d: %s", cudaGetErrorName(e),
                  cudaGetErrorString(e), file, line, expr);
    g_last_error = buf;
    return e == cudaErrorMemoryAllocation ? CHFSI_ERR_OUT_OF_MEMORY : CHFSI_ERR_CUDA;
}

}  // namespace chfsi

using namespace chfsi;

struct chfsi_ctx {
    chfsi_dims dims{};
    chfsi_config cfg{};
    int device = 0;
    cudaStream_t st = nullptr;
    std::string err;
    int nx = 0, ny = 0, nz = 0, n_pw = 0, nb = 0, np = 0, nions = 0;
    size_t ng = 0;
    bool basis_set = false, veff_set = false, psi_set = false, proj_set = false;
    bool have_vloc = false;
    double kin_max = 0.0, omega = 0.0, n_elec = 0.0, e_ewald = 0.0, n_atoms = 1.0;
    double recip[9] = {};
    double lattice[9] = {};
    // geometry
    HGeom geo{};
    AxisPlan ax{}, ay{}, az{};
    std::vector<int> dr[3];
    int* d_col_start = nullptr; int* d_col_pos = nullptr; int* d_pw_col = nullptr;
    int* d_pw_zpos = nullptr; int* d_xact = nullptr; int* d_colidx = nullptr; int* d_idr[3] = {nullptr, nullptr, nullptr};
    int* d_perm = nullptr; bool perm_identity = true;
    double2* d_twd = nullptr;  // twiddle tables x | y | z, FP64
    float2* d_twf = nullptr;   // same, FP32
    double* d_kin = nullptr;
    // potentials
    double* d_veff = nullptr; double* d_vloc = nullptr; double* d_minmax = nullptr;
    // projectors
    double2* d_beta = nullptr; double2* d_dmat = nullptr;
    int* d_proj_ion = nullptr; int* d_poff = nullptr; int* d_doff = nullptr;
    double2* d_cp = nullptr; double2* d_cd = nullptr;
    // wavefunctions
    double2* d_psi = nullptr; double2* d_psi2 = nullptr; double2* d_hpsi = nullptr;
    double2* d_nl = nullptr; double2* d_work = nullptr; double2* d_part = nullptr;
    size_t part_elems = 0;
    // Rayleigh-Ritz
    double2* d_H = nullptr; double2* d_S = nullptr; double2* d_T1 = nullptr;
    double2* d_T2 = nullptr; double2* d_V = nullptr;
    double* d_eig = nullptr; double* d_eig_prev = nullptr; double* d_jac = nullptr;
    int* d_flags = nullptr;  // [0] cholesky info, [1] norm-guard degree, [2] jacobi sweeps
    int jac_max_sweeps = 40;
    // filter
    double* d_coef = nullptr; double* d_nsq = nullptr; int max_deg = 64;
    double h_coef[6] = {};
    std::vector<double> h_nsq;
    int last_ndeg = 0;
    // Lanczos
    double2* d_lz_v = nullptr; double2* d_lz_v0 = nullptr; double2* d_lz_f = nullptr;
    double2* d_lz_start = nullptr; double* d_lz = nullptr;
    bool lz_carry = false;       // d_lz holds the tridiagonal of a Lanczos run carried by a filter
    int lz_carry_k = 0;
    // density / SCF
    double* d_occ = nullptr; std::vector<double> occ;
    std::vector<double> kin_host;  // 1/2 |G+k|^2 in the internal plane-wave order
    // band-by-band CG refinement (band_cg.rs)
    double* d_tpa = nullptr;       // TPA preconditioner diagonal
    double2* d_cgR = nullptr;      // conj((-q^-1 - beta^H T beta)^-1), ultrasoft only
    double2* d_cgv = nullptr;      // 10 work vectors of n_pw
    double2* d_cgc = nullptr;      // 3 x n_proj projections
    double2* d_cgov = nullptr;     // 2 x n_bands overlaps with the refined lower bands
    double2* d_cgG = nullptr;      // <psi_j|S psi_i> of the refined bands, j > i (n_bands^2)
    double2* d_cgpart = nullptr;   // split-K partials of the CG GEMVs
    double* d_cgdot = nullptr;     // 16 dot-product accumulators
    bool cg_ready = false;
    double2* d_psi_save = nullptr; // start of a mixed-precision pass (FP64 retry)
    // R-ChFSI (residual filter): H X, residual, FP64 recurrence pair, FP32 residual copy
    double2* d_rc_hx = nullptr; double2* d_rc_y = nullptr;
    double2* d_rc_r0 = nullptr; double2* d_rc_r1 = nullptr;
    float2* d_rc_y32 = nullptr; double* d_rc_coef = nullptr; double* d_rc_lam = nullptr;
    double* d_rho_in = nullptr; double* d_rho_out = nullptr; double* d_rho_next = nullptr;
    double2* d_cgrid = nullptr; double* d_acc = nullptr;
    double* d_hist = nullptr;  // 2 * kPulayMax * ng
    double** d_hist_ptrs = nullptr;
    double* d_dots = nullptr;
    // ultrasoft overlap S = 1 + beta q beta^H
    bool uspp = false;
    double s_min = 1.0;
    double2* d_qmat = nullptr;   // per-ion q blocks (layout of D)
    double2* d_sinvT = nullptr;  // M^T, M = q (1 + B q)^-1, S^-1 = 1 - beta M beta^H
    double2* d_bmatT = nullptr;  // B^T = conj(B), B = beta^H beta
    double2* d_cq = nullptr;     // n_proj x n_bands scratch
    double2* d_sx = nullptr;     // n_bands x n_pw scratch
    // mixed precision (FP32 filter, tcgen05 BF16x3 GEMMs)
    bool mixed = false;          // configured precision
    bool scf_done = false;       // a chfsi_scf_run left density, psi and eigenvalues
    double scf_e_last = 0.0;     // its last total energy (restart reference)
    bool mixed_active = false;   // current filter precision (SCF may switch to FP64)
    float2* d_psi32a = nullptr; float2* d_psi32b = nullptr; float2* d_psi32 = nullptr;
    float2* d_hpsi32 = nullptr; float2* d_nl32 = nullptr; float2* d_work32 = nullptr;
    void* d_planes = nullptr;    // all bf16 plane storage
    TcPlanes tp_beta_a, tp_betaT_b, tp_psi_b, tp_small_a;
    float* d_tc_part = nullptr; int* d_tc_err = nullptr;
    bool beta_planes_ready = false;
    // tcgen05 launch shapes of the projection and the expansion (-1: time
    // them at the first mixed filter)
    int tc_shape[2] = {-1, -1};
    bool last_pass_fp32 = false;  // the last filter ran in FP32
    int last_sweeps = 0;          // Jacobi sweeps of the last Rayleigh-Ritz
    // density grid: density, potentials, mixing and augmentation live here.
    // It is the wavefunction grid unless chfsi_set_density_grid chose a
    // finer one; then the smooth density is interpolated up by zero padding
    // in G and V_eff comes back by truncation.
    int fnx = 0, fny = 0, fnz = 0; size_t fng = 0;
    AxisPlan fax{}, fay{}, faz{};
    std::vector<int> fdr[3];
    int* d_fidr[3] = {nullptr, nullptr, nullptr};
    bool fine = false;
    int* d_gmap_w = nullptr; int* d_gmap_f = nullptr; int n_gmap = 0;  // shared G vectors
    double* d_veff_d = nullptr;   // V_eff on the density grid
    // exchange-correlation functional; PBE scratch: three complex density
    // grids (gradient, then 2 de/dsigma grad rho) and de/drho
    int xc = CHFSI_XC_LDA_PZ;
    double2* d_gga = nullptr; double* d_gga_v1 = nullptr;
    // ions for forces (chfsi_set_ions)
    int n_ion_atoms = 0;
    std::vector<double> atom_pos, atom_z, atom_rc;
    double ion_kpt[3] = {0.0, 0.0, 0.0};
    double* d_ion = nullptr;      // positions (3n), z (n), rc (n), forces (3n)
    double* d_qvec = nullptr;     // Cartesian G + k per plane wave, 3 x n_pw
    int* d_atom_of_ion = nullptr;
    std::vector<int32_t> miller_ctx;  // Miller indices in the context's plane-wave order
    double* d_rho_w = nullptr;    // smooth density on the wavefunction grid
    double2* d_wgrid = nullptr;   // wavefunction-grid complex scratch
    // ultrasoft augmentation Q_ij(r) = q_ij g(|r - R_I|)
    bool aug = false; double aug_width = 0.0;
    std::vector<double> ion_pos;  // ions with projectors, x 3 (bohr)
    double2* d_phase = nullptr;   // per ion e^{-i 2 pi f_d h}: [ion][fnx | fny | fnz]
    double2* d_dmat0 = nullptr;   // unscreened D
    double* d_cion = nullptr;     // per ion sum_n f_n C^H q C
    double* d_vion = nullptr;     // per ion int V_eff g(r - R_I)
    // learned density mixer (G-space residual history on the density grid)
    chfsi_mixer* mixer = nullptr;
    unsigned char* d_shell = nullptr;  // |G| shell per grid point (digit-reversed layout)
    double2* d_mix_c = nullptr;        // 7 complex grids: R_0..R_3 ring, D, E, work
    double* d_mix_r = nullptr;         // 4 real grids: prev rho_in, rho*, two uploads
    double* d_mix_acc = nullptr;       // kMixShells x kShellAcc
    float* d_mix_x = nullptr;          // features, targets, outputs
    // pinned host scratch
    double* h_pin = nullptr; size_t h_pin_n = 0;

    chfsi_status fail(chfsi_status s, const std::string& m) {
        err = m;
        g_last_error = m;
        return s;
    }
};

#define CK(expr)                                                                   \
    do {                                                                           \
        cudaError_t _e = (expr);                                                   \
        if (_e != cudaSuccess) {                                                   \
            chfsi_status _s = cuda_fail(_e, #expr, __FILE__, __LINE__);            \
            ctx->err = g_last_error;                                               \
            return _s;                                                             \
        }                                                                          \
    } while (0)

namespace {

chfsi_status ensure_pinned(chfsi_ctx* ctx, size_t n) {
    if (ctx->h_pin_n >= n) return CHFSI_OK;
    if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
    ctx->h_pin = nullptr;
    ctx->h_pin_n = 0;
    CK(cudaMallocHost((void**)&ctx->h_pin, n * sizeof(double)));
    ctx->h_pin_n = n;
    return CHFSI_OK;
}

// ---------------------------------------------------------------- H|psi>
// out = epilogue(H psi) for nb bands of psi (ld n_pw, context PW order).
// Coefficients of one residual (R-ChFSI) step for the kEpiResid epilogue.
struct ResidStep {
    const double* rc;   // {a, b, c}
    const double* lam;  // per band
    const void* y;      // residual, ld n_pw
};

chfsi_status apply_h_dev(chfsi_ctx* ctx, const double2* psi, double2* out, int nb, int mode,
                         double* norm_acc, int plain_band = -1, double2* plain_out = nullptr,
                         const ResidStep* rs = nullptr, bool with_nl = true) {
    Epilogue e{};
    e.mode = mode;
    e.plain_band = plain_band;
    e.plain_out = plain_out;
    if (rs) { e.rc = rs->rc; e.lam = rs->lam; e.yres = rs->y; }
    e.kin = ctx->d_kin;
    e.coef = ctx->d_coef;
    e.nl = nullptr;
    e.norm_acc = norm_acc;
    e.inv_n = 1.0 / (double)ctx->ng;
    if (ctx->np > 0 && with_nl) {
        // C = beta^H psi, C <- D C, nl = beta C  (chebyshev.rs:416-500)
        gemm_cn(ctx->d_beta, ctx->n_pw, psi, ctx->n_pw, ctx->np, nb, ctx->n_pw, ctx->d_part,
                ctx->d_cp, ctx->st);
        count_launch();
        k_apply_dmat<<<grid_for((size_t)ctx->np * nb), 256, 0, ctx->st>>>(
            ctx->d_cp, ctx->d_cd, ctx->np, nb, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff,
            ctx->d_dmat);
        gemm_tn(ctx->d_cd, nb, ctx->d_beta, ctx->n_pw, ctx->d_nl, ctx->n_pw, nb, ctx->n_pw,
                ctx->np, 1.0, 0.0, ctx->st);
        e.nl = ctx->d_nl;
    }
    launch_zsticks_inverse<double2>(psi, ctx->n_pw, ctx->d_work, nb, ctx->geo, ctx->st);
    launch_planes_vloc<double2>(ctx->d_work, ctx->d_veff, nb, ctx->geo, ctx->st);
    launch_zsticks_forward<double2>(ctx->d_work, psi, ctx->n_pw, out, ctx->n_pw, nb, ctx->geo, e,
                                    ctx->st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// S^-1 H x of the generalised (ultrasoft) problem as d_hpsi - d_sx:
//   H x = H_loc x + beta G,  G = D C,  C = beta^H x,
//   S^-1 = 1 - beta M beta^H,  M = q (1 + B q)^-1,  B = beta^H beta,
//   S^-1 H x = H_loc x - beta F,  F = M (E + B G) - G,  E = beta^H (H_loc x),
// so one application takes two n_pw-long projections (C, E) and one
// expansion (beta F); B G and M (.) are n_proj-sized products.  d_hpsi gets
// H_loc x for ncols columns, d_sx gets beta F for the first nout of them;
// d_cd keeps G (ld ncols).
chfsi_status sinv_h_parts(chfsi_ctx* ctx, const double2* x, int ncols, int nout) {
    cudaStream_t st = ctx->st;
    const int np = ctx->np, npw = ctx->n_pw;
    gemm_cn(ctx->d_beta, npw, x, npw, np, ncols, npw, ctx->d_part, ctx->d_cp, st);
    count_launch();
    k_apply_dmat<<<grid_for((size_t)np * ncols), 256, 0, st>>>(
        ctx->d_cp, ctx->d_cd, np, ncols, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff, ctx->d_dmat);
    chfsi_status s = apply_h_dev(ctx, x, ctx->d_hpsi, ncols, kEpiApply, nullptr, -1, nullptr,
                                 nullptr, false);
    if (s) return s;
    gemm_cn(ctx->d_beta, npw, ctx->d_hpsi, npw, np, ncols, npw, ctx->d_part, ctx->d_cp, st);
    gemm_tn(ctx->d_bmatT, np, ctx->d_cd, ncols, ctx->d_cp, ncols, np, ncols, np, 1.0, 1.0, st);
    CK(cudaMemcpyAsync(ctx->d_cq, ctx->d_cd, sizeof(double2) * (size_t)np * ncols,
                       cudaMemcpyDeviceToDevice, st));
    gemm_tn(ctx->d_sinvT, np, ctx->d_cp, ncols, ctx->d_cq, ncols, np, ncols, np, 1.0, -1.0, st);
    gemm_tn(ctx->d_cq, ncols, ctx->d_beta, npw, ctx->d_sx, npw, nout, npw, np, 1.0, 0.0, st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// One filter operator application: H x, or S^-1 H x for the generalised
// (ultrasoft) problem (sinv_h_parts), with the recurrence epilogue in
// k_cheb_combine.
// lz_col: row nb of x holds the carried Lanczos vector v; H v goes to d_lz_f
// (the H of the generalised problem's pencil, without S^-1, like the
// separate Lanczos run).
chfsi_status apply_op_dev(chfsi_ctx* ctx, const double2* x, double2* out, int nb, int mode,
                          double* norm_acc, bool lz_col = false) {
    if (!ctx->uspp || mode == kEpiApply) {
        if (!lz_col) return apply_h_dev(ctx, x, out, nb, mode, norm_acc);
        return apply_h_dev(ctx, x, out, nb + 1, mode, norm_acc, nb, ctx->d_lz_f);
    }
    const int ncols = nb + (lz_col ? 1 : 0);
    chfsi_status s = sinv_h_parts(ctx, x, ncols, nb);
    if (s) return s;
    cudaStream_t st = ctx->st;
    if (lz_col) {
        // H v = H_loc v + beta G_v
        CK(cudaMemcpyAsync(ctx->d_lz_f, ctx->d_hpsi + (size_t)nb * ctx->n_pw,
                           sizeof(double2) * ctx->n_pw, cudaMemcpyDeviceToDevice, st));
        gemm_tn(ctx->d_cd + nb, ncols, ctx->d_beta, ctx->n_pw, ctx->d_lz_f, ctx->n_pw, 1,
                ctx->n_pw, ctx->np, 1.0, 1.0, st);
    }
    const size_t n = (size_t)nb * ctx->n_pw;
    count_launch();
    k_cheb_combine<double2><<<grid_for(n), 256, 0, st>>>(ctx->d_hpsi, ctx->d_sx, x, out, n, ctx->d_coef,
                                                 mode == kEpiChebFirst ? 1 : 2, norm_acc);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// ---------------------------------------------------------------- bounds
chfsi_status lanczos_bound(chfsi_ctx* ctx) {
    const int k = std::max(2, std::min(ctx->cfg.lanczos_steps, 60));
    const size_t n = ctx->n_pw;
    CK(cudaMemsetAsync(ctx->d_lz, 0, sizeof(double) * 2 * k, ctx->st));
    CK(cudaMemcpyAsync(ctx->d_lz_v, ctx->d_lz_start, n * sizeof(double2), cudaMemcpyDeviceToDevice,
                       ctx->st));
    double* fn0 = ctx->d_lz + 2 * k - 1;  // reuse last slot for |v0|^2 before the loop
    sumsq(ctx->d_lz_v, n, fn0, ctx->st);
    scale_by_rsqrt(ctx->d_lz_v, n, fn0, ctx->st);
    CK(cudaMemsetAsync(fn0, 0, sizeof(double), ctx->st));
    for (int j = 0; j < k; ++j) {
        chfsi_status s = apply_h_dev(ctx, ctx->d_lz_v, ctx->d_lz_f, 1, kEpiApply, nullptr);
        if (s) return s;
        lanczos_a(ctx->d_lz_f, ctx->d_lz_v, ctx->d_lz_v0, j > 0 ? ctx->d_lz + k + j - 1 : nullptr,
                  n, ctx->d_lz + j, ctx->st);
        lanczos_b(ctx->d_lz_f, ctx->d_lz_v, ctx->d_lz + j, n, ctx->d_lz + k + j, ctx->st);
        if (j < k - 1) lanczos_c(ctx->d_lz_f, ctx->d_lz_v, ctx->d_lz_v0, n, ctx->d_lz + k + j, ctx->st);
    }
    bounds(ctx->kin_max, ctx->d_minmax, nullptr, 0, ctx->d_lz, k, 1.0 / ctx->s_min, ctx->d_coef,
           ctx->st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

chfsi_status compute_bounds(chfsi_ctx* ctx, const double* eig_dev, int n_eig) {
    if (ctx->cfg.bound_mode == CHFSI_BOUND_LANCZOS_FUSED && ctx->lz_carry) {
        // tridiagonal left by the Lanczos vector the previous filter carried
        bounds(ctx->kin_max, ctx->d_minmax, eig_dev, n_eig, ctx->d_lz, ctx->lz_carry_k,
               1.0 / ctx->s_min, ctx->d_coef, ctx->st);
        ctx->lz_carry = false;
        CK(cudaGetLastError());
        return CHFSI_OK;
    }
    if (ctx->cfg.bound_mode == CHFSI_BOUND_LANCZOS ||
        ctx->cfg.bound_mode == CHFSI_BOUND_LANCZOS_FUSED) {
        chfsi_status s = lanczos_bound(ctx);
        if (s) return s;
        // the cut still comes from the previous eigenvalues
        const int k = std::max(2, std::min(ctx->cfg.lanczos_steps, 60));
        bounds(ctx->kin_max, ctx->d_minmax, eig_dev, n_eig, ctx->d_lz, k, 1.0 / ctx->s_min,
               ctx->d_coef, ctx->st);
    } else {
        bounds(ctx->kin_max, ctx->d_minmax, eig_dev, n_eig, nullptr, 0, 1.0 / ctx->s_min, ctx->d_coef,
               ctx->st);
    }
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// ---------------------------------------------------------------- filter
chfsi_status filter_dev(chfsi_ctx* ctx, int ndeg, const double* eig_dev, int n_eig) {
    if (ndeg < 0 || ndeg > ctx->max_deg) return ctx->fail(CHFSI_ERR_BAD_INPUT, "ndeg out of range");
    chfsi_status s = compute_bounds(ctx, eig_dev, n_eig);
    if (s) return s;
    const size_t n = (size_t)ctx->nb * ctx->n_pw;
    CK(cudaMemsetAsync(ctx->d_nsq, 0, sizeof(double) * (ndeg + 1), ctx->st));
    sumsq(ctx->d_psi, n, ctx->d_nsq, ctx->st);
    double2* A = ctx->d_psi;   // psi_{k-2}
    double2* B = ctx->d_psi2;  // psi_{k-1}
    // k-step Lanczos carried as column nb of the first k applies (its bound
    // serves the next filter): v_0 is the shared start vector, normalised
    const int klz = ctx->cfg.bound_mode == CHFSI_BOUND_LANCZOS_FUSED
                        ? std::min(std::max(2, std::min(ctx->cfg.lanczos_steps, 60)), ndeg) : 0;
    const size_t npw = ctx->n_pw;
    if (klz >= 2) {
        CK(cudaMemsetAsync(ctx->d_lz, 0, sizeof(double) * 2 * klz, ctx->st));
        CK(cudaMemcpyAsync(ctx->d_lz_v, ctx->d_lz_start, npw * sizeof(double2),
                           cudaMemcpyDeviceToDevice, ctx->st));
        double* fn0 = ctx->d_lz + 2 * klz - 1;
        sumsq(ctx->d_lz_v, npw, fn0, ctx->st);
        scale_by_rsqrt(ctx->d_lz_v, npw, fn0, ctx->st);
        CK(cudaMemsetAsync(fn0, 0, sizeof(double), ctx->st));
        CK(cudaMemcpyAsync(A + (size_t)ctx->nb * npw, ctx->d_lz_v, npw * sizeof(double2),
                           cudaMemcpyDeviceToDevice, ctx->st));
    }
    // Lanczos step j on H v_j (in d_lz_f); v_{j+1} goes to row nb of `next`
    auto lz_step = [&](int j, double2* next) {
        lanczos_a(ctx->d_lz_f, ctx->d_lz_v, ctx->d_lz_v0, j > 0 ? ctx->d_lz + klz + j - 1 : nullptr,
                  npw, ctx->d_lz + j, ctx->st);
        lanczos_b(ctx->d_lz_f, ctx->d_lz_v, ctx->d_lz + j, npw, ctx->d_lz + klz + j, ctx->st);
        if (j < klz - 1) {
            lanczos_c(ctx->d_lz_f, ctx->d_lz_v, ctx->d_lz_v0, npw, ctx->d_lz + klz + j, ctx->st);
            return cudaMemcpyAsync(next + (size_t)ctx->nb * npw, ctx->d_lz_v, npw * sizeof(double2),
                                   cudaMemcpyDeviceToDevice, ctx->st);
        }
        return cudaSuccess;
    };
    if (ndeg >= 1) {
        s = apply_op_dev(ctx, A, B, ctx->nb, kEpiChebFirst, ctx->d_nsq + 1, klz > 0);
        if (s) return s;
        if (klz > 0) CK(lz_step(0, B));
    }
    for (int k = 2; k <= ndeg; ++k) {
        // psi_k = 2 sigma(H) psi_{k-1} - psi_{k-2}, written over psi_{k-2}
        const bool lz = k - 1 < klz;
        s = apply_op_dev(ctx, B, A, ctx->nb, kEpiCheb, ctx->d_nsq + k, lz);
        if (s) return s;
        if (lz) CK(lz_step(k - 1, A));
        std::swap(A, B);
    }
    if (klz >= 2) {
        ctx->lz_carry = true;
        ctx->lz_carry_k = klz;
    }
    double2* fin = ndeg >= 1 ? B : A;
    double2* other = fin == ctx->d_psi ? ctx->d_psi2 : ctx->d_psi;
    ctx->d_psi = fin;
    ctx->d_psi2 = other;
    s = apply_h_dev(ctx, ctx->d_psi, ctx->d_hpsi, ctx->nb, kEpiApply, nullptr);
    if (s) return s;
    norm_guard(ctx->d_nsq, ndeg, ctx->d_flags + 1, ctx->st);
    ctx->last_ndeg = ndeg;
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// ---------------------------------------------------------------- Rayleigh-Ritz
// fp32_block: the block comes from the FP32 filter, whose d_hpsi holds the
// local part only; the non-local part enters the subspace matrix as C^H D C
// (C = beta^H psi, shared with the ultrasoft overlap), which is how the
// mixed-precision passes run their FP64 Rayleigh-Ritz.
chfsi_status rr_dev(chfsi_ctx* ctx, bool fp32_block) {
    const int n = ctx->nb, np = ctx->np;
    cudaStream_t st = ctx->st;
    const bool nl_sub = fp32_block && np > 0;
    const bool aug_s = ctx->uspp && np > 0;
    if (nl_sub || aug_s) {
        // C = beta^H psi and its conjugate
        gemm_cn(ctx->d_beta, ctx->n_pw, ctx->d_psi, ctx->n_pw, np, n, ctx->n_pw, ctx->d_part,
                ctx->d_cp, st);
        count_launch();
        k_conj<<<grid_for((size_t)np * n), 256, 0, st>>>(ctx->d_cp, ctx->d_cq, (size_t)np * n);
    }
    // psi^H H psi and psi^H psi are Hermitian: upper tiles only
    gemm_cn_herm(ctx->d_psi, ctx->n_pw, ctx->d_hpsi, ctx->n_pw, n, ctx->n_pw, ctx->d_part, ctx->d_T1, st);
    if (nl_sub) {
        // H_sub += C^H D C
        count_launch();
        k_apply_dmat<<<grid_for((size_t)np * n), 256, 0, st>>>(
            ctx->d_cp, ctx->d_cd, np, n, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff, ctx->d_dmat);
        gemm_tn(ctx->d_cq, n, ctx->d_cd, n, ctx->d_T1, n, n, n, np, 1.0, 1.0, st);
    }
    symmetrize(ctx->d_T1, ctx->d_H, n, st);
    gemm_cn_herm(ctx->d_psi, ctx->n_pw, ctx->d_psi, ctx->n_pw, n, ctx->n_pw, ctx->d_part, ctx->d_T1, st);
    if (aug_s) {
        // S_sub = psi^H psi + C^H q C
        count_launch();
        k_apply_dmat<<<grid_for((size_t)np * n), 256, 0, st>>>(
            ctx->d_cp, ctx->d_cd, np, n, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff, ctx->d_qmat);
        gemm_tn(ctx->d_cq, n, ctx->d_cd, n, ctx->d_T1, n, n, n, np, 1.0, 1.0, st);
    }
    symmetrize(ctx->d_T1, ctx->d_S, n, st);
    cholesky(ctx->d_S, n, ctx->d_flags + 0, st);                   // S -> L
    tri_inv(ctx->d_S, ctx->d_T1, n, st);                            // T1 = L^-1
    small_gemm(0, 0, ctx->d_T1, ctx->d_H, ctx->d_T2, n, st);        // T2 = Li H
    small_gemm(0, 1, ctx->d_T2, ctx->d_T1, ctx->d_H, n, st);        // H = Li H Li^H
    symmetrize(ctx->d_H, ctx->d_T2, n, st);                         // T2 = B
    CK(jacobi(ctx->d_T2, ctx->d_V, n, ctx->jac_max_sweeps, 1e-26, ctx->d_jac, ctx->d_flags + 2, st));
    sort_eig(ctx->d_T2, ctx->d_V, n, ctx->d_eig, ctx->d_H, st);     // H = U (sorted)
    small_gemm(1, 0, ctx->d_T1, ctx->d_H, ctx->d_T2, n, st);        // T2 = Li^H U
    gemm_tn(ctx->d_T2, n, ctx->d_psi, ctx->n_pw, ctx->d_psi2, ctx->n_pw, n, ctx->n_pw, n, 1.0, 0.0, st);
    if (fp32_block) {
        // copy back instead of swapping the pointers: a mixed pass captured
        // into a CUDA graph (chfsi_batch_capture) replays on fixed buffers
        CK(cudaMemcpyAsync(ctx->d_psi, ctx->d_psi2, sizeof(double2) * (size_t)n * ctx->n_pw,
                           cudaMemcpyDeviceToDevice, st));
    } else {
        std::swap(ctx->d_psi, ctx->d_psi2);
    }
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// ---------------------------------------------------------------- mixed precision
// FP32 filter with the projector GEMMs on tcgen05 (BF16 3-way split, FP32
// accumulation in TMEM); the Rayleigh-Ritz of the filtered block runs in
// FP64 (rr_dev with the non-local part as C^H D C).  Long-K sums accumulated
// in the tensor core's FP32 accumulator drift low (the diagonal of psi^H psi
// over n_pw terms loses ~1e-4 relative at n_pw ~ 1.7e5), which in an FP32
// overlap shows up as a charge excess of ~0.1 electron and a total-energy
// bias of ~1e-4 Ha/atom; the filter itself tolerates such errors.

chfsi_status alloc_mixed(chfsi_ctx* ctx, int ncol) {
    const int nb = ctx->nb, np = ctx->np, npw = ctx->n_pw;
    const size_t nbpw = (size_t)nb * npw;
    CK(dalloc(&ctx->d_psi32a, nbpw));
    CK(dalloc(&ctx->d_psi32b, nbpw));
    CK(dalloc(&ctx->d_hpsi32, nbpw));
    if (np > 0) CK(dalloc(&ctx->d_nl32, nbpw));
    CK(dalloc(&ctx->d_work32, (size_t)nb * ctx->nz * ncol));
    struct Spec { TcPlanes* t; int rows_alloc; int kp; };
    const int kp_pw = tc_kpad(npw);
    std::vector<Spec> specs = {
        {&ctx->tp_psi_b, tc_rows_alloc(nb, false, nb), kp_pw},
        {&ctx->tp_small_a, tc_rows_alloc(2 * nb, true, 0), std::max(tc_kpad(std::max(np, 1)), tc_kpad(nb))},
    };
    if (np > 0) {
        specs.push_back({&ctx->tp_beta_a, tc_rows_alloc(2 * np, true, 0), kp_pw});
        specs.push_back({&ctx->tp_betaT_b, tc_rows_alloc(npw, false, npw), tc_kpad(np)});
    }
    size_t total = 0;
    for (auto& s : specs) total += 3 * (size_t)s.rows_alloc * s.kp;
    CK(cudaMalloc(&ctx->d_planes, total * 2));
    CK(cudaMemsetAsync(ctx->d_planes, 0, total * 2, ctx->st));
    char* p = (char*)ctx->d_planes;
    for (auto& s : specs) {
        for (int i = 0; i < 3; ++i) {
            s.t->p[i] = p;
            p += (size_t)s.rows_alloc * s.kp * 2;
        }
        s.t->rows_alloc = s.rows_alloc;
        s.t->kp = s.kp;
    }
    // the projector GEMM may see any band count 1..nb (chfsi_apply_h), and
    // the K-split count depends on it: size for the largest
    size_t pf = 1;
    for (int b = 1; b <= nb && np > 0; ++b) pf = std::max(pf, tc_partial_floats(np, b, npw));
    CK(dalloc(&ctx->d_tc_part, pf));
    CK(dalloc(&ctx->d_tc_err, 4));
    CK(cudaMemsetAsync(ctx->d_tc_err, 0, 4 * sizeof(int), ctx->st));
    return CHFSI_OK;
}

static_assert(CHFSI_TC_SHAPES == kTcVariantCount, "tcgen05 shape count");

// The context's launch shape of the projection (which 0) or the expansion
// (which 1) tcgen05 GEMM; shape 0 until the autotuner has run.
int tc_shape(const chfsi_ctx* ctx, int which) {
    return ctx->tc_shape[which] < 0 ? 0 : ctx->tc_shape[which];
}

// Autotuner of the projector GEMMs: every launch shape of the tcgen05 kernel
// on this context's projection (n_proj x n_b x n_pw) and expansion
// (n_b x n_pw x n_proj), one warm-up and two timed launches each (CUDA events
// on the context stream); the fastest is kept.  The operands are the packed
// projector planes and whatever the band planes hold (the timing does not
// depend on values); the outputs land in scratch the filter overwrites.
// Skipped while the stream is being captured (shape 0 then).
// Choices are kept per device and size class (which GEMM, M, N, K), so every
// context of one size uses the same shape and gives the same numbers.
std::mutex g_tc_shape_mu;
std::map<std::array<int, 5>, int> g_tc_shape_cache;

chfsi_status tune_tc_shapes(chfsi_ctx* ctx) {
    if (ctx->tc_shape[0] >= 0 && ctx->tc_shape[1] >= 0) return CHFSI_OK;
    const int np = ctx->np, nb = ctx->nb, npw = ctx->n_pw;
    const std::array<int, 5> key[2] = {{ctx->device, 0, np, nb, npw}, {ctx->device, 1, nb, npw, np}};
    {
        std::lock_guard<std::mutex> lk(g_tc_shape_mu);
        for (int which = 0; which < 2; ++which) {
            auto it = g_tc_shape_cache.find(key[which]);
            if (ctx->tc_shape[which] < 0 && it != g_tc_shape_cache.end())
                ctx->tc_shape[which] = it->second;
        }
    }
    if (ctx->tc_shape[0] >= 0 && ctx->tc_shape[1] >= 0) return CHFSI_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CK(cudaStreamIsCapturing(ctx->st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return CHFSI_OK;
    cudaStream_t st = ctx->st;
    // band-side operands as the filter packs them (their planes may not have
    // been packed yet: zero-filled planes of the right shape time the same)
    TcPlanes psi_b = ctx->tp_psi_b, small_a = ctx->tp_small_a;
    psi_b.rows = nb;
    psi_b.kp = tc_kpad(npw);
    small_a.rows = 2 * nb;
    small_a.kp = tc_kpad(np);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    cudaError_t e = cudaSuccess;
    int tuned[2] = {ctx->tc_shape[0], ctx->tc_shape[1]};
    for (int which = 0; which < 2 && e == cudaSuccess; ++which) {
        if (tuned[which] >= 0) continue;
        float best = 1e30f;
        int best_v = 0;
        for (int v = 0; v < kTcVariantCount && e == cudaSuccess; ++v) {
            auto run = [&]() {
                return which == 0
                           ? tc_gemm(ctx->tp_beta_a, psi_b, np, nb, npw, kTcOutPartial,
                                     ctx->d_cp, nb, ctx->d_tc_part, ctx->d_tc_err, st, v)
                           : tc_gemm(small_a, ctx->tp_betaT_b, nb, npw, np,
                                     kTcOutComplexF32, ctx->d_nl32, npw, nullptr, ctx->d_tc_err,
                                     st, v);
            };
            e = run();
            if (e == cudaSuccess) e = cudaEventRecord(e0, st);
            for (int r = 0; r < 2 && e == cudaSuccess; ++r) e = run();
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && ms < best) { best = ms; best_v = v; }
        }
        tuned[which] = best_v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CK(e);
    int herr = 0;
    CK(copy_sync(&herr, ctx->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (herr) {
        // a timed-out launch makes the timings meaningless: tune again later
        CK(cudaMemsetAsync(ctx->d_tc_err, 0, 4 * sizeof(int), st));
        return ctx->fail(CHFSI_ERR_TIMEOUT, "tensor-core GEMM pipeline wait timed out");
    }
    std::lock_guard<std::mutex> lk(g_tc_shape_mu);
    for (int which = 0; which < 2; ++which) {
        ctx->tc_shape[which] = tuned[which];
        g_tc_shape_cache.emplace(key[which], tuned[which]);
    }
    return CHFSI_OK;
}

chfsi_status pack_beta_planes(chfsi_ctx* ctx) {
    if (!ctx->mixed || ctx->np == 0) return CHFSI_OK;
    // beta^H psi: A operand = beta rows (doubled); back-projection: B operand = beta^T
    tc_pack<double2>(ctx->d_beta, ctx->n_pw, ctx->np, ctx->n_pw, true, kSrcPlain, ctx->tp_beta_a, ctx->st);
    tc_pack<double2>(ctx->d_beta, ctx->n_pw, ctx->n_pw, ctx->np, false, kSrcT, ctx->tp_betaT_b, ctx->st);
    CK(cudaGetLastError());
    ctx->beta_planes_ready = true;
    return tune_tc_shapes(ctx);
}

chfsi_status apply_h_dev32(chfsi_ctx* ctx, const float2* psi, float2* out, int nb, int mode,
                           double* norm_acc, bool local_only = false,
                           const ResidStep* rs = nullptr) {
    Epilogue e{};
    e.mode = mode;
    if (rs) { e.rc = rs->rc; e.lam = rs->lam; e.yres = rs->y; }
    e.kin = ctx->d_kin;
    e.coef = ctx->d_coef;
    e.nl = nullptr;
    e.norm_acc = norm_acc;
    e.inv_n = 1.0 / (double)ctx->ng;
    cudaStream_t st = ctx->st;
    if (ctx->np > 0 && !local_only) {
        // C = beta^H psi (tcgen05), C <- D C (FP64), nl = beta C (tcgen05, FP32 out)
        tc_pack<float2>(psi, ctx->n_pw, nb, ctx->n_pw, false, kSrcPlain, ctx->tp_psi_b, st);
        CK(tc_gemm(ctx->tp_beta_a, ctx->tp_psi_b, ctx->np, nb, ctx->n_pw, kTcOutPartial, ctx->d_cp,
                   nb, ctx->d_tc_part, ctx->d_tc_err, st, tc_shape(ctx, 0)));
        count_launch();
        k_apply_dmat<<<grid_for((size_t)ctx->np * nb), 256, 0, st>>>(
            ctx->d_cp, ctx->d_cd, ctx->np, nb, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff, ctx->d_dmat);
        tc_pack<double2>(ctx->d_cd, nb, nb, ctx->np, true, kSrcConjT, ctx->tp_small_a, st);
        CK(tc_gemm(ctx->tp_small_a, ctx->tp_betaT_b, nb, ctx->n_pw, ctx->np, kTcOutComplexF32,
                   ctx->d_nl32, ctx->n_pw, nullptr, ctx->d_tc_err, st, tc_shape(ctx, 1)));
        e.nl = ctx->d_nl32;
    }
    launch_zsticks_inverse<float2>(psi, ctx->n_pw, ctx->d_work32, nb, ctx->geo, st);
    launch_planes_vloc<float2>(ctx->d_work32, ctx->d_veff, nb, ctx->geo, st);
    launch_zsticks_forward<float2>(ctx->d_work32, psi, ctx->n_pw, out, ctx->n_pw, nb, ctx->geo, e, st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// S^-1 H x for the FP32 filter of the generalised problem as
// d_hpsi32 - d_nl32, in the form of sinv_h_parts: C = beta^H x and
// E = beta^H (H_loc x) on tcgen05, F = M (E + B G) - G in FP64, beta F on
// tcgen05 (FP32 out).
chfsi_status sinv_h_parts32(chfsi_ctx* ctx, const float2* x, int nb) {
    cudaStream_t st = ctx->st;
    const int np = ctx->np, npw = ctx->n_pw;
    tc_pack<float2>(x, npw, nb, npw, false, kSrcPlain, ctx->tp_psi_b, st);
    CK(tc_gemm(ctx->tp_beta_a, ctx->tp_psi_b, np, nb, npw, kTcOutPartial, ctx->d_cp, nb,
               ctx->d_tc_part, ctx->d_tc_err, st, tc_shape(ctx, 0)));
    count_launch();
    k_apply_dmat<<<grid_for((size_t)np * nb), 256, 0, st>>>(
        ctx->d_cp, ctx->d_cd, np, nb, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff, ctx->d_dmat);
    chfsi_status s = apply_h_dev32(ctx, x, ctx->d_hpsi32, nb, kEpiApply, nullptr, true);
    if (s) return s;
    tc_pack<float2>(ctx->d_hpsi32, npw, nb, npw, false, kSrcPlain, ctx->tp_psi_b, st);
    CK(tc_gemm(ctx->tp_beta_a, ctx->tp_psi_b, np, nb, npw, kTcOutPartial, ctx->d_cp, nb,
               ctx->d_tc_part, ctx->d_tc_err, st, tc_shape(ctx, 0)));
    gemm_tn(ctx->d_bmatT, np, ctx->d_cd, nb, ctx->d_cp, nb, np, nb, np, 1.0, 1.0, st);
    CK(cudaMemcpyAsync(ctx->d_cq, ctx->d_cd, sizeof(double2) * (size_t)np * nb,
                       cudaMemcpyDeviceToDevice, st));
    gemm_tn(ctx->d_sinvT, np, ctx->d_cp, nb, ctx->d_cq, nb, np, nb, np, 1.0, -1.0, st);
    tc_pack<double2>(ctx->d_cq, nb, nb, np, true, kSrcConjT, ctx->tp_small_a, st);
    CK(tc_gemm(ctx->tp_small_a, ctx->tp_betaT_b, nb, npw, np, kTcOutComplexF32, ctx->d_nl32, npw,
               nullptr, ctx->d_tc_err, st, tc_shape(ctx, 1)));
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// S^-1 H x for the FP32 filter of the generalised problem (sinv_h_parts32),
// then the recurrence epilogue in k_cheb_combine<float2>.
chfsi_status apply_op_dev32(chfsi_ctx* ctx, const float2* x, float2* out, int nb, int mode,
                            double* norm_acc) {
    if (!ctx->uspp || mode == kEpiApply) return apply_h_dev32(ctx, x, out, nb, mode, norm_acc);
    chfsi_status s = sinv_h_parts32(ctx, x, nb);
    if (s) return s;
    cudaStream_t st = ctx->st;
    const size_t n = (size_t)nb * ctx->n_pw;
    count_launch();
    k_cheb_combine<float2><<<grid_for(n), 256, 0, st>>>(ctx->d_hpsi32, ctx->d_nl32, x, out, n,
                                                         ctx->d_coef, mode == kEpiChebFirst ? 1 : 2,
                                                         norm_acc);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

chfsi_status filter_dev32(chfsi_ctx* ctx, int ndeg, const double* eig_dev, int n_eig) {
    if (ndeg < 0 || ndeg > ctx->max_deg) return ctx->fail(CHFSI_ERR_BAD_INPUT, "ndeg out of range");
    if (ctx->np > 0) {
        chfsi_status s = ctx->beta_planes_ready ? CHFSI_OK : pack_beta_planes(ctx);
        if (!s) s = tune_tc_shapes(ctx);
        if (s) return s;
    }
    chfsi_status s = compute_bounds(ctx, eig_dev, n_eig);
    if (s) return s;
    const size_t n = (size_t)ctx->nb * ctx->n_pw;
    cudaStream_t st = ctx->st;
    count_launch();
    k_f64_to_f32<<<grid_for(n), 256, 0, st>>>(ctx->d_psi, ctx->d_psi32a, n);
    CK(cudaMemsetAsync(ctx->d_nsq, 0, sizeof(double) * (ndeg + 1), st));
    count_launch();
    k_sumsq32<<<grid_for(n), 256, 0, st>>>(ctx->d_psi32a, n, ctx->d_nsq);
    float2* A = ctx->d_psi32a;
    float2* B = ctx->d_psi32b;
    if (ndeg >= 1) {
        s = apply_op_dev32(ctx, A, B, ctx->nb, kEpiChebFirst, ctx->d_nsq + 1);
        if (s) return s;
    }
    for (int k = 2; k <= ndeg; ++k) {
        s = apply_op_dev32(ctx, B, A, ctx->nb, kEpiCheb, ctx->d_nsq + k);
        if (s) return s;
        std::swap(A, B);
    }
    float2* fin = ndeg >= 1 ? B : A;
    ctx->d_psi32 = fin;
    // local H of the filtered block for the FP64 Rayleigh-Ritz (the non-local
    // part enters its subspace matrix as C^H D C)
    s = apply_h_dev32(ctx, fin, ctx->d_hpsi32, ctx->nb, kEpiApply, nullptr, true);
    if (s) return s;
    count_launch();
    k_f32_to_f64<<<grid_for(n), 256, 0, st>>>(fin, ctx->d_psi, n);
    count_launch();
    k_f32_to_f64<<<grid_for(n), 256, 0, st>>>(ctx->d_hpsi32, ctx->d_hpsi, n);
    norm_guard(ctx->d_nsq, ndeg, ctx->d_flags + 1, st);
    ctx->last_ndeg = ndeg;
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// ---------------------------------------------------------------- R-ChFSI
// Residual-based Chebyshev filter (reference_paper/2025 main.tex Algorithm 3)
// of the current Ritz pairs (X = d_psi, S-orthonormal; Lam = eig_dev), with
// the exact Woodbury S^-1 as the approximate inverse, in the form with the
// operator S^-1 H on unweighted residuals:
//   Y = S^-1 (H X - S X Lam)                                   (FP64)
//   R_1 = (s_1/e) Y, R_0 = 0
//   R_k = a_k S^-1 H R_{k-1} + b_k R_{k-1} + c_k R_{k-2} + a_k Y L_{k-1}
//   X_p = R_p + X L_p,  H X_p = H R_p + (H X) L_p              (FP64 out)
// The recurrence runs in FP32 (tcgen05 projector products) when fp32: its
// rounding enters through R, whose size falls with the residual of the Ritz
// pairs, so the filtered block keeps FP64 accuracy as the SCF converges
// (the plain FP32 filter stalls at its rounding level).  The Rayleigh-Ritz
// that follows gets the full H X_p in FP64.
chfsi_status alloc_rchfsi(chfsi_ctx* ctx, bool fp32) {
    const size_t n = (size_t)ctx->nb * ctx->n_pw;
    if (!ctx->d_rc_hx) CK(dalloc(&ctx->d_rc_hx, n));
    if (!ctx->d_rc_y) CK(dalloc(&ctx->d_rc_y, n));
    if (!ctx->d_rc_coef) CK(dalloc(&ctx->d_rc_coef, (size_t)3 * (ctx->max_deg + 1)));
    if (!ctx->d_rc_lam) CK(dalloc(&ctx->d_rc_lam, (size_t)(ctx->max_deg + 1) * ctx->nb));
    if (fp32) {
        if (!ctx->d_rc_y32) CK(dalloc(&ctx->d_rc_y32, n));
    } else {
        if (!ctx->d_rc_r0) CK(dalloc(&ctx->d_rc_r0, n));
        if (!ctx->d_rc_r1) CK(dalloc(&ctx->d_rc_r1, n));
    }
    return CHFSI_OK;
}

// out = a op(x) + b x + c out + a L y  (op = H, or S^-1 H when ultrasoft)
chfsi_status rc_step64(chfsi_ctx* ctx, const double2* x, double2* out, const ResidStep& rs) {
    const int nb = ctx->nb;
    if (!ctx->uspp) return apply_h_dev(ctx, x, out, nb, kEpiResid, nullptr, -1, nullptr, &rs);
    chfsi_status s = sinv_h_parts(ctx, x, nb, nb);
    if (s) return s;
    cudaStream_t st = ctx->st;
    const size_t n = (size_t)nb * ctx->n_pw;
    count_launch();
    k_cheb_combine<double2><<<grid_for(n), 256, 0, st>>>(
        ctx->d_hpsi, ctx->d_sx, x, out, n, ctx->d_coef, 3, nullptr,
        reinterpret_cast<const double2*>(rs.y), rs.lam, rs.rc, ctx->n_pw);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

chfsi_status rc_step32(chfsi_ctx* ctx, const float2* x, float2* out, const ResidStep& rs) {
    const int nb = ctx->nb;
    if (!ctx->uspp) return apply_h_dev32(ctx, x, out, nb, kEpiResid, nullptr, false, &rs);
    chfsi_status s = sinv_h_parts32(ctx, x, nb);
    if (s) return s;
    cudaStream_t st = ctx->st;
    const size_t n = (size_t)nb * ctx->n_pw;
    count_launch();
    k_cheb_combine<float2><<<grid_for(n), 256, 0, st>>>(
        ctx->d_hpsi32, ctx->d_nl32, x, out, n, ctx->d_coef, 3, nullptr,
        reinterpret_cast<const float2*>(rs.y), rs.lam, rs.rc, ctx->n_pw);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

chfsi_status filter_rchfsi(chfsi_ctx* ctx, int ndeg, const double* eig_dev, int n_eig, bool fp32) {
    const int nb = ctx->nb, npw = ctx->n_pw, np = ctx->np;
    if (!eig_dev || n_eig != nb || ndeg < 1 || ndeg > ctx->max_deg)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "R-ChFSI needs the Ritz values of every band");
    chfsi_status s = alloc_rchfsi(ctx, fp32);
    if (s) return s;
    if (fp32 && np > 0 && !ctx->beta_planes_ready && (s = pack_beta_planes(ctx))) return s;
    if (fp32 && np > 0 && (s = tune_tc_shapes(ctx))) return s;
    if ((s = compute_bounds(ctx, eig_dev, n_eig))) return s;
    cudaStream_t st = ctx->st;
    const size_t n = (size_t)nb * npw;
    CK(cudaMemsetAsync(ctx->d_flags + 1, 0, sizeof(int), st));
    CK(cudaMemsetAsync(ctx->d_nsq, 0, sizeof(double) * (ndeg + 1), st));
    count_launch();
    k_rc_tables<<<1, 256, 0, st>>>(ctx->d_coef, eig_dev, nb, ndeg, ctx->d_rc_coef, ctx->d_rc_lam);
    // residual of the Ritz pairs, FP64
    if ((s = apply_h_dev(ctx, ctx->d_psi, ctx->d_rc_hx, nb, kEpiApply, nullptr))) return s;
    if (ctx->uspp) {
        // S X - X = beta q beta^H X, then Y = S^-1 (H X - S X Lam)
        gemm_cn(ctx->d_beta, npw, ctx->d_psi, npw, np, nb, npw, ctx->d_part, ctx->d_cp, st);
        count_launch();
        k_apply_dmat<<<grid_for((size_t)np * nb), 256, 0, st>>>(
            ctx->d_cp, ctx->d_cd, np, nb, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff, ctx->d_qmat);
        gemm_tn(ctx->d_cd, nb, ctx->d_beta, npw, ctx->d_sx, npw, nb, npw, np, 1.0, 0.0, st);
        count_launch();
        k_rc_resid<<<grid_for(n), 256, 0, st>>>(ctx->d_rc_hx, ctx->d_psi, ctx->d_sx, eig_dev, npw, n,
                                                ctx->d_rc_y);
        gemm_cn(ctx->d_beta, npw, ctx->d_rc_y, npw, np, nb, npw, ctx->d_part, ctx->d_cp, st);
        gemm_tn(ctx->d_sinvT, np, ctx->d_cp, nb, ctx->d_cq, nb, np, nb, np, 1.0, 0.0, st);
        gemm_tn(ctx->d_cq, nb, ctx->d_beta, npw, ctx->d_sx, npw, nb, npw, np, 1.0, 0.0, st);
        count_launch();
        k_cheb_combine<double2><<<grid_for(n), 256, 0, st>>>(ctx->d_rc_y, ctx->d_sx, ctx->d_rc_y,
                                                             ctx->d_rc_y, n, ctx->d_coef, 0, nullptr);
    } else {
        count_launch();
        k_rc_resid<<<grid_for(n), 256, 0, st>>>(ctx->d_rc_hx, ctx->d_psi, nullptr, eig_dev, npw, n,
                                                ctx->d_rc_y);
    }
    const double* lam = ctx->d_rc_lam;
    if (fp32) {
        float2* A = ctx->d_psi32a;  // R_{k-2}
        float2* B = ctx->d_psi32b;  // R_{k-1}
        count_launch();
        k_rc_scale<float2><<<grid_for(n), 256, 0, st>>>(ctx->d_rc_y, ctx->d_rc_coef, n, B, ctx->d_rc_y32);
        CK(cudaMemsetAsync(A, 0, n * sizeof(float2), st));
        for (int k = 2; k <= ndeg; ++k) {
            const ResidStep rs{ctx->d_rc_coef + 3 * k, lam + (size_t)(k - 1) * nb, ctx->d_rc_y32};
            if ((s = rc_step32(ctx, B, A, rs))) return s;
            std::swap(A, B);
        }
        if ((s = apply_h_dev32(ctx, B, ctx->d_hpsi32, nb, kEpiApply, nullptr))) return s;
        count_launch();
        k_rc_final<float2><<<grid_for(n), 256, 0, st>>>(B, ctx->d_hpsi32, ctx->d_psi, ctx->d_rc_hx,
                                                        lam + (size_t)ndeg * nb, npw, n,
                                                        ctx->d_psi2, ctx->d_hpsi);
    } else {
        double2* A = ctx->d_rc_r0;
        double2* B = ctx->d_rc_r1;
        count_launch();
        k_rc_scale<double2><<<grid_for(n), 256, 0, st>>>(ctx->d_rc_y, ctx->d_rc_coef, n, B, nullptr);
        CK(cudaMemsetAsync(A, 0, n * sizeof(double2), st));
        for (int k = 2; k <= ndeg; ++k) {
            const ResidStep rs{ctx->d_rc_coef + 3 * k, lam + (size_t)(k - 1) * nb, ctx->d_rc_y};
            if ((s = rc_step64(ctx, B, A, rs))) return s;
            std::swap(A, B);
        }
        if ((s = apply_h_dev(ctx, B, A, nb, kEpiApply, nullptr))) return s;
        count_launch();
        k_rc_final<double2><<<grid_for(n), 256, 0, st>>>(B, A, ctx->d_psi, ctx->d_rc_hx,
                                                         lam + (size_t)ndeg * nb, npw, n,
                                                         ctx->d_psi2, ctx->d_hpsi);
    }
    // copy back (fixed buffers, as a captured mixed pass needs)
    CK(cudaMemcpyAsync(ctx->d_psi, ctx->d_psi2, n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    ctx->last_ndeg = ndeg;
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// A pass without previous eigenvalues (the random start) filters with the
// cut at lambda_max / 3, where the deepest states grow by ~1e9 over degree
// 16 relative to the cut: FP32 rounding of the weakly amplified top bands
// would swamp them, so such passes always run in FP64.
// The residual form runs the FP32 passes of a mixed-precision context (where
// it keeps the filtered block's error proportional to the Ritz residuals) and
// every pass of an FP64 context; the FP64 passes of a mixed context (the
// passes that confirm convergence) run the reference's Chebyshev filter.
chfsi_status filter_any(chfsi_ctx* ctx, int ndeg, const double* eig_dev, int n_eig) {
    ctx->last_pass_fp32 = ctx->mixed_active && eig_dev != nullptr && n_eig > 0;
    if (ctx->cfg.filter_form == CHFSI_FILTER_RESIDUAL && (ctx->last_pass_fp32 || !ctx->mixed) &&
        eig_dev && n_eig == ctx->nb && ndeg >= 1) {
        ctx->d_psi32 = nullptr;  // the Rayleigh-Ritz gets the full H psi in FP64
        return filter_rchfsi(ctx, ndeg, eig_dev, n_eig, ctx->last_pass_fp32);
    }
    if (ctx->last_pass_fp32) return filter_dev32(ctx, ndeg, eig_dev, n_eig);
    ctx->d_psi32 = nullptr;
    return filter_dev(ctx, ndeg, eig_dev, n_eig);
}

chfsi_status rr_any(chfsi_ctx* ctx) {
    const bool fp32_block = ctx->mixed_active && ctx->d_psi32;
    ctx->d_psi32 = nullptr;
    return rr_dev(ctx, fp32_block);
}

// Read back eigenvalues, flags, bounds and norms; translate device flags into
// the reference's error variants.
chfsi_status finish_diag(chfsi_ctx* ctx, double* eig_out, bool have_rr) {
    const int n = ctx->nb;
    chfsi_status s = ensure_pinned(ctx, (size_t)n + 16 + ctx->max_deg + 1);
    if (s) return s;
    double* h = ctx->h_pin;
    CK(cudaMemcpyAsync(h, ctx->d_eig, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(h + n, ctx->d_coef, sizeof(double) * 6, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(h + n + 6, ctx->d_flags, sizeof(int) * 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(h + n + 8, ctx->d_nsq, sizeof(double) * (ctx->last_ndeg + 1),
                       cudaMemcpyDeviceToHost, ctx->st));
    int tc_err = 0;
    if (ctx->d_tc_err)
        CK(cudaMemcpyAsync(&tc_err, ctx->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (tc_err) {
        CK(cudaMemsetAsync(ctx->d_tc_err, 0, sizeof(int), ctx->st));
        return ctx->fail(CHFSI_ERR_TIMEOUT, "tensor-core GEMM pipeline wait timed out");
    }
    std::memcpy(ctx->h_coef, h + n, sizeof(double) * 6);
    int flags[4];
    std::memcpy(flags, h + n + 6, sizeof(flags));
    ctx->h_nsq.assign(h + n + 8, h + n + 8 + ctx->last_ndeg + 1);
    if (flags[1] != 0) {
        char buf[256];
        int k = flags[1];
        double np_ = std::sqrt(ctx->h_nsq[k - 1]), nc = std::sqrt(ctx->h_nsq[k]);
        std::snprintf(buf, sizeof(buf),
                      "Chebyshev filtering diverged: norm grew %.2ex at iteration %d", nc / np_, k);
        return ctx->fail(CHFSI_ERR_CHEB_DIVERGED, buf);
    }
    if (have_rr) {
        if (flags[0] != 0) {
            char buf[128];
            std::snprintf(buf, sizeof(buf), "Rayleigh-Ritz failed: info=%d (overlap not positive definite)", flags[0]);
            return ctx->fail(CHFSI_ERR_RR_FAILED, buf);
        }
        ctx->last_sweeps = flags[2];
        if (flags[2] >= ctx->jac_max_sweeps) {
            return ctx->fail(CHFSI_ERR_RR_FAILED, "Rayleigh-Ritz failed: eigensolver did not converge");
        }
        for (int i = 0; i < n; ++i)
            if (!std::isfinite(h[i])) return ctx->fail(CHFSI_ERR_NUMERIC, "non-finite eigenvalue");
        // after an FP32 filter, a top Ritz value well inside the damped
        // interval [cut, lambda_max] means rounding swamped the top of the
        // subspace (reported so that the pass can be redone in FP64)
        if (ctx->last_pass_fp32 &&
            h[n - 1] > ctx->h_coef[1] + 0.1 * (ctx->h_coef[0] - ctx->h_coef[1]))
            return ctx->fail(CHFSI_ERR_RR_FAILED, "Rayleigh-Ritz failed: Ritz value inside the damped interval");
        if (eig_out) std::memcpy(eig_out, h, sizeof(double) * n);
    }
    return CHFSI_OK;
}

// ---------------------------------------------------------------- potentials
// 3D FFT on the density grid (unnormalised; digit-reversed G layout)
void grid_fft3(chfsi_ctx* ctx, double2* g, bool forward) {
    launch_axis_fft<double2>(g, ctx->fnx, ctx->fny, ctx->fnz, 0, forward, ctx->fax, ctx->st);
    launch_axis_fft<double2>(g, ctx->fnx, ctx->fny, ctx->fnz, 1, forward, ctx->fay, ctx->st);
    launch_axis_fft<double2>(g, ctx->fnx, ctx->fny, ctx->fnz, 2, forward, ctx->faz, ctx->st);
}

// 3D FFT on the wavefunction grid
void wave_fft3(chfsi_ctx* ctx, double2* g, bool forward) {
    launch_axis_fft<double2>(g, ctx->nx, ctx->ny, ctx->nz, 0, forward, ctx->ax, ctx->st);
    launch_axis_fft<double2>(g, ctx->nx, ctx->ny, ctx->nz, 1, forward, ctx->ay, ctx->st);
    launch_axis_fft<double2>(g, ctx->nx, ctx->ny, ctx->nz, 2, forward, ctx->az, ctx->st);
}

GridRecip grid_recip(chfsi_ctx* ctx) {
    GridRecip gr{};
    gr.nx = ctx->fnx; gr.ny = ctx->fny; gr.nz = ctx->fnz;
    gr.idr_x = ctx->d_fidr[0]; gr.idr_y = ctx->d_fidr[1]; gr.idr_z = ctx->d_fidr[2];
    std::memcpy(gr.b, ctx->recip, sizeof(gr.b));
    return gr;
}

// V_eff of the density grid -> the wavefunction grid (G truncation) + min/max
void project_veff(chfsi_ctx* ctx) {
    cudaStream_t st = ctx->st;
    if (!ctx->fine) {
        cudaMemcpyAsync(ctx->d_veff, ctx->d_veff_d, sizeof(double) * ctx->ng,
                        cudaMemcpyDeviceToDevice, st);
    } else {
        launch_real_to_complex(ctx->d_veff_d, ctx->d_cgrid, ctx->fng, st);
        grid_fft3(ctx, ctx->d_cgrid, true);
        cudaMemsetAsync(ctx->d_wgrid, 0, sizeof(double2) * ctx->ng, st);
        launch_scatter_g(ctx->d_cgrid, ctx->d_gmap_f, ctx->d_gmap_w, ctx->n_gmap,
                         1.0 / (double)ctx->fng, ctx->d_wgrid, st);
        wave_fft3(ctx, ctx->d_wgrid, false);
        launch_take_real(ctx->d_wgrid, ctx->d_veff, ctx->ng, st);
    }
    minmax(ctx->d_veff, ctx->ng, ctx->d_minmax, st);
}

// Screened D = D0 + q v_I from the density-grid V_eff (ultrasoft only).
chfsi_status screen_dmat(chfsi_ctx* ctx) {
    if (!ctx->aug) return CHFSI_OK;
    cudaStream_t st = ctx->st;
    launch_real_to_complex(ctx->d_veff_d, ctx->d_cgrid, ctx->fng, st);
    grid_fft3(ctx, ctx->d_cgrid, true);
    CK(cudaMemsetAsync(ctx->d_vion, 0, sizeof(double) * ctx->nions, st));
    launch_ion_potential(ctx->d_cgrid, grid_recip(ctx), ctx->d_phase, ctx->nions, ctx->aug_width,
                         1.0 / (double)ctx->fng, ctx->d_vion, st);
    launch_screen_d(ctx->d_dmat0, ctx->d_qmat, ctx->d_vion, ctx->d_poff, ctx->d_doff, ctx->nions,
                    ctx->d_dmat, st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// veff = vloc + V_H[rho] + V_xc[rho]; acc[0] += E_H[rho], acc[1] += E_xc[rho]
// grad rho of the density whose forward FFT is in d_cgrid: real parts of the
// three d_gga grids (PBE)
void gga_gradient(chfsi_ctx* ctx) {
    const size_t ng = ctx->fng;
    double2* g0 = ctx->d_gga;
    launch_grad_gspace(ctx->d_cgrid, grid_recip(ctx), g0, g0 + ng, g0 + 2 * ng, ctx->st);
    for (int a = 0; a < 3; ++a) grid_fft3(ctx, g0 + a * ng, false);
}

chfsi_status build_veff_dev(chfsi_ctx* ctx, const double* rho, double* acc) {
    const size_t ng = ctx->fng;
    const double dv = ctx->omega / (double)ng;
    launch_real_to_complex(rho, ctx->d_cgrid, ng, ctx->st);
    grid_fft3(ctx, ctx->d_cgrid, true);
    const bool gga = ctx->xc == CHFSI_XC_PBE;
    if (gga) gga_gradient(ctx);
    launch_hartree_gspace(ctx->d_cgrid, grid_recip(ctx), ctx->omega, acc + 0, ctx->st);
    grid_fft3(ctx, ctx->d_cgrid, false);
    if (!gga) {
        launch_assemble_veff(ctx->d_vloc, ctx->d_cgrid, rho, ctx->d_veff_d, ng, dv, acc + 1, ctx->st);
    } else {
        // V_xc = de/drho - div(2 de/dsigma grad rho)
        double2* g0 = ctx->d_gga;
        launch_pbe_point(rho, g0, g0 + ng, g0 + 2 * ng, ctx->d_gga_v1, ng, dv, acc + 1, true, ctx->st);
        for (int a = 0; a < 3; ++a) grid_fft3(ctx, g0 + a * ng, true);
        launch_div_gspace(g0, g0 + ng, g0 + 2 * ng, grid_recip(ctx), g0, ctx->st);
        grid_fft3(ctx, g0, false);
        launch_assemble_gga(ctx->d_vloc, ctx->d_cgrid, ctx->d_gga_v1, g0, ctx->d_veff_d, ng, ctx->st);
    }
    project_veff(ctx);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// rho (density grid) = sum_n f_n |psi_n|^2 (+ augmentation)
chfsi_status density_dev(chfsi_ctx* ctx, double* rho) {
    int nocc = 0;
    for (int b = 0; b < ctx->nb; ++b)
        if (ctx->occ[b] != 0.0) nocc = b + 1;
    cudaStream_t st = ctx->st;
    const bool direct = !ctx->fine && !ctx->aug;
    double* rw = direct ? rho : ctx->d_rho_w;
    CK(cudaMemsetAsync(rw, 0, sizeof(double) * ctx->ng, st));
    if (nocc > 0) {
        launch_zsticks_inverse<double2>(ctx->d_psi, ctx->n_pw, ctx->d_work, nocc, ctx->geo, st);
        launch_planes_density<double2>(ctx->d_work, ctx->d_occ, nocc, 1.0 / ctx->omega, rw,
                                       ctx->geo, st);
    }
    if (direct) {
        CK(cudaGetLastError());
        return CHFSI_OK;
    }
    // Fourier coefficients of the smooth part on the density grid
    launch_real_to_complex(rw, ctx->d_wgrid, ctx->ng, st);
    wave_fft3(ctx, ctx->d_wgrid, true);
    if (ctx->fine) {
        CK(cudaMemsetAsync(ctx->d_cgrid, 0, sizeof(double2) * ctx->fng, st));
        launch_scatter_g(ctx->d_wgrid, ctx->d_gmap_w, ctx->d_gmap_f, ctx->n_gmap,
                         1.0 / (double)ctx->ng, ctx->d_cgrid, st);
    } else {
        launch_scale_copy(ctx->d_wgrid, 1.0 / (double)ctx->ng, ctx->d_cgrid, ctx->ng, st);
    }
    if (ctx->aug && nocc > 0) {
        // c_I = sum_n f_n C_n^H q C_n with C = beta^H psi
        gemm_cn(ctx->d_beta, ctx->n_pw, ctx->d_psi, ctx->n_pw, ctx->np, ctx->nb, ctx->n_pw,
                ctx->d_part, ctx->d_cp, st);
        count_launch();
        k_apply_dmat<<<grid_for((size_t)ctx->np * ctx->nb), 256, 0, st>>>(
            ctx->d_cp, ctx->d_cd, ctx->np, ctx->nb, ctx->d_proj_ion, ctx->d_poff, ctx->d_doff,
            ctx->d_qmat);
        CK(cudaMemsetAsync(ctx->d_cion, 0, sizeof(double) * ctx->nions, st));
        launch_aug_coeffs(ctx->d_cp, ctx->d_cd, ctx->d_occ, ctx->nb, ctx->d_proj_ion, ctx->np,
                          ctx->d_cion, st);
        launch_aug_add(ctx->d_cgrid, grid_recip(ctx), ctx->d_phase, ctx->d_cion, ctx->nions,
                       ctx->aug_width, 1.0 / ctx->omega, st);
    }
    grid_fft3(ctx, ctx->d_cgrid, false);
    launch_take_real(ctx->d_cgrid, rho, ctx->fng, st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// (Re)allocate every density-grid buffer for the current fnx, fny, fnz.
chfsi_status alloc_density(chfsi_ctx* ctx) {
    void* old[] = {ctx->d_veff_d, ctx->d_vloc, ctx->d_rho_in, ctx->d_rho_out, ctx->d_rho_next,
                   ctx->d_cgrid, ctx->d_hist, ctx->d_shell, ctx->d_mix_c, ctx->d_mix_r,
                   ctx->d_fidr[0], ctx->d_fidr[1], ctx->d_fidr[2], ctx->d_phase};
    for (void* p : old)
        if (p) cudaFree(p);
    ctx->d_veff_d = ctx->d_vloc = ctx->d_rho_in = ctx->d_rho_out = ctx->d_rho_next = nullptr;
    ctx->d_cgrid = ctx->d_mix_c = nullptr;
    ctx->d_hist = ctx->d_mix_r = nullptr;
    ctx->d_shell = nullptr;
    ctx->d_phase = nullptr;
    for (int d = 0; d < 3; ++d) ctx->d_fidr[d] = nullptr;
    const size_t ng = ctx->fng;
    CK(dalloc(&ctx->d_veff_d, ng));
    CK(dalloc(&ctx->d_vloc, ng));
    CK(dalloc(&ctx->d_rho_in, ng)); CK(dalloc(&ctx->d_rho_out, ng));
    CK(dalloc(&ctx->d_rho_next, ng));
    CK(dalloc(&ctx->d_cgrid, ng));
    CK(dalloc(&ctx->d_hist, 2 * (size_t)kPulayMax * ng));
    std::vector<double*> hp(2 * kPulayMax);
    for (int i = 0; i < 2 * kPulayMax; ++i) hp[i] = ctx->d_hist + (size_t)i * ng;
    CK(copy_sync(ctx->d_hist_ptrs, hp.data(), hp.size() * sizeof(double*), cudaMemcpyHostToDevice,
                 ctx->st));
    CK(cudaMemsetAsync(ctx->d_vloc, 0, sizeof(double) * ng, ctx->st));
    const int n3[3] = {ctx->fnx, ctx->fny, ctx->fnz};
    for (int d = 0; d < 3; ++d) {
        const std::vector<int>& p = ctx->fdr[d];
        std::vector<int> inv(p.size());
        for (size_t k = 0; k < p.size(); ++k) inv[p[k]] = (int)k;
        CK(dalloc(&ctx->d_fidr[d], (size_t)n3[d]));
        CK(copy_sync(ctx->d_fidr[d], inv.data(), inv.size() * sizeof(int), cudaMemcpyHostToDevice,
                     ctx->st));
    }
    ctx->have_vloc = false;
    return CHFSI_OK;
}

// Per-ion axis phase tables e^{-i 2 pi f_d h} on the density grid.
chfsi_status upload_phases(chfsi_ctx* ctx) {
    if (!ctx->aug) return CHFSI_OK;
    double inv[9];
    {
        // fractional coordinates f = R . b / 2 pi (rows of recip are b_i)
        for (int i = 0; i < 9; ++i) inv[i] = ctx->recip[i] / (2.0 * 3.14159265358979323846);
    }
    const int n3[3] = {ctx->fnx, ctx->fny, ctx->fnz};
    const int stride = n3[0] + n3[1] + n3[2];
    std::vector<double2> ph((size_t)ctx->nions * stride);
    for (int I = 0; I < ctx->nions; ++I) {
        const double* R = &ctx->ion_pos[3 * I];
        int off = 0;
        for (int d = 0; d < 3; ++d) {
            const double f = R[0] * inv[3 * d] + R[1] * inv[3 * d + 1] + R[2] * inv[3 * d + 2];
            for (int h = 0; h < n3[d]; ++h) {
                const int hs = h >= (n3[d] + 1) / 2 ? h - n3[d] : h;
                const double a = -2.0 * 3.14159265358979323846 * f * hs;
                ph[(size_t)I * stride + off + h] = make_double2(std::cos(a), std::sin(a));
            }
            off += n3[d];
        }
    }
    if (ctx->d_phase) cudaFree(ctx->d_phase);
    ctx->d_phase = nullptr;
    CK(dalloc(&ctx->d_phase, ph.size()));
    CK(copy_sync(ctx->d_phase, ph.data(), ph.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    return CHFSI_OK;
}

// ---------------------------------------------------------------- learned mixer
chfsi_status alloc_mix(chfsi_ctx* ctx) {
    if (ctx->d_mix_c) return CHFSI_OK;
    const size_t ng = ctx->fng;
    CK(dalloc(&ctx->d_shell, ng));
    CK(dalloc(&ctx->d_mix_c, 7 * ng));
    CK(dalloc(&ctx->d_mix_r, 4 * ng));
    if (!ctx->d_mix_acc) CK(dalloc(&ctx->d_mix_acc, (size_t)kMixShells * kShellAcc));
    if (!ctx->d_mix_x) CK(dalloc(&ctx->d_mix_x, (size_t)kMixIn + kMixShells * kMixTargets + kMixOut));
    launch_shell_index(grid_recip(ctx), ctx->d_shell, ctx->st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

// Residual history R_0 (newest) .. R_3 in G space: complex grids 0..3 of d_mix_c.
struct MixRing {
    int n = 0, head = -1;
    double2* slot(const chfsi_ctx* ctx, int age) const {
        return ctx->d_mix_c + (size_t)((head - age + 4) % 4) * ctx->fng;
    }
};
double2* mix_grid(const chfsi_ctx* ctx, int k) { return ctx->d_mix_c + (size_t)k * ctx->fng; }
double* mix_real(const chfsi_ctx* ctx, int k) { return ctx->d_mix_r + (size_t)k * ctx->fng; }
constexpr int kGridD = 4, kGridE = 5, kGridW = 6;  // complex grid slots
float* mix_y(const chfsi_ctx* ctx) { return ctx->d_mix_x + kMixIn + kMixShells * kMixTargets; }

// FFT(out - in) becomes the newest residual.
void ring_push(chfsi_ctx* ctx, MixRing& r, const double* out, const double* in) {
    r.head = (r.head + 1) % 4;
    r.n = std::min(r.n + 1, 4);
    double2* dst = r.slot(ctx, 0);
    launch_diff_complex(out, in, dst, ctx->fng, ctx->st);
    grid_fft3(ctx, dst, true);
}

// Shell features of the ring (and targets when E != nullptr) into d_mix_x.
chfsi_status mix_features(chfsi_ctx* ctx, const MixRing& r, const double2* D, const double2* E) {
    CK(cudaMemsetAsync(ctx->d_mix_acc, 0, sizeof(double) * kMixShells * kShellAcc, ctx->st));
    const double2* R[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int a = 0; a < r.n; ++a) R[a] = r.slot(ctx, a);
    launch_shell_acc(R[0], R[1], R[2], R[3], D, E, ctx->d_shell, ctx->fng, ctx->d_mix_acc, ctx->st);
    launch_shell_features(ctx->d_mix_acc, ctx->d_mix_x, E ? ctx->d_mix_x + kMixIn : nullptr,
                          ctx->st);
    CK(cudaGetLastError());
    return CHFSI_OK;
}

chfsi_status alloc_all(chfsi_ctx* ctx) {
    // band buffers keep one spare row: the Lanczos vector that the filter
    // carries along as an extra column (CHFSI_BOUND_LANCZOS_FUSED)
    const int nbx = ctx->nb + 1;
    const size_t nbpw = (size_t)nbx * ctx->n_pw;
    CK(dalloc(&ctx->d_kin, ctx->n_pw));
    CK(dalloc(&ctx->d_perm, ctx->n_pw));
    CK(dalloc(&ctx->d_pw_col, ctx->n_pw));
    CK(dalloc(&ctx->d_pw_zpos, ctx->n_pw));
    CK(dalloc(&ctx->d_veff, ctx->ng));
    CK(dalloc(&ctx->d_rho_w, ctx->ng));
    CK(dalloc(&ctx->d_wgrid, ctx->ng));
    CK(dalloc(&ctx->d_minmax, 2));
    CK(dalloc(&ctx->d_psi, nbpw));
    CK(dalloc(&ctx->d_psi2, nbpw));
    CK(dalloc(&ctx->d_hpsi, nbpw));
    if (ctx->np > 0) {
        CK(dalloc(&ctx->d_nl, nbpw));
        CK(dalloc(&ctx->d_beta, (size_t)ctx->np * ctx->n_pw));
        CK(dalloc(&ctx->d_cp, (size_t)ctx->np * nbx));
        CK(dalloc(&ctx->d_cd, (size_t)ctx->np * nbx));
        CK(dalloc(&ctx->d_cq, (size_t)ctx->np * nbx));
        CK(dalloc(&ctx->d_proj_ion, ctx->np));
        CK(dalloc(&ctx->d_poff, ctx->nions + 1));
        CK(dalloc(&ctx->d_doff, ctx->nions));
    }
    const size_t nn = (size_t)ctx->nb * ctx->nb;
    CK(dalloc(&ctx->d_H, nn)); CK(dalloc(&ctx->d_S, nn)); CK(dalloc(&ctx->d_T1, nn));
    CK(dalloc(&ctx->d_T2, nn)); CK(dalloc(&ctx->d_V, nn));
    CK(dalloc(&ctx->d_eig, ctx->nb)); CK(dalloc(&ctx->d_eig_prev, ctx->nb));
    CK(dalloc(&ctx->d_jac, jacobi_scratch_doubles(ctx->nb, ctx->jac_max_sweeps)));
    CK(dalloc(&ctx->d_flags, 8));
    CK(cudaMemsetAsync(ctx->d_flags, 0, 8 * sizeof(int), ctx->st));
    CK(dalloc(&ctx->d_coef, 8));
    CK(dalloc(&ctx->d_nsq, ctx->max_deg + 2));
    CK(dalloc(&ctx->d_lz_v, ctx->n_pw)); CK(dalloc(&ctx->d_lz_v0, ctx->n_pw));
    CK(dalloc(&ctx->d_lz_f, ctx->n_pw)); CK(dalloc(&ctx->d_lz_start, ctx->n_pw));
    CK(dalloc(&ctx->d_lz, 2 * 64));
    CK(dalloc(&ctx->d_occ, ctx->nb));
    CK(dalloc(&ctx->d_acc, 8));
    CK(dalloc(&ctx->d_hist_ptrs, 2 * kPulayMax));
    CK(dalloc(&ctx->d_dots, kPulayMax));
    // split-K partials: max over the GEMMs that use them
    // (any band count 1..nb may reach the projector GEMM through chfsi_apply_h)
    size_t pe = std::max(splitk_partial_elems(ctx->nb, ctx->nb, ctx->n_pw),
                         splitk_partial_elems_herm(ctx->nb, ctx->n_pw));
    if (ctx->np > 0)
        for (int n = 1; n <= nbx; ++n)
            pe = std::max(pe, splitk_partial_elems(ctx->np, n, ctx->n_pw));
    ctx->part_elems = pe;
    CK(dalloc(&ctx->d_part, pe));
    // Lanczos start vector: SplitMix64(0x5EED) uniform pairs in [-1/2, 1/2)
    {
        std::vector<double2> v(ctx->n_pw);
        uint64_t s = 0x5EEDULL;
        auto next = [&s]() {
            uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
            return z ^ (z >> 31);
        };
        for (int g = 0; g < ctx->n_pw; ++g) {
            double re = (double)(next() >> 11) * (1.0 / 9007199254740992.0) - 0.5;
            double im = (double)(next() >> 11) * (1.0 / 9007199254740992.0) - 0.5;
            v[g] = make_double2(re, im);
        }
        CK(copy_sync(ctx->d_lz_start, v.data(), v.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    }
    ctx->occ.assign(ctx->nb, 0.0);
    CK(cudaMemsetAsync(ctx->d_occ, 0, sizeof(double) * ctx->nb, ctx->st));
    return alloc_density(ctx);
}

void free_all(chfsi_ctx* ctx) {
    void* ptrs[] = {ctx->d_col_start, ctx->d_col_pos, ctx->d_pw_col, ctx->d_pw_zpos, ctx->d_xact,
                    ctx->d_idr[0], ctx->d_idr[1], ctx->d_idr[2], ctx->d_perm, ctx->d_kin,
                    ctx->d_veff, ctx->d_vloc, ctx->d_minmax, ctx->d_beta, ctx->d_dmat,
                    ctx->d_proj_ion, ctx->d_poff, ctx->d_doff, ctx->d_cp, ctx->d_cd, ctx->d_psi,
                    ctx->d_psi2, ctx->d_hpsi, ctx->d_nl, ctx->d_work, ctx->d_part, ctx->d_H,
                    ctx->d_S, ctx->d_T1, ctx->d_T2, ctx->d_V, ctx->d_eig, ctx->d_eig_prev,
                    ctx->d_jac, ctx->d_flags, ctx->d_coef, ctx->d_nsq, ctx->d_lz_v, ctx->d_lz_v0,
                    ctx->d_lz_f, ctx->d_lz_start, ctx->d_lz, ctx->d_occ, ctx->d_rho_in,
                    ctx->d_rho_out, ctx->d_rho_next, ctx->d_cgrid, ctx->d_acc, ctx->d_hist,
                    ctx->d_hist_ptrs, ctx->d_dots};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    void* mp[] = {ctx->d_twd, ctx->d_twf, ctx->d_psi32a, ctx->d_psi32b, ctx->d_hpsi32, ctx->d_nl32, ctx->d_work32,
                  ctx->d_planes, ctx->d_tc_part, ctx->d_tc_err, ctx->d_qmat, ctx->d_sinvT,
                  ctx->d_cq, ctx->d_sx, ctx->d_shell, ctx->d_mix_c, ctx->d_mix_r,
                  ctx->d_mix_acc, ctx->d_mix_x, ctx->d_fidr[0], ctx->d_fidr[1], ctx->d_fidr[2],
                  ctx->d_gmap_w, ctx->d_gmap_f, ctx->d_veff_d, ctx->d_rho_w, ctx->d_wgrid,
                  ctx->d_phase, ctx->d_dmat0, ctx->d_cion, ctx->d_vion, ctx->d_tpa, ctx->d_cgR,
                  ctx->d_cgv, ctx->d_cgc, ctx->d_cgov, ctx->d_cgpart, ctx->d_cgdot, ctx->d_cgG,
                  ctx->d_psi_save, ctx->d_rc_hx, ctx->d_rc_y, ctx->d_rc_r0, ctx->d_rc_r1,
                  ctx->d_rc_y32, ctx->d_rc_coef, ctx->d_rc_lam, ctx->d_gga, ctx->d_gga_v1,
                  ctx->d_ion, ctx->d_qvec, ctx->d_atom_of_ion, ctx->d_colidx, ctx->d_bmatT};
    for (void* p : mp)
        if (p) cudaFree(p);
    if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
    if (ctx->st) cudaStreamDestroy(ctx->st);
}

// ---------------------------------------------------------------- band-CG
// Band-by-band preconditioned CG refinement after the filter
// (band_cg_minimize, src/eigensolver/band_cg.rs:157-437): steepest descent
// for two steps, then the modified Fletcher-Reeves direction
// d = (Re<g|r> / Re<g_old|r_old>) d_old - g; the preconditioned gradient is
// S-orthogonalised against the refined lower bands (cg_helpers.rs:161-216)
// and S-normalised; the direction is S-orthogonalised against the band; the
// step comes from the closed-form 2x2 line search (line_search.rs:57-212).
// The preconditioner is the TPA diagonal plus, with q, the ultrasoft
// Woodbury term (uspp_preconditioner.rs:80-131).  Vector work runs on the
// device; the handful of scalars per step come back to the host.
struct CgLineSearch { double step, eig, norm; int status; };

// Closed-form minimum of E(t) = (a + b t + c t^2) / (1 + d t^2), b = -2 Re<H psi|d>,
// with the step of the lower root clamped to 15 (line_search.rs:57-212).
CgLineSearch cg_line_search(double a, double hpsi_dir, double c, double d) {
    const double b = -2.0 * hpsi_dir;
    CgLineSearch out{0.0, a, 1.0, 0};
    double t = 0.0, e = a;
    if (std::fabs(d) > 2.2250738585072014e-308) {
        const double ad = a * d, bd = b * d;
        if (std::fabs(bd) < 1e-30) return {0.0, a, 1.0, -2};
        const double disc = ad * ad - 2.0 * ad * c + c * c + b * bd;
        if (disc < 0.0) return {0.0, a, 1.0, -1};
        const double sq = std::sqrt(disc);
        const double roots[2] = {(-ad + c + sq) / bd, (-ad + c - sq) / bd};
        double ev[2];
        bool ok[2];
        for (int i = 0; i < 2; ++i) {
            const double den = 1.0 + d * roots[i] * roots[i];
            ok[i] = den > 0.0;
            ev[i] = ok[i] ? (a + b * roots[i] + c * roots[i] * roots[i]) / den : 0.0;
        }
        int pick = -1;
        if (ok[0] && ok[1]) pick = ev[0] < ev[1] ? 0 : 1;
        else if (ok[0] && ev[0] < a) pick = 0;
        else if (ok[1] && ev[1] < a) pick = 1;
        if (pick < 0) return {0.0, a, 1.0, -1};
        t = -roots[pick];
        e = ev[pick];
    } else {
        if (!(c > 0.0)) return {0.0, a, 1.0, -1};
        t = -b / (2.0 * c);
        e = (a + b * t + c * t * t) / (1.0 + d * t * t);
    }
    if (t > 15.0) {
        t = 15.0;
        e = (a + b * t + c * t * t) / (1.0 + d * t * t);
        out.status = 1;
    } else if (t < 0.0) {
        out.status = -1;
    }
    const double nn = 1.0 + d * t * t;
    out.step = t;
    out.eig = e;
    out.norm = nn > 0.0 ? std::sqrt(nn) : 0.0;
    if (!(nn > 0.0)) out.status = 2;
    return out;
}

struct Cg {
    chfsi_ctx* ctx;
    size_t n;
    double2 *hpsi, *spsi, *r, *g, *sg, *d, *dold, *hd, *sd, *tmp;
    std::vector<std::complex<double>> dots(std::initializer_list<std::pair<const double2*, const double2*>> l) {
        DotSet ds{};
        int k = 0;
        for (auto& pr : l) { ds.a[k] = pr.first; ds.b[k] = pr.second; ++k; }
        cudaMemsetAsync(ctx->d_cgdot, 0, sizeof(double) * 2 * k, ctx->st);
        count_launch();
        k_multi_dot<<<grid_for(n), 256, 0, ctx->st>>>(ds, k, n, ctx->d_cgdot);
        double h[12];
        cudaMemcpyAsync(h, ctx->d_cgdot, sizeof(double) * 2 * k, cudaMemcpyDeviceToHost, ctx->st);
        cudaStreamSynchronize(ctx->st);
        std::vector<std::complex<double>> out(k);
        for (int j = 0; j < k; ++j) out[j] = {h[2 * j], h[2 * j + 1]};
        return out;
    }
    void lin(double2* y, std::complex<double> a, const double2* x, std::complex<double> b) {
        count_launch();
        k_lincomb<<<grid_for(n), 256, 0, ctx->st>>>(y, make_double2(a.real(), a.imag()), x,
                                                    make_double2(b.real(), b.imag()), n);
    }
    void copy(double2* dst, const double2* src) {
        cudaMemcpyAsync(dst, src, n * sizeof(double2), cudaMemcpyDeviceToDevice, ctx->st);
    }
    // S x = x + beta q beta^H x
    void apply_s(const double2* x, double2* sx) {
        copy(sx, x);
        if (!ctx->uspp) return;
        const int np = ctx->np;
        gemm_cn(ctx->d_beta, (int)n, x, (int)n, np, 1, (int)n, ctx->d_cgpart, ctx->d_cgc, ctx->st);
        count_launch();
        k_apply_dmat<<<grid_for((size_t)np), 256, 0, ctx->st>>>(ctx->d_cgc, ctx->d_cgc + np, np, 1,
                                                               ctx->d_proj_ion, ctx->d_poff,
                                                               ctx->d_doff, ctx->d_qmat);
        gemm_tn(ctx->d_cgc + np, 1, ctx->d_beta, (int)n, sx, (int)n, 1, (int)n, np, 1.0, 1.0, ctx->st);
    }
    chfsi_status apply_hs(const double2* x, double2* hx, double2* sx) {
        chfsi_status st = apply_h_dev(ctx, x, hx, 1, kEpiApply, nullptr);
        if (st) return st;
        apply_s(x, sx);
        return CHFSI_OK;
    }
    // out = T r + T beta R beta^H T r
    void precond(const double2* rr, double2* out) {
        count_launch();
        k_diag_apply<<<grid_for(n), 256, 0, ctx->st>>>(ctx->d_tpa, rr, nullptr, out, n);
        if (!ctx->d_cgR) return;
        const int np = ctx->np;
        gemm_cn(ctx->d_beta, (int)n, out, (int)n, np, 1, (int)n, ctx->d_cgpart, ctx->d_cgc, ctx->st);
        gemm_cn(ctx->d_cgR, np, ctx->d_cgc, np, np, 1, np, ctx->d_cgpart, ctx->d_cgc + np, ctx->st);
        gemm_tn(ctx->d_cgc + np, 1, ctx->d_beta, (int)n, tmp, (int)n, 1, (int)n, np, 1.0, 0.0, ctx->st);
        count_launch();
        k_diag_apply<<<grid_for(n), 256, 0, ctx->st>>>(ctx->d_tpa, rr, tmp, out, n);
    }
};

chfsi_status cg_prepare(chfsi_ctx* ctx) {
    if (ctx->cg_ready) return CHFSI_OK;
    const size_t n = ctx->n_pw;
    const int np = ctx->np, nb = ctx->nb;
    if (!ctx->d_tpa) CK(dalloc(&ctx->d_tpa, n));
    if (!ctx->d_cgv) CK(dalloc(&ctx->d_cgv, 10 * n));
    if (!ctx->d_cgc) CK(dalloc(&ctx->d_cgc, (size_t)3 * std::max(np, 1)));
    if (!ctx->d_cgov) CK(dalloc(&ctx->d_cgov, 2 * (size_t)nb));
    if (!ctx->d_cgG) CK(dalloc(&ctx->d_cgG, (size_t)nb * nb));
    if (!ctx->d_cgdot) CK(dalloc(&ctx->d_cgdot, 16));
    size_t pe = 0;
    for (int k = 1; k <= nb; ++k)
        pe = std::max({pe, splitk_partial_elems(k, 1, (int)n), splitk_partial_elems(1, k, (int)n)});
    if (np > 0) {
        pe = std::max(pe, splitk_partial_elems(np, 1, (int)n));
        pe = std::max(pe, splitk_partial_elems(np, 1, np));
    }
    if (!ctx->d_cgpart) CK(dalloc(&ctx->d_cgpart, pe));
    double sum = 0.0;
    for (double k : ctx->kin_host) sum += k;
    const double mean = n ? sum / (double)n : 0.0;
    count_launch();
    k_tpa<<<grid_for(n), 256, 0, ctx->st>>>(ctx->d_kin, mean > 0.0 ? 1.0 / mean : 1.0, ctx->d_tpa, n);
    if (ctx->uspp && np > 0) {
        // R = (-q^-1 - beta^H T beta)^-1 on the host (once per context)
        double2 *bt = nullptr, *part = nullptr, *cm = nullptr;
        CK(cudaMalloc((void**)&bt, (size_t)np * n * sizeof(double2)));
        cudaError_t e = cudaMalloc((void**)&part, splitk_partial_elems(np, np, (int)n) * sizeof(double2));
        if (e == cudaSuccess) e = cudaMalloc((void**)&cm, (size_t)np * np * sizeof(double2));
        if (e != cudaSuccess) {
            cudaFree(bt); cudaFree(part); cudaFree(cm);
            CK(e);
        }
        for (int p = 0; p < np; ++p) {
            count_launch();
            k_diag_apply<<<grid_for(n), 256, 0, ctx->st>>>(ctx->d_tpa, ctx->d_beta + (size_t)p * n,
                                                           nullptr, bt + (size_t)p * n, n);
        }
        gemm_cn(ctx->d_beta, (int)n, bt, (int)n, np, np, (int)n, part, cm, ctx->st);
        std::vector<std::complex<double>> C((size_t)np * np), Q((size_t)np * np, 0.0);
        std::vector<double2> qh;
        std::vector<int> poff(ctx->nions + 1), doff(ctx->nions);
        e = cudaMemcpyAsync(C.data(), cm, C.size() * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(poff.data(), ctx->d_poff, poff.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(doff.data(), ctx->d_doff, doff.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->st);
        size_t dt = 0;
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
        cudaFree(bt); cudaFree(part); cudaFree(cm);
        CK(e);
        for (int i = 0; i < ctx->nions; ++i) dt += (size_t)(poff[i + 1] - poff[i]) * (poff[i + 1] - poff[i]);
        qh.resize(dt);
        CK(copy_sync(qh.data(), ctx->d_qmat, dt * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st));
        for (int i = 0; i < ctx->nions; ++i) {
            const int p0 = poff[i], ne = poff[i + 1] - p0;
            for (int a = 0; a < ne; ++a)
                for (int b = 0; b < ne; ++b) {
                    const double2 q = qh[doff[i] + a * ne + b];
                    Q[(size_t)(p0 + a) * np + p0 + b] = {q.x, q.y};
                }
        }
        if (!invert_complex(Q, np)) return ctx->fail(CHFSI_ERR_NUMERIC, "q is singular");
        for (size_t i = 0; i < Q.size(); ++i) Q[i] = -Q[i] - C[i];
        if (!invert_complex(Q, np)) return ctx->fail(CHFSI_ERR_NUMERIC, "preconditioner matrix is singular");
        // gemm_cn conjugates its first operand: store conj(R)
        std::vector<double2> rc(Q.size());
        for (size_t i = 0; i < Q.size(); ++i) rc[i] = make_double2(Q[i].real(), -Q[i].imag());
        if (!ctx->d_cgR) CK(dalloc(&ctx->d_cgR, (size_t)np * np));
        CK(copy_sync(ctx->d_cgR, rc.data(), rc.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    }
    CK(cudaGetLastError());
    ctx->cg_ready = true;
    return CHFSI_OK;
}

// y -= sum_j w_j L_j for the first k rows L_j of a band-major block
void gemm_tn_complex_axpy(chfsi_ctx* ctx, const double2* w, int k, const double2* L, double2* y) {
    const int n = ctx->n_pw;
    gemm_tn(w, 1, L, n, y, n, 1, n, k, -1.0, 1.0, ctx->st);
}

// Refine every band of d_psi in turn; d_sx holds S psi of the refined bands
// (ultrasoft), eig[b] the band energy, steps[b] the steps taken.
chfsi_status band_cg_dev(chfsi_ctx* ctx, int max_steps, double tol, double* eig, int* steps,
                         int* n_conv) {
    chfsi_status st = cg_prepare(ctx);
    if (st) return st;
    Cg c{};
    c.ctx = ctx;
    c.n = ctx->n_pw;
    double2* V = ctx->d_cgv;
    c.hpsi = V; c.spsi = V + c.n; c.r = V + 2 * c.n; c.g = V + 3 * c.n; c.sg = V + 4 * c.n;
    c.d = V + 5 * c.n; c.dold = V + 6 * c.n; c.hd = V + 7 * c.n; c.sd = V + 8 * c.n;
    c.tmp = V + 9 * c.n;
    const size_t n = c.n;
    const int nb = ctx->nb;
    const double2* lower_s = ctx->uspp ? ctx->d_sx : ctx->d_psi;
    int nconv = 0;
    for (int b = 0; b < nb; ++b) {
        double2* psi = ctx->d_psi + (size_t)b * n;
        if ((st = c.apply_hs(psi, c.hpsi, c.spsi))) return st;
        const double s0 = c.dots({{psi, c.spsi}})[0].real();
        const double inv0 = 1.0 / std::sqrt(s0);
        c.lin(psi, inv0, nullptr, 0.0);
        c.lin(c.hpsi, inv0, nullptr, 0.0);
        c.lin(c.spsi, inv0, nullptr, 0.0);
        auto residual = [&](double& e_out) {
            const auto dd = c.dots({{psi, c.hpsi}, {psi, c.spsi}});
            const double he = dd[0].real(), se = dd[1].real();
            e_out = he;
            c.copy(c.r, c.hpsi);
            c.lin(c.r, 1.0, c.spsi, -he / se);
        };
        double e = 0.0;
        residual(e);
        double beta_old = 0.0;
        int taken = max_steps;
        bool conv = false;
        for (int step = 1; step <= max_steps; ++step) {
            c.precond(c.r, c.g);
            const double gn0 = std::sqrt(c.dots({{c.g, c.g}})[0].real());
            if (gn0 < 2.220446049250313e-16 * 1000.0) { taken = step - 1; conv = true; break; }
            const double prev = e;
            c.apply_s(c.g, c.sg);
            if (b > 0) {
                // modified Gram-Schmidt against the refined lower bands
                // (s_orthogonalize_against, cg_helpers.rs:161-216) in closed
                // form: v = Psi^H S g, ov = (1 + L)^-1 v with L the strictly
                // lower part of Psi^H S Psi, then g -= Psi ov, S g -= S Psi ov
                gemm_cn(ctx->d_psi, (int)n, c.sg, (int)n, b, 1, (int)n, ctx->d_cgpart, ctx->d_cgov, ctx->st);
                count_launch();
                k_mgs_overlaps<<<1, 32, 0, ctx->st>>>(ctx->d_cgov, ctx->d_cgG, nb, b, ctx->d_cgov + nb);
                gemm_tn_complex_axpy(ctx, ctx->d_cgov + nb, b, ctx->d_psi, c.g);
                gemm_tn_complex_axpy(ctx, ctx->d_cgov + nb, b, lower_s, c.sg);
            }
            const auto gd = c.dots({{c.g, c.sg}, {c.g, c.r}});
            const double gn = std::sqrt(std::max(gd[0].real(), 1e-300));
            c.lin(c.g, 1.0 / gn, nullptr, 0.0);
            c.lin(c.sg, 1.0 / gn, nullptr, 0.0);
            const double beta = gd[1].real() / gn;
            if (step <= 2) {
                c.copy(c.d, c.g);
                beta_old = beta;
            } else {
                const double gamma = std::fabs(beta_old) > 1e-300 ? beta / beta_old : 0.0;
                c.copy(c.d, c.dold);
                c.lin(c.d, gamma, c.g, -1.0);
                beta_old = beta;
            }
            if ((st = c.apply_hs(c.d, c.hd, c.sd))) return st;
            const auto od = c.dots({{psi, c.sd}, {c.r, c.r}});
            const std::complex<double> ov = od[0];
            if (std::abs(ov) > 1e-30) {
                c.lin(c.d, 1.0, psi, -ov);
                c.lin(c.hd, 1.0, c.hpsi, -ov);
                c.lin(c.sd, 1.0, c.spsi, -ov);
            }
            c.copy(c.dold, c.d);
            const double rn = std::sqrt(od[1].real());
            if (rn < tol * 0.01 && rn < 1e-12 * std::max(std::fabs(e), 1.0)) {
                taken = step - 1;
                conv = true;
                break;
            }
            const auto ld = c.dots({{c.hpsi, c.d}, {c.hd, c.d}, {c.sd, c.d}});
            const CgLineSearch ls = cg_line_search(e, ld[0].real(), ld[1].real(), ld[2].real());
            const double inv = ls.norm > 0.0 ? 1.0 / ls.norm : 1.0;
            c.lin(psi, inv, c.d, ls.step * inv);
            c.lin(c.hpsi, inv, c.hd, ls.step * inv);
            c.lin(c.spsi, inv, c.sd, ls.step * inv);
            double e_new = 0.0;
            residual(e_new);
            if (std::fabs(e_new - prev) < tol) {
                e = e_new;
                taken = step;
                conv = true;
                break;
            }
            e = e_new;
        }
        if (ctx->uspp) c.copy(ctx->d_sx + (size_t)b * n, c.spsi);
        if (b > 0) {
            // row b of the lower Gram matrix: G[b][i] = <psi_b|S psi_i>, i < b
            gemm_cn(psi, (int)n, lower_s, (int)n, 1, b, (int)n, ctx->d_cgpart,
                    ctx->d_cgG + (size_t)b * nb, ctx->st);
        }
        if (eig) eig[b] = e;
        if (steps) steps[b] = taken;
        nconv += conv;
    }
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaGetLastError());
    if (n_conv) *n_conv = nconv;
    return CHFSI_OK;
}

}  // namespace

// ============================================================== C ABI
extern "C" {

chfsi_status chfsi_default_config(chfsi_config* c) {
    if (!c) return CHFSI_ERR_BAD_INPUT;
    std::memset(c, 0, sizeof(*c));
    c->device = 0;
    c->precision = CHFSI_PREC_FP64;
    c->bound_mode = CHFSI_BOUND_HEURISTIC;
    c->lanczos_steps = 10;
    c->check_norms = 1;
    return CHFSI_OK;
}

const char* chfsi_last_error(const chfsi_ctx* ctx) {
    if (ctx && !ctx->err.empty()) return ctx->err.c_str();
    return g_last_error.c_str();
}

chfsi_status chfsi_create(const chfsi_dims* dims, const chfsi_config* cfg, chfsi_ctx** out) {
    if (!dims || !out) return CHFSI_ERR_BAD_INPUT;
    *out = nullptr;
    if (dims->n_pw <= 0 || dims->n_bands <= 0 || dims->n_bands > dims->n_pw || dims->n_proj < 0 ||
        (dims->n_proj > 0 && dims->n_ions <= 0))
        return CHFSI_ERR_BAD_INPUT;
    for (int d = 0; d < 3; ++d)
        if (dims->ngrid[d] <= 0 || dims->ngrid[d] > 256) return CHFSI_ERR_BAD_INPUT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g_last_error = "no CUDA device visible";
        return CHFSI_ERR_NO_DEVICE;
    }
    chfsi_ctx* ctx = new (std::nothrow) chfsi_ctx();
    if (!ctx) return CHFSI_ERR_OUT_OF_MEMORY;
    ctx->dims = *dims;
    if (cfg) ctx->cfg = *cfg; else chfsi_default_config(&ctx->cfg);
    if (ctx->cfg.filter_form != CHFSI_FILTER_CHEBYSHEV && ctx->cfg.filter_form != CHFSI_FILTER_RESIDUAL) {
        delete ctx;
        g_last_error = "unknown filter form";
        return CHFSI_ERR_BAD_INPUT;
    }
    if (ctx->cfg.bound_mode < CHFSI_BOUND_HEURISTIC || ctx->cfg.bound_mode > CHFSI_BOUND_LANCZOS_FUSED) {
        delete ctx;
        g_last_error = "unknown bound mode";
        return CHFSI_ERR_BAD_INPUT;
    }
    if (ctx->cfg.precision != CHFSI_PREC_FP64 && ctx->cfg.precision != CHFSI_PREC_MIXED) {
        delete ctx;
        g_last_error = "unknown precision mode";
        return CHFSI_ERR_BAD_INPUT;
    }
    ctx->mixed = ctx->mixed_active = ctx->cfg.precision == CHFSI_PREC_MIXED;
    ctx->device = ctx->cfg.device;
    chfsi_status s = CHFSI_OK;
    auto bail = [&](chfsi_status e) { free_all(ctx); delete ctx; return e; };
    if (cudaSetDevice(ctx->device) != cudaSuccess) { g_last_error = "cudaSetDevice failed"; return bail(CHFSI_ERR_CUDA); }
    if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess) return bail(CHFSI_ERR_CUDA);
    ctx->nx = dims->ngrid[0]; ctx->ny = dims->ngrid[1]; ctx->nz = dims->ngrid[2];
    ctx->ng = (size_t)ctx->nx * ctx->ny * ctx->nz;
    ctx->n_pw = dims->n_pw; ctx->nb = dims->n_bands; ctx->np = dims->n_proj; ctx->nions = dims->n_ions;
    if (!plan_axis(ctx->nx, ctx->ax) || !plan_axis(ctx->ny, ctx->ay) || !plan_axis(ctx->nz, ctx->az)) {
        g_last_error = "FFT grid dimensions must be 2,3,5-smooth";
        return bail(CHFSI_ERR_BAD_INPUT);
    }
    digit_reversal(ctx->ax, ctx->dr[0]);
    digit_reversal(ctx->ay, ctx->dr[1]);
    digit_reversal(ctx->az, ctx->dr[2]);
    ctx->fnx = ctx->nx; ctx->fny = ctx->ny; ctx->fnz = ctx->nz; ctx->fng = ctx->ng;
    ctx->fax = ctx->ax; ctx->fay = ctx->ay; ctx->faz = ctx->az;
    for (int d = 0; d < 3; ++d) ctx->fdr[d] = ctx->dr[d];
    s = alloc_all(ctx);
    if (s) return bail(s);
    // inverse digit reversal tables (position -> frequency) for the potential kernels
    for (int d = 0; d < 3; ++d) {
        const std::vector<int>& p = ctx->dr[d];
        std::vector<int> inv(p.size());
        for (size_t k = 0; k < p.size(); ++k) inv[p[k]] = (int)k;
        if (cudaMalloc((void**)&ctx->d_idr[d], inv.size() * sizeof(int)) != cudaSuccess) return bail(CHFSI_ERR_OUT_OF_MEMORY);
        if (copy_sync(ctx->d_idr[d], inv.data(), inv.size() * sizeof(int), cudaMemcpyHostToDevice,
                      ctx->st) != cudaSuccess)
            return bail(CHFSI_ERR_CUDA);
    }
    *out = ctx;
    return CHFSI_OK;
}

void chfsi_destroy(chfsi_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    free_all(ctx);
    delete ctx;
}

chfsi_status chfsi_set_basis(chfsi_ctx* ctx, const int32_t* miller, const double* kinetic,
                             double gmax) {
    if (!ctx || !miller || !kinetic) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    const int n = ctx->n_pw, nx = ctx->nx, ny = ctx->ny, nz = ctx->nz;
    auto wrap = [](int h, int m) { return h >= 0 ? h : h + m; };
    std::vector<int> ix(n), iy(n), iz(n);
    for (int g = 0; g < n; ++g) {
        int h = miller[3 * g], k = miller[3 * g + 1], l = miller[3 * g + 2];
        if (std::abs(2 * h) >= nx + (nx & 1) || std::abs(2 * k) >= ny + (ny & 1) ||
            std::abs(2 * l) >= nz + (nz & 1))
            return ctx->fail(CHFSI_ERR_BAD_INPUT, "Miller index outside the FFT grid");
        ix[g] = wrap(h, nx); iy[g] = wrap(k, ny); iz[g] = wrap(l, nz);
    }
    // internal order: by column (iy, ix), then l ascending
    std::vector<int> perm(n);
    for (int g = 0; g < n; ++g) perm[g] = g;
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
        int ca = iy[a] * nx + ix[a], cb = iy[b] * nx + ix[b];
        if (ca != cb) return ca < cb;
        return miller[3 * a + 2] < miller[3 * b + 2];
    });
    ctx->perm_identity = true;
    for (int g = 0; g < n; ++g)
        if (perm[g] != g) { ctx->perm_identity = false; break; }
    ctx->miller_ctx.resize(3 * (size_t)n);
    for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) ctx->miller_ctx[3 * (size_t)i + d] = miller[3 * (size_t)perm[i] + d];
    if (ctx->d_qvec) { cudaFree(ctx->d_qvec); ctx->d_qvec = nullptr; }
    std::vector<int> col_start, col_pos, pw_col(n), pw_zpos(n), xact, col_px, col_py;
    std::vector<double> kin(n);
    std::vector<char> xused(nx, 0);
    int last = -1;
    for (int i = 0; i < n; ++i) {
        const int g = perm[i];
        const int c = iy[g] * nx + ix[g];
        if (c != last) {
            col_start.push_back(i);
            const int px = ctx->dr[0][ix[g]], py = ctx->dr[1][iy[g]];
            // plane rows and elements are XOR-swizzled in shared memory
            col_pos.push_back(swz(py, ny) * (nx | 1) + swz(px, nx));
            col_px.push_back(px);
            col_py.push_back(py);
            xused[px] = 1;
            last = c;
        } else if (i > 0 && miller[3 * g + 2] == miller[3 * perm[i - 1] + 2]) {
            return ctx->fail(CHFSI_ERR_BAD_INPUT, "duplicate plane wave");
        }
        pw_col[i] = (int)col_start.size() - 1;
        pw_zpos[i] = ctx->dr[2][iz[g]];
        kin[i] = kinetic[g];
    }
    const int ncol = (int)col_start.size();
    col_start.push_back(n);
    std::vector<int> line_of(nx, -1);
    for (int x = 0; x < nx; ++x)
        if (xused[x]) {
            line_of[x] = (int)xact.size();
            xact.push_back(swz(x, nx));
        }
    // direct column I/O table of the compile-time plane kernel:
    // colidx[line * ny + py] = column at (active x line, digit-reversed y)
    std::vector<int> colidx(xact.size() * (size_t)ny, -1);
    for (int c = 0; c < (int)col_px.size(); ++c)
        colidx[(size_t)line_of[col_px[c]] * ny + col_py[c]] = c;
    double kmax = 0.0;
    for (int g = 0; g < n; ++g) kmax = std::max(kmax, kinetic[g]);
    // kinetic bound of the reference: 1/2 Gmax^2 (chebyshev.rs:232)
    ctx->kin_max = gmax > 0.0 ? 0.5 * gmax * gmax : kmax;
    if (ctx->d_col_start) cudaFree(ctx->d_col_start);
    if (ctx->d_col_pos) cudaFree(ctx->d_col_pos);
    if (ctx->d_xact) cudaFree(ctx->d_xact);
    if (ctx->d_colidx) cudaFree(ctx->d_colidx);
    ctx->d_colidx = nullptr;
    if (ctx->d_work) cudaFree(ctx->d_work);
    ctx->d_col_start = ctx->d_col_pos = ctx->d_xact = nullptr;
    ctx->d_work = nullptr;
    CK(dalloc(&ctx->d_col_start, ncol + 1));
    CK(dalloc(&ctx->d_col_pos, ncol));
    CK(dalloc(&ctx->d_xact, xact.size()));
    CK(dalloc(&ctx->d_colidx, colidx.size()));
    CK(copy_sync(ctx->d_colidx, colidx.data(), sizeof(int) * colidx.size(), cudaMemcpyHostToDevice, ctx->st));
    CK(dalloc(&ctx->d_work, (size_t)(ctx->nb + 1) * nz * ncol));
    CK(copy_sync(ctx->d_col_start, col_start.data(), sizeof(int) * (ncol + 1), cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_col_pos, col_pos.data(), sizeof(int) * ncol, cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_xact, xact.data(), sizeof(int) * xact.size(), cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_pw_col, pw_col.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_pw_zpos, pw_zpos.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_kin, kin.data(), sizeof(double) * n, cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_perm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, ctx->st));
    // twiddle tables exp(+2 pi i j / n) of the three axes (cos/sin in FP64)
    if (!ctx->d_twd) {
        std::vector<double2> twd(nx + ny + nz);
        std::vector<float2> twf(nx + ny + nz);
        int o = 0;
        for (int m : {nx, ny, nz})
            for (int j = 0; j < m; ++j, ++o) {
                const double a = 2.0 * 3.14159265358979323846 * (double)j / (double)m;
                twd[o] = make_double2(std::cos(a), std::sin(a));
                twf[o] = make_float2((float)twd[o].x, (float)twd[o].y);
            }
        CK(dalloc(&ctx->d_twd, twd.size()));
        CK(dalloc(&ctx->d_twf, twf.size()));
        CK(copy_sync(ctx->d_twd, twd.data(), twd.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
        CK(copy_sync(ctx->d_twf, twf.data(), twf.size() * sizeof(float2), cudaMemcpyHostToDevice, ctx->st));
    }
    HGeom& g = ctx->geo;
    g.twd_x = ctx->d_twd; g.twd_y = ctx->d_twd + nx; g.twd_z = ctx->d_twd + nx + ny;
    g.twf_x = ctx->d_twf; g.twf_y = ctx->d_twf + nx; g.twf_z = ctx->d_twf + nx + ny;
    g.nx = nx; g.ny = ny; g.nz = nz; g.n_pw = n; g.ncol = ncol;
    g.lsz = nz | 1; g.lsx = nx | 1; g.nxact = (int)xact.size();
    g.col_start = ctx->d_col_start; g.col_pos = ctx->d_col_pos; g.pw_col = ctx->d_pw_col;
    g.pw_zpos = ctx->d_pw_zpos; g.xact = ctx->d_xact;
    g.colidx = nx <= 256 ? ctx->d_colidx : nullptr;
    for (int w = 0; w < 8; ++w) g.xbits[w] = 0u;
    for (int x = 0; x < nx && x < 256; ++x)
        if (xused[x]) g.xbits[x >> 5] |= 1u << (x & 31);
    g.ax = ctx->ax; g.ay = ctx->ay; g.az = ctx->az;
    if (planes_smem_bytes(g, sizeof(double2)) > 227 * 1024)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "xy plane does not fit in shared memory");
    if ((size_t)nx * ny > kDensityPlanePoints)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "xy plane too large for the density kernel");
    if (ctx->mixed) {
        chfsi_status s = alloc_mixed(ctx, ncol);
        if (s) return s;
    }
    ctx->kin_host = kin;
    ctx->cg_ready = false;
    ctx->basis_set = true;
    return CHFSI_OK;
}

chfsi_status chfsi_set_projectors(chfsi_ctx* ctx, const chfsi_c128* beta,
                                  const int32_t* proj_offsets, const chfsi_c128* dmat) {
    if (!ctx || !ctx->basis_set) return CHFSI_ERR_BAD_INPUT;
    if (ctx->np == 0) return CHFSI_OK;
    if (!beta || !proj_offsets || !dmat) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    const int ni = ctx->nions;
    if (proj_offsets[0] != 0 || proj_offsets[ni] != ctx->np)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "projector offsets do not cover n_proj");
    std::vector<int> pion(ctx->np), doff(ni);
    size_t dt = 0;
    for (int i = 0; i < ni; ++i) {
        const int ne = proj_offsets[i + 1] - proj_offsets[i];
        if (ne <= 0) return ctx->fail(CHFSI_ERR_BAD_INPUT, "empty projector block");
        for (int p = proj_offsets[i]; p < proj_offsets[i + 1]; ++p) pion[p] = i;
        doff[i] = (int)dt;
        dt += (size_t)ne * ne;
    }
    if (ctx->d_dmat) cudaFree(ctx->d_dmat);
    if (ctx->d_dmat0) cudaFree(ctx->d_dmat0);
    ctx->d_dmat = ctx->d_dmat0 = nullptr;
    CK(dalloc(&ctx->d_dmat, dt));
    CK(dalloc(&ctx->d_dmat0, dt));
    CK(copy_sync(ctx->d_dmat, dmat, dt * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->d_dmat0, ctx->d_dmat, dt * sizeof(double2), cudaMemcpyDeviceToDevice,
                       ctx->st));
    CK(copy_sync(ctx->d_proj_ion, pion.data(), sizeof(int) * ctx->np, cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_poff, proj_offsets, sizeof(int) * (ni + 1), cudaMemcpyHostToDevice, ctx->st));
    CK(copy_sync(ctx->d_doff, doff.data(), sizeof(int) * ni, cudaMemcpyHostToDevice, ctx->st));
    const size_t nbeta = (size_t)ctx->np * ctx->n_pw;
    if (ctx->perm_identity) {
        CK(copy_sync(ctx->d_beta, beta, nbeta * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    } else {
        // stage in the hpsi buffer when it is large enough, else in a temporary
        double2* stage = nullptr;
        CK(cudaMalloc((void**)&stage, nbeta * sizeof(double2)));
        if (cudaError_t e = copy_sync(stage, beta, nbeta * sizeof(double2), cudaMemcpyHostToDevice,
                                      ctx->st)) {
            cudaFree(stage);
            return cuda_fail(e, "copy_sync(stage)", __FILE__, __LINE__);
        }
        count_launch();
        k_gather_rows<<<grid_for(nbeta), 256, 0, ctx->st>>>(stage, ctx->n_pw, ctx->d_perm,
                                                           ctx->d_beta, ctx->n_pw, ctx->np);
        cudaStreamSynchronize(ctx->st);
        cudaFree(stage);
        CK(cudaGetLastError());
    }
    ctx->proj_set = true;
    ctx->beta_planes_ready = false;
    return pack_beta_planes(ctx);
}

chfsi_status chfsi_set_qmat(chfsi_ctx* ctx, const chfsi_c128* qmat) {
    if (!ctx || !qmat || !ctx->proj_set || ctx->np == 0) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    const int np = ctx->np, ni = ctx->nions;
    std::vector<int> poff(ni + 1), doff(ni);
    CK(copy_sync(poff.data(), ctx->d_poff, sizeof(int) * (ni + 1), cudaMemcpyDeviceToHost, ctx->st));
    CK(copy_sync(doff.data(), ctx->d_doff, sizeof(int) * ni, cudaMemcpyDeviceToHost, ctx->st));
    size_t dt = 0;
    for (int i = 0; i < ni; ++i) dt += (size_t)(poff[i + 1] - poff[i]) * (poff[i + 1] - poff[i]);
    if (!ctx->d_qmat) CK(dalloc(&ctx->d_qmat, dt));
    CK(copy_sync(ctx->d_qmat, qmat, dt * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    // B = beta^H beta on the device
    double2 *part = nullptr, *dB = nullptr;
    CK(cudaMalloc((void**)&part, splitk_partial_elems(np, np, ctx->n_pw) * sizeof(double2)));
    CK(cudaMalloc((void**)&dB, (size_t)np * np * sizeof(double2)));
    gemm_cn(ctx->d_beta, ctx->n_pw, ctx->d_beta, ctx->n_pw, np, np, ctx->n_pw, part, dB, ctx->st);
    std::vector<std::complex<double>> B((size_t)np * np), Q((size_t)np * np, 0.0);
    cudaError_t e = cudaMemcpyAsync(B.data(), dB, B.size() * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess && !ctx->d_bmatT) e = dalloc(&ctx->d_bmatT, (size_t)np * np);
    if (e == cudaSuccess) {
        count_launch();
        k_conj<<<grid_for((size_t)np * np), 256, 0, ctx->st>>>(dB, ctx->d_bmatT, (size_t)np * np);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    cudaFree(part);
    cudaFree(dB);
    CK(e);
    const std::complex<double>* qh = reinterpret_cast<const std::complex<double>*>(qmat);
    for (int i = 0; i < ni; ++i) {
        const int p0 = poff[i], ne = poff[i + 1] - p0;
        for (int a = 0; a < ne; ++a)
            for (int b = 0; b < ne; ++b) Q[(size_t)(p0 + a) * np + p0 + b] = qh[doff[i] + a * ne + b];
    }
    // s_min = 1 - max row sum |q B|; A = 1 + B q; M = q A^-1
    double rs = 0.0;
    std::vector<std::complex<double>> A((size_t)np * np, 0.0);
    for (int i = 0; i < np; ++i) {
        double r = 0.0;
        for (int j = 0; j < np; ++j) {
            std::complex<double> qb = 0.0, bq = 0.0;
            const int ion_i = std::upper_bound(poff.begin(), poff.end(), i) - poff.begin() - 1;
            const int ion_j = std::upper_bound(poff.begin(), poff.end(), j) - poff.begin() - 1;
            for (int k = poff[ion_i]; k < poff[ion_i + 1]; ++k) qb += Q[(size_t)i * np + k] * B[(size_t)k * np + j];
            for (int k = poff[ion_j]; k < poff[ion_j + 1]; ++k) bq += B[(size_t)i * np + k] * Q[(size_t)k * np + j];
            r += std::abs(qb);
            A[(size_t)i * np + j] = bq + (i == j ? 1.0 : 0.0);
        }
        rs = std::max(rs, r);
    }
    ctx->s_min = std::max(0.1, 1.0 - rs);
    if (!invert_complex(A, np)) return ctx->fail(CHFSI_ERR_NUMERIC, "1 + B q is singular");
    std::vector<std::complex<double>> MT((size_t)np * np, 0.0);
    for (int i = 0; i < np; ++i) {
        const int ion_i = std::upper_bound(poff.begin(), poff.end(), i) - poff.begin() - 1;
        for (int j = 0; j < np; ++j) {
            std::complex<double> m = 0.0;
            for (int k = poff[ion_i]; k < poff[ion_i + 1]; ++k) m += Q[(size_t)i * np + k] * A[(size_t)k * np + j];
            MT[(size_t)j * np + i] = m;
        }
    }
    if (!ctx->d_sinvT) CK(dalloc(&ctx->d_sinvT, (size_t)np * np));
    if (!ctx->d_cq) CK(dalloc(&ctx->d_cq, (size_t)np * ctx->nb));
    if (!ctx->d_sx) CK(dalloc(&ctx->d_sx, (size_t)ctx->nb * ctx->n_pw));
    CK(copy_sync(ctx->d_sinvT, MT.data(), MT.size() * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    ctx->uspp = true;
    return CHFSI_OK;
}

chfsi_status chfsi_get_s_min(chfsi_ctx* ctx, double* out) {
    if (!ctx || !out) return CHFSI_ERR_BAD_INPUT;
    *out = ctx->s_min;
    return CHFSI_OK;
}

chfsi_status chfsi_set_veff(chfsi_ctx* ctx, const double* veff) {
    if (!ctx || !veff) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    CK(cudaMemcpyAsync(ctx->d_veff, veff, ctx->ng * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    minmax(ctx->d_veff, ctx->ng, ctx->d_minmax, ctx->st);
    CK(cudaGetLastError());
    ctx->veff_set = true;
    return CHFSI_OK;
}

chfsi_status chfsi_set_psi(chfsi_ctx* ctx, const chfsi_c128* psi) {
    if (!ctx || !psi || !ctx->basis_set) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)ctx->nb * ctx->n_pw;
    if (ctx->perm_identity) {
        CK(cudaMemcpyAsync(ctx->d_psi, psi, n * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    } else {
        CK(cudaMemcpyAsync(ctx->d_psi2, psi, n * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
        count_launch();
        k_gather_rows<<<grid_for(n), 256, 0, ctx->st>>>(ctx->d_psi2, ctx->n_pw, ctx->d_perm,
                                                       ctx->d_psi, ctx->n_pw, ctx->nb);
        CK(cudaGetLastError());
    }
    ctx->psi_set = true;
    return CHFSI_OK;
}

chfsi_status chfsi_get_psi(chfsi_ctx* ctx, chfsi_c128* psi) {
    if (!ctx || !psi) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)ctx->nb * ctx->n_pw;
    if (ctx->perm_identity) {
        CK(cudaMemcpyAsync(psi, ctx->d_psi, n * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st));
    } else {
        count_launch();
        k_scatter_rows<<<grid_for(n), 256, 0, ctx->st>>>(ctx->d_psi, ctx->d_perm, ctx->d_psi2,
                                                        ctx->n_pw, ctx->n_pw, ctx->nb);
        CK(cudaMemcpyAsync(psi, ctx->d_psi2, n * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));
    return CHFSI_OK;
}

chfsi_status chfsi_psi_device_ptr(chfsi_ctx* ctx, chfsi_c128** out) {
    if (!ctx || !out) return CHFSI_ERR_BAD_INPUT;
    *out = reinterpret_cast<chfsi_c128*>(ctx->d_psi);
    return CHFSI_OK;
}

static chfsi_status ready(chfsi_ctx* ctx) {
    if (!ctx) return CHFSI_ERR_BAD_INPUT;
    if (!ctx->basis_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "basis not set");
    if (!ctx->veff_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "V_eff not set");
    if (ctx->np > 0 && !ctx->proj_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "projectors not set");
    cudaSetDevice(ctx->device);
    return CHFSI_OK;
}

chfsi_status chfsi_apply_h_local(chfsi_ctx* ctx, const chfsi_c128* psi_dev, chfsi_c128* hpsi_dev,
                                 int nb) {
    chfsi_status s = ready(ctx);
    if (s) return s;
    if (!psi_dev || !hpsi_dev || nb <= 0 || nb > ctx->nb) return CHFSI_ERR_BAD_INPUT;
    const int np = ctx->np;
    ctx->np = 0;  // local part only: T + V_loc
    s = apply_h_dev(ctx, reinterpret_cast<const double2*>(psi_dev),
                    reinterpret_cast<double2*>(hpsi_dev), nb, kEpiApply, nullptr);
    ctx->np = np;
    if (s) return s;
    CK(cudaStreamSynchronize(ctx->st));
    return CHFSI_OK;
}

chfsi_status chfsi_get_stream(chfsi_ctx* ctx, void** out) {
    if (!ctx || !out) return CHFSI_ERR_BAD_INPUT;
    *out = (void*)ctx->st;
    return CHFSI_OK;
}

long long chfsi_launch_count(void) { return g_launch_count.load(); }

// S^-1 H x of the generalised (ultrasoft) problem, the operator the filter
// applies (Woodbury inverse S^-1 = 1 - beta M beta^H); H x alone without q.
chfsi_status chfsi_apply_sinv_h(chfsi_ctx* ctx, const chfsi_c128* psi_dev, chfsi_c128* out_dev,
                                int nb) {
    chfsi_status s = ready(ctx);
    if (s) return s;
    if (!psi_dev || !out_dev || nb <= 0 || nb > ctx->nb) return CHFSI_ERR_BAD_INPUT;
    const double2* x = reinterpret_cast<const double2*>(psi_dev);
    double2* out = reinterpret_cast<double2*>(out_dev);
    if (!ctx->uspp) {
        s = apply_h_dev(ctx, x, out, nb, kEpiApply, nullptr);
    } else {
        s = sinv_h_parts(ctx, x, nb, nb);
        if (s) return s;
        cudaStream_t st = ctx->st;
        const size_t n = (size_t)nb * ctx->n_pw;
        count_launch();
        k_cheb_combine<double2><<<grid_for(n), 256, 0, st>>>(ctx->d_hpsi, ctx->d_sx, x, out, n,
                                                             ctx->d_coef, 0, nullptr);
        CK(cudaGetLastError());
    }
    if (s) return s;
    CK(cudaStreamSynchronize(ctx->st));
    return CHFSI_OK;
}

chfsi_status chfsi_apply_h(chfsi_ctx* ctx, const chfsi_c128* psi_dev, chfsi_c128* hpsi_dev, int nb) {
    chfsi_status s = ready(ctx);
    if (s) return s;
    if (!psi_dev || !hpsi_dev || nb <= 0 || nb > ctx->nb) return CHFSI_ERR_BAD_INPUT;
    s = apply_h_dev(ctx, reinterpret_cast<const double2*>(psi_dev),
                    reinterpret_cast<double2*>(hpsi_dev), nb, kEpiApply, nullptr);
    if (s) return s;
    CK(cudaStreamSynchronize(ctx->st));
    return CHFSI_OK;
}

static chfsi_status upload_eig(chfsi_ctx* ctx, const double* eig_prev, int n_eig,
                               const double** dev) {
    *dev = nullptr;
    if (!eig_prev || n_eig <= 0) return CHFSI_OK;
    if (n_eig > ctx->nb) return CHFSI_ERR_BAD_INPUT;
    CK(cudaMemcpyAsync(ctx->d_eig_prev, eig_prev, sizeof(double) * n_eig, cudaMemcpyHostToDevice,
                       ctx->st));
    *dev = ctx->d_eig_prev;
    return CHFSI_OK;
}

chfsi_status chfsi_chebyshev_filter(chfsi_ctx* ctx, int ndeg, const double* eig_prev, int n_eig) {
    chfsi_status s = ready(ctx);
    if (s) return s;
    if (!ctx->psi_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "psi not set");
    const double* ed = nullptr;
    s = upload_eig(ctx, eig_prev, n_eig, &ed);
    if (s) return s;
    s = filter_any(ctx, ndeg, ed, ed ? n_eig : 0);
    if (s) return s;
    return finish_diag(ctx, nullptr, false);
}

chfsi_status chfsi_rayleigh_ritz(chfsi_ctx* ctx, double* eig_out) {
    chfsi_status s = ready(ctx);
    if (s) return s;
    s = rr_any(ctx);
    if (s) return s;
    return finish_diag(ctx, eig_out, true);
}

chfsi_status chfsi_diagonalize(chfsi_ctx* ctx, int ndeg, const double* eig_prev, int n_eig,
                               double* eig_out) {
    chfsi_status s = ready(ctx);
    if (s) return s;
    if (!ctx->psi_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "psi not set");
    const double* ed = nullptr;
    s = upload_eig(ctx, eig_prev, n_eig, &ed);
    if (s) return s;
    s = filter_any(ctx, ndeg, ed, ed ? n_eig : 0);
    if (s) return s;
    s = rr_any(ctx);
    if (s) return s;
    return finish_diag(ctx, eig_out, true);
}

chfsi_status chfsi_get_bounds(chfsi_ctx* ctx, double* out4) {
    if (!ctx || !out4) return CHFSI_ERR_BAD_INPUT;
    for (int i = 0; i < 4; ++i) out4[i] = ctx->h_coef[i];
    return CHFSI_OK;
}

chfsi_status chfsi_get_filter_norms(chfsi_ctx* ctx, double* out, int n) {
    if (!ctx || !out) return CHFSI_ERR_BAD_INPUT;
    for (int i = 0; i < n && i < (int)ctx->h_nsq.size(); ++i) out[i] = std::sqrt(ctx->h_nsq[i]);
    return CHFSI_OK;
}

chfsi_status chfsi_create_from_system(const chfsi_system* sys, const chfsi_config* cfg,
                                      chfsi_ctx** out) {
    if (!sys || !out) return CHFSI_ERR_BAD_INPUT;
    const System& s = *reinterpret_cast<const System*>(sys);
    chfsi_dims d{};
    for (int i = 0; i < 3; ++i) d.ngrid[i] = s.ngrid[i];
    d.n_pw = s.n_pw; d.n_bands = s.n_bands; d.n_proj = s.n_proj; d.n_ions = s.n_ions_proj;
    chfsi_ctx* ctx = nullptr;
    chfsi_status st = chfsi_create(&d, cfg, &ctx);
    if (st) return st;
    auto bail = [&](chfsi_status e) { chfsi_destroy(ctx); return e; };
    if ((st = chfsi_set_basis(ctx, s.miller.data(), s.kinetic.data(), s.gmax))) return bail(st);
    if (s.n_proj > 0 &&
        (st = chfsi_set_projectors(ctx, reinterpret_cast<const chfsi_c128*>(s.beta.data()),
                                   s.proj_offsets.data(),
                                   reinterpret_cast<const chfsi_c128*>(s.dmat.data()))))
        return bail(st);
    if ((st = chfsi_set_psi(ctx, reinterpret_cast<const chfsi_c128*>(s.psi0.data())))) return bail(st);
    if ((st = chfsi_set_occupations(ctx, s.occ.data()))) return bail(st);
    double lat[9];
    std::memcpy(lat, s.lattice, sizeof(lat));
    if ((st = chfsi_set_cell(ctx, lat, s.e_ewald, s.n_atoms))) return bail(st);
    if (s.ngrid_density[0] != s.ngrid[0] || s.ngrid_density[1] != s.ngrid[1] ||
        s.ngrid_density[2] != s.ngrid[2])
        if ((st = chfsi_set_density_grid(ctx, s.ngrid_density))) return bail(st);
    if ((st = chfsi_set_vloc_g(ctx, reinterpret_cast<const chfsi_c128*>(s.vloc_g.data())))) return bail(st);
    if (s.uspp && s.n_proj > 0) {
        if ((st = chfsi_set_qmat(ctx, reinterpret_cast<const chfsi_c128*>(s.qmat.data()))))
            return bail(st);
        if ((st = chfsi_set_augmentation(ctx, s.pos.data(), s.q_width))) return bail(st);
    }
    {
        // ions of the analytic local model, for forces
        std::vector<double> rc(s.n_atoms, s.params.rc_loc);
        if ((st = chfsi_set_ions(ctx, s.n_atoms, s.pos.data(), s.zion.data(), rc.data(),
                                 s.params.kpt)))
            return bail(st);
    }
    // a usable V_eff before the first SCF step: V_loc alone
    if (cudaError_t e = cudaMemcpyAsync(ctx->d_veff_d, ctx->d_vloc, sizeof(double) * ctx->fng,
                                        cudaMemcpyDeviceToDevice, ctx->st))
        return bail(cuda_fail(e, "cudaMemcpyAsync(vloc)", __FILE__, __LINE__));
    project_veff(ctx);
    if (cudaError_t e = cudaStreamSynchronize(ctx->st))
        return bail(cuda_fail(e, "project_veff", __FILE__, __LINE__));
    ctx->veff_set = true;
    *out = ctx;
    return CHFSI_OK;
}

// ---------------------------------------------------------------- SCF pieces
chfsi_status chfsi_set_occupations(chfsi_ctx* ctx, const double* occ) {
    if (!ctx || !occ) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    ctx->occ.assign(occ, occ + ctx->nb);
    ctx->n_elec = 0.0;
    for (double f : ctx->occ) ctx->n_elec += f;
    CK(copy_sync(ctx->d_occ, occ, sizeof(double) * ctx->nb, cudaMemcpyHostToDevice, ctx->st));
    return CHFSI_OK;
}

chfsi_status chfsi_set_cell(chfsi_ctx* ctx, const double* lattice, double e_ewald, int n_atoms) {
    if (!ctx || !lattice || n_atoms <= 0) return CHFSI_ERR_BAD_INPUT;
    const double* a = lattice;
    const double vol = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    if (!(std::fabs(vol) > 0.0)) return CHFSI_ERR_BAD_INPUT;
    ctx->omega = std::fabs(vol);
    // b_i = 2 pi (a_j x a_k) / vol
    const double tp = 2.0 * 3.14159265358979323846 / vol;
    auto cross = [](const double* u, const double* v, double* w) {
        w[0] = u[1] * v[2] - u[2] * v[1];
        w[1] = u[2] * v[0] - u[0] * v[2];
        w[2] = u[0] * v[1] - u[1] * v[0];
    };
    cross(a + 3, a + 6, ctx->recip + 0);
    cross(a + 6, a + 0, ctx->recip + 3);
    cross(a + 0, a + 3, ctx->recip + 6);
    for (int i = 0; i < 9; ++i) ctx->recip[i] *= tp;
    std::memcpy(ctx->lattice, lattice, sizeof(ctx->lattice));
    ctx->e_ewald = e_ewald;
    ctx->n_atoms = n_atoms;
    return CHFSI_OK;
}

chfsi_status chfsi_set_vloc_g(chfsi_ctx* ctx, const chfsi_c128* vloc_g) {
    if (!ctx || !vloc_g) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    // natural G order of the wavefunction grid -> digit-reversed layout of
    // the density grid (zero where the density grid has G the wavefunction
    // grid lacks, and at the wavefunction grid's Nyquist planes when the
    // grids differ), then inverse transform
    std::vector<double2> h(ctx->fng, make_double2(0.0, 0.0));
    const double2* src = reinterpret_cast<const double2*>(vloc_g);
    const int n[3] = {ctx->nx, ctx->ny, ctx->nz};
    const int f[3] = {ctx->fnx, ctx->fny, ctx->fnz};
    auto fpos = [&](int d, int i) -> int {
        if (!ctx->fine) return ctx->fdr[d][i];
        const int hs = i >= (n[d] + 1) / 2 ? i - n[d] : i;
        if ((n[d] % 2 == 0) && i == n[d] / 2) return -1;
        return ctx->fdr[d][(hs + f[d]) % f[d]];
    };
    for (int iz = 0; iz < ctx->nz; ++iz) {
        const int pz = fpos(2, iz);
        if (pz < 0) continue;
        for (int iy = 0; iy < ctx->ny; ++iy) {
            const int py = fpos(1, iy);
            if (py < 0) continue;
            for (int ix = 0; ix < ctx->nx; ++ix) {
                const int px = fpos(0, ix);
                if (px < 0) continue;
                const size_t from = ix + (size_t)ctx->nx * (iy + (size_t)ctx->ny * iz);
                h[px + (size_t)ctx->fnx * (py + (size_t)ctx->fny * pz)] = src[from];
            }
        }
    }
    CK(copy_sync(ctx->d_cgrid, h.data(), sizeof(double2) * ctx->fng, cudaMemcpyHostToDevice, ctx->st));
    grid_fft3(ctx, ctx->d_cgrid, false);
    launch_take_real(ctx->d_cgrid, ctx->d_vloc, ctx->fng, ctx->st);
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaGetLastError());
    ctx->have_vloc = true;
    return CHFSI_OK;
}

chfsi_status chfsi_get_vloc(chfsi_ctx* ctx, double* out) {
    if (!ctx || !out) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    CK(copy_sync(out, ctx->d_vloc, sizeof(double) * ctx->fng, cudaMemcpyDeviceToHost, ctx->st));
    return CHFSI_OK;
}

chfsi_status chfsi_get_veff(chfsi_ctx* ctx, double* out) {
    if (!ctx || !out) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    CK(cudaStreamSynchronize(ctx->st));
    CK(copy_sync(out, ctx->d_veff, sizeof(double) * ctx->ng, cudaMemcpyDeviceToHost, ctx->st));
    return CHFSI_OK;
}

chfsi_status chfsi_construct_density(chfsi_ctx* ctx, double* rho_out) {
    if (!ctx || !ctx->basis_set) return CHFSI_ERR_BAD_INPUT;
    if (ctx->omega <= 0.0) return ctx->fail(CHFSI_ERR_BAD_INPUT, "cell not set");
    cudaSetDevice(ctx->device);
    chfsi_status s = density_dev(ctx, ctx->d_rho_out);
    if (s) return s;
    if (rho_out) {
        CK(cudaMemcpyAsync(rho_out, ctx->d_rho_out, sizeof(double) * ctx->fng, cudaMemcpyDeviceToHost, ctx->st));
    }
    CK(cudaStreamSynchronize(ctx->st));
    return CHFSI_OK;
}

chfsi_status chfsi_build_veff(chfsi_ctx* ctx, const double* rho, double* e2) {
    if (!ctx || !rho) return CHFSI_ERR_BAD_INPUT;
    if (!ctx->have_vloc || ctx->omega <= 0.0) return ctx->fail(CHFSI_ERR_BAD_INPUT, "V_loc / cell not set");
    cudaSetDevice(ctx->device);
    CK(cudaMemcpyAsync(ctx->d_rho_in, rho, sizeof(double) * ctx->fng, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemsetAsync(ctx->d_acc, 0, sizeof(double) * 8, ctx->st));
    chfsi_status s = build_veff_dev(ctx, ctx->d_rho_in, ctx->d_acc);
    if (s) return s;
    double acc[2];
    CK(cudaMemcpyAsync(acc, ctx->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->veff_set = true;
    if (e2) { e2[0] = acc[0]; e2[1] = acc[1]; }
    return CHFSI_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ SCF loop
namespace {

struct PulayState {
    int m = 0;            // entries in history
    int head = 0;         // ring slot of the oldest entry
    double M[kPulayMax][kPulayMax] = {};
};

// Fermi-Dirac occupations f_i = 2 / (1 + exp((e_i - mu)/kT)), mu by
// bisection on sum f = n_elec (the occupation step planned for
// construct_density, PROJECT_ROOT_PLAN.md:582-589; SmearingParams
// src/types.rs:204-211).  kT <= 0: aufbau.  Returns -kT S.
double fermi_occupations(const double* e, int n, double n_elec, double kT, double* f, double* mu_out) {
    if (kT <= 0.0) {
        double left = n_elec;
        for (int i = 0; i < n; ++i) {
            f[i] = std::min(2.0, std::max(0.0, left));
            left -= f[i];
        }
        if (mu_out) *mu_out = 0.0;
        return 0.0;
    }
    double lo = e[0], hi = e[0];
    for (int i = 0; i < n; ++i) { lo = std::min(lo, e[i]); hi = std::max(hi, e[i]); }
    lo -= 40.0 * kT + 1.0;
    hi += 40.0 * kT + 1.0;
    auto count = [&](double mu) {
        double s = 0.0;
        for (int i = 0; i < n; ++i) {
            const double x = std::min(700.0, std::max(-700.0, (e[i] - mu) / kT));
            s += 2.0 / (1.0 + std::exp(x));
        }
        return s;
    };
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (count(mid) < n_elec) lo = mid; else hi = mid;
    }
    const double mu = 0.5 * (lo + hi);
    double ts = 0.0;
    for (int i = 0; i < n; ++i) {
        const double x = std::min(700.0, std::max(-700.0, (e[i] - mu) / kT));
        f[i] = 2.0 / (1.0 + std::exp(x));
        const double ft = 0.5 * f[i];
        if (ft > 1e-300 && ft < 1.0 - 1e-16)
            ts += -2.0 * (ft * std::log(ft) + (1.0 - ft) * std::log(1.0 - ft));
    }
    if (mu_out) *mu_out = mu;
    return -kT * ts;
}

// Solve the bordered Pulay system; returns false if singular.
bool pulay_coefficients(int m, const double M[kPulayMax][kPulayMax], double* c) {
    const int n = m + 1;
    double A[kPulayMax + 1][kPulayMax + 2];
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) A[i][j] = M[i][j];
        A[i][m] = 1.0;
        A[i][n] = 0.0;
    }
    for (int j = 0; j < m; ++j) A[m][j] = 1.0;
    A[m][m] = 0.0;
    A[m][n] = 1.0;
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (std::fabs(A[r][col]) > std::fabs(A[piv][col])) piv = r;
        if (piv != col)
            for (int k = 0; k <= n; ++k) std::swap(A[col][k], A[piv][k]);
        const double d = A[col][col];
        if (d == 0.0) return false;
        for (int r = col + 1; r < n; ++r) {
            const double f = A[r][col] / d;
            for (int k = col; k <= n; ++k) A[r][k] -= f * A[col][k];
        }
    }
    double x[kPulayMax + 1];
    for (int i = n - 1; i >= 0; --i) {
        double s = A[i][n];
        for (int k = i + 1; k < n; ++k) s -= A[i][k] * x[k];
        x[i] = s / A[i][i];
    }
    for (int i = 0; i < m; ++i) c[i] = x[i];
    return true;
}

}  // namespace

extern "C" chfsi_status chfsi_scf_run(chfsi_ctx* ctx, const chfsi_scf_params* p,
                                      chfsi_scf_result* r) {
    if (!ctx || !p || !r) return CHFSI_ERR_BAD_INPUT;
    if (!ctx->basis_set || !ctx->psi_set || !ctx->have_vloc || ctx->omega <= 0.0)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "context not fully initialised");
    if (ctx->np > 0 && !ctx->proj_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "projectors not set");
    if (p->max_hist < 1 || p->max_hist > kPulayMax || p->max_iter < 1 || p->ndeg < 0)
        return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    const bool learned = p->mixer == CHFSI_MIXER_LEARNED || p->mixer == CHFSI_MIXER_LEARNED_PULAY;
    if (p->mixer < CHFSI_MIXER_PULAY || p->mixer > CHFSI_MIXER_LEARNED_PULAY)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "unknown mixer");
    if (learned && !ctx->mixer)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "learned mixer requested but none set (chfsi_set_mixer)");
    if (learned && ctx->mixer->mlp.device != ctx->device)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "mixer lives on another device");
    double* r_energies = r->energies;
    double* r_eigs = r->eigenvalues;
    double* r_res = r->residuals;
    std::memset(r, 0, sizeof(*r));
    r->energies = r_energies;
    r->eigenvalues = r_eigs;
    r->residuals = r_res;
    const size_t ng = ctx->fng;  // density grid
    const double dv = ctx->omega / (double)ng;
    cudaStream_t st = ctx->st;
    const double n_elec = ctx->n_elec;
    const bool restart = p->restart != 0 && ctx->scf_done;
    if (!restart) {
        count_launch();
        k_fill<<<grid_for(ng), 256, 0, st>>>(ctx->d_rho_in, ng, n_elec / ctx->omega);
    }
    PulayState ps;
    chfsi_status s = ensure_pinned(ctx, (size_t)ctx->nb + 64 + ctx->max_deg);
    if (s) return s;
    if (learned && (s = alloc_mix(ctx))) return s;
    MixRing ring;
    int low_mixed = 0;  // mixed iterations in a row with |dE| below the switch
    std::vector<double> mixed_deig;  // eigenvalue changes of the mixed iterations
    constexpr int kMaxReverts = 3;
    int reverts = 0;
    bool have_prev = false, fell_back = false;
    int rises = 0;
    bool restart_pulay = false;
    double r_prev = -1.0;
    constexpr int kStallWindow = 10;
    std::vector<double> rhist;
    std::vector<double> eig(ctx->nb), eig_prev(ctx->nb);
    bool have_eig = restart;
    if (restart)
        CK(copy_sync(eig.data(), ctx->d_eig, sizeof(double) * ctx->nb, cudaMemcpyDeviceToHost, st));
    eig_prev = eig;
    double e_prev = restart ? ctx->scf_e_last : 0.0;
    chfsi_status status = CHFSI_NOT_CONVERGED;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, st);
    int it;
    for (it = 1; it <= p->max_iter; ++it) {
        // build_v_eff (scf.rs:157)
        CK(cudaMemsetAsync(ctx->d_acc, 0, sizeof(double) * 8, st));
        s = build_veff_dev(ctx, ctx->d_rho_in, ctx->d_acc);
        if (!s) s = screen_dmat(ctx);
        if (s) { status = s; break; }
        ctx->veff_set = true;
        // diagonalize (scf.rs:169)
        const int passes = it == 1 && !restart ? std::max(1, p->first_passes) : 1;
        for (int q = 0; q < passes; ++q) {
            const bool mixed_pass = ctx->mixed_active;
            const size_t npsi = (size_t)ctx->nb * ctx->n_pw;
            if (mixed_pass) {
                // psi and the eigenvalues the bounds come from, for an FP64 retry
                if (!ctx->d_psi_save) CK(dalloc(&ctx->d_psi_save, npsi + (ctx->nb + 1) / 2));
                CK(cudaMemcpyAsync(ctx->d_psi_save, ctx->d_psi, npsi * sizeof(double2),
                                   cudaMemcpyDeviceToDevice, st));
                CK(cudaMemcpyAsync(ctx->d_psi_save + npsi, ctx->d_eig, ctx->nb * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st));
            }
            s = filter_any(ctx, p->ndeg, have_eig ? ctx->d_eig : nullptr, have_eig ? ctx->nb : 0);
            if (!s) s = rr_any(ctx);
            if (!s) s = finish_diag(ctx, eig.data(), true);
            if (s && mixed_pass && (s == CHFSI_ERR_RR_FAILED || s == CHFSI_ERR_CHEB_DIVERGED)) {
                // the FP32 filter lost the conditioning of the subspace (the
                // overlap is no longer positive definite): redo this pass in FP64
                // from the saved psi and eigenvalues (the failed pass's
                // Rayleigh-Ritz has overwritten both)
                if (p->verbose) {
                    std::fprintf(stderr, "scf %3d pass %d fp32 failed: lm %.4f cut %.4f: %s; |psi_k|:", it,
                                 q, ctx->h_coef[0], ctx->h_coef[1], g_last_error.c_str());
                    for (double v : ctx->h_nsq) std::fprintf(stderr, " %.3e", std::sqrt(v));
                    std::fprintf(stderr, "\n");
                }
                CK(cudaMemcpyAsync(ctx->d_psi, ctx->d_psi_save, npsi * sizeof(double2),
                                   cudaMemcpyDeviceToDevice, st));
                CK(cudaMemcpyAsync(ctx->d_eig, ctx->d_psi_save + npsi, ctx->nb * sizeof(double),
                                   cudaMemcpyDeviceToDevice, st));
                ctx->mixed_active = false;
                s = filter_any(ctx, p->ndeg, have_eig ? ctx->d_eig : nullptr, have_eig ? ctx->nb : 0);
                if (!s) s = rr_any(ctx);
                if (!s) s = finish_diag(ctx, eig.data(), true);
                ctx->mixed_active = true;
                ++r->n_fp64_retries;
                if (p->verbose)
                    std::fprintf(stderr, "scf %3d pass %d: mixed pass failed, redone in FP64 -> %d\n",
                                 it, q, (int)s);
            }
            if (p->verbose)
                std::fprintf(stderr, "scf %3d pass %d %s status %d eig [%.5f, %.5f] lm %.4f cut %.4f %s\n",
                             it, q, ctx->last_pass_fp32 ? "fp32" : "fp64", (int)s, eig[0],
                             eig[ctx->nb - 1], ctx->h_coef[0], ctx->h_coef[1],
                             s ? g_last_error.c_str() : "");
            if (s) break;
            have_eig = true;
        }
        if (!s && p->cg_steps > 0) {
            // a few band-CG steps per band after the filter; the band energies
            // feed the occupations and the next filter's bounds
            int nc = 0;
            s = band_cg_dev(ctx, p->cg_steps, 1e-10, eig.data(), nullptr, &nc);
            if (!s) {
                CK(cudaMemcpyAsync(ctx->d_eig, eig.data(), sizeof(double) * ctx->nb,
                                   cudaMemcpyHostToDevice, st));
                CK(cudaStreamSynchronize(st));
            }
        }
        if (s) { status = s; break; }
        // occupations from the new eigenvalues, then construct_density (scf.rs:275)
        double mu = 0.0;
        const double e_ts = fermi_occupations(eig.data(), ctx->nb, n_elec, p->kT, ctx->occ.data(), &mu);
        CK(cudaMemcpyAsync(ctx->d_occ, ctx->occ.data(), sizeof(double) * ctx->nb, cudaMemcpyHostToDevice, st));
        s = density_dev(ctx, ctx->d_rho_out);
        if (s) { status = s; break; }
        // energy of rho_out: E_H, E_xc, double counting
        CK(cudaMemsetAsync(ctx->d_acc, 0, sizeof(double) * 8, st));
        launch_real_to_complex(ctx->d_rho_out, ctx->d_cgrid, ng, st);
        grid_fft3(ctx, ctx->d_cgrid, true);
        if (ctx->xc == CHFSI_XC_PBE) gga_gradient(ctx);
        launch_hartree_gspace(ctx->d_cgrid, grid_recip(ctx), ctx->omega, ctx->d_acc + 0, st);
        launch_energy_terms(ctx->d_rho_out, ctx->d_veff_d, ctx->d_vloc, ng, dv, ctx->d_acc + 1,
                            ctx->d_acc + 2, st);
        if (ctx->xc == CHFSI_XC_PBE) {
            // E_xc of rho_out from the gradient formed above (the LDA sum is discarded)
            CK(cudaMemsetAsync(ctx->d_acc + 1, 0, sizeof(double), st));
            double2* g0 = ctx->d_gga;
            launch_pbe_point(ctx->d_rho_out, g0, g0 + ng, g0 + 2 * ng, nullptr, ng, dv,
                             ctx->d_acc + 1, false, st);
        }
        CK(cudaGetLastError());
        double acc[3];
        CK(cudaMemcpyAsync(acc, ctx->d_acc, sizeof(acc), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double eband = 0.0;
        for (int b = 0; b < ctx->nb; ++b) eband += ctx->occ[b] * eig[b];
        const double etot = eband - acc[2] + acc[0] + acc[1] + ctx->e_ewald + e_ts;
        r->e_entropy = e_ts;
        r->mu = mu;
        if (r->energies) r->energies[it - 1] = etot;
        r->e_band = eband; r->e_hartree = acc[0]; r->e_xc = acc[1]; r->e_dc = acc[2];
        r->e_total = etot;
        r->n_iter = it;
        if (p->verbose) {
            // integrated charge of rho_out against the electron count
            std::vector<double> h(ng);
            CK(cudaMemcpyAsync(h.data(), ctx->d_rho_out, sizeof(double) * ng, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            double q = 0.0;
            for (double v : h) q += v;
            std::fprintf(stderr,
                         "scf %3d %s E %.10f dE/atom %.3e eig [%.5f, %.5f] bounds lm %.4f cut %.4f "
                         "retries %d learned %d charge-N %.3e eband %.8f\n",
                         it, ctx->mixed_active ? "mixed" : "fp64 ", etot,
                         it > 1 ? std::fabs(etot - e_prev) / ctx->n_atoms : 0.0, eig[0],
                         eig[ctx->nb - 1], ctx->h_coef[0], ctx->h_coef[1], r->n_fp64_retries,
                         r->n_iter_learned, q * dv - n_elec, eband);
        }
        if (p->trace) {
            double* tr = p->trace + (size_t)2 * (it - 1) * ng;
            CK(cudaMemcpyAsync(tr, ctx->d_rho_in, sizeof(double) * ng, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(tr + ng, ctx->d_rho_out, sizeof(double) * ng, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
        }
        // check (scf.rs:328): |dE| per atom below tolerance, declared on an
        // FP64 iteration only (the last filter pass before convergence is
        // FP64).  Mixed passes run an FP64 Rayleigh-Ritz, so their energies
        // carry no precision bias and the change from a mixed iteration to
        // the FP64 one after it counts.
        const double de = it > 1 || restart ? std::fabs(etot - e_prev) / ctx->n_atoms : 1e300;
        // largest change of an occupied eigenvalue since the previous iteration
        double deig = 0.0;
        if (it > 1 || restart) {
            for (int b = 0; b < ctx->nb; ++b)
                if (ctx->occ[b] > 0.01) deig = std::max(deig, std::fabs(eig[b] - eig_prev[b]));
        } else {
            deig = 1e300;
        }
        eig_prev = eig;
        const bool eig_ok = p->tol_eig <= 0.0 || deig < p->tol_eig;
        // the mixed iterations' eigenvalue changes carry ~2e-7 Ha of FP32
        // noise (measured on the 216-atom cell): the switch to FP64 takes at
        // least twice the tolerance, the FP64 iterations after it the tolerance
        const double sw_eig = std::max(2.0 * p->tol_eig, p->fp64_switch_eig);
        const bool eig_near = p->tol_eig <= 0.0 || deig < sw_eig;
        if (ctx->mixed_active) ++r->n_iter_mixed;
        if (p->verbose && p->tol_eig > 0.0)
            std::fprintf(stderr, "scf %3d max |d eig_occ| %.3e\n", it, deig);
        if (de < p->tol_per_atom && eig_ok && !ctx->mixed_active) {
            status = CHFSI_OK;
            e_prev = etot;
            break;
        }
        // switch to FP64 after two mixed iterations in a row with |dE| below
        // the switch threshold (a single one falls below it by chance where
        // the energy turns); an FP64 iteration whose |dE| is still ten times
        // above it hands the run back to mixed precision (at most kMaxReverts
        // times, so the two can never alternate for ever).  Eigenvalue changes
        // do not hand a run back: the first FP64 iterations move the
        // eigenvalues by up to ~1e-4 Ha while the density relaxes from the
        // mixed-precision iterate (its FP32 rounding, ~1e-7 relative in the
        // density, shifts V_eff), which is the work the FP64 iterations do.
        // The mixed iterations' eigenvalue changes level off at the FP32
        // filter's floor: once the best change of the last eight mixed
        // iterations is below three times the switch but not below half the
        // best of the mixed iterations before them (a plateau), the eigenvalue
        // test of the switch counts as met.
        const double sw = std::max(p->fp64_switch_per_atom, p->tol_per_atom);
        if (ctx->mixed_active) {
            if (p->tol_eig > 0.0 && it > 1) mixed_deig.push_back(deig);
            bool plateau = false;
            const int nm = (int)mixed_deig.size();
            if (nm >= 12) {
                const double recent = *std::min_element(mixed_deig.end() - 8, mixed_deig.end());
                const double before = *std::min_element(mixed_deig.begin(), mixed_deig.end() - 8);
                plateau = recent < 3.0 * sw_eig && recent > 0.5 * before;
            }
            low_mixed = de < sw && (eig_near || plateau) ? low_mixed + 1 : 0;
            if (low_mixed >= 2) {
                if (p->verbose)
                    std::fprintf(stderr, "scf %3d: FP64 filter from here (%s)\n", it,
                                 eig_near ? "eigenvalue changes below the switch"
                                          : "mixed eigenvalue changes level off");
                ctx->mixed_active = false;
                low_mixed = 0;
                mixed_deig.clear();
            }
        } else if (ctx->mixed && de > 10.0 * sw &&
                   reverts < kMaxReverts) {
            ctx->mixed_active = true;
            ++reverts;
            if (p->verbose) std::fprintf(stderr, "scf %3d: |dE| %.3e, back to mixed precision\n", it, de);
        }
        e_prev = etot;
        // mix (mixing.rs:24): Pulay over (rho_in, rho_out - rho_in)
        if (ps.m == p->max_hist) {
            // drop the oldest entry
            for (int i = 0; i + 1 < ps.m; ++i)
                for (int j = 0; j + 1 < ps.m; ++j) ps.M[i][j] = ps.M[i + 1][j + 1];
            ps.head = (ps.head + 1) % kPulayMax;
            --ps.m;
        }
        const int slot = (ps.head + ps.m) % kPulayMax;
        double* hr = ctx->d_hist + (size_t)slot * ng;
        double* hres = ctx->d_hist + (size_t)(kPulayMax + slot) * ng;
        pulay_push(ctx->d_rho_in, ctx->d_rho_out, hr, hres, ng, st);
        ++ps.m;
        // ordered pointer lists (oldest first): residual pointers for dots,
        // then the combine needs both lists
        std::vector<double*> lr(ps.m), lres(ps.m);
        for (int i = 0; i < ps.m; ++i) {
            const int sl = (ps.head + i) % kPulayMax;
            lr[i] = ctx->d_hist + (size_t)sl * ng;
            lres[i] = ctx->d_hist + (size_t)(kPulayMax + sl) * ng;
        }
        CK(cudaMemcpyAsync(ctx->d_hist_ptrs, lres.data(), sizeof(double*) * ps.m, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(ctx->d_hist_ptrs + kPulayMax, lr.data(), sizeof(double*) * ps.m, cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(ctx->d_dots, 0, sizeof(double) * kPulayMax, st));
        dots(hres, ctx->d_hist_ptrs, ps.m, ng, ctx->d_dots, st);
        double dd[kPulayMax];
        CK(cudaMemcpyAsync(dd, ctx->d_dots, sizeof(double) * ps.m, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        const int nw = ps.m - 1;
        for (int j = 0; j < ps.m; ++j) { ps.M[nw][j] = dd[j]; ps.M[j][nw] = dd[j]; }
        double c[kPulayMax] = {};
        if (ps.m == 1 || !pulay_coefficients(ps.m, ps.M, c)) {
            for (int j = 0; j < ps.m; ++j) c[j] = 0.0;
            c[ps.m - 1] = 1.0;
        }
        // residual norm |rho_out - rho_in|_2 and the fallback rule of the
        // learned mixers: two rises in a row hand the run to Pulay
        const double rnorm = std::sqrt(std::max(0.0, dd[nw]) * dv);
        if (r->residuals) r->residuals[it - 1] = rnorm;
        rhist.push_back(rnorm);
        if (learned && !fell_back) {
            rises = (r_prev >= 0.0 && rnorm > r_prev) ? rises + 1 : 0;
            // a learned run that stalls (the best residual of the last ten
            // iterations is not below half the best before them) is handed
            // over as well: the network's steps stop helping near convergence
            bool stalled = false;
            const int nh = (int)rhist.size();
            if (nh >= kStallWindow + 3) {
                const double recent = *std::min_element(rhist.end() - kStallWindow, rhist.end());
                const double before = *std::min_element(rhist.begin(), rhist.end() - kStallWindow);
                stalled = recent > 0.5 * before;
            }
            if (rises >= 2 || stalled) {
                if (p->verbose)
                    std::fprintf(stderr, "scf %3d: learned mixer %s, Pulay from here\n", it,
                                 rises >= 2 ? "residual rose twice" : "stalled");
                // Pulay takes over from the current input density with a fresh
                // history: the learned steps' entries span a subspace that
                // stalls the extrapolation (observed on the 216-atom cell)
                fell_back = true;
                restart_pulay = true;
            }
        }
        r_prev = rnorm;
        if (learned) ring_push(ctx, ring, ctx->d_rho_out, ctx->d_rho_in);
        double2* Dg = nullptr;
        if (learned && !fell_back) {
            if (have_prev) {
                Dg = mix_grid(ctx, kGridD);
                launch_diff_complex(ctx->d_rho_in, mix_real(ctx, 0), Dg, ng, st);
                grid_fft3(ctx, Dg, true);
            }
            if ((s = mix_features(ctx, ring, Dg, nullptr))) { status = s; break; }
            mlp_forward(ctx->mixer->mlp, ctx->d_mix_x, 1, mix_y(ctx), st);
            // a network whose output is not finite (diverged weights, a NaN in
            // the residual history) hands the run to Pulay like a residual rise
            float yh[kMixOut];
            CK(cudaMemcpyAsync(yh, mix_y(ctx), sizeof(yh), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            for (float v : yh)
                if (!std::isfinite(v)) {
                    fell_back = true;
                    restart_pulay = true;
                    if (p->verbose)
                        std::fprintf(stderr, "scf %3d: learned mixer output not finite, Pulay from here\n", it);
                    break;
                }
        }
        if (restart_pulay) {
            // keep only the newest entry (rho_in, R): a linear-mixing step now,
            // Pulay extrapolation over a new history from the next iteration
            const int newest = (ps.head + ps.m - 1) % kPulayMax;
            ps.head = newest;
            ps.m = 1;
            ps.M[0][0] = dd[nw];
            for (int j = 0; j < kPulayMax; ++j) c[j] = 0.0;
            c[0] = 1.0;
            double* pr = ctx->d_hist + (size_t)newest * ng;
            double* pres = ctx->d_hist + (size_t)(kPulayMax + newest) * ng;
            CK(cudaMemcpyAsync(ctx->d_hist_ptrs, &pres, sizeof(double*), cudaMemcpyHostToDevice, st));
            CK(cudaMemcpyAsync(ctx->d_hist_ptrs + kPulayMax, &pr, sizeof(double*), cudaMemcpyHostToDevice, st));
            restart_pulay = false;
        }
        if (!learned || fell_back) {
            pulay_combine(ctx->d_hist_ptrs + kPulayMax, ctx->d_hist_ptrs, ps.m, c, p->alpha, ng,
                          ctx->d_rho_next, st);
        } else {
            double2* W = mix_grid(ctx, kGridW);
            if (p->mixer == CHFSI_MIXER_LEARNED) {
                // rho_in + a_s R_0 + b_s D per shell
                launch_diff_complex(ctx->d_rho_in, nullptr, W, ng, st);
                grid_fft3(ctx, W, true);
                launch_shell_update(W, ring.slot(ctx, 0), Dg, mix_y(ctx), ctx->d_shell, ng, st);
            } else {
                // Pulay extrapolation with a_s in place of alpha:
                // sum c_j rho_j + a_s (sum c_j R_j)
                double* rbar = mix_real(ctx, 2);
                pulay_combine(ctx->d_hist_ptrs + kPulayMax, ctx->d_hist_ptrs, ps.m, c, 0.0, ng,
                              ctx->d_rho_next, st);
                pulay_combine(ctx->d_hist_ptrs, ctx->d_hist_ptrs, ps.m, c, 0.0, ng, rbar, st);
                double2* Rg = mix_grid(ctx, kGridE);
                launch_diff_complex(ctx->d_rho_next, nullptr, W, ng, st);
                grid_fft3(ctx, W, true);
                launch_diff_complex(rbar, nullptr, Rg, ng, st);
                grid_fft3(ctx, Rg, true);
                launch_shell_update(W, Rg, nullptr, mix_y(ctx), ctx->d_shell, ng, st);
            }
            grid_fft3(ctx, W, false);
            launch_take_real_scaled(W, ctx->d_rho_next, ng, 1.0 / (double)ng, st);
            ++r->n_iter_learned;
        }
        if (learned) {
            CK(cudaMemcpyAsync(mix_real(ctx, 0), ctx->d_rho_in, sizeof(double) * ng,
                               cudaMemcpyDeviceToDevice, st));
            have_prev = true;
        }
        std::swap(ctx->d_rho_in, ctx->d_rho_next);
        CK(cudaGetLastError());
    }
    ctx->mixed_active = ctx->mixed;
    ctx->scf_done = have_eig;
    ctx->scf_e_last = e_prev;
    r->fell_back = fell_back ? 1 : 0;
    cudaEventRecord(t1, st);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    r->seconds = ms * 1e-3;
    r->status = status;
    if (r->eigenvalues) std::memcpy(r->eigenvalues, eig.data(), sizeof(double) * ctx->nb);
    return status;
}

extern "C" chfsi_status chfsi_set_xc(chfsi_ctx* ctx, int functional) {
    if (!ctx) return CHFSI_ERR_BAD_INPUT;
    if (functional != CHFSI_XC_LDA_PZ && functional != CHFSI_XC_PBE)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "unknown exchange-correlation functional");
    cudaSetDevice(ctx->device);
    if (functional == CHFSI_XC_PBE) {
        if (!ctx->d_gga) CK(dalloc(&ctx->d_gga, 3 * ctx->fng));
        if (!ctx->d_gga_v1) CK(dalloc(&ctx->d_gga_v1, ctx->fng));
    }
    ctx->xc = functional;
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_set_ions(chfsi_ctx* ctx, int n_atoms, const double* positions,
                                       const double* zion, const double* rc_loc, const double* kpt) {
    if (!ctx || n_atoms <= 0 || !positions || !zion || !rc_loc)
        return CHFSI_ERR_BAD_INPUT;
    if (ctx->np > 0 && ctx->nions > n_atoms)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "more ions with projectors than atoms");
    cudaSetDevice(ctx->device);
    ctx->n_ion_atoms = n_atoms;
    ctx->atom_pos.assign(positions, positions + 3 * (size_t)n_atoms);
    ctx->atom_z.assign(zion, zion + n_atoms);
    ctx->atom_rc.assign(rc_loc, rc_loc + n_atoms);
    for (int d = 0; d < 3; ++d) ctx->ion_kpt[d] = kpt ? kpt[d] : 0.0;
    if (ctx->d_ion) cudaFree(ctx->d_ion);
    if (ctx->d_atom_of_ion) cudaFree(ctx->d_atom_of_ion);
    ctx->d_ion = nullptr;
    ctx->d_atom_of_ion = nullptr;
    CK(dalloc(&ctx->d_ion, 8 * (size_t)n_atoms));
    std::vector<double> h(5 * (size_t)n_atoms);
    std::memcpy(h.data(), positions, sizeof(double) * 3 * n_atoms);
    std::memcpy(h.data() + 3 * n_atoms, zion, sizeof(double) * n_atoms);
    std::memcpy(h.data() + 4 * n_atoms, rc_loc, sizeof(double) * n_atoms);
    CK(copy_sync(ctx->d_ion, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, ctx->st));
    if (ctx->nions > 0) {
        std::vector<int> map(ctx->nions);
        for (int i = 0; i < ctx->nions; ++i) map[i] = i;
        CK(dalloc(&ctx->d_atom_of_ion, ctx->nions));
        CK(copy_sync(ctx->d_atom_of_ion, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice,
                     ctx->st));
    }
    if (ctx->d_qvec) { cudaFree(ctx->d_qvec); ctx->d_qvec = nullptr; }
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_forces(chfsi_ctx* ctx, double* forces) {
    if (!ctx || !forces) return CHFSI_ERR_BAD_INPUT;
    if (ctx->n_ion_atoms == 0) return ctx->fail(CHFSI_ERR_BAD_INPUT, "ions not set (chfsi_set_ions)");
    if (ctx->omega <= 0.0 || !ctx->basis_set || !ctx->psi_set)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "context not fully initialised");
    if (ctx->uspp)
        return ctx->fail(CHFSI_ERR_NOT_IMPLEMENTED, "forces of ultrasoft cells are not built");
    if (ctx->fng != ctx->ng)
        return ctx->fail(CHFSI_ERR_NOT_IMPLEMENTED, "forces need the density grid equal to the FFT grid");
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->st;
    const int na = ctx->n_ion_atoms, nb = ctx->nb, npw = ctx->n_pw, np = ctx->np;
    double* d_pos = ctx->d_ion;
    double* d_z = d_pos + 3 * na;
    double* d_rc = d_z + na;
    double* d_f = d_rc + na;
    CK(cudaMemsetAsync(d_f, 0, sizeof(double) * 3 * na, st));
    // local part from rho_out in G space
    const size_t ng = ctx->fng;
    launch_real_to_complex(ctx->d_rho_out, ctx->d_cgrid, ng, st);
    grid_fft3(ctx, ctx->d_cgrid, true);
    const int wave[3] = {ctx->nx, ctx->ny, ctx->nz};
    launch_force_local(ctx->d_cgrid, grid_recip(ctx), wave, d_pos, d_z, d_rc, na, ctx->omega, d_f, st);
    // non-local part: C = beta^H psi, B_a = beta^H (q_a psi)
    if (np > 0) {
        if (!ctx->d_qvec) {
            std::vector<double> q(3 * (size_t)npw);
            for (int i = 0; i < npw; ++i) {
                const double m[3] = {ctx->miller_ctx[3 * (size_t)i] + ctx->ion_kpt[0],
                                     ctx->miller_ctx[3 * (size_t)i + 1] + ctx->ion_kpt[1],
                                     ctx->miller_ctx[3 * (size_t)i + 2] + ctx->ion_kpt[2]};
                for (int d = 0; d < 3; ++d)
                    q[(size_t)d * npw + i] = m[0] * ctx->recip[d] + m[1] * ctx->recip[3 + d] +
                                             m[2] * ctx->recip[6 + d];
            }
            CK(dalloc(&ctx->d_qvec, q.size()));
            CK(copy_sync(ctx->d_qvec, q.data(), sizeof(double) * q.size(), cudaMemcpyHostToDevice, st));
        }
        gemm_cn(ctx->d_beta, npw, ctx->d_psi, npw, np, nb, npw, ctx->d_part, ctx->d_cp, st);
        for (int a = 0; a < 3; ++a) {
            launch_scale_pw(ctx->d_psi, ctx->d_qvec + (size_t)a * npw, npw, nb, ctx->d_hpsi, st);
            gemm_cn(ctx->d_beta, npw, ctx->d_hpsi, npw, np, nb, npw, ctx->d_part, ctx->d_cd, st);
            launch_force_nl(ctx->d_cp, ctx->d_cd, nb, ctx->d_occ, ctx->d_poff, ctx->d_doff,
                            ctx->d_dmat, ctx->nions, a, ctx->d_atom_of_ion, d_f, st);
        }
    }
    CK(cudaGetLastError());
    std::vector<double> f(3 * (size_t)na);
    CK(copy_sync(f.data(), d_f, sizeof(double) * f.size(), cudaMemcpyDeviceToHost, st));
    // ion-ion part
    double lat[9];
    for (int i = 0; i < 9; ++i) lat[i] = ctx->lattice[i];
    std::vector<double> fe;
    ewald_forces(lat, ctx->recip, ctx->atom_pos, ctx->atom_z, fe);
    for (size_t i = 0; i < f.size(); ++i) forces[i] = f[i] + fe[i];
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_get_density(chfsi_ctx* ctx, double* rho) {
    if (!ctx || !rho) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(ctx->device);
    CK(cudaStreamSynchronize(ctx->st));
    CK(copy_sync(rho, ctx->d_rho_out, sizeof(double) * ctx->fng, cudaMemcpyDeviceToHost, ctx->st));
    return CHFSI_OK;
}

// Density (augmentation) grid: must be set before V_loc, the cell's
// augmentation and any density work; it may not be coarser than the
// wavefunction grid.
extern "C" chfsi_status chfsi_set_density_grid(chfsi_ctx* ctx, const int* ngrid) {
    if (!ctx || !ngrid) return CHFSI_ERR_BAD_INPUT;
    const int n[3] = {ctx->nx, ctx->ny, ctx->nz};
    for (int d = 0; d < 3; ++d)
        if (ngrid[d] < n[d]) return ctx->fail(CHFSI_ERR_BAD_INPUT, "density grid coarser than the wavefunction grid");
    cudaSetDevice(ctx->device);
    AxisPlan pl[3];
    for (int d = 0; d < 3; ++d)
        if (!plan_axis(ngrid[d], pl[d]))
            return ctx->fail(CHFSI_ERR_BAD_INPUT, "density grid dimensions must be 2,3,5-smooth");
    CK(cudaStreamSynchronize(ctx->st));
    ctx->fnx = ngrid[0]; ctx->fny = ngrid[1]; ctx->fnz = ngrid[2];
    ctx->fng = (size_t)ngrid[0] * ngrid[1] * ngrid[2];
    ctx->fax = pl[0]; ctx->fay = pl[1]; ctx->faz = pl[2];
    digit_reversal(ctx->fax, ctx->fdr[0]);
    digit_reversal(ctx->fay, ctx->fdr[1]);
    digit_reversal(ctx->faz, ctx->fdr[2]);
    ctx->fine = ngrid[0] != n[0] || ngrid[1] != n[1] || ngrid[2] != n[2];
    chfsi_status s = alloc_density(ctx);
    if (s) return s;
    // G vectors the two grids share: every wavefunction-grid frequency except
    // the Nyquist planes of even axes
    if (ctx->d_gmap_w) cudaFree(ctx->d_gmap_w);
    if (ctx->d_gmap_f) cudaFree(ctx->d_gmap_f);
    ctx->d_gmap_w = ctx->d_gmap_f = nullptr;
    ctx->n_gmap = 0;
    if (ctx->fine) {
        std::vector<int> wp, fp;
        const int f[3] = {ctx->fnx, ctx->fny, ctx->fnz};
        auto sgn = [&](int d, int i) { return i >= (n[d] + 1) / 2 ? i - n[d] : i; };
        auto nyq = [&](int d, int i) { return n[d] % 2 == 0 && i == n[d] / 2; };
        for (int iz = 0; iz < n[2]; ++iz) {
            if (nyq(2, iz)) continue;
            for (int iy = 0; iy < n[1]; ++iy) {
                if (nyq(1, iy)) continue;
                for (int ix = 0; ix < n[0]; ++ix) {
                    if (nyq(0, ix)) continue;
                    const int w = ctx->dr[0][ix] + n[0] * (ctx->dr[1][iy] + n[1] * ctx->dr[2][iz]);
                    const int fx = ctx->fdr[0][(sgn(0, ix) + f[0]) % f[0]];
                    const int fy = ctx->fdr[1][(sgn(1, iy) + f[1]) % f[1]];
                    const int fz = ctx->fdr[2][(sgn(2, iz) + f[2]) % f[2]];
                    wp.push_back(w);
                    fp.push_back(fx + f[0] * (fy + f[1] * fz));
                }
            }
        }
        ctx->n_gmap = (int)wp.size();
        CK(dalloc(&ctx->d_gmap_w, wp.size()));
        CK(dalloc(&ctx->d_gmap_f, fp.size()));
        CK(copy_sync(ctx->d_gmap_w, wp.data(), wp.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
        CK(copy_sync(ctx->d_gmap_f, fp.data(), fp.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    }
    return upload_phases(ctx);
}

// Jacobi sweeps of the last Rayleigh-Ritz eigensolve (diagnostics).
extern "C" chfsi_status chfsi_get_rr_sweeps(chfsi_ctx* ctx, int* sweeps) {
    if (!ctx || !sweeps) return CHFSI_ERR_BAD_INPUT;
    *sweeps = ctx->last_sweeps;
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_get_density_grid(chfsi_ctx* ctx, int* ngrid) {
    if (!ctx || !ngrid) return CHFSI_ERR_BAD_INPUT;
    ngrid[0] = ctx->fnx; ngrid[1] = ctx->fny; ngrid[2] = ctx->fnz;
    return CHFSI_OK;
}

// Ultrasoft augmentation charges Q_ij(r) = q_ij g(|r - R_I|) (unit Gaussian
// of the given width) for the ions that carry projectors; needs the cell,
// the projectors and q (chfsi_set_qmat).
extern "C" chfsi_status chfsi_set_augmentation(chfsi_ctx* ctx, const double* positions,
                                               double width) {
    if (!ctx || !positions || !(width > 0.0)) return CHFSI_ERR_BAD_INPUT;
    if (!ctx->uspp || !ctx->proj_set || ctx->omega <= 0.0)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "augmentation needs the cell, projectors and q");
    cudaSetDevice(ctx->device);
    ctx->ion_pos.assign(positions, positions + 3 * (size_t)ctx->nions);
    ctx->aug_width = width;
    ctx->aug = true;
    if (!ctx->d_cion) CK(dalloc(&ctx->d_cion, (size_t)ctx->nions));
    if (!ctx->d_vion) CK(dalloc(&ctx->d_vion, (size_t)ctx->nions));
    return upload_phases(ctx);
}

// ---------------------------------------------------------------- batches
// Many independent contexts (k-points of one cell, independent cells of
// uneven size) advanced together: one diagonalisation pass of every member
// (FP32 filter with bounds from the member's previous eigenvalues, FP64
// Rayleigh-Ritz) is captured once into a CUDA graph, each member on its own
// stream forked from and joined to the batch's origin stream, so a replay is
// one graph launch with the members' kernels free to overlap on the SMs.
struct chfsi_batch {
    std::vector<chfsi_ctx*> members;
    cudaStream_t origin = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> events;
    int ndeg = 0;
    size_t nodes = 0;
    std::string err;
};

extern "C" chfsi_status chfsi_batch_create(chfsi_ctx* const* ctxs, int n, chfsi_batch** out) {
    if (!ctxs || n <= 0 || !out) return CHFSI_ERR_BAD_INPUT;
    *out = nullptr;
    const int dev = ctxs[0] ? ctxs[0]->device : 0;
    for (int i = 0; i < n; ++i) {
        chfsi_ctx* c = ctxs[i];
        if (!c || c->device != dev) return CHFSI_ERR_BAD_INPUT;
        if (!c->mixed) {
            set_last_error("batched passes run the mixed-precision path (FP32 filter, FP64 Rayleigh-Ritz)");
            return CHFSI_ERR_BAD_INPUT;
        }
    }
    cudaSetDevice(dev);
    chfsi_batch* b = new chfsi_batch();
    b->members.assign(ctxs, ctxs + n);
    if (cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) != cudaSuccess) {
        delete b;
        return CHFSI_ERR_CUDA;
    }
    *out = b;
    return CHFSI_OK;
}

extern "C" void chfsi_batch_destroy(chfsi_batch* b) {
    if (!b) return;
    if (b->origin) cudaStreamSynchronize(b->origin);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (cudaEvent_t e : b->events) cudaEventDestroy(e);
    if (b->origin) cudaStreamDestroy(b->origin);
    delete b;
}

// Capture one pass of every member.  Each member must have run one
// uncaptured diagonalisation first (it sets up the projector planes and the
// eigenvalues the captured filter takes its bounds from).
extern "C" chfsi_status chfsi_batch_capture(chfsi_batch* b, int ndeg) {
    if (!b || ndeg < 1) return CHFSI_ERR_BAD_INPUT;
    for (chfsi_ctx* c : b->members) {
        if (!c->veff_set || !c->psi_set || ndeg > c->max_deg) return CHFSI_ERR_BAD_INPUT;
        if (!c->mixed_active || (c->np > 0 && !c->beta_planes_ready)) {
            set_last_error("run one diagonalisation of every member before capturing");
            return CHFSI_ERR_BAD_INPUT;
        }
        cudaStreamSynchronize(c->st);
    }
    cudaSetDevice(b->members[0]->device);
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    for (cudaEvent_t e : b->events) cudaEventDestroy(e);
    b->events.assign(b->members.size() + 1, nullptr);
    for (auto& e : b->events)
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return CHFSI_ERR_CUDA;
    cudaError_t e = cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamBeginCapture", __FILE__, __LINE__);
    cudaEventRecord(b->events[0], b->origin);
    chfsi_status st = CHFSI_OK;
    for (size_t i = 0; i < b->members.size() && !st; ++i) {
        chfsi_ctx* c = b->members[i];
        cudaStreamWaitEvent(c->st, b->events[0], 0);
        st = filter_any(c, ndeg, c->d_eig, c->nb);
        if (!st) st = rr_any(c);
        cudaEventRecord(b->events[i + 1], c->st);
        cudaStreamWaitEvent(b->origin, b->events[i + 1], 0);
    }
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(b->origin, &g);
    if (st) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    b->graph = g;
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate", __FILE__, __LINE__);
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    b->nodes = nn;
    b->ndeg = ndeg;
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_batch_graph_nodes(chfsi_batch* b, size_t* nodes) {
    if (!b || !nodes) return CHFSI_ERR_BAD_INPUT;
    *nodes = b->nodes;
    return CHFSI_OK;
}

// Replay the captured pass; eig_out (optional) receives every member's
// n_bands eigenvalues in member order, status_out (optional) each member's
// status (filter divergence, failed Rayleigh-Ritz).
extern "C" chfsi_status chfsi_batch_run(chfsi_batch* b, double* eig_out, int* status_out) {
    if (!b || !b->exec) return CHFSI_ERR_BAD_INPUT;
    cudaSetDevice(b->members[0]->device);
    cudaError_t e = cudaGraphLaunch(b->exec, b->origin);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch", __FILE__, __LINE__);
    e = cudaStreamSynchronize(b->origin);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize", __FILE__, __LINE__);
    chfsi_status worst = CHFSI_OK;
    size_t off = 0;
    for (size_t i = 0; i < b->members.size(); ++i) {
        chfsi_ctx* c = b->members[i];
        c->last_ndeg = b->ndeg;
        const chfsi_status s = finish_diag(c, eig_out ? eig_out + off : nullptr, true);
        if (status_out) status_out[i] = s;
        if (s && !worst) worst = s;
        off += c->nb;
    }
    return worst;
}

// Launch configurations of the local H|psi> for this context's sizes: the
// xy-plane kernel at 128, 256 or 512 threads per block and the z-stick
// kernels at 16, 32 or 64 columns per block, each with the compile-time plane
// kernel (choices 0-8, where the grid has one) and with the generic one
// (9-17), timed on the current psi (all bands); the fastest is kept.
// times_ms (optional, kLaunchConfigs entries) gets every timing.
constexpr int kLaunchConfigs = 18;
static void apply_launch_config(chfsi_ctx* ctx, int i) {
    ctx->geo.fixed_planes = i < 9 ? 1 : 0;
    ctx->geo.tune_planes = (i % 9) / 3;
    ctx->geo.tune_cols = 16 << (i % 3);
}
extern "C" chfsi_status chfsi_autotune(chfsi_ctx* ctx, int* choice, float* times_ms) {
    chfsi_status s = ready(ctx);
    if (s) return s;
    if (!ctx->psi_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "psi not set");
    cudaSetDevice(ctx->device);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int np = ctx->np;
    ctx->np = 0;  // the launch configurations only concern the local part
    float best = 1e30f;
    int best_i = 0;
    for (int i = 0; i < kLaunchConfigs && !s; ++i) {
        apply_launch_config(ctx, i);
        for (int r = 0; r < 2 && !s; ++r) s = apply_h_dev(ctx, ctx->d_psi, ctx->d_hpsi, ctx->nb, kEpiApply, nullptr);
        cudaEventRecord(e0, ctx->st);
        for (int r = 0; r < 3 && !s; ++r) s = apply_h_dev(ctx, ctx->d_psi, ctx->d_hpsi, ctx->nb, kEpiApply, nullptr);
        cudaEventRecord(e1, ctx->st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ms /= 3.f;
        if (times_ms) times_ms[i] = ms;
        if (ms < best) { best = ms; best_i = i; }
    }
    ctx->np = np;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    apply_launch_config(ctx, best_i);
    if (s) return s;
    CK(cudaGetLastError());
    if (choice) *choice = best_i;
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_get_tc_shapes(chfsi_ctx* ctx, int* projection, int* expansion) {
    if (!ctx || !projection || !expansion) return CHFSI_ERR_BAD_INPUT;
    *projection = ctx->tc_shape[0];
    *expansion = ctx->tc_shape[1];
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_set_tc_shapes(chfsi_ctx* ctx, int projection, int expansion) {
    if (!ctx || projection < -1 || projection >= kTcVariantCount || expansion < -1 ||
        expansion >= kTcVariantCount) {
        set_last_error("chfsi_set_tc_shapes: shape outside -1..CHFSI_TC_SHAPES-1");
        return CHFSI_ERR_BAD_INPUT;
    }
    ctx->tc_shape[0] = projection;
    ctx->tc_shape[1] = expansion;
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_set_launch_config(chfsi_ctx* ctx, int choice) {
    if (!ctx || choice < 0 || choice >= kLaunchConfigs) return CHFSI_ERR_BAD_INPUT;
    apply_launch_config(ctx, choice);
    return CHFSI_OK;
}

// Band-by-band CG refinement of the current wavefunctions (band_cg.rs).
extern "C" chfsi_status chfsi_band_cg(chfsi_ctx* ctx, int max_steps, double tol, double* eig_out,
                                      int* steps_out, int* n_converged) {
    if (!ctx || max_steps < 0 || !(tol > 0.0)) return CHFSI_ERR_BAD_INPUT;
    if (!ctx->basis_set || !ctx->psi_set || !ctx->veff_set)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "context not ready");
    if (ctx->np > 0 && !ctx->proj_set) return ctx->fail(CHFSI_ERR_BAD_INPUT, "projectors not set");
    cudaSetDevice(ctx->device);
    std::vector<double> e(ctx->nb);
    std::vector<int> st(ctx->nb);
    int nc = 0;
    chfsi_status s = band_cg_dev(ctx, max_steps, tol, e.data(), st.data(), &nc);
    if (s) return s;
    if (eig_out) std::memcpy(eig_out, e.data(), sizeof(double) * ctx->nb);
    if (steps_out) std::memcpy(steps_out, st.data(), sizeof(int) * ctx->nb);
    if (n_converged) *n_converged = nc;
    return CHFSI_OK;
}

extern "C" chfsi_status chfsi_set_mixer(chfsi_ctx* ctx, chfsi_mixer* m) {
    if (!ctx) return CHFSI_ERR_BAD_INPUT;
    if (m && m->mlp.device != ctx->device)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "mixer lives on another device");
    ctx->mixer = m;
    return CHFSI_OK;
}

// Features and least-squares targets of one recorded SCF trajectory, with
// the same shell reductions the SCF loop uses for inference.
extern "C" chfsi_status chfsi_mixer_samples(chfsi_ctx* ctx, const double* rho_in,
                                            const double* rho_out, int n_iter,
                                            const double* rho_star, float* x, float* t) {
    if (!ctx || !rho_in || !rho_out || !rho_star || !x || !t || n_iter <= 0)
        return CHFSI_ERR_BAD_INPUT;
    if (!ctx->basis_set || ctx->omega <= 0.0)
        return ctx->fail(CHFSI_ERR_BAD_INPUT, "context not fully initialised");
    cudaSetDevice(ctx->device);
    chfsi_status s = alloc_mix(ctx);
    if (s) return s;
    const size_t ng = ctx->fng;
    cudaStream_t st = ctx->st;
    double* prev = mix_real(ctx, 0);
    double* star = mix_real(ctx, 1);
    double* a = mix_real(ctx, 2);
    double* b = mix_real(ctx, 3);
    CK(cudaMemcpyAsync(star, rho_star, sizeof(double) * ng, cudaMemcpyHostToDevice, st));
    MixRing ring;
    for (int it = 0; it < n_iter; ++it) {
        CK(cudaMemcpyAsync(a, rho_in + (size_t)it * ng, sizeof(double) * ng, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(b, rho_out + (size_t)it * ng, sizeof(double) * ng, cudaMemcpyHostToDevice, st));
        ring_push(ctx, ring, b, a);
        double2* Dg = nullptr;
        if (it > 0) {
            Dg = mix_grid(ctx, kGridD);
            launch_diff_complex(a, prev, Dg, ng, st);
            grid_fft3(ctx, Dg, true);
        }
        double2* Eg = mix_grid(ctx, kGridE);
        launch_diff_complex(star, a, Eg, ng, st);
        grid_fft3(ctx, Eg, true);
        if ((s = mix_features(ctx, ring, Dg, Eg))) return s;
        CK(cudaMemcpyAsync(x + (size_t)it * kMixIn, ctx->d_mix_x, sizeof(float) * kMixIn,
                           cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(t + (size_t)it * kMixShells * kMixTargets, ctx->d_mix_x + kMixIn,
                           sizeof(float) * kMixShells * kMixTargets, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(prev, a, sizeof(double) * ng, cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaStreamSynchronize(st));
    return CHFSI_OK;
}

// Largest K of the GEMM entry points: the split-K chunk arithmetic is 32-bit.
constexpr int kGemmMaxK = 1 << 30;

// C[m][n] = sum_k conj(A[m][k]) B[n][k] on device pointers (row-major,
// leading dimensions lda, ldb; C dense m x n) — the op::C ZGEMM of the
// reference's BlasHandle::gemm_c64 (src/device/blas.rs:79-102) as used for
// beta^H psi and the subspace matrices.  Split-K partials go to stream-
// ordered scratch (cudaMallocAsync / cudaFreeAsync on `stream`).
extern "C" chfsi_status chfsi_zgemm_cn(const chfsi_c128* a_dev, int lda, const chfsi_c128* b_dev,
                                       int ldb, int m, int n, int k, chfsi_c128* c_dev,
                                       void* stream) {
    if (!a_dev || !b_dev || !c_dev || m <= 0 || n <= 0 || k <= 0 || lda < k || ldb < k ||
        k > kGemmMaxK) {
        g_last_error = "chfsi_zgemm_cn: null pointer, size outside 1..2^30 or lda/ldb < k";
        return CHFSI_ERR_BAD_INPUT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    double2* part = nullptr;
    const size_t pe = splitk_partial_elems(m, n, k);
    cudaError_t e = cudaMallocAsync((void**)&part, pe * sizeof(double2), st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    gemm_cn(reinterpret_cast<const double2*>(a_dev), lda, reinterpret_cast<const double2*>(b_dev),
            ldb, m, n, k, part, reinterpret_cast<double2*>(c_dev), st);
    e = cudaGetLastError();
    cudaFreeAsync(part, st);
    if (e != cudaSuccess) return cuda_fail(e, "gemm_cn", __FILE__, __LINE__);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize", __FILE__, __LINE__);
    return CHFSI_OK;
}

// Mixed-precision variant of chfsi_zgemm_cn: tcgen05 BF16 3-way split
// products with FP32 accumulation (partials summed in FP64).  Plane and
// partial scratch are stream-ordered allocations on `stream`.
extern "C" chfsi_status chfsi_zgemm_cn_bf16x3(const chfsi_c128* a_dev, int lda,
                                              const chfsi_c128* b_dev, int ldb, int m, int n,
                                              int k, chfsi_c128* c_dev, void* stream) {
    return chfsi_zgemm_cn_bf16x3_shape(a_dev, lda, b_dev, ldb, m, n, k, c_dev, stream, 0);
}

extern "C" chfsi_status chfsi_zgemm_cn_bf16x3_shape(const chfsi_c128* a_dev, int lda,
                                                    const chfsi_c128* b_dev, int ldb, int m,
                                                    int n, int k, chfsi_c128* c_dev, void* stream,
                                                    int shape) {
    if (!a_dev || !b_dev || !c_dev || m <= 0 || n <= 0 || k <= 0 || lda < k || ldb < k ||
        k > kGemmMaxK) {
        g_last_error = "chfsi_zgemm_cn_bf16x3: null pointer, size outside 1..2^30 or lda/ldb < k";
        return CHFSI_ERR_BAD_INPUT;
    }
    if (shape < 0 || shape >= kTcVariantCount) {
        g_last_error = "chfsi_zgemm_cn_bf16x3_shape: shape outside 0..CHFSI_TC_SHAPES-1";
        return CHFSI_ERR_BAD_INPUT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int kp = tc_kpad(k);
    TcPlanes pa, pb;
    pa.rows_alloc = tc_rows_alloc(2 * m, true, n);
    pb.rows_alloc = tc_rows_alloc(n, false, n);
    const size_t na = (size_t)pa.rows_alloc * kp, nbe = (size_t)pb.rows_alloc * kp;
    char* buf = nullptr;
    const size_t part_f = tc_partial_floats(m, n, k);
    const size_t bytes = 3 * (na + nbe) * 2 + part_f * 4 + 256;
    cudaError_t e = cudaMallocAsync((void**)&buf, bytes, st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    cudaMemsetAsync(buf, 0, 3 * (na + nbe) * 2 + 256, st);
    for (int i = 0; i < 3; ++i) {
        pa.p[i] = buf + (size_t)i * na * 2;
        pb.p[i] = buf + 3 * na * 2 + (size_t)i * nbe * 2;
    }
    int* err = (int*)(buf + 3 * (na + nbe) * 2);
    float* part = (float*)(buf + 3 * (na + nbe) * 2 + 256);
    tc_pack<double2>(reinterpret_cast<const double2*>(a_dev), lda, m, k, true, kSrcPlain, pa, st);
    tc_pack<double2>(reinterpret_cast<const double2*>(b_dev), ldb, n, k, false, kSrcPlain, pb, st);
    e = tc_gemm(pa, pb, m, n, k, kTcOutPartial, c_dev, n, part, err, st, shape);
    int herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(buf, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "tc_gemm", __FILE__, __LINE__);
    if (herr) {
        g_last_error = "tensor-core GEMM pipeline wait timed out";
        return CHFSI_ERR_TIMEOUT;
    }
    return CHFSI_OK;
}

// O[m][n] = alpha sum_k W[k][m] X[k][n] + beta O[m][n] on device pointers: the
// ZGEMM of the subspace rotation psi <- psi V (rayleigh_ritz.rs:209-227) and
// the projector back-substitution beta (D C) (chebyshev.rs:480-497).
extern "C" chfsi_status chfsi_zgemm_tn(const chfsi_c128* w_dev, int ldw, const chfsi_c128* x_dev,
                                       int ldx, chfsi_c128* o_dev, int ldo, int m, int n, int k,
                                       double alpha, double beta, void* stream) {
    if (!w_dev || !x_dev || !o_dev || m <= 0 || n <= 0 || k <= 0 || k > kGemmMaxK || ldw < m ||
        ldx < n || ldo < n) {
        g_last_error = "chfsi_zgemm_tn: null pointer, size outside 1..2^30 or leading dimension too small";
        return CHFSI_ERR_BAD_INPUT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    gemm_tn(reinterpret_cast<const double2*>(w_dev), ldw, reinterpret_cast<const double2*>(x_dev),
            ldx, reinterpret_cast<double2*>(o_dev), ldo, m, n, k, alpha, beta, st);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "gemm_tn", __FILE__, __LINE__);
    return CHFSI_OK;
}

// Generalised Hermitian eigenproblem H x = e S x of an n x n subspace pair on
// the device (the ZHEGVD itype-1 contract of src/device/solver.rs:47-95, by
// the Cholesky reduction of subspace_diag.rs:275-363): S = L L^H,
// B = L^-1 H L^-H, B U = U diag(w), V = L^-H U.  h_dev, s_dev: row-major
// n x n (read only); w_host: n eigenvalues ascending; v_dev: n x n with
// column i the eigenvector of w[i] (row-major, V[j][i]).  Scratch is a
// stream-ordered allocation on `stream`.  CHFSI_ERR_RR_FAILED when S is not
// positive definite or the eigensolver does not converge.
extern "C" chfsi_status chfsi_hegv_dev(const chfsi_c128* h_dev, const chfsi_c128* s_dev, int n,
                                       double* w_host, chfsi_c128* v_dev, void* stream) {
    if (!h_dev || !s_dev || !w_host || !v_dev || n <= 0 || n > 4096) {
        g_last_error = "chfsi_hegv_dev: null pointer or n outside 1..4096";
        return CHFSI_ERR_BAD_INPUT;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const size_t nn = (size_t)n * n;
    const int max_sweeps = 60;
    const size_t jac = jacobi_scratch_doubles(n, max_sweeps);
    char* buf = nullptr;
    const size_t bytes = 5 * nn * sizeof(double2) + (jac + n) * sizeof(double) + 64;
    cudaError_t e = cudaMallocAsync((void**)&buf, bytes, st);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    double2* H = (double2*)buf;
    double2* S = H + nn;
    double2* T1 = S + nn;
    double2* T2 = T1 + nn;
    double2* V = T2 + nn;
    double* w = (double*)(V + nn);
    double* js = w + n;
    int* flags = (int*)(js + jac);
    cudaMemsetAsync(flags, 0, 4 * sizeof(int), st);
    symmetrize(reinterpret_cast<const double2*>(h_dev), H, n, st);
    symmetrize(reinterpret_cast<const double2*>(s_dev), S, n, st);
    cholesky(S, n, flags + 0, st);
    tri_inv(S, T1, n, st);                       // T1 = L^-1
    small_gemm(0, 0, T1, H, T2, n, st);          // T2 = L^-1 H
    small_gemm(0, 1, T2, T1, H, n, st);          // H = L^-1 H L^-H
    symmetrize(H, T2, n, st);
    e = jacobi(T2, V, n, max_sweeps, 1e-26, js, flags + 2, st);
    if (e == cudaSuccess) {
        sort_eig(T2, V, n, w, H, st);            // H = U (sorted)
        small_gemm(1, 0, T1, H, reinterpret_cast<double2*>(v_dev), n, st);  // V = L^-H U
        e = cudaGetLastError();
    }
    int fl[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(w_host, w, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fl, flags, sizeof(fl), cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(buf, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "chfsi_hegv_dev", __FILE__, __LINE__);
    if (fl[0] != 0) {
        g_last_error = "Rayleigh-Ritz failed: overlap not positive definite";
        return CHFSI_ERR_RR_FAILED;
    }
    if (fl[2] >= max_sweeps) {
        g_last_error = "Rayleigh-Ritz failed: eigensolver did not converge";
        return CHFSI_ERR_RR_FAILED;
    }
    return CHFSI_OK;
}

// Device pointer of the context's H|psi> (n_bands x n_pw): after
// chfsi_chebyshev_filter it holds H of the filtered block (the second output
// of the reference's chebyshev_filter, chebyshev.rs:626-643).
extern "C" chfsi_status chfsi_hpsi_device_ptr(chfsi_ctx* ctx, chfsi_c128** out) {
    if (!ctx || !out) return CHFSI_ERR_BAD_INPUT;
    *out = reinterpret_cast<chfsi_c128*>(ctx->d_hpsi);
    return CHFSI_OK;
}

// Host-side fault injection for the error-path tests (no GPU fault is made:
// an injected tensor-core timeout is a producer that issues no loads, so the
// consumer's bounded wait runs out with nothing in flight).
extern "C" chfsi_status chfsi_test_inject(int what, long long arg) {
    switch (what) {
        case CHFSI_INJECT_NONE:
            tc_inject_no_loads(0);
            g_alloc_fail_in.store(-1);
            return CHFSI_OK;
        case CHFSI_INJECT_TC_NO_LOADS:
            if (arg < 0 || arg > (1 << 20)) return CHFSI_ERR_BAD_INPUT;
            tc_inject_no_loads((int)arg);
            return CHFSI_OK;
        case CHFSI_INJECT_ALLOC_FAIL:
            g_alloc_fail_in.store(arg < 0 ? -1 : arg);
            return CHFSI_OK;
        default:
            return CHFSI_ERR_BAD_INPUT;
    }
}
