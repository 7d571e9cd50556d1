// Learned density mixer kernels: the MLP (forward, backward, Adam) and the
// |G|-shell reductions that turn density residual history into its inputs
// and into least-squares training targets.  No counterpart exists in the
// reference crate, whose DensityHistory::mix (src/mixing.rs:24) is a todo!();
// Pulay (the crate's planned mixer) stays the fallback in chfsi_scf_run.
#include "mixer.hpp"

#include <cmath>
#include <cstring>
#include <vector>

#include "launch_count.hpp"

namespace chfsi {
namespace {

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }

__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// C[M x N] = op(A)[M x K] op(B)[K x N], FP32 accumulation.
//   A(m, k) = TRA ? A[k lda + m] : A[m lda + k]
//   B(k, n) = TRB ? B[n ldb + k] : B[k ldb + n]
// EPI 0: C = acc + bias[n]        EPI 1: C = acc + bias[n], H = gelu(C)
// EPI 2: C = acc * gelu'(Z[m ldc + n])
// 64 x 64 tile per block, 16-deep K slices staged in shared memory, 4 x 4
// outputs per thread.  Loads are mapped so that consecutive threads read
// consecutive addresses for either transpose.
template <typename TA, bool TRA, typename TB, bool TRB, int EPI>
__global__ void __launch_bounds__(256)
k_mm(const TA* __restrict__ A, int lda, const TB* __restrict__ B, int ldb, float* __restrict__ C,
     int ldc, int M, int N, int K, const float* __restrict__ bias, float* __restrict__ H,
     const float* __restrict__ Z) {
    __shared__ float As[16][64 + 4];
    __shared__ float Bs[16][64 + 4];
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int e = tid + 256 * i;
            int mm, kk;
            if (TRA) { kk = e >> 6; mm = e & 63; } else { mm = e >> 4; kk = e & 15; }
            const int gm = m0 + mm, gk = k0 + kk;
            float a = 0.f;
            if (gm < M && gk < K) a = to_f(TRA ? A[(size_t)gk * lda + gm] : A[(size_t)gm * lda + gk]);
            As[kk][mm] = a;
            int nn;
            if (TRB) { nn = e >> 4; kk = e & 15; } else { kk = e >> 6; nn = e & 63; }
            const int gn = n0 + nn, gk2 = k0 + kk;
            float b = 0.f;
            if (gn < N && gk2 < K) b = to_f(TRB ? B[(size_t)gn * ldb + gk2] : B[(size_t)gk2 * ldb + gn]);
            Bs[kk][nn] = b;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            const size_t o = (size_t)m * ldc + n;
            float c = acc[i][j];
            if (EPI == 2) {
                c *= gelu_grad(Z[o]);
            } else if (bias) {
                c += bias[n];
            }
            C[o] = c;
            if (EPI == 1) H[o] = gelu(c);
        }
    }
}

template <typename TA, bool TRA, typename TB, bool TRB, int EPI>
void mm(const TA* A, int lda, const TB* B, int ldb, float* C, int ldc, int M, int N, int K,
        const float* bias, float* H, const float* Z, cudaStream_t st) {
    count_launch();
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    k_mm<TA, TRA, TB, TRB, EPI><<<grid, 256, 0, st>>>(A, lda, B, ldb, C, ldc, M, N, K, bias, H, Z);
}

// db[n] = sum_b dZ[b, n]
__global__ void k_colsum(const float* __restrict__ dz, int B, int N, float* __restrict__ db) {
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int b = 0; b < B; ++b) s += dz[(size_t)b * N + n];
    db[n] = s;
}

// Loss of the per-shell update (a, b) against the least-squares optimum
// (a*, b*) in the metric M of that shell (relative density error after the
// update, up to the part no (a, b) can remove), averaged over the batch.
__global__ void k_loss_grad(const float* __restrict__ y, const float* __restrict__ t, int B,
                            float* __restrict__ dy, float* __restrict__ loss) {
    __shared__ float red[256];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (i < B * kMixShells) {
        const int b = i / kMixShells, s = i % kMixShells;
        const float* tt = t + (size_t)b * kMixShells * kMixTargets + s * kMixTargets;
        const float ea = y[(size_t)b * kMixOut + 2 * s] - tt[0];
        const float eb = y[(size_t)b * kMixOut + 2 * s + 1] - tt[1];
        const float m00 = tt[2], m01 = tt[3], m11 = tt[4];
        l = ea * ea * m00 + 2.f * ea * eb * m01 + eb * eb * m11;
        const float sc = 2.f / (float)B;
        dy[(size_t)b * kMixOut + 2 * s] = sc * (m00 * ea + m01 * eb);
        dy[(size_t)b * kMixOut + 2 * s + 1] = sc * (m01 * ea + m11 * eb);
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / (float)B);
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, __nv_bfloat16* __restrict__ wb, size_t n, float lr,
                       float bc1, float bc2) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
        w[i] = wi;
        wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void k_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

__global__ void k_gather_rows(const float* __restrict__ dx, const float* __restrict__ dt,
                              const int* __restrict__ idx, int B, float* __restrict__ x,
                              float* __restrict__ t) {
    const int b = blockIdx.x;
    if (b >= B) return;
    const size_t r = (size_t)idx[b];
    for (int j = threadIdx.x; j < kMixIn; j += blockDim.x) x[(size_t)b * kMixIn + j] = dx[r * kMixIn + j];
    for (int j = threadIdx.x; j < kMixShells * kMixTargets; j += blockDim.x)
        t[(size_t)b * kMixShells * kMixTargets + j] = dt[r * kMixShells * kMixTargets + j];
}

// ---------------------------------------------------------------- shells
__device__ __forceinline__ int shell_of(const GridRecip& gr, size_t i) {
    const int ix = (int)(i % gr.nx);
    const int iy = (int)((i / gr.nx) % gr.ny);
    const int iz = (int)(i / ((size_t)gr.nx * gr.ny));
    int h = gr.idr_x[ix], k = gr.idr_y[iy], l = gr.idr_z[iz];
    if (h >= (gr.nx + 1) / 2) h -= gr.nx;
    if (k >= (gr.ny + 1) / 2) k -= gr.ny;
    if (l >= (gr.nz + 1) / 2) l -= gr.nz;
    if (h == 0 && k == 0 && l == 0) return 255;
    const double gx = h * gr.b[0] + k * gr.b[3] + l * gr.b[6];
    const double gy = h * gr.b[1] + k * gr.b[4] + l * gr.b[7];
    const double gz = h * gr.b[2] + k * gr.b[5] + l * gr.b[8];
    const double g = sqrt(gx * gx + gy * gy + gz * gz);
    const int s = (int)floor(kMixShells * sqrt(g / kShellGmax));
    return s < kMixShells - 1 ? s : kMixShells - 1;
}

__global__ void k_shell_index(GridRecip gr, unsigned char* __restrict__ shell) {
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        shell[i] = (unsigned char)shell_of(gr, i);
}

__device__ __forceinline__ double re_cdot(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }

__global__ void __launch_bounds__(256)
k_shell_acc(const double2* __restrict__ R0, const double2* __restrict__ R1,
            const double2* __restrict__ R2, const double2* __restrict__ R3,
            const double2* __restrict__ D, const double2* __restrict__ E,
            const unsigned char* __restrict__ shell, size_t ng, double* __restrict__ acc) {
    __shared__ double sacc[kMixShells * kShellAcc];
    for (int i = threadIdx.x; i < kMixShells * kShellAcc; i += blockDim.x) sacc[i] = 0.0;
    __syncthreads();
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ng;
         i += (size_t)gridDim.x * blockDim.x) {
        const int s = shell[i];
        if (s == 255) continue;
        double* a = sacc + s * kShellAcc;
        const double2 r0 = R0[i];
        atomicAdd(a + 0, re_cdot(r0, r0));
        const double2* hist[3] = {R1, R2, R3};
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            if (!hist[t]) continue;
            const double2 rt = hist[t][i];
            atomicAdd(a + 1 + t, re_cdot(r0, rt));
            atomicAdd(a + 4 + t, re_cdot(rt, rt));
        }
        double2 d = make_double2(0.0, 0.0);
        if (D) {
            d = D[i];
            atomicAdd(a + 7, re_cdot(d, d));
            atomicAdd(a + 8, re_cdot(r0, d));
        }
        if (E) {
            const double2 e = E[i];
            atomicAdd(a + 9, re_cdot(r0, e));
            atomicAdd(a + 10, re_cdot(d, e));
            atomicAdd(a + 11, re_cdot(e, e));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kMixShells * kShellAcc; i += blockDim.x)
        if (sacc[i] != 0.0) atomicAdd(acc + i, sacc[i]);
}

__device__ __forceinline__ float slog(double x) {
    return (float)(x >= 0.0 ? log1p(x) : -log1p(-x));
}

// One block of 64 threads (one per shell).
__global__ void k_shell_features(const double* __restrict__ acc, float* __restrict__ x,
                                 float* __restrict__ t) {
    __shared__ double tot[2][kMixShells];
    const int s = threadIdx.x;
    const double* a = acc + s * kShellAcc;
    tot[0][s] = a[0];
    tot[1][s] = a[11];
    __syncthreads();
    for (int o = kMixShells / 2; o > 0; o >>= 1) {
        if (s < o) { tot[0][s] += tot[0][s + o]; tot[1][s] += tot[1][s + o]; }
        __syncthreads();
    }
    const double r2 = tot[0][0], e2 = tot[1][0];
    const double sc = r2 > 0.0 ? (double)kMixShells / r2 : 0.0;
    float* xs = x + (size_t)s * kMixHist * 2;
    xs[0] = slog(a[0] * sc);
    xs[1] = slog(a[8] * sc);
    for (int h = 1; h < kMixHist; ++h) {
        xs[2 * h] = slog(a[h] * sc);
        xs[2 * h + 1] = slog(a[3 + h] * sc);
    }
    if (!t) return;
    float* ts = t + (size_t)s * kMixTargets;
    double m00 = 0.0, m01 = 0.0, m11 = 0.0, ra = 0.0, rb = 0.0;
    if (e2 > 0.0) {
        m00 = a[0] / e2; m01 = a[8] / e2; m11 = a[7] / e2; ra = a[9] / e2; rb = a[10] / e2;
    }
    double ca = 0.0, cb = 0.0;
    if (m00 > 0.0) {
        if (m11 <= 1e-12 * m00) {
            ca = ra / m00;
        } else {
            const double lam = 1e-9 * (m00 + m11);
            const double det = (m00 + lam) * (m11 + lam) - m01 * m01;
            ca = ((m11 + lam) * ra - m01 * rb) / det;
            cb = ((m00 + lam) * rb - m01 * ra) / det;
        }
    }
    ca = fmin(10.0, fmax(-10.0, ca));
    cb = fmin(10.0, fmax(-10.0, cb));
    ts[0] = (float)ca; ts[1] = (float)cb;
    ts[2] = (float)m00; ts[3] = (float)m01; ts[4] = (float)m11;
}

__global__ void k_shell_update(double2* __restrict__ out, const double2* __restrict__ R0,
                               const double2* __restrict__ D, const float* __restrict__ y,
                               const unsigned char* __restrict__ shell, size_t ng) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < ng;
         i += (size_t)gridDim.x * blockDim.x) {
        const int s = shell[i];
        if (s == 255) continue;
        const double a = y[2 * s];
        double2 o = out[i];
        const double2 r = R0[i];
        o.x += a * r.x;
        o.y += a * r.y;
        if (D) {
            const double b = y[2 * s + 1];
            const double2 d = D[i];
            o.x += b * d.x;
            o.y += b * d.y;
        }
        out[i] = o;
    }
}

__global__ void k_diff_complex(const double* __restrict__ a, const double* __restrict__ b,
                               double2* __restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = make_double2(b ? a[i] - b[i] : a[i], 0.0);
}

__global__ void k_take_real_scaled(const double2* __restrict__ c, double* __restrict__ r, size_t n,
                                   double scale) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        r[i] = scale * c[i].x;
}

int blocks_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 148 * 4 ? (b ? b : 1) : 148 * 4);
}

// SplitMix64 uniform in [0, 1)
struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
};

}  // namespace

cudaError_t mlp_alloc(Mlp& M, int cap) {
    auto fa = [](float** p, size_t n) { return cudaMalloc((void**)p, n * sizeof(float)); };
    cudaError_t e;
    if (!M.w) {
        if ((e = fa(&M.w, kMixParams)) || (e = fa(&M.g, kMixParams)) || (e = fa(&M.m, kMixParams)) ||
            (e = fa(&M.v, kMixParams)) || (e = fa(&M.loss, 1)))
            return e;
        if ((e = cudaMalloc((void**)&M.wb, kMixParams * sizeof(__nv_bfloat16)))) return e;
        cudaMemsetAsync(M.m, 0, kMixParams * sizeof(float), M.st);
        cudaMemsetAsync(M.v, 0, kMixParams * sizeof(float), M.st);
    }
    if (cap > M.cap) {
        float** bufs[] = {&M.x, &M.t, &M.z1, &M.h1, &M.z2, &M.h2, &M.y, &M.dy, &M.d2, &M.d1};
        for (float** b : bufs) { cudaFree(*b); *b = nullptr; }
        const size_t c = (size_t)cap;
        if ((e = fa(&M.x, c * kMixIn)) || (e = fa(&M.t, c * kMixShells * kMixTargets)) ||
            (e = fa(&M.z1, c * kMixHidden)) || (e = fa(&M.h1, c * kMixHidden)) ||
            (e = fa(&M.z2, c * kMixHidden)) || (e = fa(&M.h2, c * kMixHidden)) ||
            (e = fa(&M.y, c * kMixOut)) || (e = fa(&M.dy, c * kMixOut)) ||
            (e = fa(&M.d2, c * kMixHidden)) || (e = fa(&M.d1, c * kMixHidden)))
            return e;
        M.cap = cap;
    }
    return cudaSuccess;
}

void mlp_free(Mlp& M) {
    float* bufs[] = {M.w, M.g, M.m, M.v, M.loss, M.x, M.t, M.z1, M.h1, M.z2, M.h2, M.y, M.dy,
                     M.d2, M.d1, M.data_x, M.data_t};
    for (float* b : bufs) cudaFree(b);
    cudaFree(M.wb);
    cudaFree(M.idx);
    M = Mlp{};
}

// Uniform in +-sqrt(3 / fan_in) (unit-variance preactivations), biases zero;
// the output layer is scaled by 0.01 with bias a_s = 0.3, b_s = 0, so an
// untrained network mixes like plain linear mixing with alpha = 0.3.
void mlp_init_host(float* w, uint64_t seed) {
    Rng r{seed * 0x2545F4914F6CDD1Dull + 7};
    auto fill = [&](size_t off, int fan_out, int fan_in, float scale) {
        const double lim = std::sqrt(3.0 / fan_in) * scale;
        for (size_t i = 0; i < (size_t)fan_out * fan_in; ++i)
            w[off + i] = (float)((2.0 * r.uniform() - 1.0) * lim);
    };
    fill(kOffW1, kMixHidden, kMixIn, 1.f);
    fill(kOffW2, kMixHidden, kMixHidden, 1.f);
    fill(kOffW3, kMixOut, kMixHidden, 0.01f);
    std::memset(w + kOffB1, 0, kMixHidden * sizeof(float));
    std::memset(w + kOffB2, 0, kMixHidden * sizeof(float));
    for (int s = 0; s < kMixShells; ++s) {
        w[kOffB3 + 2 * s] = 0.3f;
        w[kOffB3 + 2 * s + 1] = 0.f;
    }
}

void mlp_sync_bf16(Mlp& M, cudaStream_t st) {
    count_launch();
    k_to_bf16<<<blocks_for(kMixParams), 256, 0, st>>>(M.w, M.wb, kMixParams);
}

void mlp_forward(Mlp& M, const float* x, int B, float* y, cudaStream_t st) {
    mm<float, false, __nv_bfloat16, true, 1>(x, kMixIn, M.wb + kOffW1, kMixIn, M.z1, kMixHidden, B,
                                             kMixHidden, kMixIn, M.w + kOffB1, M.h1, nullptr, st);
    mm<float, false, __nv_bfloat16, true, 1>(M.h1, kMixHidden, M.wb + kOffW2, kMixHidden, M.z2,
                                             kMixHidden, B, kMixHidden, kMixHidden, M.w + kOffB2,
                                             M.h2, nullptr, st);
    mm<float, false, __nv_bfloat16, true, 0>(M.h2, kMixHidden, M.wb + kOffW3, kMixHidden, y, kMixOut,
                                             B, kMixOut, kMixHidden, M.w + kOffB3, nullptr, nullptr,
                                             st);
}

void mlp_backward(Mlp& M, int B, cudaStream_t st) {
    mlp_forward(M, M.x, B, M.y, st);
    cudaMemsetAsync(M.loss, 0, sizeof(float), st);
    count_launch();
    k_loss_grad<<<(B * kMixShells + 255) / 256, 256, 0, st>>>(M.y, M.t, B, M.dy, M.loss);
    // layer 3
    mm<float, true, float, false, 0>(M.dy, kMixOut, M.h2, kMixHidden, M.g + kOffW3, kMixHidden,
                                     kMixOut, kMixHidden, B, nullptr, nullptr, nullptr, st);
    count_launch();
    k_colsum<<<1, kMixOut, 0, st>>>(M.dy, B, kMixOut, M.g + kOffB3);
    mm<float, false, __nv_bfloat16, false, 2>(M.dy, kMixOut, M.wb + kOffW3, kMixHidden, M.d2,
                                              kMixHidden, B, kMixHidden, kMixOut, nullptr, nullptr,
                                              M.z2, st);
    // layer 2
    mm<float, true, float, false, 0>(M.d2, kMixHidden, M.h1, kMixHidden, M.g + kOffW2, kMixHidden,
                                     kMixHidden, kMixHidden, B, nullptr, nullptr, nullptr, st);
    count_launch();
    k_colsum<<<1, kMixHidden, 0, st>>>(M.d2, B, kMixHidden, M.g + kOffB2);
    mm<float, false, __nv_bfloat16, false, 2>(M.d2, kMixHidden, M.wb + kOffW2, kMixHidden, M.d1,
                                              kMixHidden, B, kMixHidden, kMixHidden, nullptr,
                                              nullptr, M.z1, st);
    // layer 1
    mm<float, true, float, false, 0>(M.d1, kMixHidden, M.x, kMixIn, M.g + kOffW1, kMixIn,
                                     kMixHidden, kMixIn, B, nullptr, nullptr, nullptr, st);
    count_launch();
    k_colsum<<<1, kMixHidden, 0, st>>>(M.d1, B, kMixHidden, M.g + kOffB1);
}

void mlp_adam(Mlp& M, float lr, cudaStream_t st) {
    ++M.step;
    const float bc1 = 1.f - std::pow(0.9f, (float)M.step);
    const float bc2 = 1.f - std::pow(0.999f, (float)M.step);
    count_launch();
    k_adam<<<blocks_for(kMixParams), 256, 0, st>>>(M.w, M.g, M.m, M.v, M.wb, kMixParams, lr, bc1,
                                                   bc2);
}

void mlp_gather_batch(Mlp& M, const int* idx, int B, cudaStream_t st) {
    count_launch();
    k_gather_rows<<<B, 128, 0, st>>>(M.data_x, M.data_t, idx, B, M.x, M.t);
}

void launch_shell_index(const GridRecip& gr, unsigned char* shell, cudaStream_t st) {
    count_launch();
    k_shell_index<<<blocks_for((size_t)gr.nx * gr.ny * gr.nz), 256, 0, st>>>(gr, shell);
}

void launch_shell_acc(const double2* R0, const double2* R1, const double2* R2, const double2* R3,
                      const double2* D, const double2* E, const unsigned char* shell, size_t ng,
                      double* acc, cudaStream_t st) {
    count_launch();
    k_shell_acc<<<blocks_for(ng), 256, 0, st>>>(R0, R1, R2, R3, D, E, shell, ng, acc);
}

void launch_shell_features(const double* acc, float* features, float* targets, cudaStream_t st) {
    count_launch();
    k_shell_features<<<1, kMixShells, 0, st>>>(acc, features, targets);
}

void launch_shell_update(double2* out, const double2* R0, const double2* D, const float* y,
                         const unsigned char* shell, size_t ng, cudaStream_t st) {
    count_launch();
    k_shell_update<<<blocks_for(ng), 256, 0, st>>>(out, R0, D, y, shell, ng);
}

void launch_diff_complex(const double* a, const double* b, double2* out, size_t n, cudaStream_t st) {
    count_launch();
    k_diff_complex<<<blocks_for(n), 256, 0, st>>>(a, b, out, n);
}

void launch_take_real_scaled(const double2* c, double* r, size_t n, double scale, cudaStream_t st) {
    count_launch();
    k_take_real_scaled<<<blocks_for(n), 256, 0, st>>>(c, r, n, scale);
}

}  // namespace chfsi
