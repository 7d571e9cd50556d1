// Complex FP64 GEMMs of the ChFSI path (role of the reference's cuBLAS
// ZGEMM calls: chebyshev.rs:432-497 projectors, rayleigh_ritz.rs:74-142
// subspace matrices, rayleigh_ritz.rs:209-227 rotation).  Two shapes:
//
//   gemm_cn:  P[s][m][n] = sum_{k in chunk s} conj(A[m][k]) B[n][k]
//             (A: M x K, B: N x K, both K-contiguous; long K split across
//             CTAs, partials reduced deterministically)
//             -> beta^H psi, psi^H H psi, psi^H psi
//   gemm_tn:  O[m][n] = alpha sum_k W[k][m] X[k][n] + beta O[m][n]
//             (W: K x M, X: K x N, N-contiguous; short K)
//             -> beta (D beta^H psi), psi V
//
// B200 FP64 has no tcgen05 kind; both run on the FP64 tensor path
// (mma.sync m8n8k4 .f64).
#include <algorithm>
#include "gemm.hpp"
#include "launch_count.hpp"

namespace chfsi {

namespace {

constexpr int BM = 64, BN = 64, BK = 16;
constexpr int kStages = 3;
// one CTA of 256 threads per SM (about 150 registers per thread, 120 KB of
// shared memory): split-K counts fill waves of 148 CTAs
constexpr int kCtasPerWave = 148;

// ---- FP64 tensor-core (DMMA) versions: mma.sync m8n8k4 .f64.  Fragments
// (PTX m8n8k4 .f64): A row (lane >> 2), col (lane & 3); B row (lane & 3), col
// (lane >> 2); C row (lane >> 2), cols 2 (lane & 3) + {0, 1}.  CTA tile
// 64 x 64, 8 warps as 2 (M) x 4 (N), warp tile 32 x 16 = 4 x 2 MMA tiles.
// Complex products by Gauss's three-multiplication form (three real MMAs per
// complex MAC instead of four):
//   conj(a) b:  t1 = ar br, t2 = ai bi, t3 = (ar - ai)(br + bi);
//               re = t1 + t2, im = t3 - t1 + t2
//   a b:        t1 = ar br, t2 = ai bi, t3 = (ar + ai)(br + bi);
//               re = t1 - t2, im = t3 - t1 - t2
// Operand tiles stream global -> shared with cp.async (16-byte complex
// elements, zero fill outside the matrix) through a 3-stage ring; each
// fragment is one 128-bit shared load of a complex element (re and im
// together).
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// 16-byte async copy global -> shared; src_bytes 0 writes zeros
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// row strides (complex elements): K-contiguous tiles 20 = 4 mod 8, M/N-
// contiguous tiles 66 = 2 mod 8, so that the 8 lanes of each quarter-warp
// fragment load hit 8 different 16-byte bank groups
constexpr int kSK = BK + 4;
constexpr int kSM = BM + 2;

// P[s][m][n] = sum_{k in chunk s} conj(A[m][k]) B[n][k]
__global__ void __launch_bounds__(256, 1)
k_zgemm_cn_dmma(const double2* __restrict__ A, int lda, const double2* __restrict__ B, int ldb,
                int M, int N, int K, int kchunk, double2* __restrict__ part, int tri) {
    extern __shared__ __align__(16) double2 sm_cn[];
    double2* As = sm_cn;                           // [kStages][BM][kSK]
    double2* Bs = sm_cn + kStages * BM * kSK;      // [kStages][BN][kSK]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;
    int tm = blockIdx.x, tn = blockIdx.y;
    if (tri > 0) {
        // Hermitian product: blockIdx.x enumerates the tile pairs tm <= tn of
        // a tri x tri tile grid, row by row
        int t = blockIdx.x, row = 0;
        while (t >= tri - row) { t -= tri - row; ++row; }
        tm = row;
        tn = row + t;
    }
    const int m0 = tm * BM, n0 = tn * BN;
    const int kb = blockIdx.z * kchunk;
    const int ke = min(K, kb + kchunk);
    const int nsteps = ke > kb ? (ke - kb + BK - 1) / BK : 0;
    // copy assignment: chunk c = threadIdx.x + 256 i (i < 4): row c / 16, col c % 16
    auto load_stage = [&](int step, int slot) {
        const int k0 = kb + step * BK;
        double2* as = As + slot * BM * kSK;
        double2* bs = Bs + slot * BN * kSK;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = threadIdx.x + 256 * i;
            const int r = c >> 4, kk = c & 15;
            const int k = k0 + kk;
            const int am = m0 + r, bn = n0 + r;
            const bool ka = k < ke;
            const double2* srca = A + ((ka && am < M) ? (size_t)am * lda + k : 0);
            const double2* srcb = B + ((ka && bn < N) ? (size_t)bn * ldb + k : 0);
            cp_async16(as + r * kSK + kk, srca, (ka && am < M) ? 16 : 0);
            cp_async16(bs + r * kSK + kk, srcb, (ka && bn < N) ? 16 : 0);
        }
    };
    double t1[4][2][2], t2[4][2][2], t3[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) t1[i][j][e] = t2[i][j][e] = t3[i][j][e] = 0.0;
#pragma unroll
    for (int st = 0; st < kStages - 1; ++st) {
        if (st < nsteps) load_stage(st, st);
        cp_async_commit();
    }
    for (int step = 0; step < nsteps; ++step) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        // refill the slot consumed one step ago
        const int nxt = step + kStages - 1;
        if (nxt < nsteps) load_stage(nxt, nxt % kStages);
        cp_async_commit();
        const double2* as = As + (step % kStages) * BM * kSK;
        const double2* bs = Bs + (step % kStages) * BN * kSK;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double br[2], bi[2], bs_[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const double2 v = bs[(wn * 16 + j * 8 + gid) * kSK + kk + tig];
                br[j] = v.x;
                bi[j] = v.y;
                bs_[j] = v.x + v.y;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double2 v = as[(wm * 32 + i * 8 + gid) * kSK + kk + tig];
                const double ad = v.x - v.y;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma(t1[i][j], v.x, br[j]);
                    dmma(t2[i][j], v.y, bi[j]);
                    dmma(t3[i][j], ad, bs_[j]);
                }
            }
        }
    }
    cp_async_wait<0>();
    double2* pp = part + (size_t)blockIdx.z * M * N;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + wm * 32 + i * 8 + gid;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int n = n0 + wn * 16 + j * 8 + 2 * tig + e;
                if (n < N)
                    pp[(size_t)m * N + n] = make_double2(t1[i][j][e] + t2[i][j][e],
                                                         t3[i][j][e] - t1[i][j][e] + t2[i][j][e]);
            }
    }
}

// O[m][n] = alpha sum_k W[k][m] X[k][n] + beta O[m][n]
__global__ void __launch_bounds__(256, 1)
k_zgemm_tn_dmma(const double2* __restrict__ W, int ldw, const double2* __restrict__ X, int ldx,
                double2* O, int ldo, int M, int N, int K, double alpha, double beta) {
    extern __shared__ __align__(16) double2 sm_tn[];
    double2* Ws = sm_tn;                           // [kStages][BK][kSM]
    double2* Xs = sm_tn + kStages * BK * kSM;      // [kStages][BK][kSM]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
    const int nsteps = (K + BK - 1) / BK;
    // chunk c = threadIdx.x + 256 i (i < 4): k row c / 64, column c % 64
    auto load_stage = [&](int step, int slot) {
        const int k0 = step * BK;
        double2* ws = Ws + slot * BK * kSM;
        double2* xs = Xs + slot * BK * kSM;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = threadIdx.x + 256 * i;
            const int r = c >> 6, col = c & 63;
            const int k = k0 + r;
            const int m = m0 + col, n = n0 + col;
            const bool kw = k < K;
            const double2* srcw = W + ((kw && m < M) ? (size_t)k * ldw + m : 0);
            const double2* srcx = X + ((kw && n < N) ? (size_t)k * ldx + n : 0);
            cp_async16(ws + r * kSM + col, srcw, (kw && m < M) ? 16 : 0);
            cp_async16(xs + r * kSM + col, srcx, (kw && n < N) ? 16 : 0);
        }
    };
    double t1[4][2][2], t2[4][2][2], t3[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) t1[i][j][e] = t2[i][j][e] = t3[i][j][e] = 0.0;
#pragma unroll
    for (int st = 0; st < kStages - 1; ++st) {
        if (st < nsteps) load_stage(st, st);
        cp_async_commit();
    }
    for (int step = 0; step < nsteps; ++step) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        const int nxt = step + kStages - 1;
        if (nxt < nsteps) load_stage(nxt, nxt % kStages);
        cp_async_commit();
        const double2* ws = Ws + (step % kStages) * BK * kSM;
        const double2* xs = Xs + (step % kStages) * BK * kSM;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double xr[2], xi[2], xsum[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const double2 v = xs[(kk + tig) * kSM + wn * 16 + j * 8 + gid];
                xr[j] = v.x;
                xi[j] = v.y;
                xsum[j] = v.x + v.y;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double2 v = ws[(kk + tig) * kSM + wm * 32 + i * 8 + gid];
                const double as_ = v.x + v.y;
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma(t1[i][j], v.x, xr[j]);
                    dmma(t2[i][j], v.y, xi[j]);
                    dmma(t3[i][j], as_, xsum[j]);
                }
            }
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + wm * 32 + i * 8 + gid;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int n = n0 + wn * 16 + j * 8 + 2 * tig + e;
                if (n >= N) continue;
                double2* o = O + (size_t)m * ldo + n;
                const double re = t1[i][j][e] - t2[i][j][e];
                const double im = t3[i][j][e] - t1[i][j][e] - t2[i][j][e];
                double2 r = make_double2(alpha * re, alpha * im);
                if (beta != 0.0) {
                    r.x += beta * o->x;
                    r.y += beta * o->y;
                }
                *o = r;
            }
    }
}

constexpr size_t kSmemCn = (size_t)kStages * (BM + BN) * kSK * sizeof(double2);
constexpr size_t kSmemTn = (size_t)kStages * 2 * BK * kSM * sizeof(double2);

void gemm_smem_setup() {
    static bool done = false;
    if (done) return;
    cudaFuncSetAttribute(k_zgemm_cn_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemCn);
    cudaFuncSetAttribute(k_zgemm_tn_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemTn);
    done = true;
}

// Hermitian product from its upper tiles: out[m][n] = sum of partials where
// tile(m) <= tile(n), out[n][m] = conj of it where tile(m) < tile(n)
__global__ void k_reduce_herm(const double2* __restrict__ part, int splits, int N,
                              double2* __restrict__ out) {
    const size_t nn = (size_t)N * N;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nn;
         i += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(i / N), n = (int)(i % N);
        if (m / BM > n / BN) continue;
        double2 s = make_double2(0.0, 0.0);
        for (int t = 0; t < splits; ++t) {
            const double2 v = part[(size_t)t * nn + i];
            s.x += v.x;
            s.y += v.y;
        }
        out[i] = s;
        if (m / BM < n / BN) out[(size_t)n * N + m] = make_double2(s.x, -s.y);
    }
}

__global__ void k_reduce_partials(const double2* __restrict__ part, int splits, size_t mn,
                                  double2* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < mn;
         i += (size_t)gridDim.x * blockDim.x) {
        double2 s = make_double2(0.0, 0.0);
        for (int t = 0; t < splits; ++t) {
            const double2 v = part[(size_t)t * mn + i];
            s.x += v.x;
            s.y += v.y;
        }
        out[i] = s;
    }
}

}  // namespace

// One CTA of k_zgemm_cn_dmma fills an SM, so the grid runs in waves of 148.
// The split count that fills the last wave best wins (a larger one only
// when it fills it 2 % better), with at least 256 k per split and 64 splits
// at most (e.g. 12 tiles of the 256-projector x 160-band product as 37
// splits: 444 CTAs in three full waves).
int splitk_count(int M, int N, int K) {
    return splitk_count_tiles(((M + BM - 1) / BM) * ((N + BN - 1) / BN), K);
}

int splitk_count_tiles(int tiles, int K) {
    const int max_splits = std::min(64, std::max(1, (K + 255) / 256));
    int best = 1;
    double best_eff = -1.0;
    for (int s = 1; s <= max_splits; ++s) {
        const long long ctas = (long long)tiles * s;
        const long long waves = (ctas + kCtasPerWave - 1) / kCtasPerWave;
        const double eff = (double)ctas / (waves * (double)kCtasPerWave);
        if (eff > best_eff + 0.02) {
            best_eff = eff;
            best = s;
        }
    }
    return best;
}

size_t splitk_partial_elems(int M, int N, int K) {
    return (size_t)splitk_count(M, N, K) * M * N;
}

size_t splitk_partial_elems_herm(int N, int K) {
    const int tn = (N + BN - 1) / BN;
    return (size_t)splitk_count_tiles(tn * (tn + 1) / 2, K) * N * N;
}

void gemm_cn(const double2* A, int lda, const double2* B, int ldb, int M, int N, int K,
             double2* part, double2* out, cudaStream_t st) {
    count_launch(2);
    const int splits = splitk_count(M, N, K);
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + BK - 1) / BK * BK;
    const int used = (K + kchunk - 1) / kchunk;
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, used);
    gemm_smem_setup();
    k_zgemm_cn_dmma<<<grid, 256, kSmemCn, st>>>(A, lda, B, ldb, M, N, K, kchunk, part, 0);
    const size_t mn = (size_t)M * N;
    int blocks = (int)((mn + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_reduce_partials<<<blocks, 256, 0, st>>>(part, used, mn, out);
}

// C = conj(A) A'^T for a Hermitian result (A' = A, or A' = H A with H
// Hermitian on the span): only the tiles on and above the diagonal are
// computed (half the flops), the rest mirrored by conjugation.
void gemm_cn_herm(const double2* A, int lda, const double2* B, int ldb, int N, int K,
                  double2* part, double2* out, cudaStream_t st) {
    count_launch(2);
    const int tn = (N + BN - 1) / BN;
    const int tiles = tn * (tn + 1) / 2;
    const int splits = splitk_count_tiles(tiles, K);
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + BK - 1) / BK * BK;
    const int used = (K + kchunk - 1) / kchunk;
    dim3 grid(tiles, 1, used);
    gemm_smem_setup();
    k_zgemm_cn_dmma<<<grid, 256, kSmemCn, st>>>(A, lda, B, ldb, N, N, K, kchunk, part, tn);
    const size_t nn = (size_t)N * N;
    int blocks = (int)((nn + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_reduce_herm<<<blocks, 256, 0, st>>>(part, used, N, out);
}

void gemm_tn(const double2* W, int ldw, const double2* X, int ldx, double2* O, int ldo, int M,
             int N, int K, double alpha, double beta, cudaStream_t st) {
    count_launch();
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    gemm_smem_setup();
    k_zgemm_tn_dmma<<<grid, 256, kSmemTn, st>>>(W, ldw, X, ldx, O, ldo, M, N, K, alpha, beta);
}

}  // namespace chfsi

namespace chfsi {

// gemm_cn with the split count capped at max_splits (>= 1); partials need
// min(splitk_count, max_splits) * M * N elements of `part`.
void gemm_cn_capped(const double2* A, int lda, const double2* B, int ldb, int M, int N, int K,
                    int max_splits, double2* part, double2* out, cudaStream_t st) {
    count_launch(2);
    int splits = splitk_count(M, N, K);
    if (splits > max_splits) splits = max_splits;
    if (splits < 1) splits = 1;
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + BK - 1) / BK * BK;
    const int used = (K + kchunk - 1) / kchunk;
    dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, used);
    gemm_smem_setup();
    k_zgemm_cn_dmma<<<grid, 256, kSmemCn, st>>>(A, lda, B, ldb, M, N, K, kchunk, part, 0);
    const size_t mn = (size_t)M * N;
    int blocks = (int)((mn + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_reduce_partials<<<blocks, 256, 0, st>>>(part, used, mn, out);
}

}  // namespace chfsi
