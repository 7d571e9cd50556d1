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

// ---- FP64 tensor-core (DMMA) versions: mma.sync m8n8k4 .f64, one warp
// issues 256 FMAs per instruction.  Complex products as four real MMAs on
// split (re, im) shared-memory planes.  Fragments (PTX m8n8k4 .f64): A row
// (lane >> 2), col (lane & 3); B row (lane & 3), col (lane >> 2); C row
// (lane >> 2), cols 2 (lane & 3) + {0, 1}.  CTA tile 64 x 64, 8 warps as
// 2 (M) x 4 (N), warp tile 32 x 16 = 4 x 2 MMA tiles.
// Not volatile: the MMA has no effect beyond its outputs, so the compiler may
// interleave independent MMAs with the fragment loads.
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

constexpr int kDS = BK + 4;  // row stride (doubles) of K-contiguous planes
constexpr int kDT = BM + 4;  // row stride (doubles) of M/N-contiguous planes

// P[s][m][n] = sum_{k in chunk s} conj(A[m][k]) B[n][k]
__global__ void __launch_bounds__(256, 2)
k_zgemm_cn_dmma(const double2* __restrict__ A, int lda, const double2* __restrict__ B, int ldb,
                int M, int N, int K, int kchunk, double2* __restrict__ part, int tri) {
    __shared__ double Ar[BM][kDS], Ai[BM][kDS], Br[BN][kDS], Bi[BN][kDS];
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
    double cr[4][2][2], ci[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
    const int lr = threadIdx.x >> 2, lk = (threadIdx.x & 3) * 4;
    const int am = m0 + lr, bn_ = n0 + lr;
    const double2* ap = A + (size_t)am * lda;
    const double2* bp = B + (size_t)bn_ * ldb;
    double2 ra[4], rb[4];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int k = k0 + lk + i;
            ra[i] = (am < M && k < ke) ? ap[k] : make_double2(0.0, 0.0);
            rb[i] = (bn_ < N && k < ke) ? bp[k] : make_double2(0.0, 0.0);
        }
    };
    if (kb < ke) fetch(kb);
    for (int k0 = kb; k0 < ke; k0 += BK) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Ar[lr][lk + i] = ra[i].x; Ai[lr][lk + i] = ra[i].y;
            Br[lr][lk + i] = rb[i].x; Bi[lr][lk + i] = rb[i].y;
        }
        __syncthreads();
        if (k0 + BK < ke) fetch(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double br[2], bi[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int n = wn * 16 + j * 8 + gid;
                br[j] = Br[n][kk + tig];
                bi[j] = Bi[n][kk + tig];
            }
            double ar[4], ai[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int m = wm * 32 + i * 8 + gid;
                ar[i] = Ar[m][kk + tig];
                ai[i] = Ai[m][kk + tig];
            }
            // two rounds of 16 independent MMAs: each accumulator's second
            // product comes 16 MMAs after its first
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma(cr[i][j], ar[i], br[j]);
                    dmma(ci[i][j], ar[i], bi[j]);
                }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma(cr[i][j], ai[i], bi[j]);
                    dmma(ci[i][j], -ai[i], br[j]);
                }
        }
        __syncthreads();
    }
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
                if (n < N) pp[(size_t)m * N + n] = make_double2(cr[i][j][e], ci[i][j][e]);
            }
    }
}

// O[m][n] = alpha sum_k W[k][m] X[k][n] + beta O[m][n]
__global__ void __launch_bounds__(256, 2)
k_zgemm_tn_dmma(const double2* __restrict__ W, int ldw, const double2* __restrict__ X, int ldx,
                double2* O, int ldo, int M, int N, int K, double alpha, double beta) {
    __shared__ double Wr[BK][kDT], Wi[BK][kDT], Xr[BK][kDT], Xi[BK][kDT];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;
    const int n0 = blockIdx.x * BN, m0 = blockIdx.y * BM;
    double cr[4][2][2], ci[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;
    const int lk = threadIdx.x >> 4, lc = (threadIdx.x & 15) * 4;
    double2 rw[4], rx[4];
    auto fetch = [&](int k0) {
        const int k = k0 + lk;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int m = m0 + lc + i, n = n0 + lc + i;
            rw[i] = (k < K && m < M) ? W[(size_t)k * ldw + m] : make_double2(0.0, 0.0);
            rx[i] = (k < K && n < N) ? X[(size_t)k * ldx + n] : make_double2(0.0, 0.0);
        }
    };
    fetch(0);
    for (int k0 = 0; k0 < K; k0 += BK) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            Wr[lk][lc + i] = rw[i].x; Wi[lk][lc + i] = rw[i].y;
            Xr[lk][lc + i] = rx[i].x; Xi[lk][lc + i] = rx[i].y;
        }
        __syncthreads();
        if (k0 + BK < K) fetch(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double xr[2], xi[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int n = wn * 16 + j * 8 + gid;
                xr[j] = Xr[kk + tig][n];
                xi[j] = Xi[kk + tig][n];
            }
            double wr[4], wi[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int m = wm * 32 + i * 8 + gid;
                wr[i] = Wr[kk + tig][m];
                wi[i] = Wi[kk + tig][m];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma(cr[i][j], wr[i], xr[j]);
                    dmma(ci[i][j], wr[i], xi[j]);
                }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma(cr[i][j], -wi[i], xi[j]);
                    dmma(ci[i][j], wi[i], xr[j]);
                }
        }
        __syncthreads();
    }
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
                double2 r = make_double2(alpha * cr[i][j][e], alpha * ci[i][j][e]);
                if (beta != 0.0) {
                    r.x += beta * o->x;
                    r.y += beta * o->y;
                }
                *o = r;
            }
    }
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

// Two CTAs of k_zgemm_cn_dmma fit an SM, so the grid runs in waves of 296.
// The split count that fills the last wave best wins (a larger one only
// when it fills it 2 % better), with at least 256 k per split and 64 splits
// at most.  E.g. the 256-projector x 160-band product (12 tiles) runs as 49
// splits, 588 CTAs in two full waves, not as 25 splits, 300 CTAs in 1.01
// waves; psi^H psi of 576 bands (81 tiles) as 18 splits, 1,458 CTAs in 4.93
// waves, not as 4 splits, 324 CTAs in 1.09 waves.
int splitk_count(int M, int N, int K) {
    return splitk_count_tiles(((M + BM - 1) / BM) * ((N + BN - 1) / BN), K);
}

int splitk_count_tiles(int tiles, int K) {
    const int max_splits = std::min(64, std::max(1, (K + 255) / 256));
    int best = 1;
    double best_eff = -1.0;
    for (int s = 1; s <= max_splits; ++s) {
        const long long ctas = (long long)tiles * s;
        const long long waves = (ctas + 295) / 296;
        const double eff = (double)ctas / (waves * 296.0);
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
    k_zgemm_cn_dmma<<<grid, 256, 0, st>>>(A, lda, B, ldb, M, N, K, kchunk, part, 0);
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
    k_zgemm_cn_dmma<<<grid, 256, 0, st>>>(A, lda, B, ldb, N, N, K, kchunk, part, tn);
    const size_t nn = (size_t)N * N;
    int blocks = (int)((nn + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_reduce_herm<<<blocks, 256, 0, st>>>(part, used, N, out);
}

void gemm_tn(const double2* W, int ldw, const double2* X, int ldx, double2* O, int ldo, int M,
             int N, int K, double alpha, double beta, cudaStream_t st) {
    count_launch();
    dim3 grid((N + BN - 1) / BN, (M + BM - 1) / BM);
    k_zgemm_tn_dmma<<<grid, 256, 0, st>>>(W, ldw, X, ldx, O, ldo, M, N, K, alpha, beta);
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
    k_zgemm_cn_dmma<<<grid, 256, 0, st>>>(A, lda, B, ldb, M, N, K, kchunk, part, 0);
    const size_t mn = (size_t)M * N;
    int blocks = (int)((mn + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_reduce_partials<<<blocks, 256, 0, st>>>(part, used, mn, out);
}

}  // namespace chfsi
