// tcgen05 (5th-generation tensor core) complex GEMM in BF16 3-way split
// precision with FP32 accumulation in TMEM, operands fed by TMA.
//
// Complex product C[m][n] = sum_k conj(A[m][k]) B[n][k] as one real GEMM:
//   A'' (2M x 2K): row 2m = (a_re, a_im) pairs, row 2m+1 = (-a_im, a_re) pairs
//   B'  ( N x 2K): row n  = (b_re, b_im) pairs (the interleaved complex row)
//   C''[2m][n] = Re C[m][n],  C''[2m+1][n] = Im C[m][n]
// Each real operand x is split x = x1 + x2 + x3 (bf16, x2 = bf16(x - x1), ...)
// and the six leading products (3,1) (2,2) (1,3) (2,1) (1,2) (1,1) are
// accumulated into one TMEM tile (small terms first): relative error at the
// FP32 level with BF16 tensor-core throughput.
//
// Kernel structure (one CTA per 128 x BN output tile and K range):
//   warp 0 lane 0: TMA producer, 3-stage ring; a stage holds all six
//                  operand tiles of one 32-wide K slice, {A1, A2, A3}
//                  128x32 and {B1, B2, B3} BNx32 bf16 with 64-byte swizzle,
//                  one mbarrier complete_tx for the six loads
//   warp 1 lane 0: MMA issuer, 6 products x 2 tcgen05.mma (M128 x N BN x
//                  K16) per stage, tcgen05.commit frees the stage; the five
//                  small products accumulate in a second TMEM accumulator
//                  (FP32 rounding of each small term against its own sum,
//                  not against the leading product's)
//   all 4 warps  : epilogue, tcgen05.ld 32 lanes x 16 columns per step
// Every plane is loaded once per K slice and feeds the products that use it
// (A1 and B1 three times, A2 and B2 twice): half the shared-memory fill of
// one {A, B} pair per product, 60-72 KB per 12 MMAs.
// Every wait is bounded in time (%globaltimer) and in iterations; on timeout
// the kernel records the failure in an error word, stops issuing work, waits
// (again bounded) for the TMA loads and MMAs it has already issued, frees its
// TMEM and returns, so the context stays usable and the host reads the error.
#include "gemm_tc.hpp"
#include "launch_count.hpp"

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <unordered_map>

namespace chfsi {

namespace {

constexpr int kBM = 128;
constexpr int kBK = 64;          // K padding and K-split granule (bf16 elements)
// Stage shapes: SK = 32 (one 64-byte swizzle row of bf16 per tile row, 3
// stages, BN up to 256) or SK = 64 (128-byte swizzle, 2 stages, BN up to 160);
// both hold the six plane tiles of one K slice per stage.
template <int SK> struct TcStage {
    static constexpr int stages = SK == 32 ? 3 : 2;
};
constexpr int kThreads = 128;
// hard cap on polls of one wait, whatever the clock says
constexpr long long kSpinLimit = 1LL << 30;
// time limit of one wait in normal operation (a whole GEMM takes milliseconds)
constexpr unsigned long long kWaitNs = 4000000000ULL;
// time limit while a test has switched the producer's loads off
constexpr unsigned long long kInjectedWaitNs = 20000000ULL;

std::atomic<int> g_inject_no_loads{0};

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Parity wait bounded by wait_ns of device time (and kSpinLimit polls);
// returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity,
                                          unsigned long long wait_ns) {
    const uint32_t a = smem_u32(bar);
    const unsigned long long t0 = global_ns();
    for (long long i = 0; i < kSpinLimit; ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 63) == 63 && global_ns() - t0 > wait_ns) return false;
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// K-major swizzled operand tile: rows of SK bf16 (SK = 32: 64 B rows, 64-byte
// swizzle, 8-row groups 512 B apart; SK = 64: 128 B rows, 128-byte swizzle,
// 8-row groups 1024 B apart), start address advanced 32 B per K=16 step.
template <int SK>
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;                  // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)((8 * SK * 2) >> 4) << 32;  // stride byte offset: 8 rows
    d |= (uint64_t)1 << 46;                  // descriptor version (sm_100)
    d |= (uint64_t)(SK == 32 ? 4 : 2) << 61; // 64-byte or 128-byte swizzle
    return d;
}

// kind::f16 instruction descriptor: BF16 x BF16 -> F32, K-major A and B.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
        "%12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct TcMaps {
    CUtensorMap a[3];
    CUtensorMap b[3];
};

// out modes
enum { kOutPartialF32 = 0, kOutComplexF32 = 1, kOutComplexF64 = 2 };

template <int MODE, int SK>
__global__ void __launch_bounds__(kThreads, 1)
k_umma_split3(const __grid_constant__ TcMaps maps, int M2, int N, int bn, int ktiles_total,
              int ktiles_per_split, void* out, long long ldo, int* err,
              unsigned long long wait_ns, int no_loads) {
    constexpr int kSK = SK;
    constexpr int kStages = TcStage<SK>::stages;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned stage ring: stage s = [A1 A2 A3 B1 B2 B3]
    unsigned char* base = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const int a_bytes = kBM * kSK * 2;
    const int b_bytes = bn * kSK * 2;
    const int stage_bytes = 3 * (a_bytes + b_bytes);
    uint64_t* full = (uint64_t*)(base + kStages * stage_bytes);
    uint64_t* empty = full + kStages;
    uint64_t* done = empty + kStages;
    uint32_t* tmem_slot = (uint32_t*)(done + 1);
    int* abort_flag = (int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * bn;
    // K slices of kSK columns: ktiles_* count kBK-wide tiles
    const int kt0 = blockIdx.z * ktiles_per_split;
    const int kt1 = min(ktiles_total, kt0 + ktiles_per_split);
    const int nk = kt1 - kt0;
    const int iters = (kBK / kSK) * (nk > 0 ? nk : 0);
    const int ks0 = (kBK / kSK) * kt0;
    // (a plane, b plane) pairs, smallest terms first
    const int pa[6] = {2, 1, 0, 1, 0, 0};
    const int pb[6] = {0, 1, 2, 0, 1, 0};
    // two accumulators of acc_cols TMEM columns each: the five small
    // products sum in the second, the leading product (1,1) in the first,
    // so that no small term is rounded against the large running sum; the
    // epilogue adds the two
    int acc_cols = 32;
    while (acc_cols < bn) acc_cols <<= 1;
    const int ncols = 2 * acc_cols;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_slot)),
                     "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0 && iters > 0 && !no_loads) {
        // ---- TMA producer (no_loads: a test switch under which nothing is
        // issued, so the MMA warp's first wait runs out with nothing in flight)
        int issued = 0;
        bool aborted = false;
        for (int it = 0; it < iters; ++it) {
            const int s = it % kStages;
            const uint32_t ph = (it / kStages) & 1;
            if (it >= kStages && !mbar_wait(&empty[s], ph ^ 1, wait_ns)) {
                atomicExch(err, 1);
                *(volatile int*)abort_flag = 1;
                aborted = true;
                break;
            }
            if (*(volatile int*)abort_flag) { aborted = true; break; }
            const int kx = (ks0 + it) * kSK;
            unsigned char* st_base = base + (size_t)s * stage_bytes;
            mbar_expect_tx(&full[s], stage_bytes);
#pragma unroll
            for (int i = 0; i < 3; ++i)
                tma_load_2d(st_base + i * a_bytes, &maps.a[i], &full[s], kx, m0);
#pragma unroll
            for (int i = 0; i < 3; ++i)
                tma_load_2d(st_base + 3 * a_bytes + i * b_bytes, &maps.b[i], &full[s], kx, n0);
            ++issued;
        }
        if (aborted) {
            // retire the loads still in flight (the last kStages issued)
            // before the CTA releases its shared memory
            for (int j = issued > kStages ? issued - kStages : 0; j < issued; ++j)
                if (!mbar_wait(&full[j % kStages], (j / kStages) & 1, wait_ns)) {
                    atomicExch(err, 4);
                    break;
                }
        }
    } else if (warp == 1 && lane == 0 && iters > 0) {
        // ---- MMA issuer
        const uint32_t idesc = idesc_bf16(kBM, bn);
        bool ok = true;
        for (int it = 0; it < iters; ++it) {
            const int s = it % kStages;
            const uint32_t ph = (it / kStages) & 1;
            if (!mbar_wait(&full[s], ph, wait_ns)) {
                atomicExch(err, 2);
                *(volatile int*)abort_flag = 1;
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t st_addr = smem_u32(base + (size_t)s * stage_bytes);
#pragma unroll
            for (int t = 0; t < 6; ++t) {
                const uint64_t da = umma_desc<SK>(st_addr + pa[t] * a_bytes);
                const uint64_t db = umma_desc<SK>(st_addr + 3 * a_bytes + pb[t] * b_bytes);
                const bool lead = t == 5;
                const uint32_t acc = lead ? tmem : tmem + (uint32_t)acc_cols;
#pragma unroll
                for (int k = 0; k < kSK / 16; ++k)
                    umma_bf16(acc, da + 2 * k, db + 2 * k, idesc,
                              (it > 0 || (!lead && t > 0) || k > 0) ? 1u : 0u);
            }
            umma_commit(&empty[s]);
        }
        (void)ok;
        // arrives once every MMA issued above has completed (also on abort)
        umma_commit(done);
    }
    __syncwarp();
    // ---- epilogue: every warp reads its 32 TMEM lanes
    bool have = iters > 0;
    if (have) {
        if (!mbar_wait(done, 0, wait_ns)) {
            atomicExch(err, 3);
            have = false;
        }
    }
    have = __all_sync(0xffffffffu, have);  // tcgen05.ld is warp-collective
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < bn; c0 += 16) {
        uint32_t r[16];
        if (have) {
            uint32_t rs[16];
            const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            tmem_ld16(ta, r);
            tmem_ld16(ta + (uint32_t)acc_cols, rs);
#pragma unroll
            for (int j = 0; j < 16; ++j)
                r[j] = __float_as_uint(__uint_as_float(r[j]) + __uint_as_float(rs[j]));
        } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) r[j] = 0u;
        }
        if (MODE == kOutPartialF32) {
            float* o = (float*)out + (long long)blockIdx.z * ldo * M2;
            if (row < M2) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + c0 + j;
                    if (col < N) o[(long long)row * ldo + col] = __uint_as_float(r[j]);
                }
            }
        } else {
            // rows 2m (real) and 2m+1 (imaginary) sit in adjacent lanes
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const float v = __uint_as_float(r[j]);
                const float w = __shfl_down_sync(0xffffffffu, v, 1);
                const int col = n0 + c0 + j;
                if ((lane & 1) == 0 && row + 1 < M2 + 1 && row < M2 && col < N) {
                    const long long m = row >> 1;
                    if (MODE == kOutComplexF32)
                        ((float2*)out)[m * ldo + col] = make_float2(v, w);
                    else
                        ((double2*)out)[m * ldo + col] = make_double2((double)v, (double)w);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
    }
}

// ---- operand packing: complex rows -> three bf16 planes (split 1 + 2 + 3)
__device__ __forceinline__ void split3(float v, __nv_bfloat16& h1, __nv_bfloat16& h2,
                                       __nv_bfloat16& h3) {
    h1 = __float2bfloat16_rn(v);
    const float r1 = v - __bfloat162float(h1);
    h2 = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(h2);
    h3 = __float2bfloat16_rn(r2);
}

// SRC: 0 element (r, k) = x[r][k]; 1 = conj(x[k][r]); 2 = x[k][r]
template <typename CIn, bool DOUBLED, int SRC>
__global__ void k_pack3(const CIn* __restrict__ x, long long ldx, int rows, int K, int kp,
                        __nv_bfloat16* __restrict__ p0, __nv_bfloat16* __restrict__ p1,
                        __nv_bfloat16* __restrict__ p2) {
    // DOUBLED: output rows 2r, 2r+1 per input row (conj-first operand)
    const long long kc = kp / 2;  // complex columns incl. padding
    const long long tot = (long long)rows * kc;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        int r, k;
        if (SRC == 0) { r = (int)(t / kc); k = (int)(t % kc); }
        else { k = (int)(t / rows); r = (int)(t % rows); }  // coalesced reads of x[k][*]
        float re = 0.f, im = 0.f;
        if (k < K) {
            if (SRC == 0) {
                const CIn v = x[(long long)r * ldx + k];
                re = (float)v.x;
                im = (float)v.y;
            } else {
                const CIn v = x[(long long)k * ldx + r];
                re = (float)v.x;
                im = SRC == 1 ? -(float)v.y : (float)v.y;
            }
        }
        __nv_bfloat16 a1, a2, a3, b1, b2, b3;
        split3(re, a1, a2, a3);
        split3(im, b1, b2, b3);
        if (DOUBLED) {
            const long long o0 = (2LL * r) * kp + 2 * k, o1 = (2LL * r + 1) * kp + 2 * k;
            p0[o0] = a1; p0[o0 + 1] = b1; p1[o0] = a2; p1[o0 + 1] = b2; p2[o0] = a3; p2[o0 + 1] = b3;
            // (-im, re)
            p0[o1] = __hneg(b1); p0[o1 + 1] = a1;
            p1[o1] = __hneg(b2); p1[o1 + 1] = a2;
            p2[o1] = __hneg(b3); p2[o1 + 1] = a3;
        } else {
            const long long o = (long long)r * kp + 2 * k;
            p0[o] = a1; p0[o + 1] = b1; p1[o] = a2; p1[o + 1] = b2; p2[o] = a3; p2[o + 1] = b3;
        }
    }
}

// sum of split-K partials -> complex (rows 2m, 2m+1 -> re, im), FP64 output
__global__ void k_reduce_tc(const float* __restrict__ part, int splits, int M, int N,
                            double2* __restrict__ out) {
    const long long mn = (long long)M * N;
    const long long stride = 2LL * M * N;  // one partial = (2M) x N
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < mn;
         t += (long long)gridDim.x * blockDim.x) {
        const long long m = t / N, n = t % N;
        double re = 0.0, im = 0.0;
        for (int s = 0; s < splits; ++s) {
            re += part[s * stride + (2 * m) * N + n];
            im += part[s * stride + (2 * m + 1) * N + n];
        }
        out[t] = make_double2(re, im);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

bool make_map(CUtensorMap* m, const void* ptr, int rows, int kp, int box_rows, int sk) {
    auto enc = get_encode();
    if (!enc || rows < box_rows) return false;
    cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
    cuuint32_t box[2] = {(cuuint32_t)sk, (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims, strides,
                     box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     sk == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// Launch shapes the autotuner chooses from: stage K width and the largest
// N tile (the N tiles of a product are balanced below that cap).
struct TcVariant { int sk; int bn_cap; };
constexpr TcVariant kTcVariants[kTcVariantCount] = {{32, 256}, {32, 128}, {64, 160}};

// Tensor maps are a pure function of (address, rows, K padding, box rows,
// stage K width); the planes of a context live as long as the context, so
// their maps are encoded once and reused.  The cache is cleared when it grows
// past kMapCacheMax entries (one-off operands of chfsi_zgemm_cn_bf16x3).
struct MapKey {
    const void* ptr;
    int rows, kp, box, sk;
    bool operator==(const MapKey& o) const {
        return ptr == o.ptr && rows == o.rows && kp == o.kp && box == o.box && sk == o.sk;
    }
};
struct MapKeyHash {
    size_t operator()(const MapKey& k) const {
        size_t h = std::hash<const void*>()(k.ptr);
        for (int v : {k.rows, k.kp, k.box, k.sk}) h = h * 1000003u ^ std::hash<int>()(v);
        return h;
    }
};
constexpr size_t kMapCacheMax = 256;
std::mutex g_map_mu;
std::unordered_map<MapKey, CUtensorMap, MapKeyHash> g_map_cache;

bool cached_map(CUtensorMap* m, const void* ptr, int rows, int kp, int box_rows, int sk) {
    const MapKey key{ptr, rows, kp, box_rows, sk};
    {
        std::lock_guard<std::mutex> lk(g_map_mu);
        auto it = g_map_cache.find(key);
        if (it != g_map_cache.end()) {
            *m = it->second;
            return true;
        }
    }
    if (!make_map(m, ptr, rows, kp, box_rows, sk)) return false;
    std::lock_guard<std::mutex> lk(g_map_mu);
    if (g_map_cache.size() >= kMapCacheMax) g_map_cache.clear();
    g_map_cache.emplace(key, *m);
    return true;
}

// Dynamic shared memory limit of a kernel, raised on a device only when a
// launch needs more than it was last set to.
std::mutex g_attr_mu;
std::unordered_map<const void*, int> g_attr_smem[64];

cudaError_t ensure_smem(const void* kernel, int bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    std::lock_guard<std::mutex> lk(g_attr_mu);
    int& have = g_attr_smem[dev][kernel];
    if (have >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}

int pick_bn(int n, int cap) {
    const int tiles = (n + cap - 1) / cap;
    int bn = (n + tiles - 1) / tiles;
    bn = (bn + 15) / 16 * 16;
    return bn < 16 ? 16 : (bn > cap ? cap : bn);
}

size_t smem_bytes(int bn, int sk) {
    const int stages = sk == 32 ? TcStage<32>::stages : TcStage<64>::stages;
    return 1024 + (size_t)stages * 3 * (kBM * sk * 2 + bn * sk * 2) + (2 * stages + 1) * 8 + 16;
}

int grid_for(long long n) {
    long long b = (n + 255) / 256;
    return (int)(b < 148 * 8 ? b : 148 * 8);
}

}  // namespace

int tc_kpad(int K) { return ((2 * K + kBK - 1) / kBK) * kBK; }

// K-split count of the partial-output mode.  One CTA fits an SM, so the
// grid runs in waves of 148; the split that fills the last wave best wins
// (a larger split only when it fills it 2 % better), with at least 8 K-tiles
// per split.  E.g. 81 tiles (the projector GEMM of 1,728 projectors x 576
// bands) run as 9 splits, 729 CTAs in 4.93 waves, instead of 2 splits, 162
// CTAs in 1.09 waves.
int tc_splits(int tiles, int ktiles) {
    const int smax = std::max(1, std::min(64, ktiles / 8));
    int best = 1;
    double best_eff = -1.0;
    for (int s = 1; s <= smax; ++s) {
        const int ctas = tiles * s;
        const int waves = (ctas + 147) / 148;
        const double eff = (double)ctas / (waves * 148.0);
        if (eff > best_eff + 0.02) {
            best_eff = eff;
            best = s;
        }
    }
    const int kps = (ktiles + best - 1) / best;
    return (ktiles + kps - 1) / kps;
}

size_t tc_partial_floats(int M, int N, int K) {
    const int kp = tc_kpad(K);
    const int ktiles = kp / kBK;
    const int mt = (2 * M + kBM - 1) / kBM;
    size_t most = 0;
    for (const TcVariant& v : kTcVariants) {
        const int bn = pick_bn(N, v.bn_cap), nt = (N + bn - 1) / bn;
        most = std::max(most, (size_t)tc_splits(mt * nt, ktiles) * 2 * M * N);
    }
    return most;
}

template <typename CIn>
void tc_pack(const CIn* x, long long ldx, int rows, int K, bool doubled, int src,
             TcPlanes& planes, cudaStream_t st) {
    count_launch();
    const int kp = tc_kpad(K);
    __nv_bfloat16* p0 = (__nv_bfloat16*)planes.p[0];
    __nv_bfloat16* p1 = (__nv_bfloat16*)planes.p[1];
    __nv_bfloat16* p2 = (__nv_bfloat16*)planes.p[2];
    const long long tot = (long long)rows * (kp / 2);
    const int g = grid_for(tot);
#define CHFSI_PACK(D, S) k_pack3<CIn, D, S><<<g, 256, 0, st>>>(x, ldx, rows, K, kp, p0, p1, p2)
    if (doubled) {
        if (src == kSrcConjT) CHFSI_PACK(true, 1);
        else if (src == kSrcT) CHFSI_PACK(true, 2);
        else CHFSI_PACK(true, 0);
    } else {
        if (src == kSrcConjT) CHFSI_PACK(false, 1);
        else if (src == kSrcT) CHFSI_PACK(false, 2);
        else CHFSI_PACK(false, 0);
    }
#undef CHFSI_PACK
    planes.rows = doubled ? 2 * rows : rows;
    planes.kp = kp;
}

int tc_rows_alloc(int rows, bool a_operand, int n_for_b) {
    // the largest TMA box of any variant (variant 0 has the largest N tiles)
    const int box = a_operand ? kBM : pick_bn(n_for_b, kTcVariants[0].bn_cap);
    return rows < box ? box : rows;
}

cudaError_t tc_gemm(const TcPlanes& a, const TcPlanes& b, int M, int N, int K, int out_mode,
                    void* out, long long ldo, float* part, int* err, cudaStream_t st, int variant) {
    if (a.kp != tc_kpad(K) || b.kp != a.kp || a.rows != 2 * M || b.rows != N)
        return cudaErrorInvalidValue;
    if (variant < 0 || variant >= kTcVariantCount) return cudaErrorInvalidValue;
    const TcVariant var = kTcVariants[variant];
    const int bn = pick_bn(N, var.bn_cap);
    if (a.rows_alloc < kBM || b.rows_alloc < bn) return cudaErrorInvalidValue;
    TcMaps maps;
    for (int i = 0; i < 3; ++i) {
        if (!cached_map(&maps.a[i], a.p[i], a.rows_alloc, a.kp, kBM, var.sk)) return cudaErrorInvalidValue;
        if (!cached_map(&maps.b[i], b.p[i], b.rows_alloc, b.kp, bn, var.sk)) return cudaErrorInvalidValue;
    }
    const int ktiles = a.kp / kBK;
    const int mt = (2 * M + kBM - 1) / kBM, nt = (N + bn - 1) / bn;
    int splits = 1;
    if (out_mode == kTcOutPartial) splits = tc_splits(mt * nt, ktiles);
    const int kps = (ktiles + splits - 1) / splits;
    splits = (ktiles + kps - 1) / kps;
    dim3 grid(mt, nt, splits);
    const size_t sm = smem_bytes(bn, var.sk);
    int no_loads = 0;
    unsigned long long wait_ns = kWaitNs;
    for (int left = g_inject_no_loads.load(); left > 0; left = g_inject_no_loads.load())
        if (g_inject_no_loads.compare_exchange_weak(left, left - 1)) {
            no_loads = 1;
            wait_ns = kInjectedWaitNs;
            break;
        }
    count_launch();
    auto launch = [&](auto kernel, void* dst, long long ld) {
        ensure_smem((const void*)kernel, (int)sm);
        kernel<<<grid, kThreads, sm, st>>>(maps, 2 * M, N, bn, ktiles, kps, dst, ld, err, wait_ns,
                                           no_loads);
    };
    const bool s64 = var.sk == 64;
    if (out_mode == kTcOutPartial) {
        if (s64) launch(k_umma_split3<kOutPartialF32, 64>, part, N);
        else launch(k_umma_split3<kOutPartialF32, 32>, part, N);
        count_launch();
        k_reduce_tc<<<grid_for((long long)M * N), 256, 0, st>>>(part, splits, M, N, (double2*)out);
    } else if (out_mode == kTcOutComplexF32) {
        if (s64) launch(k_umma_split3<kOutComplexF32, 64>, out, ldo);
        else launch(k_umma_split3<kOutComplexF32, 32>, out, ldo);
    } else {
        if (s64) launch(k_umma_split3<kOutComplexF64, 64>, out, ldo);
        else launch(k_umma_split3<kOutComplexF64, 32>, out, ldo);
    }
    return cudaGetLastError();
}

void tc_inject_no_loads(int launches) { g_inject_no_loads.store(launches < 0 ? 0 : launches); }

template void tc_pack<double2>(const double2*, long long, int, int, bool, int, TcPlanes&, cudaStream_t);
template void tc_pack<float2>(const float2*, long long, int, int, bool, int, TcPlanes&, cudaStream_t);

}  // namespace chfsi
