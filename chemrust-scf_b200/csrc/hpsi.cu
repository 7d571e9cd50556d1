// Local Hamiltonian H_loc|psi> = T psi + FFT^-1[V(r) FFT[psi]] on the
// G-sphere, as three pruned passes over a band batch (role of the reference's
// init_kinetic / zero / scatter / cuFFT Z2Z / veff_multiply / cuFFT /
// gather_add_kinetic sequence, src/eigensolver/chebyshev.rs:279-365):
//
//   pass 1  z-sticks:  scatter the sphere coefficients of a group of (x,y)
//           columns into smem z-lines, inverse FFT along z, write the sticks
//           plane-major: work[b][z][column]
//   pass 2  xy-planes: unpack one z-plane (only the columns that carry
//           plane waves), inverse FFT along y (active x lines only) and x,
//           multiply by V(r), forward FFT along x and y (active x lines),
//           pack the columns back in place
//   pass 3  z-sticks:  forward FFT along z, gather the sphere, add the
//           kinetic and non-local terms and run the Chebyshev-recurrence
//           epilogue, reducing |psi_k|^2 for the norm guard
//
// HBM traffic per band: 4 x (ncol x nz) complex words plus the sphere
// vectors, versus ~14 N^3 words for the unpruned zero/scatter/FFT/multiply/
// FFT/gather sequence.
#include "kernels.hpp"
#include "launch_count.hpp"

#include <cstdio>

namespace chfsi {

namespace {

template <typename C> __device__ __forceinline__ C czero() {
    using R = typename RealOf<C>::type;
    return mk((R)0, (R)0);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum; result valid in thread 0.  red needs blockDim/32 doubles.
__device__ __forceinline__ double block_sum(double v, double* red) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

template <typename C> __host__ __device__ __forceinline__ size_t align16(size_t n) {
    return (n * sizeof(C) + 15) & ~(size_t)15;
}

// ---- two-radix line transforms with compile-time plans (N = R0 R1; DIF
// stage 0: radix R0 with span R1; stage 1: radix R1 on blocks of R1
// consecutive elements, all twiddles 1), used by the z-stick and plane passes
// radix-R1 stage on block blk (elements blk R1 .. blk R1 + R1 - 1)
template <int R0, int R1, int SIGN, typename C>
__device__ __forceinline__ void p2_blocks(C* line, int es, int blk) {
    constexpr int N = R0 * R1;
    C x[R1];
#pragma unroll
    for (int j = 0; j < R1; ++j) x[j] = line[swz(blk * R1 + j, N) * es];
    dft_r<R1, SIGN>(x);
#pragma unroll
    for (int m = 0; m < R1; ++m) line[swz(blk * R1 + m, N) * es] = x[m];
}
template <int R0, int R1, typename C>
__device__ __forceinline__ void p2_load_span(const C* line, int es, int n1, C* x) {
#pragma unroll
    for (int j = 0; j < R0; ++j) x[j] = line[swz(n1 + j * R1, R0 * R1) * es];
}
template <int R0, int R1, typename C>
__device__ __forceinline__ void p2_store_span(C* line, int es, int n1, const C* x) {
#pragma unroll
    for (int j = 0; j < R0; ++j) line[swz(n1 + j * R1, R0 * R1) * es] = x[j];
}
// Span twiddles in the order the lanes of a group read them:
// twm[(m - 1) R1 + n1] = w^(n1 m), w = exp(2 pi i / (R0 R1)).  For a fixed m
// the lanes n1 = 0 .. R1 - 1 read consecutive entries (no bank conflicts;
// the table w^j indexed by n1 m puts lanes on the same bank group whenever m
// shares a factor with 8).
__device__ __forceinline__ double2 tw_entry(const double2* twd, const float2*, int j, double2) {
    return twd[j];
}
__device__ __forceinline__ float2 tw_entry(const double2*, const float2* twf, int j, float2) {
    return twf[j];
}
template <int R0, int R1, typename C>
__device__ __forceinline__ void p2_twiddles(C* twm, const double2* twd, const float2* twf) {
    for (int i = threadIdx.x; i < (R0 - 1) * R1; i += blockDim.x) {
        const int m = i / R1 + 1, n1 = i - (m - 1) * R1;
        twm[i] = tw_entry(twd, twf, n1 * m, C{});
    }
}
// Lane -> (group, index in group) of the two-radix line transforms with T
// lanes per line and PW lines per warp.  Indices 0-7 of every group fill
// whole 8-lane phases (one line per phase), the higher indices follow
// packed: the 16-byte shared-memory accesses of a phase then fall on one
// line, whose XOR-swizzled elements span all eight bank groups.
template <int T, int PW>
__device__ __forceinline__ void p2_lane(int lane, int& gi, int& li) {
    if constexpr (T <= 8) {
        gi = lane / T;
        li = lane - gi * T;
    } else {
        if (lane < PW * 8) {
            gi = lane >> 3;
            li = lane & 7;
        } else {
            const int r = lane - PW * 8;
            gi = r / (T - 8);
            li = 8 + (r - gi * (T - 8));
        }
    }
}
// Span twiddle w^(n1 m) from the table w^j (TWM false) or from the
// lane-ordered table of p2_twiddles (TWM true)
template <int R1, bool TWM, typename C>
__device__ __forceinline__ C span_tw(const C* tw, int n1, int m) {
    return TWM ? tw[(m - 1) * R1 + n1] : tw[n1 * m];
}
// DIT stage 0 on span n1: twiddle w^(n1 m), radix-R0 DFT (sign +1)
template <int R0, int R1, bool TWM, typename C>
__device__ __forceinline__ void p2_span_inverse(C* x, int n1, const C* tw) {
#pragma unroll
    for (int m = 1; m < R0; ++m) x[m] = cmul(span_tw<R1, TWM>(tw, n1, m), x[m]);
    dft_r<R0, 1>(x);
}
// DIF stage 0 on span n1: radix-R0 DFT (sign -1), twiddle w^(-n1 m)
template <int R0, int R1, bool TWM, typename C>
__device__ __forceinline__ void p2_span_forward(C* x, int n1, const C* tw) {
    dft_r<R0, -1>(x);
#pragma unroll
    for (int m = 1; m < R0; ++m) x[m] = cmulc(span_tw<R1, TWM>(tw, n1, m), x[m]);
}
// whole-line transforms by one lane group (lane i); every lane of the warp
// calls them (act = false: idle)
template <int R0, int R1, bool TWM, typename C>
__device__ __forceinline__ void p2_line_inverse(C* line, bool act, int i, int es, const C* tw) {
    if (act && i < R0) p2_blocks<R0, R1, 1>(line, es, i);
    __syncwarp();
    if (act && i < R1) {
        C x[R0];
        p2_load_span<R0, R1>(line, es, i, x);
        p2_span_inverse<R0, R1, TWM>(x, i, tw);
        p2_store_span<R0, R1>(line, es, i, x);
    }
    __syncwarp();
}
template <int R0, int R1, bool TWM, typename C>
__device__ __forceinline__ void p2_line_forward(C* line, bool act, int i, int es, const C* tw) {
    if (act && i < R1) {
        C x[R0];
        p2_load_span<R0, R1>(line, es, i, x);
        p2_span_forward<R0, R1, TWM>(x, i, tw);
        p2_store_span<R0, R1>(line, es, i, x);
    }
    __syncwarp();
    if (act && i < R0) p2_blocks<R0, R1, -1>(line, es, i);
    __syncwarp();
}

// ---------------------------------------------------------------- pass 1
// z lines of a block of columns transformed by one lane group per line with
// the compile-time two-radix plan (R0 > 0) or by the generic engine
template <int R0, int R1, bool FWD, typename C>
__device__ __forceinline__ void zlines_fft(C* lines, int nl, const HGeom& g, const C* tw) {
    if constexpr (R0 > 0) {
        constexpr int T = R0 > R1 ? R0 : R1, PW = 32 / T;
        const int lane = threadIdx.x & 31, gi = lane / T, li = lane - gi * T;
        const bool ing = gi < PW;
        const int groups = (blockDim.x >> 5) * PW, gid = (threadIdx.x >> 5) * PW + gi;
        for (int l0 = 0; l0 < nl; l0 += groups) {
            const int l = l0 + gid;
            const bool act = ing && l < nl;
            C* line = lines + (act ? l * g.lsz : 0);
            if (FWD) p2_line_forward<R0, R1, false>(line, act, li, 1, tw);
            else p2_line_inverse<R0, R1, false>(line, act, li, 1, tw);
        }
        __syncthreads();
    } else {
        fft_lines_grouped<FWD>(lines, nl, LinesStrided{g.lsz}, 1, g.az, tw);
    }
}

// 3 resident blocks per SM with the compile-time plans (their registers
// allow it), 1 guaranteed with the generic engine
template <int R0> struct ZCfg { static constexpr int min_blocks = R0 > 0 ? 3 : 1; };

template <typename C, int kColsPerBlock, int R0, int R1>
__global__ void __launch_bounds__(256, ZCfg<R0>::min_blocks)
k_zsticks_inverse(const C* __restrict__ psi, int ldp, C* __restrict__ work, HGeom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* lines = reinterpret_cast<C*>(smem_raw + align16<C>(g.nz));
    const int b = blockIdx.y;
    const int c0 = blockIdx.x * kColsPerBlock;
    const int c1 = min(c0 + kColsPerBlock, g.ncol);
    const int nl = c1 - c0;
    copy_twiddles(tw, g.twd_z, g.twf_z, g.nz);
    for (int i = threadIdx.x; i < kColsPerBlock * g.lsz; i += blockDim.x) lines[i] = czero<C>();
    __syncthreads();
    const int g0 = g.col_start[c0], g1 = g.col_start[c1];
    const C* pb = psi + (size_t)b * ldp;
    for (int q = g0 + threadIdx.x; q < g1; q += blockDim.x)
        lines[(g.pw_col[q] - c0) * g.lsz + swz(g.pw_zpos[q], g.nz)] = pb[q];
    __syncthreads();
    zlines_fft<R0, R1, false>(lines, nl, g, tw);
    C* wb = work + (size_t)b * g.nz * g.ncol;
    for (int u = threadIdx.x; u < g.nz * kColsPerBlock; u += blockDim.x) {
        const int z = u / kColsPerBlock, cl = u - z * kColsPerBlock;
        if (cl < nl) wb[(size_t)z * g.ncol + c0 + cl] = lines[cl * g.lsz + swz(z, g.nz)];
    }
}

// ---------------------------------------------------------------- pass 2
// 256 threads with 2 (FP64) or 3 (FP32) resident blocks per SM: the
// global-memory phases of one plane overlap the FFT stages of another.
// Variant 0: 256 threads, 1: 128 threads, 2: 512 threads per block, with as
// many resident blocks per SM as the registers of each precision allow.
template <typename C, int V>
struct PlanesCfg {
    static constexpr int threads = V == 0 ? 256 : (V == 1 ? 128 : 512);
    static constexpr int min_blocks =
        V == 0 ? (sizeof(C) == 16 ? 2 : 3) : (V == 1 ? (sizeof(C) == 16 ? 4 : 6) : 1);
};

template <typename C, int V>
__global__ void __launch_bounds__(PlanesCfg<C, V>::threads, PlanesCfg<C, V>::min_blocks)
k_planes_vloc(C* __restrict__ work, const double* __restrict__ veff, HGeom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* twx = reinterpret_cast<C*>(smem_raw);
    C* twy = reinterpret_cast<C*>(smem_raw + align16<C>(g.nx));
    C* plane = reinterpret_cast<C*>(smem_raw + align16<C>(g.nx) + align16<C>(g.ny));
    int* xl = reinterpret_cast<int*>(plane + (size_t)g.ny * g.lsx);
    const int z = blockIdx.x, b = blockIdx.y;
    copy_twiddles(twx, g.twd_x, g.twf_x, g.nx);
    copy_twiddles(twy, g.twd_y, g.twf_y, g.ny);
    for (int i = threadIdx.x; i < g.nxact; i += blockDim.x) xl[i] = g.xact[i];
    for (int i = threadIdx.x; i < g.ny * g.lsx; i += blockDim.x) plane[i] = czero<C>();
    __syncthreads();
    C* wp = work + ((size_t)b * g.nz + z) * g.ncol;
    for (int c = threadIdx.x; c < g.ncol; c += blockDim.x) plane[g.col_pos[c]] = wp[c];
    __syncthreads();
    fft_lines_grouped<false>(plane, g.nxact, LinesListed{xl}, g.lsx, g.ay, twy);
    // x rows: inverse, x V(r), forward, all inside one lane group per row
    const double* vz = veff + (size_t)z * g.nx * g.ny;
    using R = typename RealOf<C>::type;
    {
        const LaneGroups lg(g.ax.tpl);
        const int rounds = (g.ny + lg.total - 1) / lg.total;
        for (int rd = 0; rd < rounds; ++rd) {
            const int y = rd * lg.total + lg.id;
            const bool act = lg.in_group && y < g.ny;
            C* row = plane + (act ? swz(y, g.ny) * g.lsx : 0);
            line_fft_group<false>(row, act, lg.i, 1, g.ax, twx);
            if (act) {
                const double* vr = vz + (size_t)y * g.nx;
                for (int x = lg.i; x < g.nx; x += g.ax.tpl) {
                    C& e = row[swz(x, g.nx)];
                    e = cscale(e, (R)vr[x]);
                }
            }
            __syncwarp();
            line_fft_group<true>(row, act, lg.i, 1, g.ax, twx);
        }
    }
    __syncthreads();
    fft_lines_grouped<true>(plane, g.nxact, LinesListed{xl}, g.lsx, g.ay, twy);
    for (int c = threadIdx.x; c < g.ncol; c += blockDim.x) wp[c] = plane[g.col_pos[c]];
}

// ------------------------------------------ pass 2, two-radix compile-time plans
// The same plane pipeline for axes whose plan has two radices, N = R0 R1
// (DIF stage 0: radix R0 with span R1; stage 1: radix R1 on blocks of R1
// consecutive elements, where every twiddle is 1).  Radices, spans and
// twiddle indices are compile-time constants, and along x the last inverse
// stage, the V(r) multiply and the first forward stage share registers:
// lane n1 of a row's lane group holds the R0 elements n1 + m R1, which is
// what those two stages read and write.

// Square planes (nx = ny = R0 R1, both axes on the same plan); shared memory
// layout and launch shape as k_planes_vloc.
template <typename C, int V, int R0, int R1>
__global__ void __launch_bounds__(PlanesCfg<C, V>::threads, PlanesCfg<C, V>::min_blocks)
k_planes_vloc_p2(C* __restrict__ work, const double* __restrict__ veff, HGeom g) {
    constexpr int N = R0 * R1, LS = N | 1, T = R0 > R1 ? R0 : R1, PW = 32 / T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* twx = reinterpret_cast<C*>(smem_raw);
    C* twy = reinterpret_cast<C*>(smem_raw + align16<C>(N));
    C* plane = reinterpret_cast<C*>(smem_raw + 2 * align16<C>(N));
    int* xl = reinterpret_cast<int*>(plane + (size_t)N * LS);
    const int z = blockIdx.x, b = blockIdx.y;
    const int nxact = g.nxact;
    p2_twiddles<R0, R1, C>(twx, g.twd_x, g.twf_x);
    p2_twiddles<R0, R1, C>(twy, g.twd_y, g.twf_y);
    for (int i = threadIdx.x; i < nxact; i += blockDim.x) xl[i] = g.xact[i];
    for (int i = threadIdx.x; i < N * LS; i += blockDim.x) plane[i] = czero<C>();
    __syncthreads();
    C* wp = work + ((size_t)b * g.nz + z) * g.ncol;
    for (int c = threadIdx.x; c < g.ncol; c += blockDim.x) plane[g.col_pos[c]] = wp[c];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    int gi, li;
    p2_lane<T, PW>(lane, gi, li);
    const bool ing = gi < PW;
    const int groups = (blockDim.x >> 5) * PW, gid = (threadIdx.x >> 5) * PW + gi;
    // y lines through the active x positions
    for (int l0 = 0; l0 < nxact; l0 += groups) {
        const int l = l0 + gid;
        const bool act = ing && l < nxact;
        p2_line_inverse<R0, R1, true>(plane + (act ? xl[l] : 0), act, li, LS, twy);
    }
    __syncthreads();
    // x rows: inverse, x V(r), forward
    using R = typename RealOf<C>::type;
    const double* vz = veff + (size_t)z * N * N;
    for (int y0 = 0; y0 < N; y0 += groups) {
        const int y = y0 + gid;
        const bool act = ing && y < N;
        C* row = plane + (act ? swz(y, N) * LS : 0);
        if (act && li < R0) p2_blocks<R0, R1, 1>(row, 1, li);
        __syncwarp();
        if (act && li < R1) {
            C x[R0];
            p2_load_span<R0, R1>(row, 1, li, x);
            p2_span_inverse<R0, R1, true>(x, li, twx);
            const double* vr = vz + (size_t)y * N + li;
#pragma unroll
            for (int m = 0; m < R0; ++m) x[m] = cscale(x[m], (R)vr[m * R1]);
            p2_span_forward<R0, R1, true>(x, li, twx);
            p2_store_span<R0, R1>(row, 1, li, x);
        }
        __syncwarp();
        if (act && li < R0) p2_blocks<R0, R1, -1>(row, 1, li);
        __syncwarp();
    }
    __syncthreads();
    for (int l0 = 0; l0 < nxact; l0 += groups) {
        const int l = l0 + gid;
        const bool act = ing && l < nxact;
        p2_line_forward<R0, R1, true>(plane + (act ? xl[l] : 0), act, li, LS, twy);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < g.ncol; c += blockDim.x) wp[c] = plane[g.col_pos[c]];
}

// ------------------------------- pass 2, compile-time plans, no zero fill
// The compile-time pipeline with the plane's columns read and written in
// place of the shared-memory scatter and gather: the first inverse y stage
// of every active x line loads its inputs from the column array (zero where
// (x, y) holds no column), the last forward y stage stores its outputs
// straight to the columns, the first inverse x stage reads zero for x
// positions without columns instead of loading them, and the last forward x
// stage stores only the x positions the forward y stage reads.  No position
// of the plane is ever read before this CTA writes it, so the plane is not
// zeroed, and the shared-memory traffic per plane drops by about 30 %.
template <typename C, int V, int R0, int R1>
__global__ void __launch_bounds__(PlanesCfg<C, V>::threads, PlanesCfg<C, V>::min_blocks)
k_planes_vloc_p3(C* __restrict__ work, const double* __restrict__ veff, HGeom g) {
    constexpr int N = R0 * R1, LS = N | 1, T = R0 > R1 ? R0 : R1, PW = 32 / T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* twx = reinterpret_cast<C*>(smem_raw);
    C* twy = reinterpret_cast<C*>(smem_raw + align16<C>(N));
    C* plane = reinterpret_cast<C*>(smem_raw + 2 * align16<C>(N));
    int* xl = reinterpret_cast<int*>(plane + (size_t)N * LS);
    const int z = blockIdx.x, b = blockIdx.y;
    const int nxact = g.nxact;
    p2_twiddles<R0, R1, C>(twx, g.twd_x, g.twf_x);
    p2_twiddles<R0, R1, C>(twy, g.twd_y, g.twf_y);
    for (int i = threadIdx.x; i < nxact; i += blockDim.x) xl[i] = g.xact[i];
    __syncthreads();
    C* wp = work + ((size_t)b * g.nz + z) * g.ncol;
    const int lane = threadIdx.x & 31;
    int gi, li;
    p2_lane<T, PW>(lane, gi, li);
    const bool ing = gi < PW;
    const int groups = (blockDim.x >> 5) * PW, gid = (threadIdx.x >> 5) * PW + gi;
    using R = typename RealOf<C>::type;
    // y lines through the active x positions: inverse, inputs from the columns
    for (int l0 = 0; l0 < nxact; l0 += groups) {
        const int l = l0 + gid;
        const bool act = ing && l < nxact;
        C* line = plane + (act ? xl[l] : 0);
        if (act && li < R0) {
            const int* ci = g.colidx + (size_t)l * N + li * R1;
            C x[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const int c = __ldg(ci + j);
                x[j] = c >= 0 ? wp[c] : czero<C>();
            }
            dft_r<R1, 1>(x);
#pragma unroll
            for (int m = 0; m < R1; ++m) line[swz(li * R1 + m, N) * LS] = x[m];
        }
        __syncwarp();
        if (act && li < R1) {
            C x[R0];
            p2_load_span<R0, R1>(line, LS, li, x);
            p2_span_inverse<R0, R1, true>(x, li, twy);
            p2_store_span<R0, R1>(line, LS, li, x);
        }
        __syncwarp();
    }
    __syncthreads();
    // x rows: inverse (x positions without columns read as zero), x V(r),
    // forward (only x positions with columns stored)
    const double* vz = veff + (size_t)z * N * N;
    for (int y0 = 0; y0 < N; y0 += groups) {
        const int y = y0 + gid;
        const bool act = ing && y < N;
        C* row = plane + (act ? swz(y, N) * LS : 0);
        if (act && li < R0) {
            C x[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const int px = li * R1 + j;
                const bool on = (g.xbits[px >> 5] >> (px & 31)) & 1u;
                x[j] = on ? row[swz(px, N)] : czero<C>();
            }
            dft_r<R1, 1>(x);
#pragma unroll
            for (int m = 0; m < R1; ++m) row[swz(li * R1 + m, N)] = x[m];
        }
        __syncwarp();
        if (act && li < R1) {
            C x[R0];
            p2_load_span<R0, R1>(row, 1, li, x);
            p2_span_inverse<R0, R1, true>(x, li, twx);
            const double* vr = vz + (size_t)y * N + li;
#pragma unroll
            for (int m = 0; m < R0; ++m) x[m] = cscale(x[m], (R)vr[m * R1]);
            p2_span_forward<R0, R1, true>(x, li, twx);
            p2_store_span<R0, R1>(row, 1, li, x);
        }
        __syncwarp();
        if (act && li < R0) {
            C x[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) x[j] = row[swz(li * R1 + j, N)];
            dft_r<R1, -1>(x);
#pragma unroll
            for (int m = 0; m < R1; ++m) {
                const int px = li * R1 + m;
                if ((g.xbits[px >> 5] >> (px & 31)) & 1u) row[swz(px, N)] = x[m];
            }
        }
        __syncwarp();
    }
    __syncthreads();
    // y lines forward, outputs to the columns
    for (int l0 = 0; l0 < nxact; l0 += groups) {
        const int l = l0 + gid;
        const bool act = ing && l < nxact;
        C* line = plane + (act ? xl[l] : 0);
        if (act && li < R1) {
            C x[R0];
            p2_load_span<R0, R1>(line, LS, li, x);
            p2_span_forward<R0, R1, true>(x, li, twy);
            p2_store_span<R0, R1>(line, LS, li, x);
        }
        __syncwarp();
        if (act && li < R0) {
            C x[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) x[j] = line[swz(li * R1 + j, N) * LS];
            dft_r<R1, -1>(x);
            const int* ci = g.colidx + (size_t)l * N + li * R1;
#pragma unroll
            for (int m = 0; m < R1; ++m) {
                const int c = __ldg(ci + m);
                if (c >= 0) wp[c] = x[m];
            }
        }
        __syncwarp();
    }
}

// ------------------------- pass 2, FP32, two bands per CTA (compile-time plans)
// The pipeline of k_planes_vloc_p3 for the FP32 filter with the same plane
// position of bands 2p and 2p + 1 in one 16-byte shared-memory element: every
// shared access is a 16-byte access in 8-lane phases, the case the lane
// mapping and lane-ordered twiddles make conflict-free (8-byte elements in
// 16-lane phases put two lines on the same bank groups), and each twiddle and
// V(r) load serves both bands.  An odd last band runs alone (its partner
// loads repeat it and are not stored).
__device__ __forceinline__ float4 pair4(float2 a, float2 b) { return make_float4(a.x, a.y, b.x, b.y); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

template <int V, int R0, int R1>
__global__ void __launch_bounds__(PlanesCfg<double2, V>::threads, PlanesCfg<double2, V>::min_blocks)
k_planes_vloc_p3x2(float2* __restrict__ work, const double* __restrict__ veff, int nb, HGeom g) {
    constexpr int N = R0 * R1, LS = N | 1, T = R0 > R1 ? R0 : R1, PW = 32 / T;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* twx = reinterpret_cast<float2*>(smem_raw);
    float2* twy = reinterpret_cast<float2*>(smem_raw + align16<float2>(N));
    float4* plane = reinterpret_cast<float4*>(smem_raw + 2 * align16<float2>(N));
    int* xl = reinterpret_cast<int*>(plane + (size_t)N * LS);
    const int z = blockIdx.x, b0 = 2 * blockIdx.y;
    const bool two = b0 + 1 < nb;
    const int nxact = g.nxact;
    p2_twiddles<R0, R1, float2>(twx, g.twd_x, g.twf_x);
    p2_twiddles<R0, R1, float2>(twy, g.twd_y, g.twf_y);
    for (int i = threadIdx.x; i < nxact; i += blockDim.x) xl[i] = g.xact[i];
    __syncthreads();
    float2* wa = work + ((size_t)b0 * g.nz + z) * g.ncol;
    float2* wb = two ? work + ((size_t)(b0 + 1) * g.nz + z) * g.ncol : wa;
    const int lane = threadIdx.x & 31;
    int gi, li;
    p2_lane<T, PW>(lane, gi, li);
    const bool ing = gi < PW;
    const int groups = (blockDim.x >> 5) * PW, gid = (threadIdx.x >> 5) * PW + gi;
    const float2 zero = make_float2(0.f, 0.f);
    // y lines through the active x positions: inverse, inputs from the columns
    for (int l0 = 0; l0 < nxact; l0 += groups) {
        const int l = l0 + gid;
        const bool act = ing && l < nxact;
        float4* line = plane + (act ? xl[l] : 0);
        if (act && li < R0) {
            const int* ci = g.colidx + (size_t)l * N + li * R1;
            float2 xa[R1], xb[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const int c = __ldg(ci + j);
                xa[j] = c >= 0 ? wa[c] : zero;
                xb[j] = c >= 0 ? wb[c] : zero;
            }
            dft_r<R1, 1>(xa);
            dft_r<R1, 1>(xb);
#pragma unroll
            for (int m = 0; m < R1; ++m) line[swz(li * R1 + m, N) * LS] = pair4(xa[m], xb[m]);
        }
        __syncwarp();
        if (act && li < R1) {
            float2 xa[R0], xb[R0];
#pragma unroll
            for (int j = 0; j < R0; ++j) {
                const float4 v = line[swz(li + j * R1, N) * LS];
                xa[j] = lo2(v);
                xb[j] = hi2(v);
            }
            p2_span_inverse<R0, R1, true>(xa, li, twy);
            p2_span_inverse<R0, R1, true>(xb, li, twy);
#pragma unroll
            for (int j = 0; j < R0; ++j) line[swz(li + j * R1, N) * LS] = pair4(xa[j], xb[j]);
        }
        __syncwarp();
    }
    __syncthreads();
    // x rows: inverse (x positions without columns read as zero), x V(r),
    // forward (only x positions with columns stored)
    const double* vz = veff + (size_t)z * N * N;
    for (int y0 = 0; y0 < N; y0 += groups) {
        const int y = y0 + gid;
        const bool act = ing && y < N;
        float4* row = plane + (act ? swz(y, N) * LS : 0);
        if (act && li < R0) {
            float2 xa[R1], xb[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const int px = li * R1 + j;
                const bool on = (g.xbits[px >> 5] >> (px & 31)) & 1u;
                const float4 v = on ? row[swz(px, N)] : make_float4(0.f, 0.f, 0.f, 0.f);
                xa[j] = lo2(v);
                xb[j] = hi2(v);
            }
            dft_r<R1, 1>(xa);
            dft_r<R1, 1>(xb);
#pragma unroll
            for (int m = 0; m < R1; ++m) row[swz(li * R1 + m, N)] = pair4(xa[m], xb[m]);
        }
        __syncwarp();
        if (act && li < R1) {
            float2 xa[R0], xb[R0];
#pragma unroll
            for (int j = 0; j < R0; ++j) {
                const float4 v = row[swz(li + j * R1, N)];
                xa[j] = lo2(v);
                xb[j] = hi2(v);
            }
            p2_span_inverse<R0, R1, true>(xa, li, twx);
            p2_span_inverse<R0, R1, true>(xb, li, twx);
            const double* vr = vz + (size_t)y * N + li;
#pragma unroll
            for (int m = 0; m < R0; ++m) {
                const float s = (float)vr[m * R1];
                xa[m] = cscale(xa[m], s);
                xb[m] = cscale(xb[m], s);
            }
            p2_span_forward<R0, R1, true>(xa, li, twx);
            p2_span_forward<R0, R1, true>(xb, li, twx);
#pragma unroll
            for (int j = 0; j < R0; ++j) row[swz(li + j * R1, N)] = pair4(xa[j], xb[j]);
        }
        __syncwarp();
        if (act && li < R0) {
            float2 xa[R1], xb[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const float4 v = row[swz(li * R1 + j, N)];
                xa[j] = lo2(v);
                xb[j] = hi2(v);
            }
            dft_r<R1, -1>(xa);
            dft_r<R1, -1>(xb);
#pragma unroll
            for (int m = 0; m < R1; ++m) {
                const int px = li * R1 + m;
                if ((g.xbits[px >> 5] >> (px & 31)) & 1u) row[swz(px, N)] = pair4(xa[m], xb[m]);
            }
        }
        __syncwarp();
    }
    __syncthreads();
    // y lines forward, outputs to the columns
    for (int l0 = 0; l0 < nxact; l0 += groups) {
        const int l = l0 + gid;
        const bool act = ing && l < nxact;
        float4* line = plane + (act ? xl[l] : 0);
        if (act && li < R1) {
            float2 xa[R0], xb[R0];
#pragma unroll
            for (int j = 0; j < R0; ++j) {
                const float4 v = line[swz(li + j * R1, N) * LS];
                xa[j] = lo2(v);
                xb[j] = hi2(v);
            }
            p2_span_forward<R0, R1, true>(xa, li, twy);
            p2_span_forward<R0, R1, true>(xb, li, twy);
#pragma unroll
            for (int j = 0; j < R0; ++j) line[swz(li + j * R1, N) * LS] = pair4(xa[j], xb[j]);
        }
        __syncwarp();
        if (act && li < R0) {
            float2 xa[R1], xb[R1];
#pragma unroll
            for (int j = 0; j < R1; ++j) {
                const float4 v = line[swz(li * R1 + j, N) * LS];
                xa[j] = lo2(v);
                xb[j] = hi2(v);
            }
            dft_r<R1, -1>(xa);
            dft_r<R1, -1>(xb);
            const int* ci = g.colidx + (size_t)l * N + li * R1;
#pragma unroll
            for (int m = 0; m < R1; ++m) {
                const int c = __ldg(ci + m);
                if (c >= 0) {
                    wa[c] = xa[m];
                    if (two) wb[c] = xb[m];
                }
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------- pass 3
template <typename C, int MODE, int kColsPerBlock, int R0, int R1>
__global__ void __launch_bounds__(256, ZCfg<R0>::min_blocks)
k_zsticks_forward(const C* __restrict__ work, const C* __restrict__ psi, int ldp, C* out, int ldo,
                  HGeom g, Epilogue e) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* lines = reinterpret_cast<C*>(smem_raw + align16<C>(g.nz));
    __shared__ double red[32];
    using R = typename RealOf<C>::type;
    const int b = blockIdx.y;
    const int c0 = blockIdx.x * kColsPerBlock;
    const int c1 = min(c0 + kColsPerBlock, g.ncol);
    const int nl = c1 - c0;
    copy_twiddles(tw, g.twd_z, g.twf_z, g.nz);
    const C* wb = work + (size_t)b * g.nz * g.ncol;
    for (int u = threadIdx.x; u < g.nz * kColsPerBlock; u += blockDim.x) {
        const int z = u / kColsPerBlock, cl = u - z * kColsPerBlock;
        lines[cl * g.lsz + swz(z, g.nz)] = cl < nl ? wb[(size_t)z * g.ncol + c0 + cl] : czero<C>();
    }
    __syncthreads();
    zlines_fft<R0, R1, true>(lines, nl, g, tw);
    const int g0 = g.col_start[c0], g1 = g.col_start[c1];
    const C* pb = psi + (size_t)b * ldp;
    C* ob = out + (size_t)b * ldo;
    const C* nlb = e.nl ? reinterpret_cast<const C*>(e.nl) + (size_t)b * ldp : nullptr;
    R ie = 0, nc = 0;
    if (MODE == kEpiChebFirst || MODE == kEpiCheb) {
        ie = (R)e.coef[4];
        nc = (R)e.coef[5];
    }
    R ra = 0, rb = 0, rcc = 0, rly = 0;
    const C* yb = nullptr;
    if (MODE == kEpiResid) {
        ra = (R)e.rc[0];
        rb = (R)e.rc[1];
        rcc = (R)e.rc[2];
        rly = (R)(e.rc[0] * e.lam[b]);
        yb = reinterpret_cast<const C*>(e.yres) + (size_t)b * ldp;
    }
    const R inv_n = (R)e.inv_n;
    // the Lanczos vector carried in the batch: plain H x, no recurrence
    const bool plain = b == e.plain_band;
    C* pob = plain ? reinterpret_cast<C*>(e.plain_out) : nullptr;
    double nacc = 0.0;
    for (int q = g0 + threadIdx.x; q < g1; q += blockDim.x) {
        const C v = lines[(g.pw_col[q] - c0) * g.lsz + swz(g.pw_zpos[q], g.nz)];
        const C p = pb[q];
        const R k = (R)e.kin[q];
        C h = mk(p.x * k, p.y * k);
        h = mk(h.x + v.x * inv_n, h.y + v.y * inv_n);
        if (nlb) h = cadd(h, nlb[q]);
        if (plain) {
            pob[q] = h;
        } else if (MODE == kEpiApply) {
            ob[q] = h;
        } else if (MODE == kEpiResid) {
            const C prev = ob[q];
            const C y = yb[q];
            ob[q] = mk(ra * h.x + rb * p.x + rcc * prev.x + rly * y.x,
                       ra * h.y + rb * p.y + rcc * prev.y + rly * y.y);
        } else {
            C s = mk(h.x * ie + nc * p.x, h.y * ie + nc * p.y);
            C o;
            if (MODE == kEpiChebFirst) o = s;
            else {
                const C prev = ob[q];
                o = mk((R)2 * s.x - prev.x, (R)2 * s.y - prev.y);
            }
            ob[q] = o;
            nacc += (double)o.x * (double)o.x + (double)o.y * (double)o.y;
        }
    }
    if (MODE != kEpiApply && e.norm_acc) {
        double s = block_sum(nacc, red);
        if (threadIdx.x == 0) atomicAdd(e.norm_acc, s);
    }
}

// ------------------------------------------------------ density (pass 2')
template <typename C, int MAXPT>
__global__ void __launch_bounds__(512)
k_planes_density(const C* __restrict__ work, const double* __restrict__ occ, int nb, int bpg,
                 double scale, double* rho, HGeom g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* twx = reinterpret_cast<C*>(smem_raw);
    C* twy = reinterpret_cast<C*>(smem_raw + align16<C>(g.nx));
    C* plane = reinterpret_cast<C*>(smem_raw + align16<C>(g.nx) + align16<C>(g.ny));
    int* xl = reinterpret_cast<int*>(plane + (size_t)g.ny * g.lsx);
    const int z = blockIdx.x;
    const int b0 = blockIdx.y * bpg, b1 = min(b0 + bpg, nb);
    copy_twiddles(twx, g.twd_x, g.twf_x, g.nx);
    copy_twiddles(twy, g.twd_y, g.twf_y, g.ny);
    for (int i = threadIdx.x; i < g.nxact; i += blockDim.x) xl[i] = g.xact[i];
    double acc[MAXPT];
#pragma unroll
    for (int k = 0; k < MAXPT; ++k) acc[k] = 0.0;
    const int npl = g.nx * g.ny;
    for (int b = b0; b < b1; ++b) {
        const double f = occ[b] * scale;
        if (f == 0.0) continue;
        for (int i = threadIdx.x; i < g.ny * g.lsx; i += blockDim.x) plane[i] = czero<C>();
        __syncthreads();
        const C* wp = work + ((size_t)b * g.nz + z) * g.ncol;
        for (int c = threadIdx.x; c < g.ncol; c += blockDim.x) plane[g.col_pos[c]] = wp[c];
        __syncthreads();
        fft_lines_grouped<false>(plane, g.nxact, LinesListed{xl}, g.lsx, g.ay, twy);
        fft_lines_grouped<false>(plane, g.ny, LinesStridedSwz{g.lsx, g.ny}, 1, g.ax, twx);
#pragma unroll
        for (int k = 0; k < MAXPT; ++k) {
            const int i = threadIdx.x + k * blockDim.x;
            if (i < npl) {
                const int y = i / g.nx, x = i - y * g.nx;
                const C v = plane[swz(y, g.ny) * g.lsx + swz(x, g.nx)];
                acc[k] += f * ((double)v.x * v.x + (double)v.y * v.y);
            }
        }
        __syncthreads();
    }
    double* rz = rho + (size_t)z * npl;
#pragma unroll
    for (int k = 0; k < MAXPT; ++k) {
        const int i = threadIdx.x + k * blockDim.x;
        if (i < npl) atomicAdd(&rz[i], acc[k]);
    }
}

// ------------------------------------------------------ full-grid axis FFT
template <typename C, bool FWD>
__global__ void __launch_bounds__(256)
k_axis_fft(C* data, int nx, int ny, int nz, int axis, AxisPlan P, int lb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = P.n;
    const int ls = n | 1;
    C* tw = reinterpret_cast<C*>(smem_raw);
    C* lines = reinterpret_cast<C*>(smem_raw + align16<C>(n));
    load_twiddles(tw, n);
    // line-batch decomposition
    size_t base;      // offset of element 0 of line 0 of the batch
    size_t lstride;   // offset between consecutive lines of the batch
    size_t estride;   // offset between consecutive elements of a line
    int nl;
    if (axis == 0) {
        const int nlines = ny * nz;
        const int l0 = blockIdx.x * lb;
        nl = min(lb, nlines - l0);
        base = (size_t)l0 * nx; lstride = nx; estride = 1;
    } else {
        const int nxb = (nx + lb - 1) / lb;
        const int x0 = (blockIdx.x % nxb) * lb;
        const int other = blockIdx.x / nxb;  // z for axis 1, y for axis 2
        nl = min(lb, nx - x0);
        lstride = 1;
        if (axis == 1) { base = (size_t)other * nx * ny + x0; estride = nx; }
        else { base = (size_t)other * nx + x0; estride = (size_t)nx * ny; }
    }
    for (int u = threadIdx.x; u < lb * n; u += blockDim.x) {
        int l, j;
        if (axis == 0) { l = u / n; j = u - l * n; }
        else { j = u / lb; l = u - j * lb; }
        lines[l * ls + swz(j, n)] = l < nl ? data[base + l * lstride + j * estride] : czero<C>();
    }
    __syncthreads();
    if (FWD) fft_lines_grouped<true>(lines, nl, LinesStrided{ls}, 1, P, tw);
    else fft_lines_grouped<false>(lines, nl, LinesStrided{ls}, 1, P, tw);
    for (int u = threadIdx.x; u < lb * n; u += blockDim.x) {
        int l, j;
        if (axis == 0) { l = u / n; j = u - l * n; }
        else { j = u / lb; l = u - j * lb; }
        if (l < nl) data[base + l * lstride + j * estride] = lines[l * ls + swz(j, n)];
    }
}

// ------------------------------------------------------ potential kernels
__device__ __forceinline__ void lda_pz(double rho, double& exc, double& vxc) {
    // Perdew-Zunger 1981 parametrisation of Ceperley-Alder, unpolarised.
    if (rho < 1e-30) { exc = 0.0; vxc = 0.0; return; }
    const double rs = cbrt(3.0 / (4.0 * 3.14159265358979323846 * rho));
    const double ex = -0.4581652932831429 / rs;
    const double vx = 4.0 / 3.0 * ex;
    double ec, vc;
    if (rs >= 1.0) {
        const double gm = -0.1423, b1 = 1.0529, b2 = 0.3334;
        const double sr = sqrt(rs);
        const double den = 1.0 + b1 * sr + b2 * rs;
        ec = gm / den;
        vc = ec * (1.0 + 7.0 / 6.0 * b1 * sr + 4.0 / 3.0 * b2 * rs) / den;
    } else {
        const double A = 0.0311, B = -0.048, Cc = 0.0020, D = -0.0116;
        const double lr = log(rs);
        ec = A * lr + B + Cc * rs * lr + D * rs;
        vc = A * lr + (B - A / 3.0) + 2.0 / 3.0 * Cc * rs * lr + (2.0 * D - Cc) / 3.0 * rs;
    }
    exc = ex + ec;
    vxc = vx + vc;
}

__global__ void k_real_to_complex(const double* r, double2* c, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        c[i] = make_double2(r[i], 0.0);
}

__global__ void k_take_real(const double2* c, double* r, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        r[i] = c[i].x;
}

__global__ void __launch_bounds__(256)
k_hartree_gspace(double2* c, GridRecip gr, double omega, double* eh_acc) {
    __shared__ double red[32];
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    const double inv_n = 1.0 / (double)n;
    const double four_pi = 4.0 * 3.14159265358979323846;
    double eh = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % gr.nx);
        const int iy = (int)((i / gr.nx) % gr.ny);
        const int iz = (int)(i / ((size_t)gr.nx * gr.ny));
        int h = gr.idr_x[ix], k = gr.idr_y[iy], l = gr.idr_z[iz];
        if (h >= (gr.nx + 1) / 2) h -= gr.nx;
        if (k >= (gr.ny + 1) / 2) k -= gr.ny;
        if (l >= (gr.nz + 1) / 2) l -= gr.nz;
        const double gx = h * gr.b[0] + k * gr.b[3] + l * gr.b[6];
        const double gy = h * gr.b[1] + k * gr.b[4] + l * gr.b[7];
        const double gz = h * gr.b[2] + k * gr.b[5] + l * gr.b[8];
        const double g2 = gx * gx + gy * gy + gz * gz;
        if (h == 0 && k == 0 && l == 0) { c[i] = make_double2(0.0, 0.0); continue; }
        const double2 rg = make_double2(c[i].x * inv_n, c[i].y * inv_n);
        eh += 0.5 * omega * four_pi * (rg.x * rg.x + rg.y * rg.y) / g2;
        c[i] = make_double2(four_pi * rg.x / g2, four_pi * rg.y / g2);
    }
    double s = block_sum(eh, red);
    if (threadIdx.x == 0) atomicAdd(eh_acc, s);
}

__global__ void __launch_bounds__(256)
k_assemble_veff(const double* vloc, const double2* vh, const double* rho, double* veff, size_t n,
                double dv, double* exc_acc) {
    __shared__ double red[32];
    double e = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double ex, vx;
        const double r = rho[i];
        lda_pz(r > 0.0 ? r : 0.0, ex, vx);
        veff[i] = vloc[i] + vh[i].x + vx;
        e += r * ex;
    }
    double s = block_sum(e, red);
    if (threadIdx.x == 0 && exc_acc) atomicAdd(exc_acc, s * dv);
}

__global__ void __launch_bounds__(256)
k_energy_terms(const double* rho_out, const double* veff, const double* vloc, size_t n, double dv,
               double* exc_acc, double* dc_acc) {
    __shared__ double red[32];
    double e = 0.0, d = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double ex, vx;
        const double r = rho_out[i];
        lda_pz(r > 0.0 ? r : 0.0, ex, vx);
        e += r * ex;
        d += (veff[i] - vloc[i]) * r;
    }
    double s = block_sum(e, red);
    if (threadIdx.x == 0) atomicAdd(exc_acc, s * dv);
    s = block_sum(d, red);
    if (threadIdx.x == 0) atomicAdd(dc_acc, s * dv);
}

// Opt a kernel into more than 48 KB of dynamic shared memory (once per
// kernel and size class).
template <typename K> void allow_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

int grid_for(size_t n, int threads) {
    size_t b = (n + threads - 1) / threads;
    return (int)(b < 148 * 8 ? b : 148 * 8);
}

}  // namespace

// ------------------------------------------------------------------ launchers
template <typename C, int COLS, int R0, int R1>
void zsticks_inverse_launch(const C* psi, int ldp, C* work, int nb, const HGeom& g, cudaStream_t st) {
    dim3 grid((g.ncol + COLS - 1) / COLS, nb);
    size_t sm = align16<C>(g.nz) + (size_t)COLS * g.lsz * sizeof(C);
    allow_smem(k_zsticks_inverse<C, COLS, R0, R1>, sm);
    k_zsticks_inverse<C, COLS, R0, R1><<<grid, 256, sm, st>>>(psi, ldp, work, g);
}

// two-radix z plans with compile-time kernels (the xy-plane list)
#define CHFSI_ZPLANS(X) X(9, 8) X(12, 9) X(8, 5) X(12, 12) X(8, 8) X(8, 6)

template <typename C, int COLS>
void zsticks_inverse_cols(const C* psi, int ldp, C* work, int nb, const HGeom& g, cudaStream_t st) {
    const int key = g.az.nst == 2 ? g.az.r[0] * 100 + g.az.r[1] : 0;
    switch (key) {
#define CHFSI_ZI(A, B) case A * 100 + B: zsticks_inverse_launch<C, COLS, A, B>(psi, ldp, work, nb, g, st); return;
        CHFSI_ZPLANS(CHFSI_ZI)
#undef CHFSI_ZI
    default: zsticks_inverse_launch<C, COLS, 0, 0>(psi, ldp, work, nb, g, st);
    }
}

template <typename C>
void launch_zsticks_inverse(const C* psi, int ldp, C* work, int nb, const HGeom& g,
                            cudaStream_t st) {
    count_launch();
    switch (g.tune_cols) {
    case 16: zsticks_inverse_cols<C, 16>(psi, ldp, work, nb, g, st); break;
    case 64: zsticks_inverse_cols<C, 64>(psi, ldp, work, nb, g, st); break;
    default: zsticks_inverse_cols<C, 32>(psi, ldp, work, nb, g, st); break;
    }
}

size_t planes_smem_bytes(const HGeom& g, size_t csize) {
    auto a16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    return a16(g.nx * csize) + a16(g.ny * csize) + (size_t)g.ny * g.lsx * csize +
           (size_t)g.nxact * sizeof(int);
}

template <typename C, int V>
void planes_vloc_variant(C* work, const double* veff, int nb, const HGeom& g, cudaStream_t st) {
    dim3 grid(g.nz, nb);
    size_t sm = planes_smem_bytes(g, sizeof(C));
    allow_smem(k_planes_vloc<C, V>, sm);
    k_planes_vloc<C, V><<<grid, PlanesCfg<C, V>::threads, sm, st>>>(work, veff, g);
}

template <typename C, int V, int R0, int R1>
void planes_vloc_p2(C* work, const double* veff, int nb, const HGeom& g, cudaStream_t st) {
    dim3 grid(g.nz, nb);
    size_t sm = planes_smem_bytes(g, sizeof(C));
    if constexpr (sizeof(C) == 8) {
        // FP32: two bands per CTA in 16-byte elements, where two such CTAs
        // still fit one SM's shared memory (planes up to 80 x 80)
        const size_t sm2 = 2 * align16<float2>(R0 * R1) +
                           (size_t)R0 * R1 * ((R0 * R1) | 1) * sizeof(float4) +
                           (size_t)g.nxact * sizeof(int);
        if (g.colidx && R0 * R1 <= 256 && sm2 <= 112 * 1024) {
            dim3 grid2(g.nz, (nb + 1) / 2);
            allow_smem(k_planes_vloc_p3x2<V, R0, R1>, sm2);
            k_planes_vloc_p3x2<V, R0, R1><<<grid2, PlanesCfg<double2, V>::threads, sm2, st>>>(
                reinterpret_cast<float2*>(work), veff, nb, g);
            return;
        }
    }
    if (g.colidx && R0 * R1 <= 256) {
        allow_smem(k_planes_vloc_p3<C, V, R0, R1>, sm);
        k_planes_vloc_p3<C, V, R0, R1><<<grid, PlanesCfg<C, V>::threads, sm, st>>>(work, veff, g);
        return;
    }
    allow_smem(k_planes_vloc_p2<C, V, R0, R1>, sm);
    k_planes_vloc_p2<C, V, R0, R1><<<grid, PlanesCfg<C, V>::threads, sm, st>>>(work, veff, g);
}

template <typename C, int R0, int R1>
void planes_vloc_p2_variant(C* work, const double* veff, int nb, const HGeom& g, cudaStream_t st) {
    switch (g.tune_planes) {
    case 1: planes_vloc_p2<C, 1, R0, R1>(work, veff, nb, g, st); break;
    case 2: planes_vloc_p2<C, 2, R0, R1>(work, veff, nb, g, st); break;
    default: planes_vloc_p2<C, 0, R0, R1>(work, veff, nb, g, st); break;
    }
}

// Radix pairs with a compile-time plane kernel (square planes only); other
// plans run the generic kernel.
static bool planes_vloc_fixed(void* work, const double* veff, int nb, const HGeom& g, cudaStream_t st,
                       bool fp32) {
    if (g.nx != g.ny || g.ax.nst != 2 || g.ay.nst != 2 || g.ax.r[0] != g.ay.r[0] ||
        g.ax.r[1] != g.ay.r[1])
        return false;
    const int key = g.ax.r[0] * 100 + g.ax.r[1];
#define CHFSI_P2(A, B)                                                                          \
    case A * 100 + B:                                                                         \
        if (fp32) planes_vloc_p2_variant<float2, A, B>((float2*)work, veff, nb, g, st);        \
        else planes_vloc_p2_variant<double2, A, B>((double2*)work, veff, nb, g, st);           \
        return true;
    switch (key) {
        CHFSI_P2(9, 8)    // 72
        CHFSI_P2(12, 9)   // 108
        CHFSI_P2(8, 5)    // 40
        CHFSI_P2(12, 12)  // 144
        CHFSI_P2(8, 8)    // 64
        CHFSI_P2(8, 6)    // 48
    default: return false;
    }
#undef CHFSI_P2
}

template <typename C>
void launch_planes_vloc(C* work, const double* veff, int nb, const HGeom& g, cudaStream_t st) {
    count_launch();
    if (g.fixed_planes && planes_vloc_fixed(work, veff, nb, g, st, sizeof(C) == 8)) return;
    switch (g.tune_planes) {
    case 1: planes_vloc_variant<C, 1>(work, veff, nb, g, st); break;
    case 2: planes_vloc_variant<C, 2>(work, veff, nb, g, st); break;
    default: planes_vloc_variant<C, 0>(work, veff, nb, g, st); break;
    }
}

template <typename C, int MODE, int COLS, int R0, int R1>
void zsticks_forward_launch(const C* work, const C* psi, int ldp, C* out, int ldo, int nb,
                            const HGeom& g, const Epilogue& e, cudaStream_t st) {
    dim3 grid((g.ncol + COLS - 1) / COLS, nb);
    size_t sm = align16<C>(g.nz) + (size_t)COLS * g.lsz * sizeof(C);
    allow_smem(k_zsticks_forward<C, MODE, COLS, R0, R1>, sm);
    k_zsticks_forward<C, MODE, COLS, R0, R1><<<grid, 256, sm, st>>>(work, psi, ldp, out, ldo, g, e);
}

template <typename C, int COLS, int R0, int R1>
void zsticks_forward_modes(const C* work, const C* psi, int ldp, C* out, int ldo, int nb,
                           const HGeom& g, const Epilogue& e, cudaStream_t st) {
    switch (e.mode) {
    case kEpiApply: zsticks_forward_launch<C, kEpiApply, COLS, R0, R1>(work, psi, ldp, out, ldo, nb, g, e, st); break;
    case kEpiChebFirst: zsticks_forward_launch<C, kEpiChebFirst, COLS, R0, R1>(work, psi, ldp, out, ldo, nb, g, e, st); break;
    case kEpiResid: zsticks_forward_launch<C, kEpiResid, COLS, R0, R1>(work, psi, ldp, out, ldo, nb, g, e, st); break;
    default: zsticks_forward_launch<C, kEpiCheb, COLS, R0, R1>(work, psi, ldp, out, ldo, nb, g, e, st); break;
    }
}

template <typename C, int COLS>
void zsticks_forward_cols(const C* work, const C* psi, int ldp, C* out, int ldo, int nb,
                          const HGeom& g, const Epilogue& e, cudaStream_t st) {
    const int key = g.az.nst == 2 ? g.az.r[0] * 100 + g.az.r[1] : 0;
    switch (key) {
#define CHFSI_ZF(A, B) case A * 100 + B: zsticks_forward_modes<C, COLS, A, B>(work, psi, ldp, out, ldo, nb, g, e, st); return;
        CHFSI_ZPLANS(CHFSI_ZF)
#undef CHFSI_ZF
    default: zsticks_forward_modes<C, COLS, 0, 0>(work, psi, ldp, out, ldo, nb, g, e, st);
    }
}

template <typename C>
void launch_zsticks_forward(const C* work, const C* psi, int ldp, C* out, int ldo, int nb,
                            const HGeom& g, const Epilogue& e, cudaStream_t st) {
    count_launch();
    switch (g.tune_cols) {
    case 16: zsticks_forward_cols<C, 16>(work, psi, ldp, out, ldo, nb, g, e, st); break;
    case 64: zsticks_forward_cols<C, 64>(work, psi, ldp, out, ldo, nb, g, e, st); break;
    default: zsticks_forward_cols<C, 32>(work, psi, ldp, out, ldo, nb, g, e, st); break;
    }
}

template <typename C>
void launch_planes_density(const C* work, const double* occ, int nb, double scale, double* rho,
                           const HGeom& g, cudaStream_t st) {
    count_launch();
    int groups = (2 * 148 + g.nz - 1) / g.nz;
    if (groups > nb) groups = nb;
    if (groups < 1) groups = 1;
    const int bpg = (nb + groups - 1) / groups;
    groups = (nb + bpg - 1) / bpg;
    dim3 grid(g.nz, groups);
    size_t sm = planes_smem_bytes(g, sizeof(C));
    allow_smem(k_planes_density<C, 24>, sm);
    k_planes_density<C, 24><<<grid, 512, sm, st>>>(work, occ, nb, bpg, scale, rho, g);
}

template <typename C>
void launch_axis_fft(C* data, int nx, int ny, int nz, int axis, bool forward, const AxisPlan& P,
                     cudaStream_t st) {
    count_launch();
    const int lb = 16;
    int blocks;
    if (axis == 0) blocks = (ny * nz + lb - 1) / lb;
    else blocks = ((nx + lb - 1) / lb) * (axis == 1 ? nz : ny);
    size_t sm = align16<C>(P.n) + (size_t)lb * (P.n | 1) * sizeof(C);
    allow_smem(k_axis_fft<C, true>, sm);
    allow_smem(k_axis_fft<C, false>, sm);
    if (forward) k_axis_fft<C, true><<<blocks, 256, sm, st>>>(data, nx, ny, nz, axis, P, lb);
    else k_axis_fft<C, false><<<blocks, 256, sm, st>>>(data, nx, ny, nz, axis, P, lb);
}

void launch_real_to_complex(const double* r, double2* c, size_t n, cudaStream_t st) {
    count_launch();
    k_real_to_complex<<<grid_for(n, 256), 256, 0, st>>>(r, c, n);
}
void launch_take_real(const double2* c, double* r, size_t n, cudaStream_t st) {
    count_launch();
    k_take_real<<<grid_for(n, 256), 256, 0, st>>>(c, r, n);
}
void launch_hartree_gspace(double2* c, const GridRecip& gr, double omega, double* eh_acc,
                           cudaStream_t st) {
    count_launch();
    size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    k_hartree_gspace<<<grid_for(n, 256), 256, 0, st>>>(c, gr, omega, eh_acc);
}
void launch_assemble_veff(const double* vloc, const double2* vh, const double* rho, double* veff,
                          size_t n, double dv, double* exc_acc, cudaStream_t st) {
    count_launch();
    k_assemble_veff<<<grid_for(n, 256), 256, 0, st>>>(vloc, vh, rho, veff, n, dv, exc_acc);
}
void launch_energy_terms(const double* rho_out, const double* veff, const double* vloc, size_t n,
                         double dv, double* exc_acc, double* dc_acc, cudaStream_t st) {
    count_launch();
    k_energy_terms<<<grid_for(n, 256), 256, 0, st>>>(rho_out, veff, vloc, n, dv, exc_acc, dc_acc);
}

#define CHFSI_INST(C)                                                                        \
    template void launch_zsticks_inverse<C>(const C*, int, C*, int, const HGeom&, cudaStream_t); \
    template void launch_planes_vloc<C>(C*, const double*, int, const HGeom&, cudaStream_t);     \
    template void launch_zsticks_forward<C>(const C*, const C*, int, C*, int, int, const HGeom&, \
                                            const Epilogue&, cudaStream_t);                      \
    template void launch_planes_density<C>(const C*, const double*, int, double, double*,        \
                                           const HGeom&, cudaStream_t);                          \
    template void launch_axis_fft<C>(C*, int, int, int, int, bool, const AxisPlan&, cudaStream_t);
CHFSI_INST(double2)
CHFSI_INST(float2)
#undef CHFSI_INST

}  // namespace chfsi
