// Shared-memory mixed-radix FFT line engine.
//
// A CTA transforms a set of lines that live in shared memory.  Line l starts
// at smem offset base(l) and its elements are es apart.  Transforms are
// in place and unnormalised:
//   forward (DIF, sign -1): natural order in  -> digit-reversed order out
//   inverse (DIT, sign +1): digit-reversed in -> natural order out
// so a forward / pointwise-multiply / inverse sequence never needs an
// explicit permutation; the digit-reversal map only enters where plane
// waves are scattered into or gathered from a grid (host-built tables).
//
// For N = r0 r1 ... r_{s-1}, the DIF stage t with block size B and span
// S = B / r_t maps, for every block b0 and n1 < S,
//   x_j = a[b0 + n1 + j S],  y_m = sum_j x_j w_r^{-jm},  a[b0 + n1 + m S] = y_m w_B^{-n1 m}
// and the DIT runs the stages in reverse order with the twiddle applied
// before the butterfly (the transpose of the DIF, hence F P^T).
#pragma once

#include "common.cuh"

namespace chfsi {

constexpr int kMaxStages = 10;

struct AxisPlan {
    int n;
    int nst;
    int r[kMaxStages];  // radices in DIF order
    int tpl;            // threads per line: max over stages of n / r (<= 32)
};

// Shared-memory position of element i of a line of length n: the low three
// bits are XORed with the next three inside every full block of 8 elements,
// so the power-of-two strides of the FFT stages spread over all banks.
__host__ __device__ __forceinline__ int swz(int i, int n) {
    return i < (n & ~7) ? (i ^ ((i >> 3) & 7)) : i;
}

// cos / sin of 2 pi e / n evaluated at compile time (Taylor series on the
// octant-reduced angle; |error| < 1e-18): inner twiddles of composite radices.
__host__ __device__ constexpr double taylor_cos(double x) {
    double t = 1.0, s = 1.0;
    for (int k = 1; k <= 12; ++k) {
        t *= -x * x / ((2 * k - 1) * (2 * k));
        s += t;
    }
    return s;
}
__host__ __device__ constexpr double taylor_sin(double x) {
    double t = x, s = x;
    for (int k = 1; k <= 12; ++k) {
        t *= -x * x / ((2 * k) * (2 * k + 1));
        s += t;
    }
    return s;
}
// cos(2 pi e / n) via exact reduction of e/n to the first octant
__host__ __device__ constexpr double tw_cos(int n, int e) {
    e = ((e % n) + n) % n;
    // angle = 2 pi e / n = (pi/4) * (8 e / n); octant o, remainder in [0, 1)
    const int num = 8 * e;
    const int o = num / n;
    const double f = (double)(num - o * n) / (double)n;  // in [0, 1)
    const double q = 0.78539816339744830962;             // pi / 4
    switch (o) {
    case 0: return taylor_cos(f * q);
    case 1: return taylor_sin((1.0 - f) * q);
    case 2: return -taylor_sin(f * q);
    case 3: return -taylor_cos((1.0 - f) * q);
    case 4: return -taylor_cos(f * q);
    case 5: return -taylor_sin((1.0 - f) * q);
    case 6: return taylor_sin(f * q);
    default: return taylor_cos((1.0 - f) * q);
    }
}
__host__ __device__ constexpr double tw_sin(int n, int e) {
    // sin(t) = cos(t - pi/2) = cos(2 pi (4 e - n) / (4 n))
    return tw_cos(4 * n, 4 * e - n);
}

// r-point DFT in registers, exponent sign SIGN (+1 or -1).
template <typename C> __device__ __forceinline__ void dft2(C* x) {
    C a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
}

template <int SIGN, typename C> __device__ __forceinline__ void dft3(C* x) {
    using R = typename RealOf<C>::type;
    const R h = (R)0.86602540378443864676;  // sin(2 pi / 3)
    C t1 = cadd(x[1], x[2]);
    C t2 = csub(x[1], x[2]);
    C y0 = cadd(x[0], t1);
    C m = mk(x[0].x - (R)0.5 * t1.x, x[0].y - (R)0.5 * t1.y);
    C u = cmul_i<SIGN>(cscale(t2, h));
    x[0] = y0;
    x[1] = cadd(m, u);
    x[2] = csub(m, u);
}
template <int SIGN, typename C> __device__ __forceinline__ void dft4(C* x) {
    C a = cadd(x[0], x[2]), b = csub(x[0], x[2]);
    C c = cadd(x[1], x[3]), d = cmul_i<SIGN>(csub(x[1], x[3]));
    x[0] = cadd(a, c);
    x[2] = csub(a, c);
    x[1] = cadd(b, d);
    x[3] = csub(b, d);
}
template <int SIGN, typename C> __device__ __forceinline__ void dft5(C* x) {
    using R = typename RealOf<C>::type;
    const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;
    const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;
    C a1 = cadd(x[1], x[4]), b1 = csub(x[1], x[4]);
    C a2 = cadd(x[2], x[3]), b2 = csub(x[2], x[3]);
    C y0 = cadd(x[0], cadd(a1, a2));
    C t1 = mk(x[0].x + c1 * a1.x + c2 * a2.x, x[0].y + c1 * a1.y + c2 * a2.y);
    C t2 = mk(x[0].x + c2 * a1.x + c1 * a2.x, x[0].y + c2 * a1.y + c1 * a2.y);
    C u1 = cmul_i<SIGN>(mk(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
    C u2 = cmul_i<SIGN>(mk(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
    x[0] = y0;
    x[1] = cadd(t1, u1);
    x[4] = csub(t1, u1);
    x[2] = cadd(t2, u2);
    x[3] = csub(t2, u2);
}
// radix 8 = 2 x 4 split: x_j, j = 4 a + b  -> DFT over a (size 2), twiddle, DFT over b (size 4)
template <int SIGN, typename C> __device__ __forceinline__ void dft8(C* x) {
    using R = typename RealOf<C>::type;
    const R r2 = (R)0.70710678118654752440;
    // stage 1: four radix-2 butterflies on (x_b, x_{b+4})
    C u[8];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        u[b] = cadd(x[b], x[b + 4]);
        u[b + 4] = csub(x[b], x[b + 4]);
    }
    // twiddle w8^{SIGN * b} on the odd half
    u[5] = mk(r2 * (u[5].x - (R)SIGN * u[5].y), r2 * (u[5].y + (R)SIGN * u[5].x));
    u[6] = cmul_i<SIGN>(u[6]);
    u[7] = mk(r2 * (-u[7].x - (R)SIGN * u[7].y), r2 * (-u[7].y + (R)SIGN * u[7].x));
    C e[4] = {u[0], u[1], u[2], u[3]}, o[4] = {u[4], u[5], u[6], u[7]};
    dft4<SIGN>(e);
    dft4<SIGN>(o);
    // output index k = 2 k' + a
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        x[2 * k] = e[k];
        x[2 * k + 1] = o[k];
    }
}

template <int R, int SIGN, typename C> __device__ __forceinline__ void dft_r(C* x);

// Compile-time table of exp(i 2 pi e / N), e < N.
template <int N> struct TwTable {
    double c[N], s[N];
    __host__ __device__ constexpr TwTable() : c(), s() {
        for (int e = 0; e < N; ++e) {
            c[e] = tw_cos(N, e);
            s[e] = tw_sin(N, e);
        }
    }
};

// DFT of size R1 R2 from R2 DFTs of size R1, inner twiddles, R1 DFTs of size
// R2: input index j = R2 j1 + j2, output index k = k1 + R1 k2 (natural order).
template <int R1, int R2, int SIGN, typename C> __device__ __forceinline__ void dft_comp(C* x) {
    using R = typename RealOf<C>::type;
    constexpr int N = R1 * R2;
    constexpr TwTable<N> tab{};
    C y[N];
#pragma unroll
    for (int j2 = 0; j2 < R2; ++j2) {
        C t[R1];
#pragma unroll
        for (int j1 = 0; j1 < R1; ++j1) t[j1] = x[R2 * j1 + j2];
        dft_r<R1, SIGN>(t);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            const int e = j2 * k1;
            if (e == 0) { y[j2 * R1 + k1] = t[k1]; continue; }
            const R c = (R)tab.c[e % N], sn = (R)(SIGN * tab.s[e % N]);
            y[j2 * R1 + k1] = mk(t[k1].x * c - t[k1].y * sn, t[k1].x * sn + t[k1].y * c);
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        C t[R2];
#pragma unroll
        for (int j2 = 0; j2 < R2; ++j2) t[j2] = y[j2 * R1 + k1];
        dft_r<R2, SIGN>(t);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) x[k1 + R1 * k2] = t[k2];
    }
}

template <int R, int SIGN, typename C> __device__ __forceinline__ void dft_r(C* x) {
    if constexpr (R == 2) dft2(x);
    else if constexpr (R == 3) dft3<SIGN>(x);
    else if constexpr (R == 4) dft4<SIGN>(x);
    else if constexpr (R == 5) dft5<SIGN>(x);
    else if constexpr (R == 8) dft8<SIGN>(x);
    else if constexpr (R == 6) dft_comp<2, 3, SIGN>(x);
    else if constexpr (R == 9) dft_comp<3, 3, SIGN>(x);
    else if constexpr (R == 10) dft_comp<2, 5, SIGN>(x);
    else if constexpr (R == 12) dft_comp<4, 3, SIGN>(x);
    else if constexpr (R == 15) dft_comp<3, 5, SIGN>(x);
}

// One DIF (FWD=true, sign -1) or DIT (FWD=false, sign +1) stage of radix R
// over nlines lines.  tw[j] = exp(+2 pi i j / n).
template <int R, bool FWD, typename C, class LineBase>
__device__ __forceinline__ void fft_stage(C* s, int nlines, LineBase lb, int es, int n, int B,
                                          const C* tw) {
    const int S = B / R;
    const int nb = n / R;
    const int step = n / B;
    const int total = nlines * nb;
    for (int u = threadIdx.x; u < total; u += blockDim.x) {
        const int l = u / nb;
        const int v = u - l * nb;
        const int blk = v / S;
        const int n1 = v - blk * S;
        C* line = s + lb(l);
        const int e0 = blk * B + n1;
        C x[R];
#pragma unroll
        for (int j = 0; j < R; ++j) x[j] = line[swz(e0 + j * S, n) * es];
        const int e = step * n1;
        if (FWD) {
            dft_r<R, -1>(x);
#pragma unroll
            for (int m = 1; m < R; ++m) x[m] = cmulc(tw[e * m], x[m]);
        } else {
#pragma unroll
            for (int m = 1; m < R; ++m) x[m] = cmul(tw[e * m], x[m]);
            dft_r<R, 1>(x);
        }
#pragma unroll
        for (int m = 0; m < R; ++m) line[swz(e0 + m * S, n) * es] = x[m];
    }
}

template <bool FWD, typename C, class LineBase>
__device__ __forceinline__ void fft_dispatch(int r, C* s, int nlines, LineBase lb, int es, int n,
                                             int B, const C* tw) {
    switch (r) {
    case 2: fft_stage<2, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 3: fft_stage<3, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 4: fft_stage<4, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 5: fft_stage<5, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 6: fft_stage<6, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 8: fft_stage<8, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 9: fft_stage<9, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 10: fft_stage<10, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 12: fft_stage<12, FWD>(s, nlines, lb, es, n, B, tw); break;
    case 15: fft_stage<15, FWD>(s, nlines, lb, es, n, B, tw); break;
    default: break;
    }
}

// Forward transform (DIF, sign -1) of nlines lines; ends with __syncthreads.
template <typename C, class LineBase>
__device__ __forceinline__ void fft_forward(C* s, int nlines, LineBase lb, int es,
                                            const AxisPlan& P, const C* tw) {
    int B = P.n;
    for (int t = 0; t < P.nst; ++t) {
        fft_dispatch<true>(P.r[t], s, nlines, lb, es, P.n, B, tw);
        __syncthreads();
        B /= P.r[t];
    }
}

// Inverse transform (DIT, sign +1); ends with __syncthreads.
template <typename C, class LineBase>
__device__ __forceinline__ void fft_inverse(C* s, int nlines, LineBase lb, int es,
                                            const AxisPlan& P, const C* tw) {
    int S = 1;
    for (int t = P.nst - 1; t >= 0; --t) {
        const int B = S * P.r[t];
        fft_dispatch<false>(P.r[t], s, nlines, lb, es, P.n, B, tw);
        __syncthreads();
        S = B;
    }
}

// One butterfly (index v of the stage) of a DIF or DIT stage on one line.
template <int R, bool FWD, typename C>
__device__ __forceinline__ void butterfly(C* line, int v, int es, int n, int B, const C* tw) {
    const int S = B / R;
    const int blk = v / S;
    const int n1 = v - blk * S;
    const int e0 = blk * B + n1;
    C x[R];
#pragma unroll
    for (int j = 0; j < R; ++j) x[j] = line[swz(e0 + j * S, n) * es];
    const int e = (n / B) * n1;
    if (FWD) {
        dft_r<R, -1>(x);
#pragma unroll
        for (int m = 1; m < R; ++m) x[m] = cmulc(tw[e * m], x[m]);
    } else {
#pragma unroll
        for (int m = 1; m < R; ++m) x[m] = cmul(tw[e * m], x[m]);
        dft_r<R, 1>(x);
    }
#pragma unroll
    for (int m = 0; m < R; ++m) line[swz(e0 + m * S, n) * es] = x[m];
}

template <bool FWD, typename C>
__device__ __forceinline__ void butterfly_dispatch(int r, C* line, int v, int es, int n, int B,
                                                   const C* tw) {
    switch (r) {
    case 2: butterfly<2, FWD>(line, v, es, n, B, tw); break;
    case 3: butterfly<3, FWD>(line, v, es, n, B, tw); break;
    case 4: butterfly<4, FWD>(line, v, es, n, B, tw); break;
    case 5: butterfly<5, FWD>(line, v, es, n, B, tw); break;
    case 6: butterfly<6, FWD>(line, v, es, n, B, tw); break;
    case 8: butterfly<8, FWD>(line, v, es, n, B, tw); break;
    case 9: butterfly<9, FWD>(line, v, es, n, B, tw); break;
    case 10: butterfly<10, FWD>(line, v, es, n, B, tw); break;
    case 12: butterfly<12, FWD>(line, v, es, n, B, tw); break;
    case 15: butterfly<15, FWD>(line, v, es, n, B, tw); break;
    default: break;
    }
}

// Transform of one line by a group of P.tpl lanes of one warp (lane index i
// within the group); stages are separated by __syncwarp only.  Every lane of
// the warp must call this the same number of times (act = false: idle).
template <bool FWD, typename C>
__device__ __forceinline__ void line_fft_group(C* line, bool act, int i, int es, const AxisPlan& P,
                                               const C* tw) {
    if (FWD) {
        int B = P.n;
        for (int t = 0; t < P.nst; ++t) {
            const int r = P.r[t];
            if (act && i < P.n / r) butterfly_dispatch<true>(r, line, i, es, P.n, B, tw);
            __syncwarp();
            B /= r;
        }
    } else {
        int S = 1;
        for (int t = P.nst - 1; t >= 0; --t) {
            const int r = P.r[t];
            const int B = S * r;
            if (act && i < P.n / r) butterfly_dispatch<false>(r, line, i, es, P.n, B, tw);
            __syncwarp();
            S = B;
        }
    }
}

// Lane groups of a CTA: groups of P.tpl lanes inside each warp.
struct LaneGroups {
    int g;        // group index within the warp
    int i;        // lane index within the group
    int per_warp; // groups per warp
    int total;    // groups in the CTA
    int id;       // CTA-wide group id (valid when in_group)
    bool in_group;
    __device__ __forceinline__ explicit LaneGroups(int tpl) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        per_warp = 32 / tpl;
        g = lane / tpl;
        i = lane - g * tpl;
        in_group = g < per_warp;
        total = (blockDim.x >> 5) * per_warp;
        id = warp * per_warp + g;
    }
};

// Transform nlines lines with lane groups; ends with __syncthreads.
template <bool FWD, typename C, class LineBase>
__device__ __forceinline__ void fft_lines_grouped(C* s, int nlines, LineBase lb, int es,
                                                  const AxisPlan& P, const C* tw) {
    if (P.tpl > 32) {  // a line needs more than one warp: CTA-wide stages
        if (FWD) fft_forward(s, nlines, lb, es, P, tw);
        else fft_inverse(s, nlines, lb, es, P, tw);
        return;
    }
    const LaneGroups lg(P.tpl);
    const int rounds = (nlines + lg.total - 1) / lg.total;
    for (int rd = 0; rd < rounds; ++rd) {
        const int l = rd * lg.total + lg.id;
        const bool act = lg.in_group && l < nlines;
        line_fft_group<FWD>(act ? s + lb(l) : s, act, lg.i, es, P, tw);
    }
    __syncthreads();
}

struct LinesStrided {
    int ls;
    __device__ __forceinline__ int operator()(int l) const { return l * ls; }
};
// line l starts at row swz(l) of a plane whose rows are swizzled too
struct LinesStridedSwz {
    int ls, n;
    __device__ __forceinline__ int operator()(int l) const { return swz(l, n) * ls; }
};
struct LinesListed {
    const int* list;
    __device__ __forceinline__ int operator()(int l) const { return list[l]; }
};

// Copy a precomputed twiddle table (global memory, L2-resident) into smem.
__device__ __forceinline__ void copy_twiddles(double2* tw, const double2* twd, const float2*, int n) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = twd[j];
}
__device__ __forceinline__ void copy_twiddles(float2* tw, const double2*, const float2* twf, int n) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) tw[j] = twf[j];
}

// tw[j] = exp(+2 pi i j / n), computed in FP64 then rounded to C.
template <typename C> __device__ __forceinline__ void load_twiddles(C* tw, int n) {
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        double sn, cs;
        sincospi(2.0 * (double)j / (double)n, &sn, &cs);
        tw[j] = to_c(make_double2(cs, sn), C{});
    }
}

}  // namespace chfsi
