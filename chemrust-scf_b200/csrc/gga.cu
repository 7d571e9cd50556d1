// GGA exchange-correlation (PBE) on the density grid: the functional the
// reference's planned V_eff builder uses (plans/phase-2/PHASE_PLAN.md:90-95),
// spin-unpolarised.
//
//   E_xc = sum_r e(rho, sigma) dV,  sigma = |grad rho|^2
//   V_xc = de/drho - div(2 de/dsigma grad rho)
//
// Exchange: Perdew, Burke, Ernzerhof, PRL 77, 3865 (1996):
//   e_x = rho e_x^unif(rho) F_x(s),  e_x^unif = -3 k_F / (4 pi),
//   k_F = (3 pi^2 rho)^(1/3),  s^2 = sigma / (4 k_F^2 rho^2),
//   F_x = 1 + kappa - kappa / (1 + mu s^2 / kappa),  kappa = 0.804,
//   mu = beta pi^2 / 3.
// Correlation: e_c = rho (eps_c^PW92(r_s) + H(r_s, t)),
//   eps_c^PW92 (Perdew & Wang, PRB 45, 13244 (1992), zeta = 0):
//     -2 A (1 + a1 r_s) ln(1 + 1 / (2 A (b1 r_s^1/2 + b2 r_s + b3 r_s^3/2 + b4 r_s^2)))
//   H = gamma ln(1 + beta/gamma t^2 (1 + A' t^2) / (1 + A' t^2 + A'^2 t^4)),
//   A' = beta/gamma / (exp(-eps_c / gamma) - 1),  t^2 = sigma / (4 k_s^2 rho^2),
//   k_s = sqrt(4 k_F / pi),  gamma = (1 - ln 2) / pi^2,  beta = 0.06672455060314922.
// The derivatives de/drho and de/dsigma are taken by forward-mode
// differentiation of the same expression (dual numbers), so energy and
// potential can never disagree.  Gradient and divergence are spectral: i G
// in the digit-reversed G layout of the density-grid FFT, Nyquist planes and
// G = 0 dropped.
#include "kernels.hpp"
#include "launch_count.hpp"

namespace chfsi {

namespace {

constexpr double kPi = 3.14159265358979323846;

// value and the two partial derivatives (d/drho, d/dsigma)
struct Dual {
    double v, dr, ds;
};
__device__ __forceinline__ Dual dconst(double c) { return {c, 0.0, 0.0}; }
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.dr + b.dr, a.ds + b.ds}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.dr - b.dr, a.ds - b.ds}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) {
    return {a.v * b.v, a.dr * b.v + a.v * b.dr, a.ds * b.v + a.v * b.ds};
}
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
    const double inv = 1.0 / b.v;
    const double q = a.v * inv;
    return {q, (a.dr - q * b.dr) * inv, (a.ds - q * b.ds) * inv};
}
__device__ __forceinline__ Dual operator*(double c, Dual a) { return {c * a.v, c * a.dr, c * a.ds}; }
__device__ __forceinline__ Dual operator+(double c, Dual a) { return {c + a.v, a.dr, a.ds}; }
__device__ __forceinline__ Dual dlog(Dual a) { return {log(a.v), a.dr / a.v, a.ds / a.v}; }
__device__ __forceinline__ Dual dexp(Dual a) {
    const double e = exp(a.v);
    return {e, e * a.dr, e * a.ds};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
    const double r = sqrt(a.v);
    const double d = 0.5 / r;
    return {r, d * a.dr, d * a.ds};
}
__device__ __forceinline__ Dual dcbrt(Dual a) {
    const double r = cbrt(a.v);
    const double d = r / (3.0 * a.v);
    return {r, d * a.dr, d * a.ds};
}

// PBE energy density per volume, with d/drho and d/dsigma
__device__ Dual pbe_density(double rho_v, double sigma_v) {
    const Dual rho{rho_v, 1.0, 0.0};
    const Dual sigma{sigma_v, 0.0, 1.0};
    const double kappa = 0.804, beta = 0.06672455060314922;
    const double mu = beta * kPi * kPi / 3.0;
    const double gamma = (1.0 - 0.69314718055994530942) / (kPi * kPi);
    const Dual kf = dcbrt(3.0 * kPi * kPi * rho);
    const Dual rho2 = rho * rho;
    // exchange
    const Dual s2 = sigma / (4.0 * (kf * kf) * rho2);
    const Dual fx = (1.0 + kappa) + dconst(0.0) - dconst(kappa) / (1.0 + (mu / kappa) * s2);
    const Dual ex = (-3.0 / (4.0 * kPi)) * (kf * rho) * fx;
    // PW92 correlation (zeta = 0)
    const double A = 0.031091, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
    const Dual rs = dcbrt(dconst(3.0 / (4.0 * kPi)) / rho);
    const Dual srs = dsqrt(rs);
    const Dual den = (2.0 * A) * (b1 * srs + b2 * rs + b3 * (rs * srs) + b4 * (rs * rs));
    const Dual ec = (-2.0 * A) * (1.0 + a1 * rs) * dlog(1.0 + dconst(1.0) / den);
    // gradient correction
    const Dual ks = dsqrt((4.0 / kPi) * kf);
    const Dual t2 = sigma / (4.0 * (ks * ks) * rho2);
    const Dual Ap = dconst(beta / gamma) / (dexp((-1.0 / gamma) * ec) - dconst(1.0));
    const Dual At2 = Ap * t2;
    const Dual frac = t2 * (1.0 + At2) / (1.0 + At2 + At2 * At2);
    const Dual H = gamma * dlog(1.0 + (beta / gamma) * frac);
    return ex + rho * (ec + H);
}

constexpr double kRhoFloor = 1e-12;

__device__ __forceinline__ bool gvec(size_t i, const GridRecip& gr, double* g) {
    const int ix = (int)(i % gr.nx);
    const int iy = (int)((i / gr.nx) % gr.ny);
    const int iz = (int)(i / ((size_t)gr.nx * gr.ny));
    int h = gr.idr_x[ix], k = gr.idr_y[iy], l = gr.idr_z[iz];
    if (h >= (gr.nx + 1) / 2) h -= gr.nx;
    if (k >= (gr.ny + 1) / 2) k -= gr.ny;
    if (l >= (gr.nz + 1) / 2) l -= gr.nz;
    // Nyquist planes carry no derivative of a real field
    if ((gr.nx % 2 == 0 && 2 * h == -gr.nx) || (gr.ny % 2 == 0 && 2 * k == -gr.ny) ||
        (gr.nz % 2 == 0 && 2 * l == -gr.nz))
        return false;
    g[0] = h * gr.b[0] + k * gr.b[3] + l * gr.b[6];
    g[1] = h * gr.b[1] + k * gr.b[4] + l * gr.b[7];
    g[2] = h * gr.b[2] + k * gr.b[5] + l * gr.b[8];
    return true;
}

// out_a = i G_a f(G) / N for a = 0, 1, 2 (f: unnormalised forward FFT of a real field)
__global__ void k_grad_gspace(const double2* __restrict__ f, GridRecip gr, double2* __restrict__ o0,
                              double2* __restrict__ o1, double2* __restrict__ o2) {
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    const double inv_n = 1.0 / (double)n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double g[3];
        if (!gvec(i, gr, g)) {
            o0[i] = o1[i] = o2[i] = make_double2(0.0, 0.0);
            continue;
        }
        const double2 v = make_double2(f[i].x * inv_n, f[i].y * inv_n);
        o0[i] = make_double2(-g[0] * v.y, g[0] * v.x);
        o1[i] = make_double2(-g[1] * v.y, g[1] * v.x);
        o2[i] = make_double2(-g[2] * v.y, g[2] * v.x);
    }
}

// pointwise PBE: v1 = de/drho; h_a = 2 de/dsigma grad_a rho (written over
// the gradient, real part); exc_acc += sum e dV
__global__ void __launch_bounds__(256)
k_pbe_point(const double* __restrict__ rho, double2* g0, double2* g1, double2* g2,
            double* __restrict__ v1, size_t n, double dv, double* exc_acc, int want_potential) {
    __shared__ double red[32];
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double r = rho[i];
        const double gx = g0[i].x, gy = g1[i].x, gz = g2[i].x;
        if (r < kRhoFloor) {
            if (want_potential) {
                v1[i] = 0.0;
                g0[i] = g1[i] = g2[i] = make_double2(0.0, 0.0);
            }
            continue;
        }
        const Dual e = pbe_density(r, gx * gx + gy * gy + gz * gz);
        acc += e.v;
        if (want_potential) {
            v1[i] = e.dr;
            const double w = 2.0 * e.ds;
            g0[i] = make_double2(w * gx, 0.0);
            g1[i] = make_double2(w * gy, 0.0);
            g2[i] = make_double2(w * gz, 0.0);
        }
    }
    // block sum
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0 && exc_acc) atomicAdd(exc_acc, s * dv);
    }
}

// div(G) = sum_a i G_a h_a(G) / N, into o (h_a: forward FFTs of real fields)
__global__ void k_div_gspace(const double2* __restrict__ h0, const double2* __restrict__ h1,
                             const double2* __restrict__ h2, GridRecip gr, double2* __restrict__ o) {
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    const double inv_n = 1.0 / (double)n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        double g[3];
        if (!gvec(i, gr, g)) {
            o[i] = make_double2(0.0, 0.0);
            continue;
        }
        const double re = g[0] * h0[i].x + g[1] * h1[i].x + g[2] * h2[i].x;
        const double im = g[0] * h0[i].y + g[1] * h1[i].y + g[2] * h2[i].y;
        o[i] = make_double2(-im * inv_n, re * inv_n);
    }
}

// veff = vloc + vh + v1 - div  (vh, div: real parts)
__global__ void k_assemble_gga(const double* __restrict__ vloc, const double2* __restrict__ vh,
                               const double* __restrict__ v1, const double2* __restrict__ div,
                               double* __restrict__ veff, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        veff[i] = vloc[i] + vh[i].x + v1[i] - div[i].x;
}

int blocks_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 148 * 8 ? b : 148 * 8);
}

}  // namespace

void launch_grad_gspace(const double2* f, const GridRecip& gr, double2* o0, double2* o1,
                        double2* o2, cudaStream_t st) {
    count_launch();
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    k_grad_gspace<<<blocks_for(n), 256, 0, st>>>(f, gr, o0, o1, o2);
}

void launch_pbe_point(const double* rho, double2* g0, double2* g1, double2* g2, double* v1,
                      size_t n, double dv, double* exc_acc, bool want_potential, cudaStream_t st) {
    count_launch();
    k_pbe_point<<<blocks_for(n), 256, 0, st>>>(rho, g0, g1, g2, v1, n, dv, exc_acc,
                                               want_potential ? 1 : 0);
}

void launch_div_gspace(const double2* h0, const double2* h1, const double2* h2,
                       const GridRecip& gr, double2* o, cudaStream_t st) {
    count_launch();
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    k_div_gspace<<<blocks_for(n), 256, 0, st>>>(h0, h1, h2, gr, o);
}

void launch_assemble_gga(const double* vloc, const double2* vh, const double* v1,
                         const double2* div, double* veff, size_t n, cudaStream_t st) {
    count_launch();
    k_assemble_gga<<<blocks_for(n), 256, 0, st>>>(vloc, vh, v1, div, veff, n);
}

}  // namespace chfsi
