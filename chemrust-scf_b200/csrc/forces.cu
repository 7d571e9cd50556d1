// Hellmann-Feynman forces on the ions of a norm-conserving (or local-only)
// cell after an SCF: F_I = -dE/dR_I with the density and wavefunctions held
// fixed (the free energy E - kT S is variational in both), the step the
// reference's planned scf_run fills into its forces output
// (PROJECT_ROOT_PLAN.md:957-1018; plans/phase-2/PHASE_PLAN.md:90-95).
//
//   local:    E_loc = Omega sum_G V(G) conj(rho(G)),
//             V(G) = sum_I v_I(G) e^{-i G.R_I},  v_I = -4 pi Z_I / (Omega G^2) e^{-G^2 rc_I^2 / 4}
//             F_I = -Omega sum_G v_I(G) G Im(e^{-i G.R_I} conj(rho(G)))
//   non-local: E_nl = sum_n f_n sum_ij conj(C_in) D_ij C_jn,  C = beta^H psi,
//             d beta_j / d R_I = -i q beta_j (q = G + k, beta_j on ion I), so
//             F_I = 2 sum_n f_n sum_{ij in I} Im(conj(C_in) D_ij B_jn),  B = beta^H (q psi)
//   ion-ion:  Ewald sum of point charges with a neutralising background.
#include "kernels.hpp"
#include "launch_count.hpp"

#include <cmath>
#include <vector>

namespace chfsi {

namespace {

constexpr double kPi = 3.14159265358979323846;

// blockIdx.y = ion; threads stride over the density-grid G points inside the
// wave grid's box (|h| < nx/2, ...), G != 0
__global__ void __launch_bounds__(256)
k_force_local(const double2* __restrict__ rhog, GridRecip gr, int wnx, int wny, int wnz,
              const double* __restrict__ pos, const double* __restrict__ zion,
              const double* __restrict__ rc, double omega, double* __restrict__ force) {
    __shared__ double red[3][8];
    const int ion = blockIdx.y;
    const double R[3] = {pos[3 * ion], pos[3 * ion + 1], pos[3 * ion + 2]};
    const double pref = -4.0 * kPi * zion[ion] / omega, rc2 = rc[ion] * rc[ion];
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    const double inv_n = 1.0 / (double)n;
    double f[3] = {0.0, 0.0, 0.0};
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % gr.nx);
        const int iy = (int)((i / gr.nx) % gr.ny);
        const int iz = (int)(i / ((size_t)gr.nx * gr.ny));
        int h = gr.idr_x[ix], k = gr.idr_y[iy], l = gr.idr_z[iz];
        if (h >= (gr.nx + 1) / 2) h -= gr.nx;
        if (k >= (gr.ny + 1) / 2) k -= gr.ny;
        if (l >= (gr.nz + 1) / 2) l -= gr.nz;
        if (2 * abs(h) >= wnx || 2 * abs(k) >= wny || 2 * abs(l) >= wnz) continue;
        if (h == 0 && k == 0 && l == 0) continue;
        const double gx = h * gr.b[0] + k * gr.b[3] + l * gr.b[6];
        const double gy = h * gr.b[1] + k * gr.b[4] + l * gr.b[7];
        const double gz = h * gr.b[2] + k * gr.b[5] + l * gr.b[8];
        const double g2 = gx * gx + gy * gy + gz * gz;
        const double v = pref / g2 * exp(-0.25 * g2 * rc2);
        double sn, cs;
        sincos(-(gx * R[0] + gy * R[1] + gz * R[2]), &sn, &cs);
        // Im(e^{-i G.R} conj(rho)) with rho = (a + i b) / N
        const double a = rhog[i].x * inv_n, b = rhog[i].y * inv_n;
        const double im = sn * a - cs * b;
        const double w = -omega * v * im;
        f[0] += w * gx;
        f[1] += w * gy;
        f[2] += w * gz;
    }
    for (int d = 0; d < 3; ++d) {
        double s = f[d];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[d][threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[threadIdx.x][w];
        atomicAdd(&force[3 * ion + threadIdx.x], s);
    }
}

// out[b][g] = q_a[g] psi[b][g]
__global__ void k_scale_pw(const double2* __restrict__ psi, const double* __restrict__ q, int npw,
                           size_t n, double2* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double s = q[i % (size_t)npw];
        out[i] = make_double2(s * psi[i].x, s * psi[i].y);
    }
}

// one block per ion: F_a += 2 sum_n f_n sum_{ij in I} Im(conj(C_in) D_ij B_jn)
// C, B: n_proj x nb (row-major); D blocks ne x ne per ion at doff[ion]
__global__ void __launch_bounds__(256)
k_force_nl(const double2* __restrict__ C, const double2* __restrict__ B, int nb,
           const double* __restrict__ occ, const int* __restrict__ poff,
           const int* __restrict__ doff, const double2* __restrict__ dmat, int axis,
           const int* __restrict__ atom_of_ion, double* __restrict__ force) {
    __shared__ double red[8];
    const int ion = blockIdx.x;
    const int p0 = poff[ion], ne = poff[ion + 1] - p0;
    const double2* D = dmat + doff[ion];
    double acc = 0.0;
    for (int t = threadIdx.x; t < ne * nb; t += blockDim.x) {
        const int i = t / nb, b = t - i * nb;
        const double fo = occ[b];
        if (fo == 0.0) continue;
        const double2 c = C[(size_t)(p0 + i) * nb + b];
        // sum_j D_ij B_jb
        double sr = 0.0, si = 0.0;
        for (int j = 0; j < ne; ++j) {
            const double2 d = D[i * ne + j];
            const double2 x = B[(size_t)(p0 + j) * nb + b];
            sr += d.x * x.x - d.y * x.y;
            si += d.x * x.y + d.y * x.x;
        }
        // Im(conj(c) (sr + i si)) = c.x si - c.y sr
        acc += 2.0 * fo * (c.x * si - c.y * sr);
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        atomicAdd(&force[3 * atom_of_ion[ion] + axis], s);
    }
}

}  // namespace

void launch_force_local(const double2* rhog, const GridRecip& gr, const int* wave_grid,
                        const double* pos, const double* zion, const double* rc, int n_ions,
                        double omega, double* force, cudaStream_t st) {
    count_launch();
    dim3 grid(48, n_ions);
    k_force_local<<<grid, 256, 0, st>>>(rhog, gr, wave_grid[0], wave_grid[1], wave_grid[2], pos,
                                        zion, rc, omega, force);
}

void launch_scale_pw(const double2* psi, const double* q, int npw, int nb, double2* out,
                     cudaStream_t st) {
    count_launch();
    const size_t n = (size_t)nb * npw;
    size_t blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_scale_pw<<<(int)blocks, 256, 0, st>>>(psi, q, npw, n, out);
}

void launch_force_nl(const double2* C, const double2* B, int nb, const double* occ,
                     const int* poff, const int* doff, const double2* dmat, int n_ions, int axis,
                     const int* atom_of_ion, double* force, cudaStream_t st) {
    count_launch();
    k_force_nl<<<n_ions, 256, 0, st>>>(C, B, nb, occ, poff, doff, dmat, axis, atom_of_ion, force);
}

// Ewald forces of point charges z_i at Cartesian positions (bohr) in the cell
// with lattice rows a1, a2, a3 and reciprocal rows b1, b2, b3 (2 pi inv(A)^T):
// splitting eta = 5 / Omega^(1/3), real-space images |n_d| <= 2, reciprocal
// |m_d| <= 10 (erfc(10) and exp(-39) of the cubic cells' sums: converged).
void ewald_forces(const double* lat, const double* rec, const std::vector<double>& pos,
                  const std::vector<double>& z, std::vector<double>& f) {
    const int na = (int)z.size();
    const double omega = std::fabs(lat[0] * (lat[4] * lat[8] - lat[5] * lat[7]) -
                                   lat[1] * (lat[3] * lat[8] - lat[5] * lat[6]) +
                                   lat[2] * (lat[3] * lat[7] - lat[4] * lat[6]));
    const double eta = 5.0 / std::cbrt(omega);
    f.assign(3 * (size_t)na, 0.0);
    const int nimg = 2;
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < na; ++j)
            for (int lx = -nimg; lx <= nimg; ++lx)
                for (int ly = -nimg; ly <= nimg; ++ly)
                    for (int lz = -nimg; lz <= nimg; ++lz) {
                        if (i == j && lx == 0 && ly == 0 && lz == 0) continue;
                        double d[3];
                        for (int c = 0; c < 3; ++c)
                            d[c] = pos[3 * i + c] - pos[3 * j + c] + lx * lat[c] + ly * lat[3 + c] +
                                   lz * lat[6 + c];
                        const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                        // -d/dr [erfc(eta r) / r]
                        const double g = std::erfc(eta * r) / (r * r) +
                                         2.0 * eta / std::sqrt(kPi) * std::exp(-eta * eta * r * r) / r;
                        const double w = z[i] * z[j] * g / r;
                        for (int c = 0; c < 3; ++c) f[3 * i + c] += w * d[c];
                    }
    const int gm = 10;
    for (int h = -gm; h <= gm; ++h)
        for (int k = -gm; k <= gm; ++k)
            for (int l = -gm; l <= gm; ++l) {
                if (h == 0 && k == 0 && l == 0) continue;
                double g[3];
                for (int c = 0; c < 3; ++c) g[c] = h * rec[c] + k * rec[3 + c] + l * rec[6 + c];
                const double g2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
                const double wg = (4.0 * kPi / omega) * std::exp(-g2 / (4.0 * eta * eta)) / g2;
                double sr = 0.0, si = 0.0;
                for (int i = 0; i < na; ++i) {
                    const double ph = g[0] * pos[3 * i] + g[1] * pos[3 * i + 1] + g[2] * pos[3 * i + 2];
                    sr += z[i] * std::cos(ph);
                    si += z[i] * std::sin(ph);
                }
                // F_i = (4 pi / Omega) sum_G e^{-G^2/4eta^2}/G^2 z_i G Im(conj(S) e^{i G.R_i})
                for (int i = 0; i < na; ++i) {
                    const double ph = g[0] * pos[3 * i] + g[1] * pos[3 * i + 1] + g[2] * pos[3 * i + 2];
                    const double im = sr * std::sin(ph) - si * std::cos(ph);
                    for (int c = 0; c < 3; ++c) f[3 * i + c] += wg * z[i] * g[c] * im;
                }
            }
}

}  // namespace chfsi
