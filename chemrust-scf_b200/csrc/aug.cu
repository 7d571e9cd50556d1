// Ultrasoft augmentation and the density (augmentation) grid.
//
// Augmentation functions are Q_ij(r) = q_ij g(|r - R_I|) with g a unit
// Gaussian of width w, g(r) = exp(-r^2/w^2) / (pi^{3/2} w^3), whose
// transform is g^(G) = exp(-G^2 w^2 / 4), so int Q_ij = q_ij and the
// overlap S = 1 + sum beta q beta^H of the generalised problem conserves
// charge.  The density on the density grid is
//   rho(G) = rho_smooth(G) + (1/Omega) g^(G) sum_I c_I e^{-i G.R_I},
//   c_I = sum_n f_n sum_{ij in I} conj(<beta_i|psi_n>) q_ij <beta_j|psi_n>,
// and the screened nonlocal strengths are D_I = D0_I + q_I v_I with
//   v_I = int V_eff(r) g(r - R_I) dr = sum_G V_G g^(G) e^{i G.R_I}.
// The reference crate's phase-0 gate builds the same S from q_ij
// (tests/phase0_gate2_convergence.rs:279-322); its augmentation charges come
// from chemrust-hamiltonian-core, which is not available, so the Gaussian
// form is the synthetic model of the 216-atom ultrasoft configuration.
//
// The smooth density is formed on the wavefunction grid and interpolated
// to the density grid by zero padding in G; V_eff goes back by truncation
// (downsample_array_to_wave_grid, src/scf.rs:413-454).
#include <cuda_runtime.h>

#include "kernels.hpp"
#include "launch_count.hpp"

namespace chfsi {
namespace {

int blocks_for(size_t n) {
    size_t b = (n + 255) / 256;
    return (int)(b < 148 * 8 ? (b ? b : 1) : 148 * 8);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void k_scatter_g(const double2* __restrict__ src, const int* __restrict__ src_pos,
                            const int* __restrict__ dst_pos, int n, double scale,
                            double2* __restrict__ dst) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double2 v = src[src_pos[i]];
        dst[dst_pos[i]] = make_double2(scale * v.x, scale * v.y);
    }
}

__global__ void k_scale_copy(const double2* __restrict__ src, double scale, double2* __restrict__ dst,
                             size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        dst[i] = make_double2(scale * src[i].x, scale * src[i].y);
}

struct GFreq {
    int h, k, l;
    double g2;
};
__device__ __forceinline__ GFreq freq_of(const GridRecip& gr, int ix, int iy, int iz) {
    GFreq f;
    f.h = gr.idr_x[ix];
    f.k = gr.idr_y[iy];
    f.l = gr.idr_z[iz];
    int h = f.h, k = f.k, l = f.l;
    if (h >= (gr.nx + 1) / 2) h -= gr.nx;
    if (k >= (gr.ny + 1) / 2) k -= gr.ny;
    if (l >= (gr.nz + 1) / 2) l -= gr.nz;
    const double gx = h * gr.b[0] + k * gr.b[3] + l * gr.b[6];
    const double gy = h * gr.b[1] + k * gr.b[4] + l * gr.b[7];
    const double gz = h * gr.b[2] + k * gr.b[5] + l * gr.b[8];
    f.g2 = gx * gx + gy * gy + gz * gz;
    return f;
}

// One block per (y, z) row of the G grid, threads over x.  ph holds, per
// ion, e^{-i 2 pi f h} for the three fractional coordinates f of the ion and
// every frequency h of each axis: [ion][nx | ny | nz].
__global__ void __launch_bounds__(256)
k_aug_add(double2* __restrict__ F, GridRecip gr, const double2* __restrict__ ph,
          const double* __restrict__ c, int nions, double width, double scale) {
    extern __shared__ double2 yz[];  // per ion: c_I e^{-i G_y} e^{-i G_z}
    const int iy = blockIdx.x, iz = blockIdx.y;
    const int ky = gr.idr_y[iy], lz = gr.idr_z[iz];
    const int stride = gr.nx + gr.ny + gr.nz;
    for (int I = threadIdx.x; I < nions; I += blockDim.x) {
        const double2* p = ph + (size_t)I * stride;
        const double2 v = cmul(p[gr.nx + ky], p[gr.nx + gr.ny + lz]);
        yz[I] = make_double2(c[I] * v.x, c[I] * v.y);
    }
    __syncthreads();
    for (int ix = threadIdx.x; ix < gr.nx; ix += blockDim.x) {
        const GFreq f = freq_of(gr, ix, iy, iz);
        double2 s = make_double2(0.0, 0.0);
        for (int I = 0; I < nions; ++I) {
            const double2 e = cmul(yz[I], ph[(size_t)I * stride + f.h]);
            s.x += e.x;
            s.y += e.y;
        }
        const double gh = scale * exp(-0.25 * f.g2 * width * width);
        const size_t o = ix + (size_t)gr.nx * (iy + (size_t)gr.ny * iz);
        F[o].x += gh * s.x;
        F[o].y += gh * s.y;
    }
}

// v_I += scale * Re sum_G V(G) g^(G) e^{+i G.R_I}: blocks (row chunk, ion).
__global__ void __launch_bounds__(256)
k_ion_potential(const double2* __restrict__ V, GridRecip gr, const double2* __restrict__ ph,
                double width, double scale, double* __restrict__ v) {
    __shared__ double red[32];
    const int I = blockIdx.y;
    const int stride = gr.nx + gr.ny + gr.nz;
    const double2* p = ph + (size_t)I * stride;
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    double acc = 0.0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const int ix = (int)(i % gr.nx);
        const int iy = (int)((i / gr.nx) % gr.ny);
        const int iz = (int)(i / ((size_t)gr.nx * gr.ny));
        const GFreq f = freq_of(gr, ix, iy, iz);
        // e^{-i G.R} from the tables; e^{+i G.R} is its conjugate
        const double2 e = cmul(cmul(p[f.h], p[gr.nx + f.k]), p[gr.nx + gr.ny + f.l]);
        const double2 vg = V[i];
        const double gh = exp(-0.25 * f.g2 * width * width);
        acc += gh * (vg.x * e.x + vg.y * e.y);  // Re(V conj(e))
    }
    // block sum
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) red[w] = acc;
    __syncthreads();
    if (w == 0) {
        acc = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) atomicAdd(v + I, scale * acc);
    }
}

// c_I += f_n Re(conj(C_in) (qC)_in) for projector i of ion I, band n.
__global__ void k_aug_coeffs(const double2* __restrict__ C, const double2* __restrict__ qC,
                             const double* __restrict__ occ, int nb, const int* __restrict__ proj_ion,
                             int np, double* __restrict__ c) {
    const size_t n = (size_t)np * nb;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
         t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / nb), b = (int)(t % nb);
        const double f = occ[b];
        if (f == 0.0) continue;
        const double2 a = C[t], q = qC[t];
        atomicAdd(c + proj_ion[i], f * (a.x * q.x + a.y * q.y));
    }
}

// D_I = D0_I + v_I q_I over each ion's ne x ne block (offset doff[I],
// ne = poff[I + 1] - poff[I]); one block per ion.
__global__ void k_screen_d(const double2* __restrict__ D0, const double2* __restrict__ q,
                           const double* __restrict__ v, const int* __restrict__ poff,
                           const int* __restrict__ doff, double2* __restrict__ D) {
    const int I = blockIdx.x;
    const int ne = poff[I + 1] - poff[I];
    const size_t o = doff[I];
    const double vi = v[I];
    for (int t = threadIdx.x; t < ne * ne; t += blockDim.x) {
        const double2 d = D0[o + t], qq = q[o + t];
        D[o + t] = make_double2(d.x + vi * qq.x, d.y + vi * qq.y);
    }
}

}  // namespace

void launch_scatter_g(const double2* src, const int* src_pos, const int* dst_pos, int n,
                      double scale, double2* dst, cudaStream_t st) {
    count_launch();
    k_scatter_g<<<blocks_for((size_t)n), 256, 0, st>>>(src, src_pos, dst_pos, n, scale, dst);
}

void launch_scale_copy(const double2* src, double scale, double2* dst, size_t n, cudaStream_t st) {
    count_launch();
    k_scale_copy<<<blocks_for(n), 256, 0, st>>>(src, scale, dst, n);
}

void launch_aug_add(double2* F, const GridRecip& gr, const double2* ph, const double* c, int nions,
                    double width, double scale, cudaStream_t st) {
    count_launch();
    const size_t sm = (size_t)nions * sizeof(double2);
    if (sm > 48 * 1024) cudaFuncSetAttribute(k_aug_add, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    dim3 grid(gr.ny, gr.nz);
    k_aug_add<<<grid, 256, sm, st>>>(F, gr, ph, c, nions, width, scale);
}

void launch_ion_potential(const double2* V, const GridRecip& gr, const double2* ph, int nions,
                          double width, double scale, double* v, cudaStream_t st) {
    count_launch();
    const size_t n = (size_t)gr.nx * gr.ny * gr.nz;
    int chunks = (int)((n + 256 * 64 - 1) / (256 * 64));
    if (chunks < 1) chunks = 1;
    if (chunks > 256) chunks = 256;
    dim3 grid(chunks, nions);
    k_ion_potential<<<grid, 256, 0, st>>>(V, gr, ph, width, scale, v);
}

void launch_aug_coeffs(const double2* C, const double2* qC, const double* occ, int nb,
                       const int* proj_ion, int np, double* c, cudaStream_t st) {
    count_launch();
    k_aug_coeffs<<<blocks_for((size_t)np * nb), 256, 0, st>>>(C, qC, occ, nb, proj_ion, np, c);
}

void launch_screen_d(const double2* D0, const double2* q, const double* v, const int* poff,
                     const int* doff, int nions, double2* D, cudaStream_t st) {
    count_launch();
    k_screen_d<<<nions, 128, 0, st>>>(D0, q, v, poff, doff, D);
}

}  // namespace chfsi
