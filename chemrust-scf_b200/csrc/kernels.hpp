// Launch interfaces of the device kernels (host side).
#pragma once

#include <vector>

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "fft_engine.cuh"

namespace chfsi {

// Geometry of the pruned plane-wave <-> grid transforms.
struct HGeom {
    int nx, ny, nz;
    int n_pw, ncol;
    int lsz;     // smem line stride of z-sticks (odd)
    int lsx;     // smem row stride of an xy plane (odd)
    int nxact;   // x positions (digit-reversed) that carry columns
    const int* col_start;  // ncol + 1: plane-wave range per column
    const int* col_pos;    // ncol: py * lsx + px, digit-reversed plane offset
    const int* pw_col;     // n_pw: column of each plane wave
    const int* pw_zpos;    // n_pw: digit-reversed z position
    const int* xact;       // nxact: digit-reversed x positions
    AxisPlan ax, ay, az;
    // twiddle tables exp(+2 pi i j / n) per axis, precomputed once per context
    const double2* twd_x; const double2* twd_y; const double2* twd_z;
    const float2* twf_x; const float2* twf_y; const float2* twf_z;
    // launch configuration chosen by chfsi_autotune: xy-plane kernel
    // 0 = 256 threads, 1 = 128 threads, 2 = 512 threads per block; z-stick
    // kernels at tune_cols (16, 32, 64) columns per block
    int tune_planes = 0;
    int tune_cols = 32;
    // xy-plane kernels with compile-time radices where the plan has one
    // (square planes, two radices); 0 = always the generic kernel
    int fixed_planes = 1;
    // direct column I/O of the compile-time plane kernel: colidx[l * ny + py]
    // = column at (active x line l, digit-reversed y position py) or -1;
    // xbits: bit px set when digit-reversed x position px carries columns
    const int* colidx = nullptr;
    unsigned int xbits[8] = {0, 0, 0, 0, 0, 0, 0, 0};
};

// Pass-3 epilogue: what to do with (H psi)_g once it is assembled.
enum EpiMode { kEpiApply = 0, kEpiChebFirst = 1, kEpiCheb = 2, kEpiResid = 3 };

struct Epilogue {
    int mode;
    const double* kin;     // n_pw
    const double* coef;    // device: [.., .., c, e, 1/e, -c/e]
    const void* nl;        // non-local contribution (same type as psi), ld n_pw; may be null
    double* norm_acc;      // += sum |out|^2 (may be null)
    double inv_n;          // 1 / N^3
    // one band of the batch that gets plain H x written to plain_out instead
    // of the recurrence (the Lanczos vector carried along by the filter);
    // -1: none
    int plain_band = -1;
    void* plain_out = nullptr;
    // kEpiResid (residual Chebyshev step, R-ChFSI):
    //   out = a H p + b p + c prev + a lam[band] y,  {a, b, c} = rc[0..2]
    const double* rc = nullptr;
    const double* lam = nullptr;   // per band
    const void* yres = nullptr;    // residual Y (same type as psi), ld n_pw
};

// density accumulation keeps 24 plane points per thread x 512 threads
constexpr size_t kDensityPlanePoints = 24 * 512;

// psi (nb x n_pw, ld ldp) -> work (nb x nz x ncol): scatter + inverse z.
template <typename C>
void launch_zsticks_inverse(const C* psi, int ldp, C* work, int nb, const HGeom& g,
                            cudaStream_t st);
// work planes: inverse y, inverse x, x V(r), forward x, forward y (in place).
template <typename C>
void launch_planes_vloc(C* work, const double* veff, int nb, const HGeom& g, cudaStream_t st);
// work -> out: forward z + gather + kinetic + non-local + epilogue.
template <typename C>
void launch_zsticks_forward(const C* work, const C* psi, int ldp, C* out, int ldo, int nb,
                            const HGeom& g, const Epilogue& e, cudaStream_t st);
// density: rho[r] += sum_b occ[b] |psi_b(r)|^2 * scale from inverse-z work.
template <typename C>
void launch_planes_density(const C* work, const double* occ, int nb, double scale, double* rho,
                           const HGeom& g, cudaStream_t st);
size_t planes_smem_bytes(const HGeom& g, size_t csize);

// Full-grid 1D transforms along one axis (0 = x, 1 = y, 2 = z) of a
// complex grid [nz][ny][nx].
template <typename C>
void launch_axis_fft(C* data, int nx, int ny, int nz, int axis, bool forward, const AxisPlan& P,
                     cudaStream_t st);

// Potential helpers on the full grid.
struct GridRecip {
    int nx, ny, nz;
    const int* idr_x; const int* idr_y; const int* idr_z;  // digit-reversed pos -> frequency
    double b[9];       // reciprocal lattice rows b1, b2, b3
};
void launch_real_to_complex(const double* r, double2* c, size_t n, cudaStream_t st);
// ---- GGA (PBE) pieces, gga.cu
// o_a = i G_a f(G) / N (digit-reversed density-grid layout)
void launch_grad_gspace(const double2* f, const GridRecip& gr, double2* o0, double2* o1,
                        double2* o2, cudaStream_t st);
// pointwise PBE on rho and grad rho (real parts of g0..g2): exc_acc += E_xc;
// with want_potential: v1 = de/drho, g_a <- 2 de/dsigma grad_a rho
void launch_pbe_point(const double* rho, double2* g0, double2* g1, double2* g2, double* v1,
                      size_t n, double dv, double* exc_acc, bool want_potential, cudaStream_t st);
// o = sum_a i G_a h_a(G) / N
void launch_div_gspace(const double2* h0, const double2* h1, const double2* h2,
                       const GridRecip& gr, double2* o, cudaStream_t st);
// veff = vloc + Re vh + v1 - Re div
void launch_assemble_gga(const double* vloc, const double2* vh, const double* v1,
                         const double2* div, double* veff, size_t n, cudaStream_t st);
// ---- Hellmann-Feynman forces, forces.cu
void launch_force_local(const double2* rhog, const GridRecip& gr, const int* wave_grid,
                        const double* pos, const double* zion, const double* rc, int n_ions,
                        double omega, double* force, cudaStream_t st);
void launch_scale_pw(const double2* psi, const double* q, int npw, int nb, double2* out,
                     cudaStream_t st);
void launch_force_nl(const double2* C, const double2* B, int nb, const double* occ,
                     const int* poff, const int* doff, const double2* dmat, int n_ions, int axis,
                     const int* atom_of_ion, double* force, cudaStream_t st);
void ewald_forces(const double* lattice, const double* recip, const std::vector<double>& pos,
                  const std::vector<double>& z, std::vector<double>& f);
// In G space (digit-reversed layout): c <- 4 pi c / (N^3 G^2), G = 0 -> 0;
// eh_acc += 1/2 Omega 4 pi |c / N^3|^2 / G^2 (before scaling).
void launch_hartree_gspace(double2* c, const GridRecip& gr, double omega, double* eh_acc,
                           cudaStream_t st);
// veff = vloc + Re(vh) + vxc(rho);  exc_acc += sum rho eps_xc * dv.
void launch_assemble_veff(const double* vloc, const double2* vh, const double* rho, double* veff,
                          size_t n, double dv, double* exc_acc, cudaStream_t st);
// exc_acc += sum rho eps_xc(rho) dv;  dc_acc += sum (veff - vloc) rho_out dv
void launch_energy_terms(const double* rho_out, const double* veff, const double* vloc, size_t n,
                         double dv, double* exc_acc, double* dc_acc, cudaStream_t st);
void launch_take_real(const double2* c, double* r, size_t n, cudaStream_t st);

// ---- density grid and ultrasoft augmentation (aug.cu)
// dst[dst_pos[i]] = scale * src[src_pos[i]]: G vectors shared by two grids
void launch_scatter_g(const double2* src, const int* src_pos, const int* dst_pos, int n,
                      double scale, double2* dst, cudaStream_t st);
void launch_scale_copy(const double2* src, double scale, double2* dst, size_t n, cudaStream_t st);
// F(G) += scale exp(-G^2 w^2 / 4) sum_I c_I e^{-i G.R_I}; ph: per ion the
// axis phase tables e^{-i 2 pi f_d h}, [ion][nx | ny | nz] (frequency order)
void launch_aug_add(double2* F, const GridRecip& gr, const double2* ph, const double* c, int nions,
                    double width, double scale, cudaStream_t st);
// v_I += scale Re sum_G V(G) exp(-G^2 w^2 / 4) e^{+i G.R_I}  (v zeroed by caller)
void launch_ion_potential(const double2* V, const GridRecip& gr, const double2* ph, int nions,
                          double width, double scale, double* v, cudaStream_t st);
// c_I += f_n Re(conj(C_in) (qC)_in)  (C, qC: n_proj x nb; c zeroed by caller)
void launch_aug_coeffs(const double2* C, const double2* qC, const double* occ, int nb,
                       const int* proj_ion, int np, double* c, cudaStream_t st);
// D_I = D0_I + v_I q_I per ion block
void launch_screen_d(const double2* D0, const double2* q, const double* v, const int* poff,
                     const int* doff, int nions, double2* D, cudaStream_t st);

}  // namespace chfsi
