/*
 * chfsi.h — C ABI of the B200 (sm_100a) Chebyshev-filtered subspace iteration
 * (ChFSI) SCF path.
 *
 * The entry points replace, one for one, the crate-internal Rust contracts of
 * the reference crate chemrust-scf (paths relative to that project):
 *
 *   chfsi_chebyshev_filter   src/eigensolver/chebyshev.rs:626-816  chebyshev_filter()
 *   chfsi_rayleigh_ritz      src/eigensolver/rayleigh_ritz.rs:48-245 rayleigh_ritz()
 *   chfsi_diagonalize        src/scf.rs:169-265  ScfIteration<_, VEffBuilt>::diagonalize()
 *   chfsi_apply_h            src/eigensolver/chebyshev.rs:371-403 apply_full_hamiltonian()
 *   chfsi_set_veff           src/scf.rs:188-195 (V_eff upload + min/max fold)
 *   chfsi_set_basis          src/scf.rs:387-401 pw_coords_to_fft_indices()
 *   chfsi_set_projectors     src/eigensolver/vnl_data.rs:25-89 VnlBatchData::precompute()
 *   chfsi_construct_density  src/scf.rs:275-279 construct_density() (todo!() in the reference)
 *   chfsi_build_veff         src/scf.rs:157-159 build_v_eff()       (todo!() in the reference)
 *   (Pulay step of chfsi_scf_run) src/mixing.rs:24-27 DensityHistory::mix (todo!() there)
 *   chfsi_scf_run            src/scf.rs:358-376 run_scf(); shape of the planned
 *                            scf_run() C ABI (PROJECT_ROOT_PLAN.md:957-1018)
 *   chfsi_create / _destroy  planned scf_context_create/_destroy (PROJECT_ROOT_PLAN.md:860-1029)
 *
 * Conventions (identical to the reference's):
 *   - complex numbers are interleaved (re, im) doubles (CudaComplex = double2,
 *     src/device/mod.rs:27);
 *   - wavefunctions are band-major ("ColumnDistributed"): psi[b * n_pw + g]
 *     (src/layout.rs:25-26, chebyshev.rs:104-106);
 *   - the FFT grid is stored [ngz][ngy][ngx] with linear index
 *     ix + ngx * (iy + ngy * iz); negative Miller indices wrap to n + h
 *     (src/scf.rs:382-401);
 *   - both FFT directions are unnormalised; H|psi> applies 1/N^3 at the gather
 *     (chebyshev.rs:126-142, 654);
 *   - eigenvalues are returned ascending (subspace_diag.rs:335-363).
 *
 * Ownership: a context owns all of its device memory and one CUDA stream.
 * Calls on one context are not re-entrant.  Host arrays passed in are copied;
 * device pointers passed to chfsi_apply_h stay owned by the caller.
 * The context stream is created non-blocking: work on a device pointer is
 * ordered after earlier work on that stream (chfsi_get_stream) only, so a
 * caller that fills the buffer on another stream synchronises first.
 * Errors are returned as chfsi_status (mirror of the crate's Error enum,
 * src/types.rs:226-248); chfsi_last_error() gives the message.
 */
#ifndef CHFSI_H
#define CHFSI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes: mirror of src/types.rs:226-248 Error, plus the planned     */
/* scf_run convention (0 converged, -1 not converged, < -1 error).          */
/* ------------------------------------------------------------------------ */
typedef enum chfsi_status {
    CHFSI_OK                  = 0,
    CHFSI_NOT_CONVERGED       = -1,  /* scf_run hit max iterations           */
    CHFSI_ERR_NOT_IMPLEMENTED = -2,  /* Error::NotImplemented                */
    CHFSI_ERR_CHEB_DIVERGED   = -3,  /* Error::ChebyshevDiverged             */
    CHFSI_ERR_RR_FAILED       = -4,  /* Error::RayleighRitzFailed{info}      */
    CHFSI_ERR_CUDA            = -5,  /* Error::Cuda                          */
    CHFSI_ERR_BAD_INPUT       = -6,  /* shape / pointer / range violation    */
    CHFSI_ERR_NO_DEVICE       = -7,  /* no CUDA device visible               */
    CHFSI_ERR_OUT_OF_MEMORY   = -8,
    CHFSI_ERR_NUMERIC         = -9,  /* NaN/Inf detected on device           */
    CHFSI_ERR_TIMEOUT         = -10  /* a bounded device-side wait ran out
                                        (the kernel stopped, retired what it
                                        had issued and returned)             */
} chfsi_status;

typedef struct chfsi_c128 { double re, im; } chfsi_c128;

/* Precision of the filter (the Rayleigh-Ritz, its subspace matrices and the
 * rotation of the block are FP64 in both modes). */
enum { CHFSI_PREC_FP64 = 0, CHFSI_PREC_MIXED = 1 };
/* Upper spectral bound used by the filter. */
enum {
    CHFSI_BOUND_HEURISTIC = 0, /* chebyshev.rs:225-254: 1/2 Gmax^2 + (maxV - minV) */
    CHFSI_BOUND_LANCZOS   = 1, /* k-step Lanczos: lambda_max(T_k) + |f_k| (Zhou 2010) */
    CHFSI_BOUND_LANCZOS_FUSED = 2 /* the same k-step Lanczos carried as one extra column of
                                     the filter's own H applies (FP64 filter): each filter
                                     leaves the bound for the next, no separate passes; the
                                     first filter of a context, and mixed-precision filters,
                                     run the k steps separately */
};

/* Form of the filter once Ritz values of the current block are known.
 * CHEBYSHEV: the reference's three-term recurrence on the block itself
 * (chebyshev.rs:626-816).  RESIDUAL: R-ChFSI (reference_paper/2025
 * Algorithm 3), the sigma-scaled recurrence on the residuals H X - S X Lam of
 * the Ritz pairs with the Woodbury S^-1 as approximate inverse: the same
 * span in exact arithmetic, and in the mixed-precision mode an FP32/BF16x3
 * filter whose error falls with the residual instead of stalling at FP32
 * rounding.  The norm guard does not apply to the residual recurrence.  In a
 * mixed-precision context the FP64 passes (first pass, convergence checks)
 * keep the Chebyshev form. */
enum { CHFSI_FILTER_CHEBYSHEV = 0, CHFSI_FILTER_RESIDUAL = 1 };

/* ------------------------------------------------------------------------ */
/* Synthetic systems (the seeded inputs of the benchmark configurations).   */
/* The reference obtains these from chemrust-hamiltonian-core (absent);     */
/* here they come from analytic formulas, deterministic in the seed.        */
/* ------------------------------------------------------------------------ */
enum { CHFSI_LATTICE_DIAMOND = 0, CHFSI_LATTICE_SC = 1, CHFSI_LATTICE_BCC = 2 };

typedef struct chfsi_synth_params {
    int      lattice;        /* CHFSI_LATTICE_*                                   */
    int      n_rep;          /* conventional cells per axis                       */
    double   a_conv;         /* conventional cubic cell edge (bohr)               */
    double   jitter;         /* uniform +-jitter per Cartesian component (bohr)   */
    double   z_val;          /* valence charge per atom                           */
    double   rc_loc;         /* V_loc(G) = -4 pi Z/(Omega G^2) exp(-G^2 rc^2/4)   */
    double   ecut;           /* plane-wave cutoff (Ha): 1/2 |G+k|^2 <= ecut        */
    int      ngrid[3];       /* FFT grid; 0 = smallest 2,3,5-smooth >= 4 m + 1     */
    int      n_bands;        /* 0 = 1.25 x occupied, rounded up                   */
    int      n_shell;        /* radial projector shells per atom (0: local only)  */
    double   rc_proj[4];     /* beta_l(r) = r^l exp(-r^2/rc^2) per shell           */
    int      lmax;           /* projectors for l = 0..lmax (lmax <= 1)            */
    double   d_min, d_max;   /* D_ll ~ U[d_min, d_max] (Ha) per atom, shell, l    */
    int      uspp;           /* 1: augmentation charges q_ij (S = 1 + b q b^H)    */
    double   q_width;        /* Gaussian width of Q_ij(r) (bohr)                  */
    double   q_amp;          /* A_ij ~ U[-q_amp, q_amp]                           */
    double   kpt[3];         /* k in reduced (fractional) coordinates             */
    uint64_t seed;
    int      ngrid_density[3]; /* density/augmentation grid; 0 = the FFT grid     */
} chfsi_synth_params;

typedef struct chfsi_system chfsi_system;

typedef struct chfsi_system_info {
    int    ngrid[3];
    int    n_pw;
    int    n_bands;
    int    n_occ;           /* bands with occupation 2                          */
    int    n_atoms;
    int    n_proj;          /* total projectors over all atoms                  */
    int    n_ions_with_proj;
    int    n_columns;       /* (x,y) columns that hold plane waves              */
    double omega;           /* cell volume (bohr^3)                             */
    double n_elec;
    double gmax;            /* max |G+k| over the plane-wave sphere             */
    double e_ewald;         /* ion-ion energy of point charges (Ha)             */
    double lattice[9];      /* rows a1, a2, a3 (bohr)                           */
    int    ngrid_density[3];
    double q_width;         /* Gaussian width of Q_ij(r) when ultrasoft (bohr)  */
    int    uspp;
} chfsi_system_info;

chfsi_status chfsi_synth_defaults(int config_index, chfsi_synth_params* out);
chfsi_status chfsi_system_generate(const chfsi_synth_params* p, chfsi_system** out);
/* The same system with the atoms at the given Cartesian positions (n_atoms x
 * 3, bohr) in place of the seeded jittered lattice (finite-difference
 * forces, displaced geometries). */
chfsi_status chfsi_system_generate_at(const chfsi_synth_params* p, const double* positions,
                                      chfsi_system** out);
void         chfsi_system_destroy(chfsi_system* s);
chfsi_status chfsi_system_get_info(const chfsi_system* s, chfsi_system_info* out);
/* Miller indices (n_pw x 3), sorted by (iy, ix) column then iz. */
chfsi_status chfsi_system_get_miller(const chfsi_system* s, int32_t* out);
/* 1/2 |G+k|^2 per plane wave (n_pw). */
chfsi_status chfsi_system_get_kinetic(const chfsi_system* s, double* out);
/* V_loc(G) * S(G) on the full FFT grid (ngz*ngy*ngx, grid order). */
chfsi_status chfsi_system_get_vloc_g(const chfsi_system* s, chfsi_c128* out);
/* Projectors beta_p(G+k), row-major (n_proj x n_pw), grouped by ion. */
chfsi_status chfsi_system_get_beta(const chfsi_system* s, chfsi_c128* out);
/* proj_offsets[n_ions_with_proj + 1]: first projector of each ion. */
chfsi_status chfsi_system_get_proj_offsets(const chfsi_system* s, int32_t* out);
/* Per-ion D blocks (ne_i x ne_i, row-major), concatenated over ions. */
chfsi_status chfsi_system_get_dmat(const chfsi_system* s, chfsi_c128* out);
/* Per-ion q blocks (same layout as D); zero when the system is not USPP. */
chfsi_status chfsi_system_get_qmat(const chfsi_system* s, chfsi_c128* out);
/* Initial wavefunctions: complex Gaussian, band-major (n_bands x n_pw). */
chfsi_status chfsi_system_get_psi0(const chfsi_system* s, chfsi_c128* out);
/* Occupations (n_bands). */
chfsi_status chfsi_system_get_occupations(const chfsi_system* s, double* out);
/* Atom positions (n_atoms x 3, Cartesian bohr). */
chfsi_status chfsi_system_get_positions(const chfsi_system* s, double* out);

/* ------------------------------------------------------------------------ */
/* Context (device state).                                                  */
/* ------------------------------------------------------------------------ */
typedef struct chfsi_ctx chfsi_ctx;

typedef struct chfsi_dims {
    int ngrid[3];           /* ngx, ngy, ngz                                    */
    int n_pw;
    int n_bands;
    int n_proj;             /* 0: local Hamiltonian only                        */
    int n_ions;             /* ions carrying projectors                         */
} chfsi_dims;

typedef struct chfsi_config {
    int    device;          /* CUDA ordinal                                     */
    int    precision;       /* CHFSI_PREC_*                                     */
    int    bound_mode;      /* CHFSI_BOUND_*                                    */
    int    lanczos_steps;   /* k for CHFSI_BOUND_LANCZOS (default 10)          */
    int    check_norms;     /* 1: 10x norm-growth guard (chebyshev.rs:552-563) */
    int    filter_form;     /* CHFSI_FILTER_*                                  */
    int    reserved[2];
} chfsi_config;

chfsi_status chfsi_default_config(chfsi_config* out);
chfsi_status chfsi_create(const chfsi_dims* dims, const chfsi_config* cfg, chfsi_ctx** out);
void         chfsi_destroy(chfsi_ctx* ctx);
const char*  chfsi_last_error(const chfsi_ctx* ctx);
/* Convenience: create a context and upload every array of a synthetic system. */
chfsi_status chfsi_create_from_system(const chfsi_system* s, const chfsi_config* cfg,
                                      chfsi_ctx** out);

chfsi_status chfsi_set_basis(chfsi_ctx* ctx, const int32_t* miller, const double* kinetic,
                             double gmax);
chfsi_status chfsi_set_projectors(chfsi_ctx* ctx, const chfsi_c128* beta,
                                  const int32_t* proj_offsets, const chfsi_c128* dmat);
/* Ultrasoft overlap S = 1 + sum_I beta q_I beta^H (per-ion q blocks, layout of
 * dmat): the filter then runs on S^-1 H (Woodbury inverse) and Rayleigh-Ritz
 * solves H x = e S x with S_sub = psi^H S psi.  FP64 contexts only.  The GPU
 * ChFSI of the reference ignores S (it has no generalised path). */
chfsi_status chfsi_set_qmat(chfsi_ctx* ctx, const chfsi_c128* qmat);
/* Density (augmentation) grid, at least as fine as the FFT grid of the
 * wavefunctions; call before chfsi_set_vloc_g.  Density, V_eff, mixing and
 * energies then live on it: the smooth density is interpolated up by zero
 * padding in G and V_eff is brought down by truncation
 * (downsample_array_to_wave_grid, src/scf.rs:413-454). */
chfsi_status chfsi_set_density_grid(chfsi_ctx* ctx, const int* ngrid);
/* Jacobi sweeps of the last Rayleigh-Ritz eigensolve (diagnostics). */
chfsi_status chfsi_get_rr_sweeps(chfsi_ctx* ctx, int* sweeps);
chfsi_status chfsi_get_density_grid(chfsi_ctx* ctx, int* ngrid);
/* Ultrasoft augmentation: Q_ij(r) = q_ij g(|r - R_I|), g a unit Gaussian of
 * the given width (bohr), for the ions with projectors (positions n_ions x 3,
 * bohr, the order of chfsi_set_projectors).  chfsi_construct_density then
 * adds sum_ij rho_ij Q_ij and chfsi_scf_run screens D = D0 + int V_eff Q
 * every iteration.  Needs the cell, the projectors and chfsi_set_qmat. */
chfsi_status chfsi_set_augmentation(chfsi_ctx* ctx, const double* positions, double width);
/* Lower bound of the spectrum of S used to scale the filter's upper bound. */
chfsi_status chfsi_get_s_min(chfsi_ctx* ctx, double* out);
chfsi_status chfsi_set_veff(chfsi_ctx* ctx, const double* veff);
chfsi_status chfsi_set_psi(chfsi_ctx* ctx, const chfsi_c128* psi);
chfsi_status chfsi_get_psi(chfsi_ctx* ctx, chfsi_c128* psi);
/* H|psi> for nb bands; psi_dev/hpsi_dev are DEVICE pointers in the
 * context's plane-wave order (the order given to chfsi_set_basis). */
chfsi_status chfsi_apply_h(chfsi_ctx* ctx, const chfsi_c128* psi_dev, chfsi_c128* hpsi_dev,
                           int nb);
/* Chebyshev filter of the context's psi in place; leaves H|psi_filtered> on
 * the device for chfsi_rayleigh_ritz.  eig_prev may be NULL (first SCF step). */
chfsi_status chfsi_chebyshev_filter(chfsi_ctx* ctx, int ndeg, const double* eig_prev,
                                    int n_eig);
/* Rayleigh-Ritz on the filtered psi: psi <- psi V, eigenvalues ascending. */
chfsi_status chfsi_rayleigh_ritz(chfsi_ctx* ctx, double* eig_out);
/* Filter + Rayleigh-Ritz (one ChFSI iteration). */
chfsi_status chfsi_diagonalize(chfsi_ctx* ctx, int ndeg, const double* eig_prev, int n_eig,
                               double* eig_out);
/* Spectral bounds used by the last filter: {lambda_max, eps_cut, center, half_width}. */
chfsi_status chfsi_get_bounds(chfsi_ctx* ctx, double* out4);
/* Frobenius norms |psi_k| per filter degree k = 0..ndeg of the last filter. */
chfsi_status chfsi_get_filter_norms(chfsi_ctx* ctx, double* out, int n);

/* S^-1 H |psi> of the generalised (ultrasoft) problem after chfsi_set_qmat,
 * the operator the filter applies (the reference's ChFSI has no S; the
 * operator pair is tests/phase0_gate2_convergence.rs:279-322 apply_hs with
 * the Woodbury inverse noted at cg_helpers.rs:86-92); H |psi> without q.
 * Device pointers as chfsi_apply_h; overwrites the context's H|psi> buffer. */
chfsi_status chfsi_apply_sinv_h(chfsi_ctx* ctx, const chfsi_c128* psi_dev, chfsi_c128* out_dev,
                                int nb);

/* Local part only, T + V_loc (apply_v_loc_hamiltonian, chebyshev.rs:279-365). */
chfsi_status chfsi_apply_h_local(chfsi_ctx* ctx, const chfsi_c128* psi_dev,
                                 chfsi_c128* hpsi_dev, int nb);

/* Device pointer of the context's psi (n_bands x n_pw, context PW order). */
chfsi_status chfsi_psi_device_ptr(chfsi_ctx* ctx, chfsi_c128** out);
/* The context's CUDA stream (cudaStream_t), for event timing by the caller. */
chfsi_status chfsi_get_stream(chfsi_ctx* ctx, void** out);
/* Kernels launched by this library since load (all contexts). */
long long    chfsi_launch_count(void);

/* C[m][n] = sum_k conj(A[m][k]) B[n][k] on DEVICE pointers (row-major; C is
 * m x n dense), on `stream` (cudaStream_t, 0 = legacy default).  The op::C
 * ZGEMM of BlasHandle::gemm_c64 (src/device/blas.rs:79-102) that forms
 * beta^H psi, psi^H psi and psi^H H psi.  Blocks until done. */
chfsi_status chfsi_zgemm_cn(const chfsi_c128* a_dev, int lda, const chfsi_c128* b_dev, int ldb,
                            int m, int n, int k, chfsi_c128* c_dev, void* stream);
/* Same product with no device allocation, for callers that cannot call
 * cudaMalloc (a host code that gives the whole GPU to its own memory pool, or
 * a latency-critical caller for which cudaMalloc/cudaFree would synchronise
 * the device).  No counterpart in the reference.  Split-K partials use one
 * static device array of CHFSI_NOALLOC_SCRATCH_BYTES per GPU (held until the
 * process exits); m * n must not exceed CHFSI_NOALLOC_SCRATCH_BYTES / 16
 * (262144), otherwise CHFSI_ERR_BAD_INPUT.  The first call on a device sets
 * up the array's device address (make it before any stream capture).  Calls
 * share the array: calls that overlap on the GPU race.  Blocks until done. */
#define CHFSI_NOALLOC_SCRATCH_BYTES (4u * 1024u * 1024u)
chfsi_status chfsi_zgemm_cn_noalloc(const chfsi_c128* a_dev, int lda, const chfsi_c128* b_dev,
                                    int ldb, int m, int n, int k, chfsi_c128* c_dev, void* stream);
/* Same product on the tcgen05 tensor cores in BF16 3-way split precision
 * with FP32 accumulation (the mixed-precision filter's projector GEMM). */
chfsi_status chfsi_zgemm_cn_bf16x3(const chfsi_c128* a_dev, int lda, const chfsi_c128* b_dev,
                                   int ldb, int m, int n, int k, chfsi_c128* c_dev, void* stream);
/* The same with an explicit launch shape of the tcgen05 kernel:
 * 0: stages of K 32 (64-byte swizzle, 3 stages), N tiles up to 256;
 * 1: K 32, N tiles up to 128; 2: K 64 (128-byte swizzle, 2 stages), N up to 160. */
#define CHFSI_TC_SHAPES 3
chfsi_status chfsi_zgemm_cn_bf16x3_shape(const chfsi_c128* a_dev, int lda, const chfsi_c128* b_dev,
                                         int ldb, int m, int n, int k, chfsi_c128* c_dev,
                                         void* stream, int shape);
/* Launch shapes of a mixed-precision context's two projector GEMMs
 * (projection beta^H x, expansion beta F).  The context times every shape on
 * its own sizes at its first mixed-precision filter (outside stream capture)
 * and keeps the fastest; chfsi_set_tc_shapes fixes them instead (-1: tune). */
chfsi_status chfsi_get_tc_shapes(chfsi_ctx* ctx, int* projection, int* expansion);
chfsi_status chfsi_set_tc_shapes(chfsi_ctx* ctx, int projection, int expansion);


/* ------------------------------------------------------------------------ */
/* SCF pieces: V_loc, cell, occupations, density, V_eff, full SCF loop.     */
/* ------------------------------------------------------------------------ */
/* V_loc(G) S(G) on the full grid (natural grid order), transformed to V_loc(r). */
chfsi_status chfsi_set_vloc_g(chfsi_ctx* ctx, const chfsi_c128* vloc_g);
chfsi_status chfsi_get_vloc(chfsi_ctx* ctx, double* out);
chfsi_status chfsi_get_veff(chfsi_ctx* ctx, double* out);
/* lattice rows a1, a2, a3 (bohr), ion-ion energy and atom count (for dE/atom). */
chfsi_status chfsi_set_cell(chfsi_ctx* ctx, const double* lattice, double e_ewald, int n_atoms);
chfsi_status chfsi_set_occupations(chfsi_ctx* ctx, const double* occ);
/* rho(r) = sum_b f_b |psi_b(r)|^2 / Omega of the context's psi (construct_density). */
chfsi_status chfsi_construct_density(chfsi_ctx* ctx, double* rho_out);
/* V_eff = V_loc + V_H[rho] + V_xc^LDA-PZ[rho] (build_v_eff); e2 = {E_H, E_xc} or NULL. */
chfsi_status chfsi_build_veff(chfsi_ctx* ctx, const double* rho, double* e2);
/* Density of the last chfsi_construct_density / chfsi_scf_run step. */
chfsi_status chfsi_get_density(chfsi_ctx* ctx, double* rho);

/* Exchange-correlation functional of chfsi_build_veff and chfsi_scf_run:
 * LDA (Perdew-Zunger 1981, the default) or the GGA PBE (Perdew, Burke,
 * Ernzerhof 1996 with PW92 correlation), the functional of the reference's
 * planned V_eff builder (plans/phase-2/PHASE_PLAN.md:90-95). */
enum { CHFSI_XC_LDA_PZ = 0, CHFSI_XC_PBE = 1 };
chfsi_status chfsi_set_xc(chfsi_ctx* ctx, int functional);

/* Ions of the cell for forces: Cartesian positions (n_atoms x 3, bohr),
 * valence charges and the local-pseudopotential widths of the analytic
 * model v(G) = -4 pi Z/(Omega G^2) exp(-G^2 rc^2/4) that chfsi_set_vloc_g
 * received summed over ions, and k (fractional) of the context's basis.
 * Ions with projectors are the first n_ions of chfsi_set_projectors, in the
 * same order.  Set by chfsi_create_from_system. */
chfsi_status chfsi_set_ions(chfsi_ctx* ctx, int n_atoms, const double* positions,
                            const double* zion, const double* rc_loc, const double* kpt);
/* Hellmann-Feynman forces (Ha/bohr, n_atoms x 3) of the current density and
 * wavefunctions (after chfsi_scf_run): local pseudopotential, non-local
 * projectors and ion-ion Ewald terms; the forces output of the planned
 * scf_run (PROJECT_ROOT_PLAN.md:957-1018).  Norm-conserving and local cells
 * with equal density and wavefunction grids; CHFSI_ERR_NOT_IMPLEMENTED for
 * ultrasoft ones (their augmentation and overlap terms are not built). */
chfsi_status chfsi_forces(chfsi_ctx* ctx, double* forces);

typedef struct chfsi_scf_params {
    int    ndeg;          /* Chebyshev degree                                   */
    int    max_iter;      /* SCF iterations at most                             */
    double tol_per_atom;  /* converged when |E_i - E_{i-1}| / n_atoms < tol (Ha) */
    double alpha;         /* Pulay mixing parameter                             */
    int    max_hist;      /* Pulay history length, 1..8 (1 = linear mixing)     */
    int    first_passes;  /* filter + Rayleigh-Ritz passes in the first step    */
    double kT;            /* Fermi-Dirac smearing (Ha); <= 0: fixed aufbau occupations */
    double fp64_switch_per_atom; /* mixed precision: switch the filter to FP64 after
                                    two mixed steps in a row with |dE|/atom below
                                    max(this, tol); convergence is declared on FP64
                                    steps only; an FP64 step with |dE| ten times above
                                    the switch returns to mixed (at most 3 times)      */
    int    mixer;         /* CHFSI_MIXER_PULAY / _LEARNED / _LEARNED_PULAY            */
    int    cg_steps;      /* band-CG steps per band after each filter (0: none)      */
    double* trace;        /* optional host buffer of 2 * max_iter * N^3 doubles: rho_in
                             and rho_out of every iteration (training trajectories)   */
    int    verbose;       /* 1: one line per iteration on stderr                       */
    int    restart;       /* 1: continue from the context's current input density,
                             wavefunctions and eigenvalues (one pass in the first
                             step, fresh mixing history) instead of a uniform density */
    double tol_eig;       /* > 0: convergence also needs the occupied eigenvalues
                             (f > 0.01) to change by less than this (Ha) from the
                             previous iteration; mixed runs switch to FP64 only after
                             two mixed iterations with |dE| below the switch and
                             eigenvalue changes below the eigenvalue switch, or
                             levelled off below three times it (the best of the
                             last eight mixed iterations not below half the best
                             before them)                                           */
    double fp64_switch_eig; /* eigenvalue switch of mixed runs: max(this, 2 x tol_eig)
                               (on the 216-atom cell the mixed iterations' eigenvalue
                               changes level off at 1-3e-6 Ha: FP32 rounding of the
                               filtered bands, ~1e-7 relative in the density)        */
} chfsi_scf_params;

/* Density mixers of chfsi_scf_run.  PULAY: Pulay/DIIS over (rho_in,
 * rho_out - rho_in) with scalar alpha (mixing.rs:24 as planned in the crate).
 * LEARNED: rho_next(G) = rho_in(G) + a_s R(G) + b_s (rho_in - rho_in_prev)(G)
 * with (a_s, b_s) per |G| shell from the MLP of chfsi_set_mixer.
 * LEARNED_PULAY: Pulay extrapolation with the MLP's a_s as per-shell
 * preconditioner in place of alpha.  Both learned modes fall back to plain
 * Pulay for the rest of the run once the residual norm rises two steps in a
 * row, once the smallest residual of the last ten iterations is not below
 * half the smallest before them (a stall), or once the network's output is
 * not finite; Pulay then starts a fresh history from the current density. */
#define CHFSI_MIXER_PULAY 0
#define CHFSI_MIXER_LEARNED 1
#define CHFSI_MIXER_LEARNED_PULAY 2

typedef struct chfsi_scf_result {
    int     status;       /* CHFSI_OK (converged), CHFSI_NOT_CONVERGED or error */
    int     n_iter;
    int     n_iter_mixed; /* iterations whose filter ran in mixed precision       */
    double  e_total;      /* free energy: sum f eps - int (V_H+V_xc)[in] rho_out
                             + E_H + E_xc + E_ion-ion - kT S                    */
    double  e_band, e_hartree, e_xc, e_dc, e_entropy, mu;
    double  seconds;      /* device time of the whole loop                      */
    double* energies;     /* caller array of max_iter entries, or NULL          */
    double* eigenvalues;  /* caller array of n_bands entries, or NULL           */
    int     n_iter_learned; /* iterations mixed by the learned mixer            */
    int     fell_back;    /* 1 if a learned run fell back to Pulay              */
    double* residuals;    /* caller array of max_iter entries (|rho_out - rho_in|_2
                             on the grid), or NULL                              */
    int     n_fp64_retries; /* mixed-precision passes redone in FP64 after the FP32
                               filter left a non-positive-definite overlap      */
} chfsi_scf_result;

/* Full SCF from a uniform density: build_v_eff -> diagonalize -> density ->
 * energy -> check -> Pulay mix (run_scf, src/scf.rs:358-376).  Returns
 * CHFSI_OK when converged, CHFSI_NOT_CONVERGED after max_iter. */
chfsi_status chfsi_scf_run(chfsi_ctx* ctx, const chfsi_scf_params* p, chfsi_scf_result* r);

/* Band-by-band preconditioned CG refinement of the current wavefunctions
 * (band_cg_minimize, src/eigensolver/band_cg.rs:157-437): each band in turn,
 * S-orthogonalised against the already refined lower bands, at most
 * max_steps steps, stopping when its energy changes by less than tol (Ha).
 * Preconditioner: TPA diagonal, plus the ultrasoft Woodbury term when q is
 * set (uspp_preconditioner.rs).  eig_out / steps_out: n_bands entries or NULL. */
chfsi_status chfsi_band_cg(chfsi_ctx* ctx, int max_steps, double tol, double* eig_out,
                           int* steps_out, int* n_converged);

/* ---- batches of independent systems (k-points, independent cells) -------
 * One mixed-precision diagonalisation pass (FP32 filter with bounds from
 * each member's previous eigenvalues, FP64 Rayleigh-Ritz) of every member is
 * captured once into a CUDA graph, members on their own streams forked from
 * and joined to one origin stream; chfsi_batch_run replays it as a single
 * graph launch.  Members: contexts created with CHFSI_PREC_MIXED on one
 * device, each having run one chfsi_diagonalize before capture.  The
 * reference crate has no batched path (one context, one stream). */
typedef struct chfsi_batch chfsi_batch;
chfsi_status chfsi_batch_create(chfsi_ctx* const* ctxs, int n, chfsi_batch** out);
void         chfsi_batch_destroy(chfsi_batch* b);
chfsi_status chfsi_batch_capture(chfsi_batch* b, int ndeg);
/* eig_out: every member's n_bands eigenvalues in member order (or NULL);
 * status_out: per member status (or NULL); returns the first failure */
chfsi_status chfsi_batch_run(chfsi_batch* b, double* eig_out, int* status_out);
chfsi_status chfsi_batch_graph_nodes(chfsi_batch* b, size_t* nodes);
/* Autotuner: times the local H|psi> of this context at 2 x 3 x 3 launch
 * configurations (xy-plane kernel with compile-time radices where the grid's
 * plan has one, or the generic kernel; 256 / 128 / 512 threads per block;
 * z-stick kernels 16 / 32 / 64 columns per block) on its current psi and
 * keeps the fastest; choice = generic * 9 + planes * 3 + columns, times_ms
 * (18 floats) may be NULL.  chfsi_set_launch_config applies a choice (e.g.
 * one tuned per size class). */
chfsi_status chfsi_autotune(chfsi_ctx* ctx, int* choice, float* times_ms);
chfsi_status chfsi_set_launch_config(chfsi_ctx* ctx, int choice);

/* ---- learned density mixer (no counterpart in the reference crate) ------
 * MLP 512 -> 256 -> 256 -> 128 with GELU, BF16 weights and FP32 accumulation.
 * Input: the last 4 density residuals R_0..R_3 binned into 64 |G| shells:
 * per shell (|R_0|^2, Re<R_0, D>) and, for t = 1..3, (Re<R_0, R_t>, |R_t|^2),
 * each over the total |R_0|^2 (x 64) and compressed by sign(x) log(1 + |x|);
 * D = rho_in - rho_in_prev.  Output: per shell (a_s, b_s).
 * Training targets per shell (a*, b*, M00, M01, M11): the least-squares
 * (a, b) of rho* - rho_in ~ a R_0 + b D and its normal matrix M over
 * |rho* - rho_in|^2; the loss sum_s (y_s - y*_s)^T M_s (y_s - y*_s) is the
 * relative density error left after the update. */
#define CHFSI_MIXER_SHELLS 64
#define CHFSI_MIXER_FEATURES 512
#define CHFSI_MIXER_OUTPUTS 128
#define CHFSI_MIXER_TARGETS 320   /* 64 shells x 5 */
typedef struct chfsi_mixer chfsi_mixer;
chfsi_status chfsi_mixer_create(int device, uint64_t seed, chfsi_mixer** out);
void         chfsi_mixer_destroy(chfsi_mixer* m);
size_t       chfsi_mixer_num_params(void);
/* fp32 master parameters: W1 (256x512), b1, W2 (256x256), b2, W3 (128x256), b3 */
chfsi_status chfsi_mixer_get_params(chfsi_mixer* m, float* out);
chfsi_status chfsi_mixer_set_params(chfsi_mixer* m, const float* in);
/* host x (batch x 512) -> host y (batch x 128) */
chfsi_status chfsi_mixer_forward(chfsi_mixer* m, const float* x, int batch, float* y);
/* loss and gradient (num_params floats) of one batch; host arrays */
chfsi_status chfsi_mixer_gradient(chfsi_mixer* m, const float* x, const float* t, int batch,
                                  float* grad, float* loss);
/* Adam (lr, beta 0.9/0.999) over n samples resident on the device, shuffled
 * minibatches from seed; loss_per_epoch (epochs floats) may be NULL. */
chfsi_status chfsi_mixer_train(chfsi_mixer* m, const float* x, const float* t, int n, int epochs,
                               int batch, float lr, uint64_t seed, float* loss_per_epoch);
/* use m in chfsi_scf_run when params.mixer is LEARNED or LEARNED_PULAY (NULL to detach) */
chfsi_status chfsi_set_mixer(chfsi_ctx* ctx, chfsi_mixer* m);
/* features (n_iter x 512) and targets (n_iter x 320) of one SCF trajectory on
 * this context's grid: rho_in / rho_out are n_iter x N^3, rho_star N^3 */
chfsi_status chfsi_mixer_samples(chfsi_ctx* ctx, const double* rho_in, const double* rho_out,
                                 int n_iter, const double* rho_star, float* x, float* t);

/* O[m][n] = alpha sum_k W[k][m] X[k][n] + beta O[m][n] (device pointers,
 * row-major): the rotation psi <- psi V of rayleigh_ritz.rs:209-227 and the
 * projector back-substitution of chebyshev.rs:480-497.  Blocks until done. */
chfsi_status chfsi_zgemm_tn(const chfsi_c128* w_dev, int ldw, const chfsi_c128* x_dev, int ldx,
                            chfsi_c128* o_dev, int ldo, int m, int n, int k, double alpha,
                            double beta, void* stream);
/* Subspace eigenproblem H x = e S x (n x n, device, row-major), the ZHEGVD
 * itype-1 contract of src/device/solver.rs:47-95 solved by Cholesky
 * reduction and the library's Jacobi eigensolver: eigenvalues ascending to
 * w_host, eigenvectors as the columns of v_dev (V[j][i]).  Blocks until done. */
chfsi_status chfsi_hegv_dev(const chfsi_c128* h_dev, const chfsi_c128* s_dev, int n,
                            double* w_host, chfsi_c128* v_dev, void* stream);
/* Device pointer of the context's H|psi> (after chfsi_chebyshev_filter: H of
 * the filtered block, the second output of chebyshev.rs:626-643). */
chfsi_status chfsi_hpsi_device_ptr(chfsi_ctx* ctx, chfsi_c128** out);

/* ---- test hooks (host-side fault injection; no counterpart in the crate) --
 * CHFSI_INJECT_TC_NO_LOADS: the next `arg` tensor-core GEMM launches run with
 *   a producer that issues no loads; the consumer's wait runs out after 20 ms
 *   and the call returns CHFSI_ERR_TIMEOUT (no GPU fault, nothing in flight).
 * CHFSI_INJECT_ALLOC_FAIL: the arg-th device allocation of a context from now
 *   (0 = the next) fails as out of memory.
 * CHFSI_INJECT_NONE clears both. */
enum { CHFSI_INJECT_NONE = 0, CHFSI_INJECT_TC_NO_LOADS = 1, CHFSI_INJECT_ALLOC_FAIL = 2 };
chfsi_status chfsi_test_inject(int what, long long arg);

#ifdef __cplusplus
}
#endif
#endif /* CHFSI_H */
