// Host launchers of the small dense kernels (Rayleigh-Ritz, bounds, Lanczos, Pulay).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace chfsi {

constexpr int kPulayMax = 8;

void symmetrize(const double2* in, double2* out, int n, cudaStream_t st);
void cholesky(double2* A, int n, int* info, cudaStream_t st);
void tri_inv(const double2* L, double2* X, int n, cudaStream_t st);
void small_gemm(int opa, int opb, const double2* A, const double2* B, double2* C, int n,
                cudaStream_t st);
size_t jacobi_scratch_doubles(int n, int max_sweeps);
cudaError_t jacobi(double2* A, double2* V, int n, int max_sweeps, double tol2, double* scratch,
                   int* sweeps_out, cudaStream_t st);
void sort_eig(const double2* A, const double2* V, int n, double* w, double2* U, cudaStream_t st);
void minmax(const double* v, size_t n, double* out, cudaStream_t st);
void sumsq(const double2* x, size_t n, double* acc, cudaStream_t st);
void bounds(double kin_max, const double* minmax_dev, const double* eig_dev, int n_eig,
            const double* lanczos, int k, double lm_scale, double* coef, cudaStream_t st);
void norm_guard(const double* nsq, int ndeg, int* status, cudaStream_t st);
void scale_by_rsqrt(double2* v, size_t n, const double* nsq, cudaStream_t st);
void lanczos_a(double2* f, const double2* v, const double2* v0, const double* beta_sq, size_t n,
               double* alpha_acc, cudaStream_t st);
void lanczos_b(double2* f, const double2* v, const double* alpha, size_t n, double* fn_acc,
               cudaStream_t st);
void lanczos_c(const double2* f, double2* v, double2* v0, size_t n, const double* fn,
               cudaStream_t st);
void lanczos_store_beta(const double* fn, double* beta, cudaStream_t st);
void pulay_push(const double* rin, const double* rout, double* hr, double* hres, size_t n,
                cudaStream_t st);
void dots(const double* x, const double* const* ys, int m, size_t n, double* out, cudaStream_t st);
void pulay_combine(const double* const* hr, const double* const* hres, int m, const double* c,
                   double alpha, size_t n, double* out, cudaStream_t st);

}  // namespace chfsi
