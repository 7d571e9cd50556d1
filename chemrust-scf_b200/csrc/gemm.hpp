// Host launchers of the complex FP64 GEMMs.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace chfsi {

// out[m][n] = sum_k conj(A[m][k]) B[n][k]; part must hold
// splitk_partial_elems(M, N, K) elements of scratch.
void gemm_cn(const double2* A, int lda, const double2* B, int ldb, int M, int N, int K,
             double2* part, double2* out, cudaStream_t st);
int splitk_count(int M, int N, int K);
int splitk_count_tiles(int tiles, int K);
// Hermitian N x N result of conj(A) B^T from its upper tiles (B = A, or
// B = H A with H Hermitian); part: splitk_partial_elems(N, N, K) elements
void gemm_cn_herm(const double2* A, int lda, const double2* B, int ldb, int N, int K,
                  double2* part, double2* out, cudaStream_t st);
// same product with at most max_splits K-splits (partials: splits * M * N elements)
void gemm_cn_capped(const double2* A, int lda, const double2* B, int ldb, int M, int N, int K,
                    int max_splits, double2* part, double2* out, cudaStream_t st);
size_t splitk_partial_elems(int M, int N, int K);
size_t splitk_partial_elems_herm(int N, int K);

// O[m][n] = alpha sum_k W[k][m] X[k][n] + beta O[m][n]
void gemm_tn(const double2* W, int ldw, const double2* X, int ldx, double2* O, int ldo, int M,
             int N, int K, double alpha, double beta, cudaStream_t st);

}  // namespace chfsi
