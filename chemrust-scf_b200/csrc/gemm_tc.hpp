// Host interface of the tcgen05 BF16 3-way split complex GEMM.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>

namespace chfsi {

// Three bf16 planes (x = p0 + p1 + p2) of a real-ified complex operand,
// row-major rows x kp (kp = 2K padded to 64).
struct TcPlanes {
    void* p[3] = {nullptr, nullptr, nullptr};
    int rows = 0;
    int kp = 0;
    int rows_alloc = 0;  // allocated rows (>= the TMA box height), zero beyond `rows`
};

enum { kTcOutPartial = 0, kTcOutComplexF32 = 1, kTcOutComplexF64 = 2 };

int tc_kpad(int K);
// rows to allocate for a plane set: at least the TMA box height
int tc_rows_alloc(int rows, bool a_operand, int n_for_b);
// scratch floats for kTcOutPartial of an M x N x K complex product
size_t tc_partial_floats(int M, int N, int K);

// Source element (r, k) of a packed operand: x[r][k], conj(x[k][r]) or x[k][r].
enum { kSrcPlain = 0, kSrcConjT = 1, kSrcT = 2 };
// Split rows of a complex matrix into bf16 planes.  doubled: conj-first
// operand layout (2 rows per complex row).
template <typename CIn>
void tc_pack(const CIn* x, long long ldx, int rows, int K, bool doubled, int src,
             TcPlanes& planes, cudaStream_t st);

// C[m][n] = sum_k conj(A[m][k]) B[n][k]; a: doubled planes (2M rows),
// b: plain planes (N rows).  kTcOutPartial writes double2 C (M x N dense)
// through `part` scratch; the complex modes write float2 / double2 rows of
// leading dimension ldo directly.  err: device word set on a wait timeout.
// Test hook: the next `launches` tcgen05 GEMM launches run with a producer
// that issues no loads and a 20 ms wait limit (their waits run out, the
// error word is set, nothing is left in flight).
void tc_inject_no_loads(int launches);

// Launch shapes of the autotuner (stage K width, largest N tile):
// 0: K 32, N <= 256; 1: K 32, N <= 128; 2: K 64, N <= 160.
constexpr int kTcVariantCount = 3;
cudaError_t tc_gemm(const TcPlanes& a, const TcPlanes& b, int M, int N, int K, int out_mode,
                    void* out, long long ldo, float* part, int* err, cudaStream_t st,
                    int variant = 0);

}  // namespace chfsi
