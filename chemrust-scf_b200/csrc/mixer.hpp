// Learned density mixer: a 512 -> 256 -> 256 -> 128 MLP (GELU) over
// |G|-shell-binned residual history, with BF16 weights and FP32 accumulation.
// Forward, backward and Adam are hand-written kernels (mixer.cu); the shell
// reductions that build its inputs and training targets run on the density
// grid in G space (digit-reversed layout, as produced by the grid FFT).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "kernels.hpp"

namespace chfsi {

constexpr int kMixShells = 64;
constexpr int kMixHist = 4;                         // residuals R_0 .. R_3 in the input
constexpr int kMixIn = kMixShells * kMixHist * 2;  // 512 (two per shell and age)
constexpr int kMixHidden = 256;
constexpr int kMixOut = kMixShells * 2;             // per shell (a_s, b_s)
constexpr int kMixTargets = 5;                      // per shell: a*, b*, M00, M01, M11
constexpr int kShellAcc = 12;                       // per-shell accumulators (see k_shell_acc)
// |G| of shell boundaries: s = floor(64 sqrt(|G| / kShellGmax)), clamped.
constexpr double kShellGmax = 12.0;  // bohr^-1

// Parameter layout (fp32 master copy, bf16 working copy, same offsets).
constexpr size_t kOffW1 = 0;
constexpr size_t kOffB1 = kOffW1 + (size_t)kMixHidden * kMixIn;
constexpr size_t kOffW2 = kOffB1 + kMixHidden;
constexpr size_t kOffB2 = kOffW2 + (size_t)kMixHidden * kMixHidden;
constexpr size_t kOffW3 = kOffB2 + kMixHidden;
constexpr size_t kOffB3 = kOffW3 + (size_t)kMixOut * kMixHidden;
constexpr size_t kMixParams = kOffB3 + kMixOut;

struct Mlp {
    int device = 0;
    cudaStream_t st = nullptr;
    float* w = nullptr;          // master weights
    __nv_bfloat16* wb = nullptr; // BF16 weights used by forward and backward
    float* g = nullptr;          // gradient
    float* m = nullptr;          // Adam first moment
    float* v = nullptr;          // Adam second moment
    long step = 0;
    int cap = 0;                 // batch capacity of the activation buffers
    float *x = nullptr, *t = nullptr;          // batch inputs / targets
    float *z1 = nullptr, *h1 = nullptr, *z2 = nullptr, *h2 = nullptr, *y = nullptr;
    float *dy = nullptr, *d2 = nullptr, *d1 = nullptr;  // B x 128, B x 256, B x 256
    float* loss = nullptr;       // device scalar
    float* data_x = nullptr;     // resident training set
    float* data_t = nullptr;
    size_t data_cap = 0;
    int* idx = nullptr;          // minibatch row indices
    size_t idx_cap = 0;
};

cudaError_t mlp_alloc(Mlp& M, int batch_cap);
void mlp_free(Mlp& M);
void mlp_init_host(float* w, uint64_t seed);
// bf16 copy of the master weights
void mlp_sync_bf16(Mlp& M, cudaStream_t st);
// y = MLP(x) for B rows (device pointers; x is B x 512, y B x 128)
void mlp_forward(Mlp& M, const float* x, int B, float* y, cudaStream_t st);
// loss and gradient of the batch in M.x / M.t (B rows) into M.g
void mlp_backward(Mlp& M, int B, cudaStream_t st);
void mlp_adam(Mlp& M, float lr, cudaStream_t st);
void mlp_gather_batch(Mlp& M, const int* idx, int B, cudaStream_t st);

// Shell index of every grid point (G space, digit-reversed layout); 255 for G = 0.
void launch_shell_index(const GridRecip& gr, unsigned char* shell, cudaStream_t st);
// Per-shell sums over G != 0 (acc has kMixShells x kShellAcc doubles, zeroed by caller):
//  0 |R0|^2   1..3 Re conj(R0) R_t   4..6 |R_t|^2 (t = 1..3)   7 |D|^2   8 Re conj(R0) D
//  9 Re conj(R0) E   10 Re conj(D) E   11 |E|^2      (E = rho* - rho_in; optional)
// Shells hold G and -G together, so for real fields every such sum is real.
void launch_shell_acc(const double2* R0, const double2* R1, const double2* R2, const double2* R3,
                      const double2* D, const double2* E, const unsigned char* shell, size_t ng,
                      double* acc, cudaStream_t st);
// features (512 floats) and, if targets != nullptr, targets (64 x 5 floats) from acc
void launch_shell_features(const double* acc, float* features, float* targets, cudaStream_t st);
// out <- out + a_s R0 + b_s D over G != 0 (all in the units of the unnormalised
// forward FFT), with (a_s, b_s) = y[2s], y[2s+1]; D may be null
void launch_shell_update(double2* out, const double2* R0, const double2* D, const float* y,
                         const unsigned char* shell, size_t ng, cudaStream_t st);

// out = a - b (b may be null) as a complex grid with zero imaginary part
void launch_diff_complex(const double* a, const double* b, double2* out, size_t n, cudaStream_t st);
// r = scale * Re(c)
void launch_take_real_scaled(const double2* c, double* r, size_t n, double scale, cudaStream_t st);

}  // namespace chfsi

// Handle behind the C ABI's chfsi_mixer.
struct chfsi_mixer {
    chfsi::Mlp mlp;
    float* loss_hist = nullptr;  // per-minibatch losses of one epoch (device)
    int loss_cap = 0;
};
