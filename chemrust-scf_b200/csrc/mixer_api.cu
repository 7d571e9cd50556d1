// C ABI of the learned density mixer object (include/chfsi.h): creation,
// parameters, batched inference, gradients and on-device Adam training.
// The mixer has no counterpart in the reference crate (src/mixing.rs:24 is a
// todo!()); its use inside the SCF loop lives in context.cu.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "chfsi.h"
#include "mixer.hpp"

namespace chfsi {
chfsi_status cuda_fail(cudaError_t e, const char* expr, const char* file, int line);
void set_last_error(const char* msg);
}  // namespace chfsi

using namespace chfsi;

#define MK(expr)                                                              \
    do {                                                                      \
        cudaError_t e_ = (expr);                                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr, __FILE__, __LINE__); \
    } while (0)

namespace {

uint64_t mix64(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

chfsi_status ensure_batch(chfsi_mixer* m, int batch) {
    if (batch <= m->mlp.cap) return CHFSI_OK;
    MK(mlp_alloc(m->mlp, std::max(batch, 2 * m->mlp.cap)));
    return CHFSI_OK;
}

}  // namespace

extern "C" {

size_t chfsi_mixer_num_params(void) { return kMixParams; }

chfsi_status chfsi_mixer_create(int device, uint64_t seed, chfsi_mixer** out) {
    if (!out) return CHFSI_ERR_BAD_INPUT;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_last_error("no CUDA device");
        return CHFSI_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return CHFSI_ERR_BAD_INPUT;
    MK(cudaSetDevice(device));
    chfsi_mixer* m = new chfsi_mixer();
    m->mlp.device = device;
    auto bail = [&](chfsi_status s) { chfsi_mixer_destroy(m); return s; };
    if (cudaStreamCreateWithFlags(&m->mlp.st, cudaStreamNonBlocking) != cudaSuccess)
        return bail(CHFSI_ERR_CUDA);
    if (mlp_alloc(m->mlp, 256) != cudaSuccess) return bail(CHFSI_ERR_OUT_OF_MEMORY);
    std::vector<float> w(kMixParams);
    mlp_init_host(w.data(), seed);
    chfsi_status s = chfsi_mixer_set_params(m, w.data());
    if (s) return bail(s);
    *out = m;
    return CHFSI_OK;
}

void chfsi_mixer_destroy(chfsi_mixer* m) {
    if (!m) return;
    cudaSetDevice(m->mlp.device);
    cudaStream_t st = m->mlp.st;
    if (st) cudaStreamSynchronize(st);
    cudaFree(m->loss_hist);
    mlp_free(m->mlp);
    if (st) cudaStreamDestroy(st);
    delete m;
}

chfsi_status chfsi_mixer_get_params(chfsi_mixer* m, float* out) {
    if (!m || !out) return CHFSI_ERR_BAD_INPUT;
    MK(cudaSetDevice(m->mlp.device));
    MK(cudaMemcpyAsync(out, m->mlp.w, kMixParams * sizeof(float), cudaMemcpyDeviceToHost, m->mlp.st));
    MK(cudaStreamSynchronize(m->mlp.st));
    return CHFSI_OK;
}

chfsi_status chfsi_mixer_set_params(chfsi_mixer* m, const float* in) {
    if (!m || !in) return CHFSI_ERR_BAD_INPUT;
    MK(cudaSetDevice(m->mlp.device));
    MK(cudaMemcpyAsync(m->mlp.w, in, kMixParams * sizeof(float), cudaMemcpyHostToDevice, m->mlp.st));
    MK(cudaMemsetAsync(m->mlp.m, 0, kMixParams * sizeof(float), m->mlp.st));
    MK(cudaMemsetAsync(m->mlp.v, 0, kMixParams * sizeof(float), m->mlp.st));
    m->mlp.step = 0;
    mlp_sync_bf16(m->mlp, m->mlp.st);
    MK(cudaGetLastError());
    MK(cudaStreamSynchronize(m->mlp.st));
    return CHFSI_OK;
}

chfsi_status chfsi_mixer_forward(chfsi_mixer* m, const float* x, int batch, float* y) {
    if (!m || !x || !y || batch <= 0) return CHFSI_ERR_BAD_INPUT;
    MK(cudaSetDevice(m->mlp.device));
    chfsi_status s = ensure_batch(m, batch);
    if (s) return s;
    Mlp& M = m->mlp;
    MK(cudaMemcpyAsync(M.x, x, (size_t)batch * kMixIn * sizeof(float), cudaMemcpyHostToDevice, M.st));
    mlp_forward(M, M.x, batch, M.y, M.st);
    MK(cudaGetLastError());
    MK(cudaMemcpyAsync(y, M.y, (size_t)batch * kMixOut * sizeof(float), cudaMemcpyDeviceToHost, M.st));
    MK(cudaStreamSynchronize(M.st));
    return CHFSI_OK;
}

chfsi_status chfsi_mixer_gradient(chfsi_mixer* m, const float* x, const float* t, int batch,
                                  float* grad, float* loss) {
    if (!m || !x || !t || !grad || batch <= 0) return CHFSI_ERR_BAD_INPUT;
    MK(cudaSetDevice(m->mlp.device));
    chfsi_status s = ensure_batch(m, batch);
    if (s) return s;
    Mlp& M = m->mlp;
    MK(cudaMemcpyAsync(M.x, x, (size_t)batch * kMixIn * sizeof(float), cudaMemcpyHostToDevice, M.st));
    MK(cudaMemcpyAsync(M.t, t, (size_t)batch * kMixShells * kMixTargets * sizeof(float),
                       cudaMemcpyHostToDevice, M.st));
    mlp_backward(M, batch, M.st);
    MK(cudaGetLastError());
    MK(cudaMemcpyAsync(grad, M.g, kMixParams * sizeof(float), cudaMemcpyDeviceToHost, M.st));
    float l = 0.f;
    MK(cudaMemcpyAsync(&l, M.loss, sizeof(float), cudaMemcpyDeviceToHost, M.st));
    MK(cudaStreamSynchronize(M.st));
    if (loss) *loss = l;
    return CHFSI_OK;
}

chfsi_status chfsi_mixer_train(chfsi_mixer* m, const float* x, const float* t, int n, int epochs,
                               int batch, float lr, uint64_t seed, float* loss_per_epoch) {
    if (!m || !x || !t || n <= 0 || epochs < 0 || batch <= 0 || !(lr > 0.f))
        return CHFSI_ERR_BAD_INPUT;
    MK(cudaSetDevice(m->mlp.device));
    batch = std::min(batch, n);
    chfsi_status s = ensure_batch(m, batch);
    if (s) return s;
    Mlp& M = m->mlp;
    const size_t nt = (size_t)kMixShells * kMixTargets;
    if ((size_t)n > M.data_cap) {
        cudaFree(M.data_x);
        cudaFree(M.data_t);
        M.data_x = M.data_t = nullptr;
        M.data_cap = 0;
        MK(cudaMalloc((void**)&M.data_x, (size_t)n * kMixIn * sizeof(float)));
        MK(cudaMalloc((void**)&M.data_t, (size_t)n * nt * sizeof(float)));
        M.data_cap = n;
    }
    MK(cudaMemcpyAsync(M.data_x, x, (size_t)n * kMixIn * sizeof(float), cudaMemcpyHostToDevice, M.st));
    MK(cudaMemcpyAsync(M.data_t, t, (size_t)n * nt * sizeof(float), cudaMemcpyHostToDevice, M.st));
    const int nbatch = n / batch;  // drop the ragged tail of each shuffled epoch
    if ((size_t)nbatch * batch > M.idx_cap) {
        cudaFree(M.idx);
        M.idx = nullptr;
        MK(cudaMalloc((void**)&M.idx, (size_t)nbatch * batch * sizeof(int)));
        M.idx_cap = (size_t)nbatch * batch;
    }
    if (nbatch > m->loss_cap) {
        cudaFree(m->loss_hist);
        m->loss_hist = nullptr;
        MK(cudaMalloc((void**)&m->loss_hist, nbatch * sizeof(float)));
        m->loss_cap = nbatch;
    }
    std::vector<int> perm(n);
    std::vector<float> lh(nbatch);
    uint64_t rs = seed ^ 0x5DEECE66Dull;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int i = 0; i < n; ++i) perm[i] = i;
        for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[mix64(rs) % (uint64_t)(i + 1)]);
        // the host vector is pageable: the copy returns once it is staged
        MK(cudaMemcpyAsync(M.idx, perm.data(), (size_t)nbatch * batch * sizeof(int),
                           cudaMemcpyHostToDevice, M.st));
        for (int b = 0; b < nbatch; ++b) {
            mlp_gather_batch(M, M.idx + (size_t)b * batch, batch, M.st);
            mlp_backward(M, batch, M.st);
            mlp_adam(M, lr, M.st);
            MK(cudaMemcpyAsync(m->loss_hist + b, M.loss, sizeof(float), cudaMemcpyDeviceToDevice, M.st));
        }
        MK(cudaGetLastError());
        MK(cudaMemcpyAsync(lh.data(), m->loss_hist, nbatch * sizeof(float), cudaMemcpyDeviceToHost, M.st));
        MK(cudaStreamSynchronize(M.st));
        if (loss_per_epoch) {
            double a = 0.0;
            for (float v : lh) a += v;
            loss_per_epoch[ep] = (float)(a / std::max(1, nbatch));
        }
    }
    return CHFSI_OK;
}

}  // extern "C"
