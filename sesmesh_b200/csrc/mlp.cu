// Warm-start MLP of fast mode: parameters, tcgen05 forward and the training
// step (forward, backward, Adam) as hand-written kernels, behind
// smb_mlp_* in include/sesmesh_b200.h.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/sesmesh_b200.h"
#include "device/mlp.cuh"
#include "runtime.hpp"

using namespace smb;

namespace {

void set_err(char* err, size_t len, const char* fmt, ...) {
    if (!err || !len) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_err(err, errlen, "%s failed: %s", #call, cudaGetErrorString(e_));         \
            return SMB_ERR_CUDA;                                                          \
        }                                                                                 \
    } while (0)

// bf16 weight tiles in core-matrix layout from the f32 parameters.
__global__ void k_mlp_pack(const float* p, __nv_bfloat16* w1t, __nv_bfloat16* w2t) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_H * MLP_IN) {
        int o = i / MLP_IN, k = i % MLP_IN;
        w1t[umma::tile_offset(o, k, MLP_IN) / 2] = __float2bfloat16_rn(p[MLP_W1 + i]);
    }
    if (i < MLP_H * MLP_H) {
        int o = i / MLP_H, k = i % MLP_H;
        w2t[umma::tile_offset(o, k, MLP_H) / 2] = __float2bfloat16_rn(p[MLP_W2 + i]);
    }
}

__global__ void __launch_bounds__(128) k_mlp_forward(const float* x, uint32_t n, MlpDev P, float* t_out,
                                                     unsigned long long* timeouts) {
    extern __shared__ __align__(128) unsigned char smem[];
    MlpSmem& S = *reinterpret_cast<MlpSmem*>(smem);
    mlp_setup(S, P);
    uint32_t phase = 0;
    const uint32_t row = blockIdx.x * MLP_ROWS + threadIdx.x;
    float f[MLP_IN];
    for (int k = 0; k < MLP_IN; k++) f[k] = row < n ? x[size_t(row) * MLP_IN + k] : 0.0f;
    mlp_put_row(S, f);
    float t;
    bool ok = mlp_forward(S, phase, &t, nullptr, nullptr, nullptr);
    if (!ok && threadIdx.x == 0) atomicAdd(timeouts, 1ull);
    if (row < n) t_out[row] = t;
    mlp_teardown(S);
}

}  // namespace

struct smb_mlp {
    smb_device* dev = nullptr;
    DBuf p, w1t, w2t, x, y, t, counters;
};

namespace smb {
MlpDev mlp_dev(const smb_mlp* m) {
    return MlpDev{m->p.as<float>(), m->w1t.as<__nv_bfloat16>(), m->w2t.as<__nv_bfloat16>()};
}
size_t mlp_smem_bytes() { return sizeof(MlpSmem) + 128; }
}  // namespace smb

extern "C" {

int smb_mlp_new(smb_device* dev, const float* params, smb_mlp** out, char* err, size_t errlen) {
    if (!dev || !params || !out) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *out = nullptr;
    CK(cudaSetDevice(dev->index));
    auto* m = new smb_mlp();
    m->dev = dev;
    int rc;
    if ((rc = m->p.reserve(MLP_NPARAM * 4, err, errlen)) || (rc = m->w1t.reserve(MLP_H * MLP_IN * 2, err, errlen)) ||
        (rc = m->w2t.reserve(MLP_H * MLP_H * 2, err, errlen)) || (rc = m->counters.reserve(64, err, errlen))) {
        smb_mlp_free(m);
        return rc;
    }
    *out = m;
    return smb_mlp_set_params(m, params, err, errlen);
}

void smb_mlp_free(smb_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->dev->index);
    for (DBuf* b : {&m->p, &m->w1t, &m->w2t, &m->x, &m->y, &m->t, &m->counters}) b->release();
    delete m;
}

int smb_mlp_set_params(smb_mlp* m, const float* params, char* err, size_t errlen) {
    if (!m || !params) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    CK(cudaSetDevice(m->dev->index));
    cudaStream_t s = m->dev->stream;
    CK(cudaMemcpyAsync(m->p.p, params, MLP_NPARAM * 4, cudaMemcpyHostToDevice, s));
    k_mlp_pack<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(m->p.as<float>(), m->w1t.as<__nv_bfloat16>(),
                                                           m->w2t.as<__nv_bfloat16>());
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return SMB_OK;
}

int smb_mlp_get_params(const smb_mlp* m, float* params) {
    if (!m || !params) return SMB_ERR_ARG;
    cudaSetDevice(m->dev->index);
    return cudaMemcpy(params, m->p.p, MLP_NPARAM * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? SMB_OK : SMB_ERR_CUDA;
}

int smb_mlp_forward(smb_mlp* m, const float* x, size_t n, float* t, char* err, size_t errlen) {
    if (!m || (n && (!x || !t))) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    if (n == 0) return SMB_OK;
    CK(cudaSetDevice(m->dev->index));
    cudaStream_t s = m->dev->stream;
    int rc;
    if ((rc = m->x.reserve(n * MLP_IN * 4, err, errlen)) || (rc = m->t.reserve(n * 4, err, errlen))) return rc;
    CK(cudaMemcpyAsync(m->x.p, x, n * MLP_IN * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(m->counters.p, 0, 64, s));
    size_t smem = mlp_smem_bytes();
    CK(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_mlp_forward<<<uint32_t((n + MLP_ROWS - 1) / MLP_ROWS), MLP_ROWS, smem, s>>>(
        m->x.as<float>(), uint32_t(n), mlp_dev(m), m->t.as<float>(), m->counters.as<unsigned long long>());
    CK(cudaGetLastError());
    unsigned long long to = 0;
    CK(cudaMemcpyAsync(t, m->t.p, n * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&to, m->counters.p, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (to) return set_err(err, errlen, "a bounded tensor-core wait gave up"), SMB_ERR_TIMEOUT;
    return SMB_OK;
}

}  // extern "C"
