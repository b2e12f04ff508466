// Warm-start MLP of fast mode: parameters, tcgen05 forward and the training
// step (forward, backward, Adam) as hand-written kernels, behind
// smb_mlp_* in include/sesmesh_b200.h.
#include <algorithm>
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

// ---------------------------------------------------------------------------
// Training step: forward and backward of one 128-row tile per CTA, every
// matrix product on the tensor cores (tcgen05, bf16 operands, f32 TMEM
// accumulators), bias/GELU/loss terms in f32.  Each CTA writes its partial
// gradient; k_mlp_reduce_adam sums the partials in a fixed order and applies
// Adam, so a step is deterministic.
//
// Shared tiles (bf16, core-matrix layout): X 128x32, XT 32x128, A1 128x64,
// A1T 64x128, DZ2 128x64, DZ2T 128x128 (rows 64.. zero), DZ1T 128x128 (rows
// 64.. zero), W1 64x32, W2 64x64, W2T 64x64.  TMEM (256 columns): layer-1
// accumulator [0,64) (later dW1 in [0,32)), layer 2 [64,128), dA1 [128,192),
// dW2 [192,256).
struct TrainSmem {
    __nv_bfloat16 x[128 * 32], xt[32 * 128], a1[128 * 64], a1t[64 * 128], dz2[128 * 64], dz2t[128 * 128],
        dz1t[128 * 128], w1[64 * 32], w2[64 * 64], w2t[64 * 64];
    float b1[64], b2[64], w3[64], red[4][64];
    float b3;
    uint32_t tmem;
    alignas(8) uint64_t bar;
};

__device__ __forceinline__ float warp_sum(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-order block sum of one value per thread for each of the 64 columns
// (warp shuffles, then the 4 warp sums in order); result in red[0][col].
__device__ __forceinline__ void block_col_sum(TrainSmem& S, int col, float v) {
    float w = warp_sum(v);
    if ((threadIdx.x & 31) == 0) S.red[threadIdx.x >> 5][col] = w;
}

__global__ void __launch_bounds__(128) k_mlp_train(const float* x, const float* target, uint32_t n, uint32_t first,
                                                   float inv_batch, const float* p, const __nv_bfloat16* w1t,
                                                   const __nv_bfloat16* w2t, const __nv_bfloat16* w2tt, float* partial,
                                                   float* loss_partial, unsigned long long* timeouts) {
    extern __shared__ __align__(128) unsigned char smem[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem);
    const int r = threadIdx.x, warp = r >> 5;
    const uint32_t row = first + blockIdx.x * 128 + r;
    const bool valid = row < n;
    // Weights, zero padding of the transposed tiles, TMEM.
    for (int i = r; i < 64 * 32 / 8; i += 128) reinterpret_cast<uint4*>(S.w1)[i] = reinterpret_cast<const uint4*>(w1t)[i];
    for (int i = r; i < 64 * 64 / 8; i += 128) {
        reinterpret_cast<uint4*>(S.w2)[i] = reinterpret_cast<const uint4*>(w2t)[i];
        reinterpret_cast<uint4*>(S.w2t)[i] = reinterpret_cast<const uint4*>(w2tt)[i];
    }
    for (int i = r; i < 128 * 128 / 8; i += 128) {
        reinterpret_cast<uint4*>(S.dz2t)[i] = make_uint4(0, 0, 0, 0);
        reinterpret_cast<uint4*>(S.dz1t)[i] = make_uint4(0, 0, 0, 0);
    }
    if (r < 64) S.b1[r] = p[MLP_B1 + r], S.b2[r] = p[MLP_B2 + r], S.w3[r] = p[MLP_W3 + r];
    if (r == 0) {
        S.b3 = p[MLP_B3];
        umma::bar_init(&S.bar, 1);
    }
    if (r < 32) umma::tmem_alloc(&S.tmem, 256);
    // Inputs (row r) into X and XT.
    float xr[32];
    for (int k = 0; k < 32; k++) xr[k] = valid ? x[size_t(row) * 32 + k] : 0.0f;
    for (int k = 0; k < 32; k++) {
        __nv_bfloat16 b = __float2bfloat16_rn(xr[k]);
        S.x[umma::tile_offset(r, k, 32) / 2] = b;
        S.xt[umma::tile_offset(k, r, 128) / 2] = b;
    }
    umma::fence_before();
    umma::fence_smem_async();
    __syncthreads();
    umma::fence_after();
    const uint32_t T = S.tmem;
    uint32_t phase = 0;
    bool ok = true;
    auto issue = [&](uint32_t d, const void* a, uint32_t ka, const void* b, uint32_t kb, uint32_t M, uint32_t N,
                     uint32_t K) {
        if (r == 0) {
            umma::fence_after();
            const uint32_t id = umma::idesc_bf16(M, N);
            const uint32_t aa = umma::saddr(a), ba = umma::saddr(b);
            for (uint32_t k = 0; k < K / 16; k++)
                umma::mma_bf16(d, umma::desc_kmajor(aa + k * 256, ka), umma::desc_kmajor(ba + k * 256, kb), id, k > 0);
            umma::commit(&S.bar);
        }
        ok = umma::bar_wait(&S.bar, phase & 1) && ok;
        phase++;
        umma::fence_after();
    };
    auto sync_for_mma = [&]() {
        umma::fence_before();
        umma::fence_smem_async();
        __syncthreads();
    };
    // Layer 1.
    issue(T, S.x, 32, S.w1, 32, 128, 64, 32);
    for (int c = 0; c < 64; c += 8) {
        float v[8];
        umma::ld8(T, warp, c, v);
        umma::ld_wait();
        for (int i = 0; i < 8; i++) {
            __nv_bfloat16 a = __float2bfloat16_rn(gelu(v[i] + S.b1[c + i]));
            S.a1[umma::tile_offset(r, c + i, 64) / 2] = a;
            S.a1t[umma::tile_offset(c + i, r, 128) / 2] = a;
        }
    }
    sync_for_mma();
    // Layer 2 and the output.
    issue(T + 64, S.a1, 64, S.w2, 64, 128, 64, 64);
    float y = S.b3;
    for (int c = 0; c < 64; c += 8) {
        float v[8];
        umma::ld8(T, warp, 64 + c, v);
        umma::ld_wait();
        for (int i = 0; i < 8; i++) y += gelu(v[i] + S.b2[c + i]) * S.w3[c + i];
    }
    const float t = 1.0f / (1.0f + expf(-y));
    const float tg = valid ? target[row] : 0.0f;
    const float err = valid ? t - tg : 0.0f;
    const float dy = 2.0f * err * t * (1.0f - t) * inv_batch;
    // Output layer gradients and dZ2.
    float* g = partial + size_t(blockIdx.x) * MLP_NPARAM;
    for (int c = 0; c < 64; c += 8) {
        float v[8];
        umma::ld8(T, warp, 64 + c, v);
        umma::ld_wait();
        for (int i = 0; i < 8; i++) {
            float z = v[i] + S.b2[c + i];
            float dz = dy * S.w3[c + i] * gelu_grad(z);
            __nv_bfloat16 q = __float2bfloat16_rn(dz);
            S.dz2[umma::tile_offset(r, c + i, 64) / 2] = q;
            S.dz2t[umma::tile_offset(c + i, r, 128) / 2] = q;
            block_col_sum(S, c + i, gelu(z) * dy);
        }
    }
    __syncthreads();
    if (r < 64) g[MLP_W3 + r] = S.red[0][r] + S.red[1][r] + S.red[2][r] + S.red[3][r];
    __syncthreads();
    for (int c = 0; c < 64; c += 8) {
        float v[8];
        umma::ld8(T, warp, 64 + c, v);
        umma::ld_wait();
        for (int i = 0; i < 8; i++) block_col_sum(S, c + i, dy * S.w3[c + i] * gelu_grad(v[i] + S.b2[c + i]));
    }
    __syncthreads();
    if (r < 64) g[MLP_B2 + r] = S.red[0][r] + S.red[1][r] + S.red[2][r] + S.red[3][r];
    {
        float w = warp_sum(dy), e2 = warp_sum(err * err);
        __syncthreads();
        if ((r & 31) == 0) S.red[warp][0] = w, S.red[warp][1] = e2;
        __syncthreads();
        if (r == 0) {
            g[MLP_B3] = S.red[0][0] + S.red[1][0] + S.red[2][0] + S.red[3][0];
            loss_partial[blockIdx.x] = S.red[0][1] + S.red[1][1] + S.red[2][1] + S.red[3][1];
        }
    }
    sync_for_mma();
    // dA1 = dZ2 W2 and dW2 = dZ2^T A1.
    issue(T + 128, S.dz2, 64, S.w2t, 64, 128, 64, 64);
    issue(T + 192, S.dz2t, 128, S.a1t, 128, 128, 64, 128);
    // dZ1 (rows), dW2 rows 0..63, db1.
    for (int c = 0; c < 64; c += 8) {
        float v[8], z[8];
        umma::ld8(T, warp, 128 + c, v);
        umma::ld8(T, warp, c, z);
        umma::ld_wait();
        for (int i = 0; i < 8; i++) {
            float dz = v[i] * gelu_grad(z[i] + S.b1[c + i]);
            S.dz1t[umma::tile_offset(c + i, r, 128) / 2] = __float2bfloat16_rn(dz);
            block_col_sum(S, c + i, dz);
        }
    }
    for (int c = 0; c < 64; c += 8) {
        float v[8];
        umma::ld8(T, warp, 192 + c, v);
        umma::ld_wait();
        if (r < 64)
            for (int i = 0; i < 8; i++) g[MLP_W2 + r * 64 + c + i] = v[i];
    }
    __syncthreads();
    if (r < 64) g[MLP_B1 + r] = S.red[0][r] + S.red[1][r] + S.red[2][r] + S.red[3][r];
    sync_for_mma();
    // dW1 = dZ1^T X (TMEM columns [0, 32), layer 1 is consumed).
    issue(T, S.dz1t, 128, S.xt, 128, 128, 32, 128);
    for (int c = 0; c < 32; c += 8) {
        float v[8];
        umma::ld8(T, warp, c, v);
        umma::ld_wait();
        if (r < 64)
            for (int i = 0; i < 8; i++) g[MLP_W1 + r * 32 + c + i] = v[i];
    }
    if (!ok && r == 0) atomicAdd(timeouts, 1ull);
    umma::fence_before();
    __syncthreads();
    if (r < 32) umma::tmem_dealloc(T, 256);
}

// grad = sum of the CTA partials in order; Adam (bias-corrected) update.
__global__ void k_mlp_reduce_adam(const float* partial, uint32_t tiles, float* grad, float* p, float* m, float* v,
                                  float lr, float b1, float b2, float eps, float c1, float c2, int apply) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= MLP_NPARAM) return;
    float s = 0.0f;
    for (uint32_t b = 0; b < tiles; b++) s += partial[size_t(b) * MLP_NPARAM + j];
    grad[j] = s;
    if (!apply) return;
    float mj = b1 * m[j] + (1.0f - b1) * s;
    float vj = b2 * v[j] + (1.0f - b2) * s * s;
    m[j] = mj;
    v[j] = vj;
    p[j] -= lr * (mj / c1) / (sqrtf(vj / c2) + eps);
}

__global__ void k_mlp_pack_t(const float* p, __nv_bfloat16* w2tt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_H * MLP_H) {
        int o = i / MLP_H, k = i % MLP_H;  // W2[o][k]: W2^T tile row k, column o
        w2tt[umma::tile_offset(k, o, MLP_H) / 2] = __float2bfloat16_rn(p[MLP_W2 + i]);
    }
}
}  // namespace

struct smb_mlp {
    smb_device* dev = nullptr;
    DBuf p, w1t, w2t, w2tt, x, y, t, counters, partial, loss, grad, m, v;
    long step = 0;
    int use = SMB_MLP_GATE;
};

namespace smb {
MlpDev mlp_dev(const smb_mlp* m) {
    return MlpDev{m->p.as<float>(), m->w1t.as<__nv_bfloat16>(), m->w2t.as<__nv_bfloat16>()};
}
int mlp_use(const smb_mlp* m) { return m->use; }
size_t mlp_smem_bytes() { return sizeof(MlpSmem) + 128; }
const smb_device* mlp_device(const smb_mlp* m) { return m->dev; }
}  // namespace smb

extern "C" {

int smb_mlp_new(smb_device* dev, const float* params, smb_mlp** out, char* err, size_t errlen) {
    if (!dev || !params || !out) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *out = nullptr;
    CK(cudaSetDevice(dev->index));
    auto* m = new smb_mlp();
    m->dev = dev;
    dev_retain(dev);
    int rc;
    if ((rc = m->p.reserve(MLP_NPARAM * 4, err, errlen)) || (rc = m->w1t.reserve(MLP_H * MLP_IN * 2, err, errlen)) ||
        (rc = m->w2t.reserve(MLP_H * MLP_H * 2, err, errlen)) || (rc = m->w2tt.reserve(MLP_H * MLP_H * 2, err, errlen)) ||
        (rc = m->counters.reserve(64, err, errlen)) || (rc = m->grad.reserve(MLP_NPARAM * 4, err, errlen)) ||
        (rc = m->m.reserve(MLP_NPARAM * 4, err, errlen)) || (rc = m->v.reserve(MLP_NPARAM * 4, err, errlen))) {
        smb_mlp_free(m);
        return rc;
    }
    *out = m;
    return smb_mlp_set_params(m, params, err, errlen);
}

void smb_mlp_free(smb_mlp* m) {
    if (!m) return;
    cudaSetDevice(m->dev->index);
    for (DBuf* b : {&m->p, &m->w1t, &m->w2t, &m->w2tt, &m->x, &m->y, &m->t, &m->counters, &m->partial, &m->loss,
                    &m->grad, &m->m, &m->v})
        b->release();
    smb_device* d = m->dev;
    delete m;
    dev_release(d);
}

int smb_mlp_set_params(smb_mlp* m, const float* params, char* err, size_t errlen) {
    if (!m || !params) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    CK(cudaSetDevice(m->dev->index));
    cudaStream_t s = m->dev->stream;
    CK(cudaMemcpyAsync(m->p.p, params, MLP_NPARAM * 4, cudaMemcpyHostToDevice, s));
    k_mlp_pack<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(m->p.as<float>(), m->w1t.as<__nv_bfloat16>(),
                                                           m->w2t.as<__nv_bfloat16>());
    k_mlp_pack_t<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(m->p.as<float>(), m->w2tt.as<__nv_bfloat16>());
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(m->m.p, 0, MLP_NPARAM * 4, s));
    CK(cudaMemsetAsync(m->v.p, 0, MLP_NPARAM * 4, s));
    m->step = 0;
    CK(cudaStreamSynchronize(s));
    return SMB_OK;
}

int smb_mlp_set_use(smb_mlp* m, int use) {
    if (!m || (use != SMB_MLP_GATE && use != SMB_MLP_ROOT)) return SMB_ERR_ARG;
    m->use = use;
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

// One pass over (x, target) in minibatches of `batch` rows (a multiple of
// 128): per minibatch, tensor-core forward/backward tiles, the fixed-order
// gradient sum and an Adam step (apply != 0) or only the gradient of the
// whole set as one batch (apply == 0, grad_out gets it).
static int mlp_run(smb_mlp* m, const float* x, const float* target, size_t n, size_t batch, float lr, int apply,
                   float* losses, float* grad_out, char* err, size_t errlen) {
    if (!m || !x || !target || n == 0) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    if (apply && (batch == 0 || batch % 128)) return set_err(err, errlen, "batch must be a positive multiple of 128"), SMB_ERR_ARG;
    if (!apply) batch = (n + 127) / 128 * 128;
    CK(cudaSetDevice(m->dev->index));
    cudaStream_t s = m->dev->stream;
    const size_t tiles = batch / 128;
    int rc;
    if ((rc = m->x.reserve(n * MLP_IN * 4, err, errlen)) || (rc = m->y.reserve(n * 4, err, errlen)) ||
        (rc = m->partial.reserve(tiles * MLP_NPARAM * 4, err, errlen)) || (rc = m->loss.reserve(tiles * 4, err, errlen)))
        return rc;
    CK(cudaMemcpyAsync(m->x.p, x, n * MLP_IN * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(m->y.p, target, n * 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(m->counters.p, 0, 64, s));
    const size_t smem = sizeof(TrainSmem) + 128;
    CK(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const float b1 = 0.9f, b2 = 0.999f;
    std::vector<float> lp(tiles);
    size_t steps = (n + batch - 1) / batch;
    for (size_t st = 0; st < steps; st++) {
        size_t first = st * batch, rows = std::min(batch, n - first);
        uint32_t nt = uint32_t((rows + 127) / 128);
        k_mlp_train<<<nt, 128, smem, s>>>(m->x.as<float>(), m->y.as<float>(), uint32_t(first + rows), uint32_t(first),
                                         1.0f / float(rows), m->p.as<float>(), m->w1t.as<__nv_bfloat16>(),
                                         m->w2t.as<__nv_bfloat16>(), m->w2tt.as<__nv_bfloat16>(),
                                         m->partial.as<float>(), m->loss.as<float>(),
                                         m->counters.as<unsigned long long>());
        CK(cudaGetLastError());
        if (apply) m->step++;
        float c1 = apply ? 1.0f - std::pow(b1, float(m->step)) : 1.0f, c2 = apply ? 1.0f - std::pow(b2, float(m->step)) : 1.0f;
        k_mlp_reduce_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(m->partial.as<float>(), nt, m->grad.as<float>(),
                                                                    m->p.as<float>(), m->m.as<float>(),
                                                                    m->v.as<float>(), lr, b1, b2, 1e-8f, c1, c2, apply);
        if (apply) {
            k_mlp_pack<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(m->p.as<float>(), m->w1t.as<__nv_bfloat16>(),
                                                                   m->w2t.as<__nv_bfloat16>());
            k_mlp_pack_t<<<(MLP_H * MLP_H + 255) / 256, 256, 0, s>>>(m->p.as<float>(), m->w2tt.as<__nv_bfloat16>());
        }
        CK(cudaGetLastError());
        if (losses) {
            CK(cudaMemcpyAsync(lp.data(), m->loss.p, nt * 4, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            double sum = 0;
            for (uint32_t k = 0; k < nt; k++) sum += lp[k];
            losses[st] = float(sum / double(rows));
        }
    }
    unsigned long long to = 0;
    CK(cudaMemcpyAsync(&to, m->counters.p, 8, cudaMemcpyDeviceToHost, s));
    if (grad_out) CK(cudaMemcpyAsync(grad_out, m->grad.p, MLP_NPARAM * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (to) return set_err(err, errlen, "a bounded tensor-core wait gave up"), SMB_ERR_TIMEOUT;
    return SMB_OK;
}

int smb_mlp_gradient(smb_mlp* m, const float* x, const float* target, size_t n, float* loss, float* grad, char* err,
                     size_t errlen) {
    if (n > (size_t(1) << 20)) return set_err(err, errlen, "at most 2^20 rows for one gradient"), SMB_ERR_ARG;
    return mlp_run(m, x, target, n, 0, 0.0f, 0, loss, grad, err, errlen);
}

int smb_mlp_train_epoch(smb_mlp* m, const float* x, const float* target, size_t n, size_t batch, float lr,
                        float* losses, char* err, size_t errlen) {
    return mlp_run(m, x, target, n, batch, lr, 1, losses, nullptr, err, errlen);
}

}  // extern "C"
