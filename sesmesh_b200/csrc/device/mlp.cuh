// The warm-start MLP of fast mode: 32 -> 64 -> 64 -> 1, GELU hidden layers,
// sigmoid output t in [0, 1].  BF16 weights and activations on the tensor
// cores (tcgen05, FP32 accumulation in TMEM); bias, GELU and the last layer
// in FP32 on the CUDA cores.
//
// One CTA of 128 threads evaluates a tile of 128 rows (thread r owns row r).
// Shared-memory layout of a forward pass (bytes):
//   X   bf16 128 x 32  (core-matrix tile, K = 32)      8192
//   A1  bf16 128 x 64  (K = 64)                       16384
//   W1  bf16  64 x 32                                   4096
//   W2  bf16  64 x 64                                   8192
// TMEM: 128 columns (layer-1 accumulator in [0, 64), layer 2 in [64, 128)).
#pragma once
#include <cuda_bf16.h>

#include "umma.cuh"

namespace smb {

constexpr int MLP_IN = 32, MLP_H = 64, MLP_ROWS = 128;
// Parameter vector layout (f32 master copy): W1 [64][32], b1 [64],
// W2 [64][64], b2 [64], w3 [64], b3.
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_H * MLP_IN, MLP_W2 = MLP_B1 + MLP_H,
              MLP_B2 = MLP_W2 + MLP_H * MLP_H, MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H,
              MLP_NPARAM = MLP_B3 + 1;

// Device parameters: f32 vector plus the bf16 weight tiles in core-matrix
// layout (W1: 64 x 32, W2: 64 x 64), ready to copy into shared memory.
struct MlpDev {
    const float* p;
    const __nv_bfloat16* w1t;
    const __nv_bfloat16* w2t;
};

// Weights, biases, TMEM slot and barrier first (they live across tiles),
// then the per-tile input and hidden tiles (a caller may reuse those bytes
// between tiles: offsetof(MlpSmem, x) is the persistent part's size).
struct MlpSmem {
    __nv_bfloat16 w1[MLP_H * MLP_IN];
    __nv_bfloat16 w2[MLP_H * MLP_H];
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];
    float b3;
    uint32_t tmem;
    alignas(8) uint64_t bar;
    alignas(16) __nv_bfloat16 x[MLP_ROWS * MLP_IN];
    __nv_bfloat16 a1[MLP_ROWS * MLP_H];
};

// tanh on the special-function unit (one MUFU instruction, relative error
// below 2^-10, far inside the BF16 rounding of the activations it feeds).
__device__ __forceinline__ float tanh_sfu(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GELU, tanh form, and its derivative (f32 arithmetic, SFU tanh).
__device__ __forceinline__ float gelu(float z) {
    const float k = 0.7978845608028654f;
    float u = k * (z + 0.044715f * z * z * z);
    return 0.5f * z * (1.0f + tanh_sfu(u));
}
__device__ __forceinline__ float gelu_grad(float z) {
    const float k = 0.7978845608028654f;
    float u = k * (z + 0.044715f * z * z * z);
    float th = tanh_sfu(u);
    return 0.5f * (1.0f + th) + 0.5f * z * (1.0f - th * th) * k * (1.0f + 3.0f * 0.044715f * z * z);
}

// Loads the weights into shared memory and allocates `ncols` TMEM columns
// (all threads; 64 suffice for inference, see mlp_forward).
__device__ __forceinline__ void mlp_setup(MlpSmem& S, const MlpDev& P, uint32_t ncols = 128) {
    const int t = threadIdx.x;
    const uint4* w1 = reinterpret_cast<const uint4*>(P.w1t);
    const uint4* w2 = reinterpret_cast<const uint4*>(P.w2t);
    for (int i = t; i < MLP_H * MLP_IN / 8; i += blockDim.x) reinterpret_cast<uint4*>(S.w1)[i] = w1[i];
    for (int i = t; i < MLP_H * MLP_H / 8; i += blockDim.x) reinterpret_cast<uint4*>(S.w2)[i] = w2[i];
    for (int i = t; i < MLP_H; i += blockDim.x) {
        S.b1[i] = P.p[MLP_B1 + i];
        S.b2[i] = P.p[MLP_B2 + i];
        S.w3[i] = P.p[MLP_W3 + i];
    }
    if (t == 0) {
        S.b3 = P.p[MLP_B3];
        umma::bar_init(&S.bar, 1);
    }
    if (t < 32) umma::tmem_alloc(&S.tmem, ncols);
    umma::fence_before();
    __syncthreads();
    umma::fence_after();
}

__device__ __forceinline__ void mlp_teardown(MlpSmem& S, uint32_t ncols = 128) {
    umma::fence_before();
    __syncthreads();
    if (threadIdx.x < 32) umma::tmem_dealloc(S.tmem, ncols);
}

// Forward pass of the tile whose inputs thread r has placed in S.x (row r);
// returns thread r's output t and, when z1/z2 are given, the hidden
// pre-activations of its row.  `phase` is the mbarrier parity of the first of
// the two waits (it advances by 2 per call); false if a wait gave up.  Layer
// 2 accumulates at TMEM column `l2col`: 0 reuses layer 1's columns (every
// thread has read them before the layer-2 MMA is issued), 64 keeps them.
__device__ __forceinline__ bool mlp_forward(MlpSmem& S, uint32_t& phase, float* t_out, float* z1, float* z2,
                                            float* a2_out, uint32_t l2col = 64) {
    const int r = threadIdx.x, warp = r >> 5;
    umma::fence_smem_async();
    __syncthreads();
    if (r == 0) {
        umma::fence_after();
        const uint32_t id = umma::idesc_bf16(MLP_ROWS, MLP_H);
        const uint32_t xa = umma::saddr(S.x), wa = umma::saddr(S.w1);
        for (int k = 0; k < MLP_IN / 16; k++)
            umma::mma_bf16(S.tmem, umma::desc_kmajor(xa + k * 256, MLP_IN), umma::desc_kmajor(wa + k * 256, MLP_IN), id,
                           k > 0);
        umma::commit(&S.bar);
    }
    bool ok = umma::bar_wait(&S.bar, phase & 1);
    phase++;
    umma::fence_after();
    // Layer 1 epilogue: bias, GELU, bf16 into A1 (row r).
    for (int c = 0; c < MLP_H; c += 8) {
        float v[8];
        umma::ld8(S.tmem, warp, c, v);
        umma::ld_wait();
        for (int i = 0; i < 8; i++) {
            float z = v[i] + S.b1[c + i];
            if (z1) z1[c + i] = z;
            S.a1[umma::tile_offset(r, c + i, MLP_H) / 2] = __float2bfloat16_rn(gelu(z));
        }
    }
    umma::fence_before();
    umma::fence_smem_async();
    __syncthreads();
    if (r == 0) {
        umma::fence_after();
        const uint32_t id = umma::idesc_bf16(MLP_ROWS, MLP_H);
        const uint32_t aa = umma::saddr(S.a1), wa = umma::saddr(S.w2);
        for (int k = 0; k < MLP_H / 16; k++)
            umma::mma_bf16(S.tmem + l2col, umma::desc_kmajor(aa + k * 256, MLP_H), umma::desc_kmajor(wa + k * 256, MLP_H),
                           id, k > 0);
        umma::commit(&S.bar);
    }
    ok = umma::bar_wait(&S.bar, phase & 1) && ok;
    phase++;
    umma::fence_after();
    float y = S.b3;
    for (int c = 0; c < MLP_H; c += 8) {
        float v[8];
        umma::ld8(S.tmem, warp, l2col + c, v);
        umma::ld_wait();
        for (int i = 0; i < 8; i++) {
            float z = v[i] + S.b2[c + i];
            if (z2) z2[c + i] = z;
            float a = gelu(z);
            if (a2_out) a2_out[c + i] = a;
            y += a * S.w3[c + i];
        }
    }
    *t_out = 1.0f / (1.0f + expf(-y));
    umma::fence_before();
    return ok;
}

// Thread r writes its 32 features into row r of the input tile (bf16).
__device__ __forceinline__ void mlp_put_row(MlpSmem& S, const float* f) {
    const int r = threadIdx.x;
    for (int k = 0; k < MLP_IN; k++) S.x[umma::tile_offset(r, k, MLP_IN) / 2] = __float2bfloat16_rn(f[k]);
}

}  // namespace smb
