// Order-preserving scans and compactions (device-wide and block-wide).
#pragma once
#include <cstdint>

namespace smb {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Exclusive block-wide scan of one value per thread; returns the exclusive
// prefix and writes the block total to *total.  All threads must call it.
template <int NT>
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long v, unsigned long long* sh,
                                                                   unsigned long long* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long x = v;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned long long w = lane < NT / 32 ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NT / 32) sh[lane] = w;
    }
    __syncthreads();
    unsigned long long before = (warp ? sh[warp - 1] : 0) + x - v;
    *total = sh[NT / 32 - 1];
    __syncthreads();
    return before;
}

}  // namespace smb
