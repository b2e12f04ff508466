// Marching cubes over caller-owned device buffers with no allocation at all.
//
// Some callers of this library cannot allocate device memory when they mesh:
// services that reserve a fixed device-memory budget up front and must not
// grow it while they serve, and hosts whose device memory belongs to another
// framework's caching allocator (there a cudaMalloc beside it can fail once
// that allocator has reserved the free memory, or force it to give back its
// cache).  smb_mc_noalloc gives them the marching-cubes pass of a run
// (per-brick counts, offsets, ordered compaction of crossing edges and
// triangle references) with all of its scratch in one file-scope device
// array of fixed size (SCRATCH_BYTES = 524,832 bytes, 512.5 KiB, for at most
// SMB_MC_NOALLOC_MAX_BRICKS bricks); inputs and outputs are the caller's
// device buffers.
//
// The array is a host-side stand-in in host code: a kernel given its name
// would fault (or, where the GPU can reach host memory, silently use the
// wrong memory).  Its device address is therefore looked up once per
// device, with that device current, by cudaGetSymbolAddress, and passed to
// the kernels.  The call runs on the resident's device stream and returns
// once its work there has finished (it reads the totals back to check the
// caller's capacities); the caller's current device is left as it was.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/sesmesh_b200.h"
#include "device/kernels.hpp"
#include "runtime.hpp"

using namespace smb;

namespace {

constexpr size_t MAX_BRICKS = SMB_MC_NOALLOC_MAX_BRICKS;
constexpr size_t TILE_WORDS = 64;  // >= scan_tiles_needed(MAX_BRICKS) = 17
constexpr size_t SCRATCH_BYTES = (TILE_WORDS + 4) * 8 + 2 * MAX_BRICKS * 4;
static_assert(SCRATCH_BYTES == 524832, "the documented scratch size");

// Shared by every call on a device; holds the last call's contents.  Nothing
// in it needs clearing: the count pass writes every brick's two counts and
// the scans write their tiles and totals before reading them.
static __device__ __align__(256) unsigned char g_mc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_lock;
void* g_addr[MAX_DEVICES] = {};

void set_err(char* err, size_t len, const char* msg, const char* detail) {
    if (err && len) std::snprintf(err, len, "%s%s%s", msg, detail ? ": " : "", detail ? detail : "");
}

// Makes `dev` current for the call and gives the caller its own current
// device back on every return.
struct DeviceScope {
    int saved = -1;
    cudaError_t enter(int dev) {
        cudaError_t e = cudaGetDevice(&saved);
        if (e != cudaSuccess) return saved = -1, e;
        return saved == dev ? cudaSuccess : cudaSetDevice(dev);
    }
    ~DeviceScope() {
        int cur = -1;
        if (saved >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != saved) cudaSetDevice(saved);
    }
};

}  // namespace

extern "C" int smb_mc_noalloc(const smb_resident* res, float* values, const uint32_t* records, size_t n_bricks,
                              uint32_t* edge_off, uint32_t* edges, float* edge_vals, size_t edges_cap,
                              uint32_t* tri_off, uint32_t* tris, size_t tris_cap, size_t* n_edges, size_t* n_tris,
                              char* err, size_t errlen) {
    if (!res || !values || !records || !edge_off || !tri_off) return set_err(err, errlen, "null argument", nullptr), SMB_ERR_ARG;
    if (n_bricks > MAX_BRICKS) {
        char d[96];
        std::snprintf(d, sizeof d, "%zu bricks requested, at most %zu per call", n_bricks, MAX_BRICKS);
        return set_err(err, errlen, "smb_mc_noalloc", d), SMB_ERR_ARG;
    }
    const int dev = res->dev->index;
    if (dev < 0 || dev >= MAX_DEVICES) return set_err(err, errlen, "device index out of range", nullptr), SMB_ERR_ARG;
    DeviceScope scope;
    cudaError_t e = scope.enter(dev);
    if (e != cudaSuccess) return set_err(err, errlen, "cudaSetDevice", cudaGetErrorString(e)), SMB_ERR_CUDA;
    void* base;
    {
        // First call on this device: find the array's device address.
        std::lock_guard<std::mutex> g(g_lock);
        if (!g_addr[dev]) {
            e = cudaGetSymbolAddress(&g_addr[dev], g_mc_scratch);
            if (e != cudaSuccess) {
                g_addr[dev] = nullptr;
                return set_err(err, errlen, "cudaGetSymbolAddress", cudaGetErrorString(e)), SMB_ERR_CUDA;
            }
        }
        base = g_addr[dev];
    }
    unsigned long long* tiles = static_cast<unsigned long long*>(base);
    unsigned long long* totals = tiles + TILE_WORDS;
    uint32_t* counts = reinterpret_cast<uint32_t*>(totals + 4);
    cudaStream_t s = res->dev->stream;
    const uint32_t n = uint32_t(n_bricks);
    if (n == 0) {
        uint32_t zero = 0;
        if ((e = cudaMemcpyAsync(edge_off, &zero, 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaMemcpyAsync(tri_off, &zero, 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return set_err(err, errlen, "copy", cudaGetErrorString(e)), SMB_ERR_CUDA;
        if (n_edges) *n_edges = 0;
        if (n_tris) *n_tris = 0;
        return SMB_OK;
    }
    // Count pass (writes every brick's two counts: nothing to clear), scans.
    e = launch_mc(res->L, n, values, records, counts, nullptr, nullptr, nullptr, nullptr, nullptr, false, s);
    if (e != cudaSuccess) return set_err(err, errlen, "count launch", cudaGetErrorString(e)), SMB_ERR_CUDA;
    launch_scan(counts, n, edge_off, nullptr, tiles, totals + 1, s);
    launch_scan(counts + n, n, tri_off, nullptr, tiles, totals + 2, s);
    unsigned long long t[3] = {0, 0, 0};
    if ((e = cudaMemcpyAsync(t, totals, sizeof t, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return set_err(err, errlen, "count pass", cudaGetErrorString(e)), SMB_ERR_CUDA;
    if (n_edges) *n_edges = size_t(t[1]);
    if (n_tris) *n_tris = size_t(t[2]);
    // The offsets are 32-bit words: a total at or past 2^32 has wrapped them.
    if (t[1] >= (1ull << 32) || t[2] >= (1ull << 32))
        return set_err(err, errlen, "output too large for 32-bit offsets", nullptr), SMB_ERR_MEMORY;
    if (t[1] > edges_cap || t[2] > tris_cap || !edges || !edge_vals || !tris) {
        char d[128];
        std::snprintf(d, sizeof d, "%llu edges and %llu triangles, room for %zu and %zu", t[1], t[2], edges_cap, tris_cap);
        return set_err(err, errlen, "output buffers too small", d), SMB_ERR_MEMORY;
    }
    uint32_t ends[2] = {uint32_t(t[1]), uint32_t(t[2])};
    if ((e = cudaMemcpyAsync(edge_off + n, &ends[0], 4, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(tri_off + n, &ends[1], 4, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return set_err(err, errlen, "offsets", cudaGetErrorString(e)), SMB_ERR_CUDA;
    // The capacities go to the fill kernel too: a brick whose range would end
    // past them writes nothing.
    e = launch_mc(res->L, n, values, records, nullptr, edge_off, tri_off, edges, reinterpret_cast<float2*>(edge_vals),
                  tris, true, s, nullptr, edges_cap, tris_cap);
    if (e != cudaSuccess) return set_err(err, errlen, "fill launch", cudaGetErrorString(e)), SMB_ERR_CUDA;
    if ((e = cudaStreamSynchronize(s)) != cudaSuccess)
        return set_err(err, errlen, "fill pass", cudaGetErrorString(e)), SMB_ERR_CUDA;
    return SMB_OK;
}
