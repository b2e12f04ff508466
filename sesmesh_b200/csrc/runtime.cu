// Host runtime behind the C ABI of include/sesmesh_b200.h: device open and
// self-test, the resident arrangement, device-side brick classification and
// batch runs (sub-block states, gather, sampling, marching cubes).
//
// Stands in for sesmesh's CUDA back-end crate (crates/sesmesh-gpu/src/cuda/
// {mod.rs,resident.rs,memory.rs,stream.rs}): one stream per device, device
// buffers grown on demand and reused across runs, CUDA events around each
// pass.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/sesmesh_b200.h"
#include "device/kernels.hpp"
#include "device/mlp.cuh"
#include "device/sas.hpp"
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

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess) {                                                                 \
            set_err(err, errlen, "%s failed: %s", #call, cudaGetErrorString(e_));                \
            return SMB_ERR_CUDA;                                                                 \
        }                                                                                        \
    } while (0)

uint64_t splitmix(uint64_t& s) {
    s += 0x9E3779B97F4A7C15ULL;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Host recomputation of k_selftest (built without FMA contraction).
void selftest_ref(float x, float y, uint32_t out[12]) {
    float dx = x - y, dy = y * 0.75f - x, dz = x * y - 1.0f;
    float d = std::sqrt(dx * dx + dy * dy + dz * dz);
    float r[8] = {x + y, x * y, x / y, std::sqrt(std::fabs(x)), d, (d - y) / d, std::fmin(x, y), std::fabs(d - std::fabs(y))};
    for (int k = 0; k < 8; k++) std::memcpy(&out[k], &r[k], 4);
    double X = double(x) * 1.0000001, Y = double(y) - 0.3;
    double D = X * Y + X, E = std::sqrt(std::fabs(X * X + Y * Y - X)), F = X / (Y + 2.5), G = std::floor(X * 3.7);
    double rr[4] = {D, E, F, G};
    for (int k = 0; k < 4; k++) {
        uint64_t u;
        std::memcpy(&u, &rr[k], 8);
        out[8 + k] = uint32_t(u ^ (u >> 32));
    }
}

}  // namespace

namespace smb {

// Device memory cache.  Blocks a library object frees stay with the process
// and are handed to the next allocation of a similar size on the same
// device, so engines made one after another (compute_surface calls) do not
// pay cudaMalloc / cudaFree for their multi-GB buffers each time.  A free
// synchronizes the device first, as cudaFree does, so no queued kernel
// still uses a block when it is handed out again.  An allocation that fails
// releases the device's cached blocks and retries; the cache is released
// when the last handle of a device closes.
namespace {
constexpr int MAX_DEVICES = 64;
struct MemCache {
    std::mutex m;
    std::multimap<size_t, void*> free_blocks[MAX_DEVICES];
    std::unordered_map<void*, std::pair<int, size_t>> live;  // block -> (device, bytes)
    int open[MAX_DEVICES] = {};
};
MemCache& mem_cache() {
    static MemCache* c = new MemCache();  // kept to process exit: frees may run in static destructors
    return *c;
}
}  // namespace

void mem_trim(int dev) {
    if (dev < 0 || dev >= MAX_DEVICES) return;
    MemCache& C = mem_cache();
    std::vector<void*> blocks;
    {
        std::lock_guard<std::mutex> g(C.m);
        for (auto& kv : C.free_blocks[dev]) blocks.push_back(kv.second);
        C.free_blocks[dev].clear();
    }
    if (blocks.empty()) return;
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(dev);
    for (void* b : blocks) cudaFree(b);
    cudaSetDevice(cur);
}

cudaError_t mem_alloc(void** p, size_t bytes) {
    *p = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    MemCache& C = mem_cache();
    if (dev >= 0 && dev < MAX_DEVICES) {
        std::lock_guard<std::mutex> g(C.m);
        auto& fb = C.free_blocks[dev];
        auto it = fb.lower_bound(bytes);
        if (it != fb.end() && it->first <= 2 * bytes + (size_t(1) << 20)) {
            *p = it->second;
            C.live[*p] = {dev, it->first};
            fb.erase(it);
            return cudaSuccess;
        }
    }
    cudaError_t e = cudaMalloc(p, bytes);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        mem_trim(dev);
        e = cudaMalloc(p, bytes);
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> g(C.m);
    C.live[*p] = {dev, bytes};
    return cudaSuccess;
}

void mem_free_synced(void* p) {
    if (!p) return;
    MemCache& C = mem_cache();
    std::lock_guard<std::mutex> g(C.m);
    auto it = C.live.find(p);
    if (it == C.live.end()) {
        cudaFree(p);
        return;
    }
    C.free_blocks[it->second.first].emplace(it->second.second, p);
    C.live.erase(it);
}

void mem_free(void* p) {
    if (!p) return;
    MemCache& C = mem_cache();
    std::pair<int, size_t> info{-1, 0};
    {
        std::lock_guard<std::mutex> g(C.m);
        auto it = C.live.find(p);
        if (it != C.live.end()) info = it->second, C.live.erase(it);
    }
    if (info.first < 0 || info.first >= MAX_DEVICES) {
        cudaFree(p);
        return;
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != info.first) cudaSetDevice(info.first);
    cudaDeviceSynchronize();
    if (cur != info.first) cudaSetDevice(cur);
    std::lock_guard<std::mutex> g(C.m);
    C.free_blocks[info.first].emplace(info.second, p);
}

// Page-locked host memory through a cache of the same kind (no device
// synchronization needed: callers free staging only after their copies
// completed).  Released when the last device handle closes.
namespace {
struct HostCache {
    std::mutex m;
    std::multimap<size_t, void*> free_blocks;
    std::unordered_map<void*, size_t> live;
};
HostCache& host_cache() {
    static HostCache* c = new HostCache();
    return *c;
}
void host_trim() {
    std::vector<void*> blocks;
    {
        std::lock_guard<std::mutex> g(host_cache().m);
        for (auto& kv : host_cache().free_blocks) blocks.push_back(kv.second);
        host_cache().free_blocks.clear();
    }
    for (void* b : blocks) cudaFreeHost(b);
}
}  // namespace

void* pinned_alloc(size_t bytes) {
    HostCache& C = host_cache();
    {
        std::lock_guard<std::mutex> g(C.m);
        auto it = C.free_blocks.lower_bound(bytes);
        if (it != C.free_blocks.end() && it->first <= 2 * bytes + (size_t(1) << 20)) {
            void* p = it->second;
            C.live[p] = it->first;
            C.free_blocks.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        host_trim();
        if (cudaHostAlloc(&p, bytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
    }
    std::lock_guard<std::mutex> g(C.m);
    C.live[p] = bytes;
    return p;
}

void pinned_free(void* p) {
    if (!p) return;
    HostCache& C = host_cache();
    std::lock_guard<std::mutex> g(C.m);
    auto it = C.live.find(p);
    if (it == C.live.end()) {
        cudaFreeHost(p);
        return;
    }
    C.free_blocks.emplace(it->second, p);
    C.live.erase(it);
}

void mem_device_open(int dev) {
    if (dev < 0 || dev >= MAX_DEVICES) return;
    std::lock_guard<std::mutex> g(mem_cache().m);
    mem_cache().open[dev]++;
}

void mem_device_close(int dev) {
    if (dev < 0 || dev >= MAX_DEVICES) return;
    bool last;
    {
        std::lock_guard<std::mutex> g(mem_cache().m);
        last = --mem_cache().open[dev] <= 0;
    }
    if (last) mem_trim(dev);
    bool none = true;
    {
        std::lock_guard<std::mutex> g(mem_cache().m);
        for (int k = 0; k < MAX_DEVICES; k++) none &= mem_cache().open[k] <= 0;
    }
    if (none) host_trim();
}

int dev_alloc(void** p, size_t bytes, std::vector<void*>* owned, size_t* total, char* err, size_t errlen) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = mem_alloc(p, bytes);
    if (e != cudaSuccess) {
        set_err(err, errlen, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
        *p = nullptr;
        return e == cudaErrorMemoryAllocation ? SMB_ERR_MEMORY : SMB_ERR_CUDA;
    }
    if (owned) owned->push_back(*p);
    if (total) *total += bytes;
    return SMB_OK;
}

// Grows a batch buffer to at least `bytes` (contents discarded).
int DBuf::reserve(size_t bytes, char* err, size_t errlen) {
    if (bytes <= cap) return SMB_OK;
    if (p) mem_free(p);
    p = nullptr;
    cap = 0;
    size_t want = bytes + bytes / 4 + 256;
    cudaError_t e = mem_alloc(&p, want);
    if (e != cudaSuccess) {
        set_err(err, errlen, "cudaMalloc(%zu bytes) failed: %s", want, cudaGetErrorString(e));
        p = nullptr;
        return e == cudaErrorMemoryAllocation ? SMB_ERR_MEMORY : SMB_ERR_CUDA;
    }
    cap = want;
    return SMB_OK;
}

void DBuf::release_synced() {
    if (p) mem_free_synced(p);
    p = nullptr;
    cap = 0;
}

void DBuf::release() {
    if (p) mem_free(p);
    p = nullptr;
    cap = 0;
}

static void destroy_device(smb_device* d) {
    if (d->gone.exchange(true)) return;
    cudaSetDevice(d->index);
    if (d->stream) cudaStreamDestroy(d->stream);
    if (d->copy) cudaStreamDestroy(d->copy);
    mem_device_close(d->index);
    delete d;
}

void dev_retain(smb_device* d) { d->refs.fetch_add(1); }

void dev_release(smb_device* d) {
    if (d->refs.fetch_sub(1) == 1 && d->closed.load()) destroy_device(d);
}

}  // namespace smb

extern "C" {

int smb_open(int index, smb_device** out, char* err, size_t errlen) {
    if (!out) return set_err(err, errlen, "null output"), SMB_ERR_ARG;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        set_err(err, errlen, "no CUDA device: %s", e == cudaSuccess ? "count is 0" : cudaGetErrorString(e));
        return SMB_ERR_NODEVICE;
    }
    if (index < 0 || index >= count) return set_err(err, errlen, "device %d of %d", index, count), SMB_ERR_NODEVICE;
    CK(cudaSetDevice(index));
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, index));
    if (prop.major < 10) {
        set_err(err, errlen, "device %d (%s) is sm_%d%d; the library is built for sm_100a", index, prop.name, prop.major,
                prop.minor);
        return SMB_ERR_NODEVICE;
    }
    auto* d = new smb_device();
    d->index = index;
    std::snprintf(d->info.name, sizeof d->info.name, "%s", prop.name);
    d->info.major = prop.major;
    d->info.minor = prop.minor;
    d->info.multiprocessors = prop.multiProcessorCount;
    d->info.memory = prop.totalGlobalMem;
    d->smem_optin = prop.sharedMemPerBlockOptin;
    e = cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->copy, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        if (d->stream) cudaStreamDestroy(d->stream);
        delete d;
        set_err(err, errlen, "cudaStreamCreate failed: %s", cudaGetErrorString(e));
        return SMB_ERR_CUDA;
    }
    mem_device_open(index);
    int rc = smb_self_test(d, 4096, err, errlen);
    if (rc != SMB_OK) {
        smb_close(d);
        return rc;
    }
    *out = d;
    return SMB_OK;
}

void smb_close(smb_device* d) {
    if (!d) return;
    d->closed.store(true);
    if (d->refs.load() == 0) destroy_device(d);
}

int smb_device_info_get(const smb_device* d, smb_device_info* out) {
    if (!d || !out) return SMB_ERR_ARG;
    *out = d->info;
    return SMB_OK;
}

int smb_self_test(smb_device* d, uint32_t n, char* err, size_t errlen) {
    if (!d || n == 0) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    CK(cudaSetDevice(d->index));
    std::vector<float> a(n), b(n);
    uint64_t s = 0x5e5e5e5eULL + n;
    for (uint32_t i = 0; i < n; i++) {
        a[i] = float(int64_t(splitmix(s) >> 40) - (int64_t(1) << 23)) / 65536.0f;
        b[i] = 0.1f + float(splitmix(s) >> 40) / 262144.0f;
    }
    float *da = nullptr, *db = nullptr;
    uint32_t* dout = nullptr;
    std::vector<uint32_t> got(size_t(n) * 12);
    auto cleanup = [&] {
        cudaFree(da);
        cudaFree(db);
        cudaFree(dout);
    };
    if (cudaMalloc(&da, n * 4) != cudaSuccess || cudaMalloc(&db, n * 4) != cudaSuccess ||
        cudaMalloc(&dout, size_t(n) * 48) != cudaSuccess) {
        cleanup();
        return set_err(err, errlen, "self-test allocation failed"), SMB_ERR_MEMORY;
    }
    cudaMemcpyAsync(da, a.data(), n * 4, cudaMemcpyHostToDevice, d->stream);
    cudaMemcpyAsync(db, b.data(), n * 4, cudaMemcpyHostToDevice, d->stream);
    launch_selftest(da, db, dout, n, d->stream);
    cudaMemcpyAsync(got.data(), dout, size_t(n) * 48, cudaMemcpyDeviceToHost, d->stream);
    cudaError_t e = cudaStreamSynchronize(d->stream);
    cleanup();
    if (e != cudaSuccess) return set_err(err, errlen, "self-test failed: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t want[12];
        selftest_ref(a[i], b[i], want);
        for (int k = 0; k < 12; k++)
            if (want[k] != got[size_t(i) * 12 + k]) {
                set_err(err, errlen, "arithmetic self-test: pair %u op %d differs (device %08x, host %08x)", i, k,
                        got[size_t(i) * 12 + k], want[k]);
                return SMB_ERR_SELFTEST;
            }
    }
    return SMB_OK;
}

static bool csr_ok(const uint32_t* off, size_t rows, size_t items) {
    if (!off || off[0] != 0) return false;
    for (size_t i = 0; i < rows; i++)
        if (off[i + 1] < off[i]) return false;
    return off[rows] == items;
}

// Lattice constants, computed here in the CPU's f64 operation order.
static void set_lattice(DLat& L, const smb_lattice_ref* lat, double probe, int kind) {
    L.kind = kind != SMB_KIND_SES ? 1 : 0;
    L.h = lat->spacing;
    L.b = int(lat->brick);
    L.sub = L.b / 2;
    L.spb = (L.b + 1) * (L.b + 1) * (L.b + 1);
    for (int k = 0; k < 3; k++) L.frame[k] = (long long)lat->frame[k];
    L.fx = double(lat->frame[0]) * L.h, L.fy = double(lat->frame[1]) * L.h, L.fz = double(lat->frame[2]) * L.h;
    L.band = lat->band;
    L.rho_sub = 0.5 * std::sqrt(3.0) * double(L.sub) * L.h;   // kernel.rs:474
    L.rho_brick = 0.5 * std::sqrt(3.0) * double(L.b) * L.h;   // lattice.rs:78-80
    L.h32 = float(L.h);
    L.band32 = float(L.band);
    L.probe32 = float(probe);
    float cutoff = float(probe + L.band);                      // kernel.rs:425
    L.cutoff2 = cutoff * cutoff;
}

int smb_resident_new(smb_device* d, const smb_arrangement_ref* a, const smb_lattice_ref* lat, smb_resident** out,
                     char* err, size_t errlen) {
    if (!d || !a || !lat || !out) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *out = nullptr;
    if (lat->brick < 4 || lat->brick > 32 || lat->brick % 2)
        return set_err(err, errlen, "brick must be even and 4..32, got %u", lat->brick), SMB_ERR_ARG;
    if (!(lat->spacing >= 0.01) || !std::isfinite(lat->spacing))
        return set_err(err, errlen, "grid spacing must be at least 0.01"), SMB_ERR_ARG;
    size_t n = a->n_spheres, nc = a->n_circles, nv = a->n_vertices;
    if (a->kind != SMB_KIND_SES && a->kind != SMB_KIND_SAS && a->kind != SMB_KIND_VDW)
        return set_err(err, errlen, "unknown surface kind %d", a->kind), SMB_ERR_ARG;
    if (a->kind != SMB_KIND_SES && (nc || nv))
        return set_err(err, errlen, "a sphere field has no circles or vertices"), SMB_ERR_ARG;
    if (n >= (size_t(1) << 32) || nc >= (size_t(1) << 32) || nv >= (size_t(1) << 32))
        return set_err(err, errlen, "too many spheres, circles or vertices"), SMB_ERR_ARG;
    // Shapes, as batch::validate (batch.rs:323-338).
    if (n && (!a->center || !a->expanded || !a->radius || !a->status || !a->nb_off))
        return set_err(err, errlen, "missing sphere arrays"), SMB_ERR_ARG;
    if (n && !csr_ok(a->nb_off, n, a->nb_off[n])) return set_err(err, errlen, "malformed neighbour CSR"), SMB_ERR_ARG;
    if (nc && (!a->circle || !a->cb_off || !csr_ok(a->cb_off, nc, a->cb_off[nc])))
        return set_err(err, errlen, "malformed circle tables"), SMB_ERR_ARG;
    if (nv && !a->vertex) return set_err(err, errlen, "missing vertices"), SMB_ERR_ARG;
    size_t nb_items = n ? a->nb_off[n] : 0, cb_items = nc ? a->cb_off[nc] : 0;
    for (size_t i = 0; i < nb_items; i++)
        if (a->nb_items[i] >= n) return set_err(err, errlen, "neighbour index out of range"), SMB_ERR_ARG;
    for (size_t i = 0; i < cb_items; i++)
        if (a->cb_items[i] >= n) return set_err(err, errlen, "circle blocker index out of range"), SMB_ERR_ARG;
    for (size_t i = 0; i < n; i++)
        if (a->status[i] > 2) return set_err(err, errlen, "bad sphere status"), SMB_ERR_ARG;
    const smb_grid_ref* grids[3] = {&a->sphere_grid, &a->circle_grid, &a->vertex_grid};
    size_t grid_items[3] = {n, nc, nv};
    for (int g = 0; g < 3; g++) {
        const smb_grid_ref* G = grids[g];
        size_t cells = size_t(G->dims[0]) * G->dims[1] * G->dims[2];
        if (!G->dims[0] || !G->dims[1] || !G->dims[2] || !G->starts || !(G->cell > 0))
            return set_err(err, errlen, "malformed cell grid %d", g), SMB_ERR_ARG;
        if (!csr_ok(G->starts, cells, G->n_items) || G->n_items != grid_items[g])
            return set_err(err, errlen, "malformed cell grid %d table", g), SMB_ERR_ARG;
        for (size_t i = 0; i < G->n_items; i++)
            if (G->items[i] >= grid_items[g]) return set_err(err, errlen, "grid %d item out of range", g), SMB_ERR_ARG;
    }
    CK(cudaSetDevice(d->index));
    auto* r = new smb_resident();
    r->dev = d;
    dev_retain(d);
    int rc = SMB_OK;
    auto fail = [&](int code) {
        smb_resident_free(r);
        return code;
    };
    // Spheres: (x, y, z, R) f64 rows, vdW radii, status.
    std::vector<double> sph(4 * n);
    for (size_t i = 0; i < n; i++) {
        sph[4 * i] = a->center[3 * i], sph[4 * i + 1] = a->center[3 * i + 1], sph[4 * i + 2] = a->center[3 * i + 2];
        sph[4 * i + 3] = a->expanded[i];
        for (int k = 0; k < 3; k++) {
            r->lo[k] = i ? std::fmin(r->lo[k], a->center[3 * i + k]) : a->center[3 * i + k];
            r->hi[k] = i ? std::fmax(r->hi[k], a->center[3 * i + k]) : a->center[3 * i + k];
        }
    }
    std::vector<double> circ(12 * nc, 0.0);
    for (size_t c = 0; c < nc; c++)
        for (int k = 0; k < 10; k++) circ[12 * c + k] = a->circle[10 * c + k];
    std::vector<double> vert(4 * nv, 0.0);
    for (size_t v = 0; v < nv; v++)
        for (int k = 0; k < 3; k++) vert[4 * v + k] = a->vertex[3 * v + k];
    auto up = [&](void** dst, const void* src, size_t bytes) -> int {
        int c = dev_alloc(dst, bytes, &r->owned, &r->bytes, err, errlen);
        if (c != SMB_OK) return c;
        if (bytes && src) {
            cudaError_t e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, d->stream);
            if (e != cudaSuccess) return set_err(err, errlen, "upload failed: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
        }
        return SMB_OK;
    };
    DArr& A = r->A;
    A.n = uint32_t(n), A.nc = uint32_t(nc), A.nv = uint32_t(nv);
    {  // rows that ascend let the exact refinement merge instead of search
        bool sorted = true;
        for (size_t i = 0; i < n && sorted; i++)
            for (uint32_t p = a->nb_off[i] + 1; p < a->nb_off[i + 1] && sorted; p++)
                sorted = a->nb_items[p - 1] < a->nb_items[p];
        for (size_t c = 0; c < nc && sorted; c++)
            for (uint32_t p = a->cb_off[c] + 1; p < a->cb_off[c + 1] && sorted; p++)
                sorted = a->cb_items[p - 1] < a->cb_items[p];
        A.flags = (sorted ? DARR_ROWS_SORTED : 0u) | (a->kind != SMB_KIND_SES ? DARR_SPHERES : 0u);
    }
    void* p;
    if ((rc = up(&p, sph.data(), sph.size() * 8)) != SMB_OK) return fail(rc);
    A.sph = static_cast<const double4*>(p);
    if ((rc = up(&p, a->radius, n * 8)) != SMB_OK) return fail(rc);
    A.rvdw = static_cast<const double*>(p);
    if ((rc = up(&p, a->status, n * 4)) != SMB_OK) return fail(rc);
    A.status = static_cast<const uint32_t*>(p);
    std::vector<uint32_t> zero_off(1, 0);
    if ((rc = up(&p, n ? a->nb_off : zero_off.data(), (n + 1) * 4)) != SMB_OK) return fail(rc);
    A.nb_off = static_cast<const uint32_t*>(p);
    if ((rc = up(&p, a->nb_items, nb_items * 4)) != SMB_OK) return fail(rc);
    A.nb_items = static_cast<const uint32_t*>(p);
    if ((rc = up(&p, circ.data(), circ.size() * 8)) != SMB_OK) return fail(rc);
    A.circ = static_cast<const double*>(p);
    if ((rc = up(&p, nc ? a->cb_off : zero_off.data(), (nc + 1) * 4)) != SMB_OK) return fail(rc);
    A.cb_off = static_cast<const uint32_t*>(p);
    if ((rc = up(&p, a->cb_items, cb_items * 4)) != SMB_OK) return fail(rc);
    A.cb_items = static_cast<const uint32_t*>(p);
    if ((rc = up(&p, vert.data(), vert.size() * 8)) != SMB_OK) return fail(rc);
    A.vert = static_cast<const double4*>(p);
    DGrid* dg[3] = {&A.gs, &A.gc, &A.gv};
    for (int g = 0; g < 3; g++) {
        const smb_grid_ref* G = grids[g];
        DGrid& D = *dg[g];
        D.ox = G->origin[0], D.oy = G->origin[1], D.oz = G->origin[2], D.cell = G->cell;
        D.dx = G->dims[0], D.dy = G->dims[1], D.dz = G->dims[2];
        size_t cells = size_t(G->dims[0]) * G->dims[1] * G->dims[2];
        if ((rc = up(&p, G->starts, (cells + 1) * 4)) != SMB_OK) return fail(rc);
        D.starts = static_cast<const uint32_t*>(p);
        if ((rc = up(&p, G->items, G->n_items * 4)) != SMB_OK) return fail(rc);
        D.items = static_cast<const uint32_t*>(p);
    }
    A.max_expanded = a->max_expanded, A.rho_max = a->rho_max, A.probe = a->probe;
    set_lattice(r->L, lat, a->probe, a->kind);
    cudaError_t e = cudaStreamSynchronize(d->stream);
    if (e != cudaSuccess) {
        set_err(err, errlen, "upload failed: %s", cudaGetErrorString(e));
        return fail(SMB_ERR_CUDA);
    }
    *out = r;
    return SMB_OK;
}

static void destroy_resident(smb_resident* r) {
    if (r->gone.exchange(true)) return;
    smb_device* d = r->dev;
    cudaSetDevice(d->index);
    cudaStreamSynchronize(d->stream);
    for (void* p : r->owned) mem_free(p);
    if (r->keys) mem_free(r->keys);
    delete r;
    dev_release(d);
}

void smb_resident_free(smb_resident* r) {
    if (!r) return;
    r->freed.store(true);
    if (r->refs.load() == 0) destroy_resident(r);
}

size_t smb_resident_bytes(const smb_resident* r) { return r ? r->bytes : 0; }

int smb_classify(smb_resident* r, size_t* touched, size_t* surface, char* err, size_t errlen) {
    if (!r) return SMB_ERR_ARG;
    smb_device* d = r->dev;
    CK(cudaSetDevice(d->index));
    cudaStream_t s = d->stream;
    const DLat& L = r->L;
    if (r->keys) mem_free(r->keys);
    r->keys = nullptr;
    r->n_bricks = 0;
    r->classified = false;
    if (r->A.n == 0) {
        if (touched) *touched = 0;
        if (surface) *surface = 0;
        r->classified = true;
        return SMB_OK;
    }
    // Box of all bricks any sphere can touch: brick_of is monotone, so the
    // extreme centres with the largest radius bound every sphere's range.
    BrickBox box{};
    double rr = r->A.max_expanded + CLASSIFY_EPS, bh = double(L.b) * L.h;
    double ncell = 1;
    for (int k = 0; k < 3; k++) {
        double lo = std::floor((r->lo[k] - rr) / bh), hi = std::floor((r->hi[k] + rr) / bh);
        if (!(std::fabs(lo) < double(KEY_BIAS) && std::fabs(hi) < double(KEY_BIAS)))
            return set_err(err, errlen, "coordinates too far from the origin for grid spacing %g", L.h), SMB_ERR_RANGE;
        box.lo[k] = (long long)lo;
        box.n[k] = uint32_t(hi - lo + 1);
        ncell *= double(box.n[k]);
    }
    if (ncell > double(1u << 31))
        return set_err(err, errlen, "brick grid of %.0f bricks exceeds the dense classification limit", ncell), SMB_ERR_RANGE;
    uint32_t nb = uint32_t(ncell);
    DBuf flags, list, surf, cells, tiles, tot, errbuf;
    auto cleanup = [&] {
        flags.release(), list.release(), surf.release(), cells.release(), tiles.release(), tot.release(), errbuf.release();
    };
    int rc;
    if ((rc = flags.reserve(size_t(nb) * 4, err, errlen)) || (rc = list.reserve(size_t(nb) * 4, err, errlen)) ||
        (rc = surf.reserve(size_t(nb) * 4, err, errlen)) || (rc = cells.reserve(size_t(nb) * 4, err, errlen)) ||
        (rc = tiles.reserve(size_t(scan_tiles_needed(nb)) * 8, err, errlen)) || (rc = tot.reserve(16, err, errlen)) ||
        (rc = errbuf.reserve(16, err, errlen))) {
        cleanup();
        return rc;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    cudaMemsetAsync(flags.p, 0, size_t(nb) * 4, s);
    cudaMemsetAsync(surf.p, 0, size_t(nb) * 4, s);
    cudaMemsetAsync(errbuf.p, 0, 16, s);
    launch_mark_touched(r->A, L, box, flags.as<uint32_t>(), errbuf.as<int>(), s);
    launch_scan(flags.as<uint32_t>(), nb, nullptr, list.as<uint32_t>(), tiles.as<unsigned long long>(),
                tot.as<unsigned long long>(), s);
    unsigned long long n_touched = 0;
    int kerr = 0;
    cudaMemcpyAsync(&n_touched, tot.p, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&kerr, errbuf.p, 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess || kerr) {
        cleanup();
        if (e != cudaSuccess) return set_err(err, errlen, "classification failed: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
        return set_err(err, errlen, "coordinates too far from the origin for grid spacing %g", L.h), SMB_ERR_RANGE;
    }
    launch_classify_bricks(r->A, L, box, list.as<uint32_t>(), uint32_t(n_touched), surf.as<uint32_t>(), s);
    launch_scan(surf.as<uint32_t>(), nb, nullptr, cells.as<uint32_t>(), tiles.as<unsigned long long>(),
                tot.as<unsigned long long>(), s);
    unsigned long long n_surface = 0;
    cudaMemcpyAsync(&n_surface, tot.p, 8, cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && n_surface) e = mem_alloc(reinterpret_cast<void**>(&r->keys), n_surface * sizeof(int4));
    if (e == cudaSuccess) launch_cells_to_keys(box, cells.as<uint32_t>(), uint32_t(n_surface), r->keys, s);
    cudaEventRecord(e1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cleanup();
    if (e != cudaSuccess) return set_err(err, errlen, "classification failed: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    r->classify_ms = ms;
    r->n_touched = n_touched;
    r->n_bricks = uint32_t(n_surface);
    r->classified = true;
    if (touched) *touched = n_touched;
    if (surface) *surface = n_surface;
    return SMB_OK;
}

int smb_resident_bricks(const smb_resident* r, int32_t* out, size_t cap) {
    if (!r || !r->classified) return SMB_ERR_STATE;
    cudaSetDevice(r->dev->index);
    size_t n = r->n_bricks < cap ? r->n_bricks : cap;
    std::vector<int4> k(n);
    if (n && cudaMemcpy(k.data(), r->keys, n * sizeof(int4), cudaMemcpyDeviceToHost) != cudaSuccess) return SMB_ERR_CUDA;
    for (size_t i = 0; i < n; i++) out[3 * i] = k[i].x, out[3 * i + 1] = k[i].y, out[3 * i + 2] = k[i].z;
    return SMB_OK;
}

int smb_batch_new(smb_resident* r, smb_batch** out, char* err, size_t errlen) {
    if (!r || !out) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    CK(cudaSetDevice(r->dev->index));
    auto* b = new smb_batch();
    b->res = r;
    r->refs.fetch_add(1);
    for (auto& ev : b->ev) cudaEventCreate(&ev);
    {
        smb_device* d = r->dev;
        std::lock_guard<std::mutex> g(d->hint_mu);
        if (d->hint.warps && d->hint.b == r->L.b && d->hint.h == r->L.h && d->hint.probe == r->A.probe)
            b->caps = d->hint.caps, b->gather_warps = d->hint.warps;
    }
    *out = b;
    return SMB_OK;
}

void smb_batch_free(smb_batch* b) {
    if (!b) return;
    cudaSetDevice(b->res->dev->index);
    cudaStreamSynchronize(b->res->dev->stream);
    for (DBuf* p : b->bufs()) p->release();
    for (auto& ev : b->ev) cudaEventDestroy(ev);
    smb_resident* r = b->res;
    delete b;
    if (r->refs.fetch_sub(1) == 1 && r->freed.load()) destroy_resident(r);
}

int smb_run(smb_resident* r, size_t first, size_t count, smb_batch* b, smb_batch_times* times, char* err,
            size_t errlen) {
    if (!r || !b || b->res != r) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    if (!r->classified) return set_err(err, errlen, "smb_classify must run first"), SMB_ERR_STATE;
    if (first > r->n_bricks || count > r->n_bricks - first) return set_err(err, errlen, "brick range"), SMB_ERR_ARG;
    smb_device* d = r->dev;
    CK(cudaSetDevice(d->index));
    cudaStream_t s = d->stream;
    const DLat& L = r->L;
    b->n = uint32_t(count);
    b->first = first;
    b->refined = false;
    b->refined_exact = false;
    b->n_work = 0;
    b->n_edges = b->n_tris = 0;
    b->ids_words = 0;
    if (count == 0) {
        if (times) *times = smb_batch_times{};
        return SMB_OK;
    }
    const int4* keys = r->keys + first;
    const size_t nsub = count * 8;
    b->window_ok = false;
    int rc;
    if ((rc = b->rec.reserve(nsub * REC_WORDS * 4, err, errlen)) || (rc = b->sampled.reserve(nsub * 4, err, errlen)) ||
        (rc = b->work.reserve(nsub * 4, err, errlen)) || (rc = b->retry_a.reserve(nsub * 4, err, errlen)) ||
        (rc = b->retry_b.reserve(nsub * 4, err, errlen)) ||
        (rc = b->values.reserve(count * size_t(L.spb) * 4, err, errlen)) ||
        (rc = b->tiles.reserve(size_t(scan_tiles_needed(uint32_t(nsub))) * 8, err, errlen)) ||
        (rc = b->totals.reserve(64, err, errlen)) || (rc = b->counters.reserve(CNT_N * 8, err, errlen)) ||
        (rc = b->mc_counts.reserve(count * 8, err, errlen)) || (rc = b->edge_off.reserve(count * 4 + 4, err, errlen)) ||
        (rc = b->tri_off.reserve(count * 4 + 4, err, errlen)) || (rc = b->x_window.reserve(nsub, err, errlen)) ||
        (b->record_features && (rc = b->w_feats.reserve(count * size_t(L.spb) * 4, err, errlen))))
        return rc;
    b->have_features = false;
    cudaEventRecord(b->ev[0], s);
    launch_substates(r->A, L, keys, uint32_t(count), b->rec.as<uint32_t>(), b->sampled.as<uint32_t>(), s);
    launch_scan(b->sampled.as<uint32_t>(), uint32_t(nsub), nullptr, b->work.as<uint32_t>(),
                b->tiles.as<unsigned long long>(), b->totals.as<unsigned long long>(), s);
    cudaEventRecord(b->ev[1], s);
    unsigned long long n_work = 0;
    cudaMemcpyAsync(&n_work, b->totals.p, 8, cudaMemcpyDeviceToHost, s);
    CK(cudaStreamSynchronize(s));
    b->n_work = uint32_t(n_work);

    // (b) gather, with list memory grown and shared-memory caps raised as
    // needed (bit-identical results at any capacity).
    GatherCaps caps = b->caps;
    unsigned long long cnt[CNT_N];
    size_t want_ids = std::max<size_t>(b->ids.cap / 4, size_t(n_work) * 1024),
           want_pack = std::max<size_t>(b->pack.cap / 16, size_t(n_work) * 512);
    for (int attempt = 0;; attempt++) {
        if ((rc = b->ids.reserve(want_ids * 4, err, errlen)) || (rc = b->pack.reserve(want_pack * 16, err, errlen)))
            return rc;
        CK(cudaMemsetAsync(b->counters.p, 0, CNT_N * 8, s));
        GatherOut O{b->rec.as<uint32_t>(), b->ids.as<uint32_t>(), b->pack.as<uint4>(), b->retry_a.as<uint32_t>(),
                    b->counters.as<unsigned long long>(), b->ids.cap / 4, b->pack.cap / 16, ~0ull, nullptr,
                    b->x_window.as<uint8_t>()};
        cudaError_t e = launch_gather(r->A, L, keys, b->work.as<uint32_t>(), uint32_t(n_work), O, caps, b->gather_warps, s);
        if (e != cudaSuccess) return set_err(err, errlen, "gather launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
        CK(cudaMemcpyAsync(cnt, b->counters.p, CNT_N * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (cnt[CNT_NOMEM] && attempt < 4) {
            want_ids = size_t(cnt[CNT_IDS]) + size_t(cnt[CNT_IDS]) / 4 + 1024;
            want_pack = size_t(cnt[CNT_PACK]) + size_t(cnt[CNT_PACK]) / 4 + 1024;
            continue;
        }
        if (cnt[CNT_NOMEM]) return set_err(err, errlen, "candidate list memory could not be sized"), SMB_ERR_MEMORY;
        // Sub-blocks over the shared-memory caps: again with larger caps, one
        // warp per block, until every list fits.
        GatherCaps big = caps;
        DBuf* from = &b->retry_a;
        DBuf* to = &b->retry_b;
        unsigned long long pending = cnt[CNT_OVERFLOW];
        while (pending) {
            big.near *= 2, big.s *= 2, big.c *= 2, big.v *= 2;
            if (gather_smem_bytes(big) > size_t(d->smem_optin))
                return set_err(err, errlen, "a sub-block's candidate lists exceed shared memory"), SMB_ERR_MEMORY;
            CK(cudaMemsetAsync(b->counters.as<unsigned long long>() + CNT_OVERFLOW, 0, 8, s));
            GatherOut O2 = O;
            O2.retry = to->as<uint32_t>();
            e = launch_gather(r->A, L, keys, from->as<uint32_t>(), uint32_t(pending), O2, big, 1, s);
            if (e != cudaSuccess) return set_err(err, errlen, "gather launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
            CK(cudaMemcpyAsync(cnt, b->counters.p, CNT_N * 8, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            if (cnt[CNT_NOMEM]) break;
            pending = cnt[CNT_OVERFLOW];
            std::swap(from, to);
        }
        if (cnt[CNT_NOMEM] && attempt < 4) {
            want_ids = size_t(cnt[CNT_IDS]) + size_t(cnt[CNT_IDS]) / 4 + 1024;
            want_pack = size_t(cnt[CNT_PACK]) + size_t(cnt[CNT_PACK]) / 4 + 1024;
            continue;
        }
        if (cnt[CNT_NOMEM]) return set_err(err, errlen, "candidate list memory could not be sized"), SMB_ERR_MEMORY;
        break;
    }
    b->ids_words = size_t(cnt[CNT_IDS]);
    b->window_ok = true;
    b->max_pack = uint32_t(cnt[CNT_MAXPACK]);
    b->pack_units = cnt[CNT_PACK];
    {
        // Caps for the next run of this batch: the list sizes seen, with an
        // eighth to spare, rounded to 16; warps per block so that a block's
        // scratch stays near 64 KB (several blocks per SM).
        auto up = [](unsigned long long v) { return std::max(32, int((v + v / 8 + 16 + 15) / 16 * 16)); };
        GatherCaps next{up(cnt[CNT_MAXNN]), up(cnt[CNT_MAXNS]), up(cnt[CNT_MAXNC]), up(cnt[CNT_MAXNV])};
        size_t per = gather_smem_bytes(next);
        if (per <= size_t(d->smem_optin)) {
            b->caps = next;
            b->gather_warps = int(std::max<size_t>(1, std::min<size_t>(8, size_t(65536) / per)));
            std::lock_guard<std::mutex> g(d->hint_mu);
            d->hint.h = L.h, d->hint.b = L.b, d->hint.probe = r->A.probe;
            d->hint.caps = b->caps, d->hint.warps = b->gather_warps;
        }
    }
    cudaEventRecord(b->ev[2], s);

    // (c) sampling.
    if (size_t(b->max_pack) * 16 > size_t(d->smem_optin))
        return set_err(err, errlen, "a sub-block's candidates (%u x 16 bytes) exceed shared memory", b->max_pack),
               SMB_ERR_MEMORY;
    const size_t small = b->s_region ? b->s_region : SAMPLE_REGION;
    if (size_t(b->max_pack) * 16 > small && (rc = b->s_list.reserve(size_t(n_work) * 4 + 4, err, errlen)))
        return rc;
    cudaError_t e = launch_sample(L, keys, b->work.as<uint32_t>(), uint32_t(n_work), b->rec.as<uint32_t>(),
                                  b->pack.as<uint4>(), b->max_pack, b->values.as<float>(),
                                  b->counters.as<unsigned long long>(), b->use_tma, false, s, nullptr,
                                  size_t(b->max_pack) * 16 > small ? b->s_list.as<uint32_t>() : nullptr, small,
                                  b->ids.as<uint32_t>(), b->record_features ? b->w_feats.as<uint32_t>() : nullptr);
    if (e != cudaSuccess) return set_err(err, errlen, "sample launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    b->have_features = b->record_features;
    cudaEventRecord(b->ev[3], s);

    // (d) marching cubes: counts, offsets, fill.
    e = launch_mc(L, uint32_t(count), b->values.as<float>(), b->rec.as<uint32_t>(), b->mc_counts.as<uint32_t>(), nullptr,
                  nullptr, nullptr, nullptr, nullptr, false, s);
    if (e != cudaSuccess) return set_err(err, errlen, "mc launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    unsigned long long* tot = b->totals.as<unsigned long long>();
    launch_scan(b->mc_counts.as<uint32_t>(), uint32_t(count), b->edge_off.as<uint32_t>(), nullptr,
                b->tiles.as<unsigned long long>(), tot + 1, s);
    launch_scan(b->mc_counts.as<uint32_t>() + count, uint32_t(count), b->tri_off.as<uint32_t>(), nullptr,
                b->tiles.as<unsigned long long>(), tot + 2, s);
    unsigned long long t2[3];
    CK(cudaMemcpyAsync(t2, tot, 24, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpyAsync(cnt, b->counters.p, CNT_N * 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (cnt[CNT_TIMEOUT]) return set_err(err, errlen, "a bounded wait for a bulk copy gave up"), SMB_ERR_TIMEOUT;
    b->n_edges = size_t(t2[1]);
    b->n_tris = size_t(t2[2]);
    if (b->n_edges >= (size_t(1) << 32) || b->n_tris >= (size_t(1) << 32))
        return set_err(err, errlen, "batch too large for 32-bit offsets"), SMB_ERR_MEMORY;
    uint32_t ne32 = uint32_t(b->n_edges), nt32 = uint32_t(b->n_tris);
    CK(cudaMemcpyAsync(b->edge_off.as<uint32_t>() + count, &ne32, 4, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b->tri_off.as<uint32_t>() + count, &nt32, 4, cudaMemcpyHostToDevice, s));
    if ((rc = b->edges.reserve(b->n_edges * 4, err, errlen)) || (rc = b->edge_vals.reserve(b->n_edges * 8, err, errlen)) ||
        (rc = b->tris.reserve(b->n_tris * 12, err, errlen)))
        return rc;
    e = launch_mc(L, uint32_t(count), b->values.as<float>(), b->rec.as<uint32_t>(), nullptr, b->edge_off.as<uint32_t>(),
                  b->tri_off.as<uint32_t>(), b->edges.as<uint32_t>(), b->edge_vals.as<float2>(), b->tris.as<uint32_t>(),
                  true, s);
    if (e != cudaSuccess) return set_err(err, errlen, "mc launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    cudaEventRecord(b->ev[4], s);
    CK(cudaStreamSynchronize(s));
    if (times) {
        float t[4];
        for (int k = 0; k < 4; k++) cudaEventElapsedTime(&t[k], b->ev[k], b->ev[k + 1]);
        times->substates = t[0], times->gather = t[1], times->sample = t[2], times->mc = t[3];
        times->total = double(t[0]) + t[1] + t[2] + t[3];
    }
    return SMB_OK;
}

int smb_resident_set_refinement(smb_resident* r, char* err, size_t errlen) {
    if (!r) return set_err(err, errlen, "null resident"), SMB_ERR_ARG;
    // RefineRef (batch.rs:133-150; field/gpu.rs:207-221): h as an f32 pair,
    // TOL, MAX_ITER and MAX_BISECT of mesh/extract.rs:29-35.
    r->rc.h_hi = float(r->L.h);
    r->rc.h_lo = float(r->L.h - double(r->rc.h_hi));
    r->rc.tol = float(1e-5);
    r->rc.max_iter = 8;
    r->rc.max_bisect = 64;
    r->refine_ready = true;
    return SMB_OK;
}

// Lanes per edge in the f32 refinement: a warp when the sub-blocks' lists
// average 16 KiB or more (the lane loops over them diverge most), else 8.
static int refine_group(const smb_batch* b) {
    if (b->r_group) return b->r_group;
    return b->n_work && double(b->pack_units) * 16.0 >= 16384.0 * double(b->n_work) ? 32 : 8;
}

// Lanes per edge in the exact refinement: a warp for lists of 16 KiB or
// more on average, else a lane (short f64 lists gain less from groups than
// the edges lose from running one at a time).
static int exact_group(const smb_batch* b) {
    if (b->x_group) return b->x_group;
    return refine_group(b) == 32 ? 32 : 1;
}

// One refinement-kernel pass over the sampled sub-blocks of the last run:
// plain (linear start), warm (the MLP's starts: features, MLP, then the
// refinement from them) or the feature pass alone (FEATURES: the rows'
// features into e_x, evals = 1 marks the edges covered).
enum { PASS_PLAIN = 0, PASS_WARM = 1, PASS_FEATURES = 2 };
static int refine_pass(smb_resident* r, smb_batch* b, int pass, const smb_mlp* mlp, double* ms, char* err,
                       size_t errlen, bool count = false) {
    if (!r || !b || b->res != r) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    if (!r->refine_ready) return set_err(err, errlen, "smb_resident_set_refinement must run first"), SMB_ERR_STATE;
    smb_device* d = r->dev;
    if (pass == PASS_WARM && (!mlp || mlp_device(mlp) != d))
        return set_err(err, errlen, "the MLP must live on the resident's device"), SMB_ERR_ARG;
    if (pass != PASS_PLAIN && !b->have_features)
        return set_err(err, errlen, "the last run did not record the nearest features (smb_batch_record_features)"),
               SMB_ERR_STATE;
    CK(cudaSetDevice(d->index));
    cudaStream_t s = d->stream;
    size_t ne = b->n_edges;
    int rc;
    if ((rc = b->e_t.reserve(ne * 4, err, errlen)) || (rc = b->e_feat.reserve(ne * 4, err, errlen)) ||
        (rc = b->e_q.reserve(ne * 12, err, errlen)) || (rc = b->e_evals.reserve(ne * 4, err, errlen)))
        return rc;
    if ((pass == PASS_FEATURES && (rc = b->e_x.reserve(ne * 4 * 32, err, errlen))) ||
        (pass == PASS_WARM && (rc = b->w_start.reserve(ne * 8, err, errlen))))
        return rc;
    b->refined = false;
    b->refined_exact = false;
    if (ms) *ms = 0;
    if (ne == 0 || b->n_work == 0) {
        if (ne) CK(cudaMemsetAsync(b->e_evals.p, 0, ne * 4, s));
        CK(cudaStreamSynchronize(s));
        b->refined = pass != PASS_FEATURES;
        return SMB_OK;
    }
    const size_t cand = size_t(b->max_pack) * 16 + 64;
    const int mode = pass == PASS_WARM ? REFINE_WARM : REFINE_PLAIN;
    size_t smem = 0;
    launch_refine(r->A, r->L, r->rc, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0,
                  nullptr, nullptr, nullptr, nullptr, cand, mode, nullptr, nullptr, d->info.multiprocessors,
                  d->smem_optin, s, &smem);
    if (smem > size_t(d->smem_optin))
        return set_err(err, errlen, "a sub-block's candidates exceed shared memory for refinement"), SMB_ERR_MEMORY;
    const uint32_t nw = b->n_work;
    if ((rc = b->item_counts.reserve(size_t(nw) * 4, err, errlen)) ||
        (rc = b->item_off.reserve(size_t(nw) * 4 + 4, err, errlen)) ||
        (rc = b->item_edges.reserve(ne * 4, err, errlen)) ||
        (rc = b->tiles.reserve(size_t(scan_tiles_needed(nw)) * 8, err, errlen)) ||
        (rc = b->x_ovf.reserve(size_t(nw) * 4 + 8, err, errlen)))
        return rc;
    cudaEventRecord(b->ev[4], s);
    CK(cudaMemsetAsync(b->e_evals.p, 0, ne * 4, s));
    unsigned long long* cnt = b->counters.as<unsigned long long>();
    CK(cudaMemsetAsync(cnt + CNT_TIMEOUT, 0, 8, s));
    CK(cudaMemsetAsync(cnt + CNT_MAXITEM, 0, 8, s));
    if (count) CK(cudaMemsetAsync(cnt + CNT_OPS, 0, 8, s));
    launch_item_edges(r->L, b->work.as<uint32_t>(), nw, b->rec.as<uint32_t>(), b->edge_off.as<uint32_t>(),
                      b->edges.as<uint32_t>(), b->item_counts.as<uint32_t>(), b->item_off.as<uint32_t>(),
                      b->item_edges.as<uint32_t>(), b->tiles.as<unsigned long long>(),
                      b->totals.as<unsigned long long>() + 3, cnt, s);
    if (pass == PASS_FEATURES) {
        launch_warm_features(r->A, r->L, r->rc, r->keys + b->first, b->work.as<uint32_t>(), nw, b->rec.as<uint32_t>(),
                             b->edges.as<uint32_t>(), b->edge_vals.as<float2>(), b->item_off.as<uint32_t>(),
                             b->item_edges.as<uint32_t>(), b->values.as<float>(), b->w_feats.as<uint32_t>(),
                             b->e_x.as<float>(), ne, d->info.multiprocessors, s);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(s));
        return SMB_OK;
    }
    if (pass == PASS_WARM)
        CK(launch_warm_starts(r->A, r->L, r->rc, r->keys + b->first, b->work.as<uint32_t>(), nw, b->rec.as<uint32_t>(),
                              b->edges.as<uint32_t>(), b->edge_vals.as<float2>(), b->item_off.as<uint32_t>(),
                              b->item_edges.as<uint32_t>(), b->values.as<float>(), b->w_feats.as<uint32_t>(),
                              mlp_dev(mlp), mlp_use(mlp), b->w_start.as<float2>(), cnt, ne, d->info.multiprocessors,
                              s));
    cudaError_t e = launch_refine(r->A, r->L, r->rc, r->keys + b->first, b->work.as<uint32_t>(), b->rec.as<uint32_t>(),
                                  b->ids.as<uint32_t>(), b->edges.as<uint32_t>(), b->edge_vals.as<float2>(),
                                  b->item_off.as<uint32_t>(), b->item_edges.as<uint32_t>(), nw,
                                  b->e_t.as<float>(), b->e_feat.as<uint32_t>(), b->e_q.as<float>(),
                                  b->e_evals.as<uint32_t>(), cand, mode,
                                  pass == PASS_WARM ? b->w_start.as<float2>() : nullptr, cnt, d->info.multiprocessors,
                                  d->smem_optin, s, nullptr, nullptr, b->x_ovf.as<uint32_t>(), b->r_region,
                                  refine_group(b), count);
    if (e != cudaSuccess) return set_err(err, errlen, "refine launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    cudaEventRecord(b->ev[5], s);
    CK(cudaStreamSynchronize(s));
    unsigned long long timeouts = 0;
    CK(cudaMemcpy(&timeouts, cnt + CNT_TIMEOUT, 8, cudaMemcpyDeviceToHost));
    if (timeouts) return set_err(err, errlen, "tensor-core wait timed out in %llu tiles", timeouts), SMB_ERR_CUDA;
    float t = 0;
    cudaEventElapsedTime(&t, b->ev[4], b->ev[5]);
    if (ms) *ms = t;
    b->refined = true;
    return SMB_OK;
}

int smb_refine(smb_resident* r, smb_batch* b, double* ms, char* err, size_t errlen) {
    return refine_pass(r, b, PASS_PLAIN, nullptr, ms, err, errlen);
}

int smb_batch_count_refine_ops(smb_batch* b, const smb_mlp* mlp, unsigned long long* ops, char* err,
                               size_t errlen) {
    if (!b || !ops) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    int rc = refine_pass(b->res, b, mlp ? PASS_WARM : PASS_PLAIN, mlp, nullptr, err, errlen, true);
    if (rc) return rc;
    CK(cudaMemcpy(ops, b->counters.as<unsigned long long>() + CNT_OPS, 8, cudaMemcpyDeviceToHost));
    return SMB_OK;
}

int smb_refine_warm(smb_resident* r, smb_batch* b, const smb_mlp* mlp, double* ms, char* err, size_t errlen) {
    if (!mlp) return refine_pass(r, b, PASS_PLAIN, nullptr, ms, err, errlen);
    return refine_pass(r, b, PASS_WARM, mlp, ms, err, errlen);
}

int smb_batch_record_features(smb_batch* b, int on) {
    if (!b) return SMB_ERR_ARG;
    b->record_features = on != 0;
    return SMB_OK;
}

int smb_batch_sample_features(const smb_batch* b, uint32_t* out) {
    if (!b || !out) return SMB_ERR_ARG;
    if (!b->have_features) return SMB_ERR_STATE;
    const size_t n = size_t(b->n) * size_t(b->res->L.spb);
    if (n && cudaMemcpy(out, b->w_feats.p, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return SMB_ERR_CUDA;
    return SMB_OK;
}

int smb_batch_edge_features(smb_resident* r, smb_batch* b, float* features, uint8_t* covered, char* err,
                            size_t errlen) {
    int rc = refine_pass(r, b, PASS_FEATURES, nullptr, nullptr, err, errlen);
    if (rc != SMB_OK) return rc;
    const size_t ne = b->n_edges;
    if (!ne) return SMB_OK;
    if (features) std::memset(features, 0, ne * 4 * 32);
    if (covered) std::memset(covered, 0, ne);
    if (b->n_work == 0) return SMB_OK;
    // Rows (the items' edge lists) to marching-cubes edge order.
    unsigned long long n_rows = 0;
    CK(cudaMemcpy(&n_rows, b->totals.as<unsigned long long>() + 3, 8, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> k_of(n_rows);
    std::vector<float> x(n_rows * 32);
    if (n_rows) {
        CK(cudaMemcpy(k_of.data(), b->item_edges.p, n_rows * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(x.data(), b->e_x.p, n_rows * 4 * 32, cudaMemcpyDeviceToHost));
    }
    for (size_t e = 0; e < n_rows; e++) {
        const size_t k = k_of[e];
        if (k >= ne) return set_err(err, errlen, "edge list entry out of range"), SMB_ERR_STATE;
        if (features) std::memcpy(features + k * 32, x.data() + e * 32, 32 * 4);
        if (covered) covered[k] = 1;
    }
    return SMB_OK;
}

}  // extern "C"

namespace smb {

int resident_from_device(smb_device* d, DevArrangement& D, const smb_lattice_ref* lat, smb_resident** out, char* err,
                         size_t errlen) {
    if (!d || !lat || !out) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *out = nullptr;
    if (lat->brick < 4 || lat->brick > 32 || lat->brick % 2)
        return set_err(err, errlen, "brick must be even and 4..32, got %u", lat->brick), SMB_ERR_ARG;
    if (!(lat->spacing >= 0.01) || !std::isfinite(lat->spacing))
        return set_err(err, errlen, "grid spacing must be at least 0.01"), SMB_ERR_ARG;
    auto* r = new smb_resident();
    r->dev = d;
    dev_retain(d);
    r->A = D.A;
    r->owned.swap(D.owned);
    r->bytes = D.bytes;
    D.bytes = 0;
    for (int k = 0; k < 3; k++) r->lo[k] = D.lo[k], r->hi[k] = D.hi[k];
    set_lattice(r->L, lat, D.A.probe, SMB_KIND_SES);
    r->xa = ExactAttr{D.orig, D.circle_ij, D.vertex_atoms, 0.0};
    *out = r;
    return SMB_OK;
}

void resident_set_exact_tmin(smb_resident* r, double t_min) {
    r->xa.t_min = t_min;
    r->exact_ready = true;
}

}  // namespace smb

extern "C" {

int smb_resident_set_exact(smb_resident* r, const uint32_t* orig, const uint32_t* circle_ij, size_t n_circles,
                           const uint32_t* vertex_atoms, size_t n_vertices, double t_min, char* err, size_t errlen) {
    if (!r) return set_err(err, errlen, "null resident"), SMB_ERR_ARG;
    const size_t n = r->A.n;
    if ((n && !orig) || (n_circles && !circle_ij) || (n_vertices && !vertex_atoms))
        return set_err(err, errlen, "missing attribute tables"), SMB_ERR_ARG;
    if (n_circles != r->A.nc || n_vertices != r->A.nv)
        return set_err(err, errlen, "attribute tables do not match the arrangement (%zu circles, %zu vertices)",
                       size_t(r->A.nc), size_t(r->A.nv)),
               SMB_ERR_ARG;
    for (size_t i = 0; i < 2 * n_circles; i++)
        if (circle_ij[i] >= n) return set_err(err, errlen, "circle atom out of range"), SMB_ERR_ARG;
    for (size_t i = 0; i < 3 * n_vertices; i++)
        if (vertex_atoms[i] >= n) return set_err(err, errlen, "vertex atom out of range"), SMB_ERR_ARG;
    if (!(t_min >= 0.0 && t_min < 0.5)) return set_err(err, errlen, "t_min must be in [0, 0.5)"), SMB_ERR_ARG;
    smb_device* d = r->dev;
    CK(cudaSetDevice(d->index));
    const void* src[3] = {orig, circle_ij, vertex_atoms};
    const size_t bytes[3] = {n * 4, n_circles * 8, n_vertices * 12};
    const uint32_t* dst[3] = {nullptr, nullptr, nullptr};
    for (int k = 0; k < 3; k++) {
        void* p = nullptr;
        int rc = dev_alloc(&p, bytes[k], &r->owned, &r->bytes, err, errlen);
        if (rc != SMB_OK) return rc;
        if (bytes[k]) CK(cudaMemcpyAsync(p, src[k], bytes[k], cudaMemcpyHostToDevice, d->stream));
        dst[k] = static_cast<const uint32_t*>(p);
    }
    CK(cudaStreamSynchronize(d->stream));
    r->xa = ExactAttr{dst[0], dst[1], dst[2], t_min};
    r->exact_ready = true;
    return SMB_OK;
}

// The exact refinement of the last run's crossing edges (mask: only the
// edges k with mask[k] != 0; their results into the vertex buffers).
static int exact_pass(smb_resident* r, smb_batch* b, const uint8_t* mask, char* err, size_t errlen,
                      bool count = false) {
    smb_device* d = r->dev;
    cudaStream_t s = d->stream;
    const size_t ne = b->n_edges;
    const uint32_t nw = b->n_work;
    int rc;
    const size_t slab = exact_slab_bytes(d->info.multiprocessors);
    if ((rc = b->x_ovf.reserve(size_t(nw) * 4 + 8, err, errlen)) || (rc = b->x_slab.reserve(slab, err, errlen)) ||
        (rc = b->item_counts.reserve(size_t(nw) * 4, err, errlen)) ||
        (rc = b->item_off.reserve(size_t(nw) * 4 + 4, err, errlen)) ||
        (rc = b->item_edges.reserve(ne * 4, err, errlen)) ||
        (rc = b->tiles.reserve(size_t(scan_tiles_needed(nw)) * 8, err, errlen)))
        return rc;
    b->x_block_items = 0;
    if (!ne || !nw) return SMB_OK;
    unsigned long long* cnt = b->counters.as<unsigned long long>();
    CK(cudaMemsetAsync(cnt + CNT_MAXITEM, 0, 8, s));
    launch_item_edges(r->L, b->work.as<uint32_t>(), nw, b->rec.as<uint32_t>(), b->edge_off.as<uint32_t>(),
                      b->edges.as<uint32_t>(), b->item_counts.as<uint32_t>(), b->item_off.as<uint32_t>(),
                      b->item_edges.as<uint32_t>(), b->tiles.as<unsigned long long>(),
                      b->totals.as<unsigned long long>() + 3, cnt, s, nullptr, nullptr, mask, true);
    ExactOut out{b->x_pos.as<float>(), b->x_nrm.as<float>(), b->x_atom.as<uint32_t>(), b->x_patch.as<uint8_t>(),
                 b->x_t.as<float>(), b->x_evals.as<uint32_t>()};
    cudaError_t e = launch_refine_exact(r->A, r->L, r->xa, r->keys + b->first, b->work.as<uint32_t>(),
                                        b->edges.as<uint32_t>(), b->edge_vals.as<float2>(), b->item_off.as<uint32_t>(),
                                        b->item_edges.as<uint32_t>(), nw, out, b->x_ovf.as<uint32_t>(),
                                        b->x_slab.as<unsigned char>(), slab, cnt, d->info.multiprocessors,
                                        b->x_region, s, count, exact_group(b), b->rec.as<uint32_t>(), b->x_hint,
                                        b->window_ok ? b->ids.as<uint32_t>() : nullptr,
                                        b->window_ok ? b->x_window.as<uint8_t>() : nullptr);
    if (e != cudaSuccess) return set_err(err, errlen, "exact refine launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    uint32_t n_block = 0;
    CK(cudaMemcpyAsync(&n_block, b->x_ovf.p, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    b->x_block_items = n_block;
    return SMB_OK;
}

static int reserve_vertices(smb_batch* b, char* err, size_t errlen) {
    const size_t ne = b->n_edges;
    int rc;
    if ((rc = b->x_pos.reserve(ne * 12, err, errlen)) || (rc = b->x_nrm.reserve(ne * 12, err, errlen)) ||
        (rc = b->x_atom.reserve(ne * 4, err, errlen)) || (rc = b->x_patch.reserve(ne, err, errlen)) ||
        (rc = b->x_t.reserve(ne * 4, err, errlen)) || (rc = b->x_evals.reserve(ne * 4, err, errlen)) ||
        (rc = b->x_sum.reserve(16, err, errlen)))
        return rc;
    return SMB_OK;
}

int smb_refine_exact(smb_resident* r, smb_batch* b, double* ms, char* err, size_t errlen) {
    if (!r || !b || b->res != r) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    if (!r->exact_ready) return set_err(err, errlen, "smb_resident_set_exact must run first"), SMB_ERR_STATE;
    smb_device* d = r->dev;
    CK(cudaSetDevice(d->index));
    cudaStream_t s = d->stream;
    int rc;
    if ((rc = reserve_vertices(b, err, errlen))) return rc;
    b->refined_exact = false;
    b->refined = false;
    b->x_exact_edges = b->n_edges;
    if (ms) *ms = 0;
    cudaEventRecord(b->ev[4], s);
    if (b->n_edges) CK(cudaMemsetAsync(b->x_evals.p, 0, b->n_edges * 4, s));
    if ((rc = exact_pass(r, b, nullptr, err, errlen))) return rc;
    cudaEventRecord(b->ev[5], s);
    CK(cudaStreamSynchronize(s));
    float t = 0;
    cudaEventElapsedTime(&t, b->ev[4], b->ev[5]);
    if (ms) *ms = t;
    b->refined_exact = true;
    return SMB_OK;
}

int smb_batch_count_exact_ops(smb_batch* b, unsigned long long* ops, char* err, size_t errlen) {
    if (!b || !ops) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    smb_resident* r = b->res;
    if (!b->refined_exact || b->x_exact_edges != b->n_edges)
        return set_err(err, errlen, "smb_refine_exact must run first"), SMB_ERR_STATE;
    CK(cudaSetDevice(r->dev->index));
    int rc = exact_pass(r, b, nullptr, err, errlen, true);
    if (rc) return rc;
    CK(cudaMemcpy(ops, b->counters.as<unsigned long long>() + CNT_OPS, 8, cudaMemcpyDeviceToHost));
    return SMB_OK;
}

int smb_place_fast(smb_resident* r, smb_batch* b, double* ms, char* err, size_t errlen) {
    if (!r || !b || b->res != r) return set_err(err, errlen, "bad arguments"), SMB_ERR_ARG;
    if (!b->refined) return set_err(err, errlen, "smb_refine must run first"), SMB_ERR_STATE;
    if (!r->exact_ready) return set_err(err, errlen, "smb_resident_set_exact must run first"), SMB_ERR_STATE;
    smb_device* d = r->dev;
    CK(cudaSetDevice(d->index));
    cudaStream_t s = d->stream;
    const size_t ne = b->n_edges;
    int rc;
    if ((rc = reserve_vertices(b, err, errlen)) || (rc = b->x_mask.reserve(ne, err, errlen))) return rc;
    b->refined_exact = false;
    if (ms) *ms = 0;
    cudaEventRecord(b->ev[4], s);
    ExactOut out{b->x_pos.as<float>(), b->x_nrm.as<float>(), b->x_atom.as<uint32_t>(), b->x_patch.as<uint8_t>(),
                 b->x_t.as<float>(), b->x_evals.as<uint32_t>()};
    unsigned long long* marked = b->x_sum.as<unsigned long long>();
    cudaError_t e = launch_place_fast(r->A, r->L, r->xa, r->keys + b->first, b->n, b->edge_off.as<uint32_t>(),
                                      b->edges.as<uint32_t>(), b->edge_vals.as<float2>(), ne, b->e_t.as<float>(),
                                      b->e_feat.as<uint32_t>(), b->e_q.as<float>(), b->e_evals.as<uint32_t>(), out,
                                      b->x_mask.as<uint8_t>(), marked, s);
    if (e != cudaSuccess) return set_err(err, errlen, "placement launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    unsigned long long n_marked = 0;
    CK(cudaMemcpyAsync(&n_marked, marked, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    b->x_exact_edges = size_t(n_marked);
    if (n_marked && (rc = exact_pass(r, b, b->x_mask.as<uint8_t>(), err, errlen))) return rc;
    cudaEventRecord(b->ev[5], s);
    CK(cudaStreamSynchronize(s));
    float t = 0;
    cudaEventElapsedTime(&t, b->ev[4], b->ev[5]);
    if (ms) *ms = t;
    b->refined_exact = true;
    return SMB_OK;
}

int smb_batch_vertices(const smb_batch* b, float* positions, float* normals, uint32_t* atoms, uint8_t* patches,
                       float* t, uint32_t* evals) {
    if (!b || !b->refined_exact) return SMB_ERR_STATE;
    cudaSetDevice(b->res->dev->index);
    const size_t ne = b->n_edges;
    if (!ne) return SMB_OK;
    cudaStream_t s = b->res->dev->stream;
    bool ok = true;
    if (positions) ok &= cudaMemcpyAsync(positions, b->x_pos.p, ne * 12, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    if (normals) ok &= cudaMemcpyAsync(normals, b->x_nrm.p, ne * 12, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    if (atoms) ok &= cudaMemcpyAsync(atoms, b->x_atom.p, ne * 4, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    if (patches) ok &= cudaMemcpyAsync(patches, b->x_patch.p, ne, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    if (t) ok &= cudaMemcpyAsync(t, b->x_t.p, ne * 4, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    if (evals) ok &= cudaMemcpyAsync(evals, b->x_evals.p, ne * 4, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok &= cudaStreamSynchronize(s) == cudaSuccess;
    return ok ? SMB_OK : SMB_ERR_CUDA;
}

int smb_batch_exact_summary(const smb_batch* b, unsigned long long* evaluations, unsigned long long* host_edges,
                            unsigned long long* exact_edges) {
    if (!b || !b->refined_exact) return SMB_ERR_STATE;
    smb_device* d = b->res->dev;
    if (cudaSetDevice(d->index) != cudaSuccess) return SMB_ERR_CUDA;
    unsigned long long out[2] = {0, 0};
    if (b->n_edges) {
        unsigned long long* sum = b->x_sum.as<unsigned long long>();
        if (!sum || launch_exact_summary(b->x_evals.as<uint32_t>(), b->n_edges, sum, d->info.multiprocessors,
                                         d->stream) != cudaSuccess ||
            cudaMemcpyAsync(out, sum, 16, cudaMemcpyDeviceToHost, d->stream) != cudaSuccess ||
            cudaStreamSynchronize(d->stream) != cudaSuccess)
            return SMB_ERR_CUDA;
    }
    if (evaluations) *evaluations = out[0];
    if (host_edges) *host_edges = out[1];
    if (exact_edges) *exact_edges = b->x_exact_edges;
    return SMB_OK;
}

int smb_batch_set_refine_region(smb_batch* b, size_t bytes) {
    if (!b || (bytes && (bytes < 1024 || bytes > 56 * 1024))) return SMB_ERR_ARG;
    b->r_region = bytes;
    return SMB_OK;
}

int smb_batch_set_sample_region(smb_batch* b, size_t bytes) {
    if (!b || (bytes && bytes < 1024)) return SMB_ERR_ARG;
    b->s_region = bytes;
    return SMB_OK;
}

int smb_batch_set_exact_hint(smb_batch* b, int mode) {
    if (!b || mode < 0 || mode > 2) return SMB_ERR_ARG;
    b->x_hint = mode;
    return SMB_OK;
}

int smb_batch_set_exact_group(smb_batch* b, int lanes) {
    if (!b || (lanes != 0 && lanes != 1 && lanes != 8 && lanes != 32)) return SMB_ERR_ARG;
    b->x_group = lanes;
    return SMB_OK;
}

int smb_batch_set_refine_group(smb_batch* b, int lanes) {
    if (!b || (lanes != 0 && lanes != 8 && lanes != 32)) return SMB_ERR_ARG;
    b->r_group = lanes;
    return SMB_OK;
}

int smb_batch_set_exact_region(smb_batch* b, size_t bytes) {
    if (!b || bytes < 1024 || bytes > 48 * 1024) return SMB_ERR_ARG;
    b->x_region = bytes;
    return SMB_OK;
}

int smb_batch_edges(const smb_batch* b, float* t, uint32_t* feat, float* closest, uint32_t* evals) {
    if (!b || !b->refined) return SMB_ERR_STATE;
    cudaSetDevice(b->res->dev->index);
    size_t ne = b->n_edges;
    if (!ne) return SMB_OK;
    bool ok = true;
    if (t) ok &= cudaMemcpy(t, b->e_t.p, ne * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (feat) ok &= cudaMemcpy(feat, b->e_feat.p, ne * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (closest) ok &= cudaMemcpy(closest, b->e_q.p, ne * 12, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (evals) ok &= cudaMemcpy(evals, b->e_evals.p, ne * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    return ok ? SMB_OK : SMB_ERR_CUDA;
}

size_t smb_batch_bricks(const smb_batch* b) { return b ? b->n : 0; }

unsigned long long smb_kernel_launches(void) { return kernel_launches(); }

int smb_batch_info_get(const smb_batch* b, smb_batch_info* out) {
    if (!b || !out) return SMB_ERR_ARG;
    out->bricks = b->n;
    out->sampled_subblocks = b->n_work;
    out->ids_words = b->ids_words;
    out->max_pack_units = b->max_pack;
    out->edges = b->n_edges;
    out->triangles = b->n_tris;
    out->classify_ms = b->res->classify_ms;
    out->touched = b->res->n_touched;
    out->resident_bytes = b->res->bytes;
    unsigned long long c[CNT_N] = {0};
    if (b->counters.p) {
        cudaSetDevice(b->res->dev->index);
        if (cudaMemcpy(c, b->counters.p, sizeof c, cudaMemcpyDeviceToHost) != cudaSuccess) return SMB_ERR_CUDA;
    }
    out->pack_units = c[CNT_PACK];
    out->exact_block_items = b->x_block_items;
    out->gather_caps[0] = uint32_t(b->caps.near), out->gather_caps[1] = uint32_t(b->caps.s);
    out->gather_caps[2] = uint32_t(b->caps.c), out->gather_caps[3] = uint32_t(b->caps.v);
    out->gather_warps = uint32_t(b->gather_warps);
    return SMB_OK;
}

int smb_batch_count_ops(smb_batch* b, unsigned long long* ops, unsigned long long* samples, char* err, size_t errlen) {
    if (!b) return SMB_ERR_ARG;
    smb_resident* r = b->res;
    smb_device* d = r->dev;
    CK(cudaSetDevice(d->index));
    cudaStream_t s = d->stream;
    CK(cudaMemsetAsync(b->counters.as<unsigned long long>() + CNT_OPS, 0, 16, s));
    cudaError_t e = launch_sample(r->L, r->keys + b->first, b->work.as<uint32_t>(), b->n_work, b->rec.as<uint32_t>(),
                                  b->pack.as<uint4>(), b->max_pack, b->values.as<float>(),
                                  b->counters.as<unsigned long long>(), true, true, s);
    if (e != cudaSuccess) return set_err(err, errlen, "count launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    unsigned long long c[CNT_N];
    CK(cudaMemcpyAsync(c, b->counters.p, sizeof c, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (ops) *ops = c[CNT_OPS];
    if (samples) *samples = c[CNT_OWNED];
    return SMB_OK;
}

int smb_batch_records(const smb_batch* b, uint32_t* out) {
    if (!b || !out) return SMB_ERR_ARG;
    cudaSetDevice(b->res->dev->index);
    return cudaMemcpy(out, b->rec.p, size_t(b->n) * 8 * REC_WORDS * 4, cudaMemcpyDeviceToHost) == cudaSuccess
               ? SMB_OK : SMB_ERR_CUDA;
}

int smb_batch_values(const smb_batch* b, float* out) {
    if (!b || !out) return SMB_ERR_ARG;
    cudaSetDevice(b->res->dev->index);
    return cudaMemcpy(out, b->values.p, size_t(b->n) * b->res->L.spb * 4, cudaMemcpyDeviceToHost) == cudaSuccess
               ? SMB_OK : SMB_ERR_CUDA;
}

size_t smb_batch_ids_words(const smb_batch* b) { return b ? b->ids_words : 0; }

int smb_batch_ids(const smb_batch* b, uint32_t* out) {
    if (!b || !out) return SMB_ERR_ARG;
    if (!b->ids_words) return SMB_OK;
    cudaSetDevice(b->res->dev->index);
    return cudaMemcpy(out, b->ids.p, b->ids_words * 4, cudaMemcpyDeviceToHost) == cudaSuccess ? SMB_OK : SMB_ERR_CUDA;
}

int smb_batch_mc_counts(const smb_batch* b, size_t* edges, size_t* triangles) {
    if (!b) return SMB_ERR_ARG;
    if (edges) *edges = b->n_edges;
    if (triangles) *triangles = b->n_tris;
    return SMB_OK;
}

int smb_batch_mc(const smb_batch* b, uint32_t* edge_off, uint32_t* edges, float* edge_vals, uint32_t* tri_off,
                 uint32_t* tris) {
    if (!b) return SMB_ERR_ARG;
    cudaSetDevice(b->res->dev->index);
    size_t n = b->n;
    bool ok = true;
    if (edge_off) ok &= cudaMemcpy(edge_off, b->edge_off.p, (n + 1) * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (tri_off) ok &= cudaMemcpy(tri_off, b->tri_off.p, (n + 1) * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (edges && b->n_edges) ok &= cudaMemcpy(edges, b->edges.p, b->n_edges * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (edge_vals && b->n_edges)
        ok &= cudaMemcpy(edge_vals, b->edge_vals.p, b->n_edges * 8, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (tris && b->n_tris) ok &= cudaMemcpy(tris, b->tris.p, b->n_tris * 12, cudaMemcpyDeviceToHost) == cudaSuccess;
    return ok ? SMB_OK : SMB_ERR_CUDA;
}

}  // extern "C"
