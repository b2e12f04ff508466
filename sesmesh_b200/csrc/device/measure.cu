// Validation, components, area and volume, and triangle grouping of an
// assembled mesh on the device: validate_with, components_with,
// triangle_area_volume and group_by_component (crates/sesmesh/src/mesh/
// mod.rs:91-330, 638-700; mesh/post.rs:14-32), with the host mesher's
// results bit for bit (host/mesher.cpp defects, components_and_group):
//   * defects: non-finite positions, normals not of unit length, triangle
//     indices out of range (then nothing else is counted), repeated or zero-
//     area triangles, undirected edges not used exactly once in each
//     direction, duplicate triangles;
//   * union-find linking the larger root to the smaller, so every root is
//     its component's smallest vertex whatever the order of the links;
//     components numbered by their root;
//   * area and volume in f64 (the first vertex as origin) summed per
//     component within fixed 16,384-triangle chunks in triangle order, then
//     over the chunks in chunk order: the host's operations in the host's
//     order;
//   * Euler characteristic from the distinct undirected edges;
//   * triangles regrouped by component, relative order kept.
// Edges and duplicate triangles are found with open-addressing hash tables
// in HBM (linear probing, half full at most); the order-dependent parts
// (the sums, the regrouping) follow the host's order exactly.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../host/mesher.hpp"
#include "../runtime.hpp"
#include "kernels.hpp"
#include "measure.hpp"

namespace smb {
namespace {

constexpr uint64_t EMPTY = ~0ull;
constexpr uint32_t SUM_CHUNK = 1u << 14;  // triangles per area/volume chunk, as the host

__device__ __forceinline__ uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
    x ^= x >> 30;
    x *= 0xbf58476d1ce4e5b9ull;
    x ^= x >> 27;
    x *= 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ void block_add(unsigned long long* dst, unsigned long long v) {
    // Warp sums, one atomic per warp.
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// base[key] += 1 for the active threads of a warp, one atomic per distinct
// key (the counts of a large component's members come from one address).
// All threads of the warp call it.
__device__ __forceinline__ void add_by_key(unsigned long long* base, uint32_t key, bool active) {
    const unsigned m = __ballot_sync(0xffffffffu, active);
    if (!active) return;
    const unsigned peers = __match_any_sync(m, key);
    if (int(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&base[key], (unsigned long long)__popc(peers));
}

__global__ void k_vertex_checks(const float* pos, const float* nrm, uint32_t nv, unsigned long long* bad) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long b = 0;
    if (v < nv) {
        const float* p = pos + 3 * size_t(v);
        if (!(isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]))) b++;
        if (nrm) {
            const float* q = nrm + 3 * size_t(v);
            float len2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
            if (!(isfinite(q[0]) && isfinite(q[1]) && isfinite(q[2]) && fabsf(len2 - 1.0f) < 1e-3f)) b++;
        }
    }
    block_add(bad, b);
}

__device__ __forceinline__ void area_volume(const float* pos, const uint32_t* t, const double o[3], double& a,
                                            double& v) {
    double p[3][3];
    for (int q = 0; q < 3; q++)
        for (int k = 0; k < 3; k++) p[q][k] = double(pos[3 * size_t(t[q]) + k]) - o[k];
    double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    a = 0.5 * sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    double x[3] = {p[1][1] * p[2][2] - p[1][2] * p[2][1], p[1][2] * p[2][0] - p[1][0] * p[2][2],
                   p[1][0] * p[2][1] - p[1][1] * p[2][0]};
    v = (p[0][0] * x[0] + p[0][1] * x[1] + p[0][2] * x[2]) / 6.0;
}

__global__ void k_index_checks(const uint32_t* tris, uint32_t nt, uint32_t nv, unsigned long long* oob) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long b = 0;
    if (t < nt) {
        const uint32_t* T = tris + 3 * size_t(t);
        b = (T[0] >= nv || T[1] >= nv || T[2] >= nv) ? 1 : 0;
    }
    block_add(oob, b);
}

__global__ void k_triangle_checks(const float* pos, const uint32_t* tris, uint32_t nt, unsigned long long* bad) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long b = 0;
    if (t < nt) {
        const uint32_t* T = tris + 3 * size_t(t);
        double o[3] = {double(pos[0]), double(pos[1]), double(pos[2])};
        double a, v;
        area_volume(pos, T, o, a, v);
        b = (T[0] == T[1] || T[1] == T[2] || T[0] == T[2] || a == 0.0) ? 1 : 0;
    }
    block_add(bad, b);
}

// Undirected edge (lo, hi) of every triangle side a -> b: counts of uses
// a < b (low half) and a > b (high half).
__global__ void k_edge_insert(const uint32_t* tris, uint32_t nt, unsigned long long* keys, unsigned long long* cnt,
                              uint64_t mask) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const uint32_t* T = tris + 3 * size_t(t);
    for (int k = 0; k < 3; k++) {
        uint32_t a = T[k], b = T[(k + 1) % 3];
        uint64_t key = (uint64_t(min(a, b)) << 32) | max(a, b);
        for (uint64_t s = mix64(key) & mask, probes = 0; probes <= mask; s = (s + 1) & mask, probes++) {
            unsigned long long prev = atomicCAS(&keys[s], EMPTY, key);
            if (prev == EMPTY || prev == key) {
                atomicAdd(&cnt[s], a < b ? 1ull : (1ull << 32));
                break;
            }
        }
    }
}

__global__ void k_edge_check(const unsigned long long* keys, const unsigned long long* cnt, uint64_t cap,
                             unsigned long long* bad) {
    uint64_t s = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    unsigned long long b = 0;
    if (s < cap && keys[s] != EMPTY) b = (cnt[s] == ((1ull << 32) | 1ull)) ? 0 : 1;
    block_add(bad, b);
}

// Duplicate triangles (equal vertex sets): the first of each set takes a
// slot, every later one counts.
__global__ void k_duplicates(const uint32_t* tris, uint32_t nt, uint32_t* slots, uint64_t mask,
                             unsigned long long* bad) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long b = 0;
    if (t < nt) {
        const uint32_t* T = tris + 3 * size_t(t);
        uint32_t a0 = T[0], a1 = T[1], a2 = T[2], x;
        if (a0 > a1) x = a0, a0 = a1, a1 = x;
        if (a1 > a2) x = a1, a1 = a2, a2 = x;
        if (a0 > a1) x = a0, a0 = a1, a1 = x;
        uint64_t h = mix64((uint64_t(a0) << 32 | a1) ^ mix64(a2));
        for (uint64_t s = h & mask, probes = 0; probes <= mask; s = (s + 1) & mask, probes++) {
            uint32_t prev = atomicCAS(&slots[s], 0u, t + 1);
            if (prev == 0) break;
            const uint32_t* U = tris + 3 * size_t(prev - 1);
            uint32_t b0 = U[0], b1 = U[1], b2 = U[2];
            if (b0 > b1) x = b0, b0 = b1, b1 = x;
            if (b1 > b2) x = b1, b1 = b2, b2 = x;
            if (b0 > b1) x = b0, b0 = b1, b1 = x;
            if (a0 == b0 && a1 == b1 && a2 == b2) {
                b = 1;
                break;
            }
        }
    }
    block_add(bad, b);
}

// Parent pointers are read from L2 (__ldcg): other blocks change them with
// atomics, and a stale L1 copy could make a root look like a root forever.
// Links only ever lower a parent, so every retry makes progress; the loops
// are bounded all the same and report a failure (the host then measures).
constexpr uint32_t UF_LIMIT = 1u << 22;

__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t x, unsigned long long* fail) {
    for (uint32_t it = 0; it < UF_LIMIT; it++) {
        uint32_t p = __ldcg(parent + x);
        if (p == x) return x;
        uint32_t g = __ldcg(parent + p);
        if (g != p) atomicCAS(&parent[x], p, g);
        x = g;
    }
    atomicAdd(fail, 1ull);
    return x;
}

__device__ __forceinline__ void uf_unite(uint32_t* parent, uint32_t a, uint32_t b, unsigned long long* fail) {
    for (uint32_t it = 0; it < UF_LIMIT; it++) {
        uint32_t ra = uf_find(parent, a, fail), rb = uf_find(parent, b, fail);
        if (ra == rb) return;
        uint32_t lo = min(ra, rb), hi = max(ra, rb);
        if (atomicCAS(&parent[hi], hi, lo) == hi) return;
    }
    atomicAdd(fail, 1ull);
}

__global__ void k_uf_init(uint32_t* parent, uint32_t nv) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < nv) parent[v] = v;
}

__global__ void k_uf_link(const uint32_t* tris, uint32_t nt, uint32_t* parent, unsigned long long* fail) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const uint32_t* T = tris + 3 * size_t(t);
    uf_unite(parent, T[0], T[1], fail);
    uf_unite(parent, T[0], T[2], fail);
}

// Roots (a component's smallest vertex) and the root flags for numbering.
__global__ void k_uf_roots(uint32_t* parent, uint32_t nv, uint32_t* is_root, unsigned long long* fail) {
    uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    uint32_t r = uf_find(parent, v, fail);
    is_root[v] = r == v ? 1u : 0u;
}

__global__ void k_component_ids(const uint32_t* parent, const uint32_t* cid_of_root, uint32_t nv, uint32_t* id,
                                unsigned long long* comp_vertices) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t c = 0;
    if (v < nv) {
        uint32_t r = parent[v];
        for (uint32_t it = 0; it < UF_LIMIT && parent[r] != r; it++) r = parent[r];
        c = cid_of_root[r];
        id[v] = c;
    }
    add_by_key(comp_vertices, c, v < nv);
}

// Per chunk of SUM_CHUNK triangles, in order: each component's triangle
// count and area and volume partial sums (sequential, the host's order).
struct Partial {
    uint32_t comp, chunk;
    unsigned long long t;
    double a, v;
};

// Segments of the triangles sorted by component (stably: triangle order
// within a component): a new segment where the component or the 16,384-
// triangle chunk changes.  flag[p] = 1 at a segment's first position.
__global__ void k_segment_flags(const uint32_t* comp, const uint32_t* perm, uint32_t nt, uint32_t* flag) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nt) return;
    flag[p] = (p == 0 || comp[p] != comp[p - 1] || (perm[p] / SUM_CHUNK) != (perm[p - 1] / SUM_CHUNK)) ? 1u : 0u;
}

// Area and volume of each triangle, in the component-sorted order.
__global__ void k_triangle_area_volume(const float* pos, const uint32_t* tris, const uint32_t* perm, uint32_t nt,
                                       double* ta, double* tv) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nt) return;
    const double o[3] = {double(pos[0]), double(pos[1]), double(pos[2])};
    double a, v;
    area_volume(pos, tris + 3 * size_t(perm[p]), o, a, v);
    ta[p] = a, tv[p] = v;
}

// Thread per segment: its triangles' area and volume summed in triangle
// order (one (component, chunk) partial of the host's sums).
constexpr int SEG_WARPS = 4;     // warps (segments) per block of k_segment_partials
constexpr uint32_t SEG_STAGE = 256;  // values per array a warp stages at a time

// A warp per (component, chunk) segment: the lanes stage the segment's
// per-triangle areas and volumes in shared memory, coalesced, and lane 0
// sums them in triangle order (the host's order of additions).
__global__ void __launch_bounds__(32 * SEG_WARPS) k_segment_partials(const double* ta, const double* tv,
                                                                   const uint32_t* comp, const uint32_t* perm,
                                                                   uint32_t nt, const uint32_t* start, uint32_t n_seg,
                                                                   Partial* out, uint32_t* seg_comp) {
    __shared__ double sa[SEG_WARPS][SEG_STAGE], sv[SEG_WARPS][SEG_STAGE];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t s = blockIdx.x * SEG_WARPS + warp;
    if (s >= n_seg) return;
    const uint32_t p0 = start[s], p1 = s + 1 < n_seg ? start[s + 1] : nt;
    double a = 0.0, v = 0.0;
    for (uint32_t base = p0; base < p1; base += SEG_STAGE) {
        const uint32_t cnt = min(SEG_STAGE, p1 - base);
        for (uint32_t u = lane; u < cnt; u += 32) sa[warp][u] = ta[base + u], sv[warp][u] = tv[base + u];
        __syncwarp();
        if (lane == 0)
            for (uint32_t u = 0; u < cnt; u++) a += sa[warp][u], v += sv[warp][u];
        __syncwarp();
    }
    if (lane == 0) {
        out[s] = Partial{comp[p0], perm[p0] / SUM_CHUNK, (unsigned long long)(p1 - p0), a, v};
        seg_comp[s] = comp[p0];
    }
}

// Partials in (component, chunk) order (sorted_idx: their order, or null
// for the identity): each component sums its chunks in chunk order (the
// host's order).
__global__ void k_component_sums(const Partial* parts, const uint32_t* sorted_idx, uint32_t n_parts,
                                 const uint32_t* first, uint32_t n_comp, unsigned long long* tris_out, double* area,
                                 double* volume) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_comp) return;
    unsigned long long t = 0;
    double a = 0.0, v = 0.0;
    for (uint32_t i = first[c]; i < first[c + 1]; i++) {
        const Partial& p = parts[sorted_idx ? sorted_idx[i] : i];
        t += p.t, a += p.a, v += p.v;
    }
    tris_out[c] = t, area[c] = a, volume[c] = v;
}

__global__ void k_first_of_component(const uint32_t* sorted_comp, uint32_t n, uint32_t* first, uint32_t n_comp) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n) return;
    // first[c] = the first sorted index with component >= c.
    uint32_t lo = i == 0 ? 0 : sorted_comp[i - 1] + 1, hi = i == n ? n_comp : sorted_comp[i];
    for (uint32_t c = lo; c <= hi && c <= n_comp; c++) first[c] = i;
}

__global__ void k_triangle_keys(const uint32_t* tris, uint32_t nt, const uint32_t* id, uint32_t* key,
                                uint32_t* idx) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    key[t] = id[tris[3 * size_t(t)]];
    idx[t] = t;
}

__global__ void k_gather_triangles(const uint32_t* tris, const uint32_t* idx, uint32_t nt, uint32_t* out) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const uint32_t* T = tris + 3 * size_t(idx[t]);
    uint32_t* U = out + 3 * size_t(t);
    U[0] = T[0], U[1] = T[1], U[2] = T[2];
}

uint64_t pow2_at_least(uint64_t v) {
    uint64_t p = 1024;
    while (p < v) p <<= 1;
    return p;
}

// extract::assemble (mesh/extract.rs:606-691) on the device.  Packed brick
// keys (lattice.rs:93-96): the bricks must be in ascending packed order.
__device__ __forceinline__ unsigned long long pack_key(long long x, long long y, long long z) {
    const long long bias = 1ll << 20;
    return (unsigned long long)(x + bias) | ((unsigned long long)(y + bias) << 21) |
           ((unsigned long long)(z + bias) << 42);
}

__global__ void k_packed_keys(const int4* keys, uint32_t n, unsigned long long* packed, unsigned long long* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int4 k = keys[i];
    packed[i] = pack_key(k.x, k.y, k.z);
    if (i > 0) {
        const int4 p = keys[i - 1];
        if (pack_key(k.x, k.y, k.z) <= pack_key(p.x, p.y, p.z)) atomicOr(err, 4ull);
    }
}

// Thread per triangle: each corner's (neighbour code, edge id) reference
// resolved to the global vertex index edge_off[target] + position of the
// edge in the target brick's (ascending) edge list.  err |= 1: a reference
// to a missing brick; 2: to an edge without vertex.
__global__ void k_assemble(const unsigned long long* packed, const int4* keys, uint32_t n, const uint32_t* edge_off,
                           const uint32_t* edges, const uint32_t* tri_off, const uint32_t* refs, uint32_t nt,
                           uint32_t* tris, unsigned long long* err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    uint32_t lo = 0, hi = n;  // the brick holding triangle t: tri_off[lo] <= t < tri_off[lo + 1]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tri_off[mid] <= t) lo = mid;
        else hi = mid;
    }
    const int4 key = keys[lo];
    for (int c = 0; c < 3; c++) {
        const uint32_t r = refs[3 * size_t(t) + c], code = r >> 28, id = r & ((1u << 28) - 1);
        uint32_t tb = lo;
        if (code) {
            const unsigned long long want = pack_key((long long)key.x + (code & 1), (long long)key.y + ((code >> 1) & 1),
                                                     (long long)key.z + ((code >> 2) & 1));
            uint32_t a = 0, b = n;
            while (a < b) {
                const uint32_t mid = (a + b) >> 1;
                if (packed[mid] < want) a = mid + 1;
                else b = mid;
            }
            if (a == n || packed[a] != want) {
                atomicOr(err, 1ull);
                tris[3 * size_t(t) + c] = 0;
                continue;
            }
            tb = a;
        }
        uint32_t a = edge_off[tb], b = edge_off[tb + 1];
        const uint32_t e1 = b;
        while (a < b) {
            const uint32_t mid = (a + b) >> 1;
            if (edges[mid] < id) a = mid + 1;
            else b = mid;
        }
        if (a == e1 || edges[a] != id) {
            atomicOr(err, 2ull);
            tris[3 * size_t(t) + c] = 0;
            continue;
        }
        tris[3 * size_t(t) + c] = a;
    }
}

unsigned bits_for(uint32_t n) {
    unsigned b = 1;
    while (b < 32 && (uint64_t(1) << b) <= n) b++;
    return b;
}

#define MCK(call)                                                                          \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            if (msg) *msg = std::string(#call) + ": " + cudaGetErrorString(e_);            \
            return false;                                                                  \
        }                                                                                  \
    } while (0)

}  // namespace

void MeasureScratch::release(bool synced) {
    for (DBuf* b : {&pos, &nrm, &tris, &tris_out, &keys, &cnt, &dup, &parent, &flag, &cid, &id, &counters, &comp_v,
                    &comp_t, &area, &volume, &parts, &pkey, &pidx, &pkey2, &pidx2, &first, &tkey, &tidx,
                    &tkey2, &tidx2, &tiles, &cub, &packed, &err, &tri_a, &tri_v})
        synced ? b->release_synced() : b->release();
    pinned_free(host);
    host = nullptr;
    host_cap = 0;
    pinned_free(words);
    words = nullptr;
}

// The first n counters into page-locked host words, by the device itself.
__global__ void k_read_words(const unsigned long long* src, unsigned long long* dst, int n) {
    if (int(threadIdx.x) < n) dst[threadIdx.x] = src[threadIdx.x];
}

// The measure of a mesh already on the device (pos, nrm: 3 f32 per vertex,
// nrm may be null; tris: 3 u32 per triangle).  Results: comps, *bad, and,
// when there are no defects, each vertex's component into host_comp and the
// regrouped triangles into host_tris (nv and 3 nt words on the host).
static bool measure_core(smb_device* d, const float* pos, const float* nrm, const uint32_t* tris, size_t nv,
                         size_t nt, std::vector<smbh::Component>& comps, size_t* bad, MeasureScratch& S,
                         std::string* msg, uint32_t* host_comp, uint32_t* host_tris) {
    using smbh::Component;
    cudaStream_t s = d->stream;
    if (nv >= (size_t(1) << 31) || nt >= (size_t(1) << 31)) {
        if (msg) *msg = "mesh too large for the device measure";
        return false;
    }
    char e[256];
    auto R = [&](DBuf& b, size_t bytes) { return b.reserve(std::max<size_t>(bytes, 16), e, sizeof e) == 0; };
    const uint64_t ecap = pow2_at_least(uint64_t(nt) * 3 + 16), dcap = pow2_at_least(uint64_t(nt) * 2 + 16);
    if (!R(S.tris_out, nt * 12) ||
        !R(S.keys, ecap * 8) || !R(S.cnt, ecap * 8) || !R(S.dup, dcap * 4) || !R(S.parent, nv * 4) ||
        !R(S.flag, nv * 4) || !R(S.cid, nv * 4) || !R(S.id, nv * 4) || !R(S.counters, 64) ||
        !R(S.tkey, nt * 4) || !R(S.tidx, nt * 4) ||
        !R(S.tkey2, nt * 4) || !R(S.tidx2, nt * 4) || !R(S.tiles, size_t(scan_tiles_needed(uint32_t(std::max(nv, nt)))) * 8 + 64)) {
        if (msg) *msg = std::string("device memory for the measure: ") + e;
        return false;
    }
    unsigned long long* cnt = S.counters.as<unsigned long long>();  // 0 bad, 1 oob, 2 parts, 3 overflow, 4 comps, 5 union-find
    MCK(cudaMemsetAsync(cnt, 0, 64, s));
    if (!S.words && !(S.words = static_cast<unsigned long long*>(pinned_alloc(64)))) {
        if (msg) *msg = "page-locked counter words";
        return false;
    }
    // Counters 0..7 to the host once the main stream gets here (a kernel
    // writes them: a copy would wait behind the vertex copies).
    volatile unsigned long long* W = S.words;
    auto pull = [&]() -> bool {
        k_read_words<<<1, 32, 0, s>>>(cnt, S.words, 8);
        return cudaStreamSynchronize(s) == cudaSuccess;
    };
    auto blocks = [](uint64_t n) { return unsigned((n + 255) / 256); };
    if (nv) k_vertex_checks<<<blocks(nv), 256, 0, s>>>(pos, nrm, uint32_t(nv), cnt);
    if (nt) k_index_checks<<<blocks(nt), 256, 0, s>>>(tris, uint32_t(nt), uint32_t(nv), cnt + 1);
    if (!pull()) {
        if (msg) *msg = "measure checks";
        return false;
    }
    if (W[1]) {  // indices out of range: the host counts one defect more and stops there
        *bad = size_t(W[0] + 1);
        return true;
    }
    if (nt) {
        k_triangle_checks<<<blocks(nt), 256, 0, s>>>(pos, tris, uint32_t(nt), cnt);
        MCK(cudaMemsetAsync(S.keys.p, 0xFF, ecap * 8, s));
        MCK(cudaMemsetAsync(S.cnt.p, 0, ecap * 8, s));
        MCK(cudaMemsetAsync(S.dup.p, 0, dcap * 4, s));
        k_edge_insert<<<blocks(nt), 256, 0, s>>>(tris, uint32_t(nt), S.keys.as<unsigned long long>(),
                                                 S.cnt.as<unsigned long long>(), ecap - 1);
        k_edge_check<<<blocks(ecap), 256, 0, s>>>(S.keys.as<unsigned long long>(), S.cnt.as<unsigned long long>(), ecap,
                                                  cnt);
        k_duplicates<<<blocks(nt), 256, 0, s>>>(tris, uint32_t(nt), S.dup.as<uint32_t>(), dcap - 1, cnt);
    }
    if (!pull()) {
        if (msg) *msg = "measure checks";
        return false;
    }
    const unsigned long long nbad = W[0];
    *bad = size_t(nbad);
    if (nbad) return true;
    // Components.
    uint32_t* parent = S.parent.as<uint32_t>();
    if (nv) {
        k_uf_init<<<blocks(nv), 256, 0, s>>>(parent, uint32_t(nv));
        if (nt) k_uf_link<<<blocks(nt), 256, 0, s>>>(tris, uint32_t(nt), parent, cnt + 5);
        k_uf_roots<<<blocks(nv), 256, 0, s>>>(parent, uint32_t(nv), S.flag.as<uint32_t>(), cnt + 5);
        launch_scan(S.flag.as<uint32_t>(), uint32_t(nv), S.cid.as<uint32_t>(), nullptr,
                    S.tiles.as<unsigned long long>(), cnt + 4, s);
    }
    if (!pull()) {
        if (msg) *msg = "measure components";
        return false;
    }
    const unsigned long long n_comp = W[4], uf_fail = W[5];
    if (uf_fail) {
        if (msg) *msg = "union-find gave up";
        return false;
    }
    const uint32_t nc = uint32_t(n_comp);
    if (!R(S.comp_v, size_t(nc) * 8) || !R(S.comp_t, size_t(nc) * 8) ||
        !R(S.area, size_t(nc) * 8) || !R(S.volume, size_t(nc) * 8) || !R(S.first, (size_t(nc) + 1) * 4)) {
        if (msg) *msg = std::string("device memory for the measure: ") + e;
        return false;
    }
    MCK(cudaMemsetAsync(S.comp_v.p, 0, size_t(nc) * 8 + 8, s));
    uint32_t* id = S.id.as<uint32_t>();
    if (nv) k_component_ids<<<blocks(nv), 256, 0, s>>>(parent, S.cid.as<uint32_t>(), uint32_t(nv), id,
                                                       S.comp_v.as<unsigned long long>());
    // Arrays that are final go back on the copy stream while the main one
    // computes the rest; the end of this function waits for both.
    cudaStream_t cs = d->copy ? d->copy : s;
    auto to_host = [&](void* dst, const void* src, size_t bytes) -> bool {
        if (!bytes) return true;
        if (cs != s) {
            cudaEvent_t ready;
            if (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess) return false;
            const bool ok =
                cudaEventRecord(ready, s) == cudaSuccess && cudaStreamWaitEvent(cs, ready, 0) == cudaSuccess;
            cudaEventDestroy(ready);
            if (!ok) return false;
        }
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, cs) == cudaSuccess;
    };
    struct Join {
        cudaStream_t c;
        ~Join() {
            if (c) cudaStreamSynchronize(c);
        }
    } join{cs != s ? cs : nullptr};
    if (nv && !to_host(host_comp, id, nv * 4)) {
        if (msg) *msg = "component copy";
        return false;
    }
    auto sort_pairs = [&](const uint32_t* kin, uint32_t* kout, const uint32_t* vin, uint32_t* vout, uint32_t n,
                          unsigned bits) -> bool {
        size_t tmp = 0;
        if (cub::DeviceRadixSort::SortPairs(nullptr, tmp, kin, kout, vin, vout, int(n), 0, int(bits), s) !=
            cudaSuccess)
            return false;
        if (!R(S.cub, tmp)) return false;
        return cub::DeviceRadixSort::SortPairs(S.cub.p, tmp, kin, kout, vin, vout, int(n), 0, int(bits), s) ==
               cudaSuccess;
    };
    // Triangles stably sorted by component: the regrouping's order, and the
    // segments of the area/volume sums.
    if (nt) {
        k_triangle_keys<<<blocks(nt), 256, 0, s>>>(tris, uint32_t(nt), id, S.tkey.as<uint32_t>(), S.tidx.as<uint32_t>());
        if (!sort_pairs(S.tkey.as<uint32_t>(), S.tkey2.as<uint32_t>(), S.tidx.as<uint32_t>(), S.tidx2.as<uint32_t>(),
                        uint32_t(nt), bits_for(nc))) {
            if (msg) *msg = "triangle sort failed";
            return false;
        }
        // Triangles regrouped by component, relative order kept.
        k_gather_triangles<<<blocks(nt), 256, 0, s>>>(tris, S.tidx2.as<uint32_t>(), uint32_t(nt),
                                                      S.tris_out.as<uint32_t>());
        if (!to_host(host_tris, S.tris_out.p, nt * 12)) {
            if (msg) *msg = "triangle copy";
            return false;
        }
    }
    // Area and volume: one partial per (component, 16,384-triangle chunk)
    // summed in triangle order, then each component's partials in chunk
    // order (the host's operations in the host's order).  The sorted
    // triangles list the segments in (component, chunk) order.
    unsigned long long n_seg = 0;
    if (nt) {
        uint32_t* flag = S.tkey.as<uint32_t>();   // free once sorted
        uint32_t* start = S.tidx.as<uint32_t>();  // idem
        k_segment_flags<<<blocks(nt), 256, 0, s>>>(S.tkey2.as<uint32_t>(), S.tidx2.as<uint32_t>(), uint32_t(nt), flag);
        launch_scan(flag, uint32_t(nt), nullptr, start, S.tiles.as<unsigned long long>(), cnt + 2, s);
        if (!pull()) {
            if (msg) *msg = "measure segments";
            return false;
        }
        n_seg = W[2];
    }
    const uint32_t np = uint32_t(n_seg);
    if (np) {
        if (!R(S.parts, size_t(np) * sizeof(Partial)) || !R(S.pkey, size_t(np) * 4) || !R(S.tri_a, nt * 8) ||
            !R(S.tri_v, nt * 8)) {
            if (msg) *msg = std::string("device memory for the measure: ") + e;
            return false;
        }
        Partial* parts = S.parts.as<Partial>();
        k_triangle_area_volume<<<blocks(nt), 256, 0, s>>>(pos, tris, S.tidx2.as<uint32_t>(), uint32_t(nt),
                                                          S.tri_a.as<double>(), S.tri_v.as<double>());
        k_segment_partials<<<(np + SEG_WARPS - 1) / SEG_WARPS, 32 * SEG_WARPS, 0, s>>>(
            S.tri_a.as<double>(), S.tri_v.as<double>(),
                                                      S.tkey2.as<uint32_t>(), S.tidx2.as<uint32_t>(), uint32_t(nt),
                                                      S.tidx.as<uint32_t>(), np, parts, S.pkey.as<uint32_t>());
        k_first_of_component<<<blocks(uint64_t(np) + 1), 256, 0, s>>>(S.pkey.as<uint32_t>(), np,
                                                                        S.first.as<uint32_t>(), nc);
        k_component_sums<<<blocks(nc), 256, 0, s>>>(parts, nullptr, np, S.first.as<uint32_t>(), nc,
                                                    S.comp_t.as<unsigned long long>(), S.area.as<double>(),
                                                    S.volume.as<double>());
    } else if (nc) {
        MCK(cudaMemsetAsync(S.comp_t.p, 0, size_t(nc) * 8, s));
        MCK(cudaMemsetAsync(S.area.p, 0, size_t(nc) * 8, s));
        MCK(cudaMemsetAsync(S.volume.p, 0, size_t(nc) * 8, s));
    }
    // Results to the host.
    std::vector<unsigned long long> cv(nc), ct(nc);
    std::vector<double> ca(nc), cvol(nc);
    if (nc) {
        MCK(cudaMemcpyAsync(cv.data(), S.comp_v.p, size_t(nc) * 8, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(ct.data(), S.comp_t.p, size_t(nc) * 8, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(ca.data(), S.area.p, size_t(nc) * 8, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(cvol.data(), S.volume.p, size_t(nc) * 8, cudaMemcpyDeviceToHost, s));
    }
    MCK(cudaStreamSynchronize(s));
    comps.assign(nc, Component());
    size_t start = 0;
    for (uint32_t c = 0; c < nc; c++) {
        Component& C = comps[c];
        C.vertices = size_t(cv[c]);
        C.triangles = size_t(ct[c]);
        C.area = ca[c];
        C.volume = cvol[c];
        // The mesh passed the edge check: every edge is used once in each
        // direction, by two triangles of one component, so the component has
        // 3 T / 2 distinct edges.
        C.euler = int64_t(cv[c]) - int64_t(3 * ct[c] / 2) + int64_t(ct[c]);
        C.first_triangle = start;
        start += C.triangles;
    }
    return true;
}

bool measure_on_device(smb_device* d, smbh::Mesh& m, std::vector<smbh::Component>& comps, size_t* bad,
                       MeasureScratch& S, std::string* msg) {
    cudaStream_t s = d->stream;
    const size_t nv = m.positions.size(), nt = m.triangles.size();
    char e[256];
    auto R = [&](DBuf& b, size_t bytes) { return b.reserve(std::max<size_t>(bytes, 16), e, sizeof e) == 0; };
    if (!R(S.pos, nv * 12) || !R(S.nrm, nv * 12) || !R(S.tris, nt * 12)) {
        if (msg) *msg = std::string("device memory for the measure: ") + e;
        return false;
    }
    MCK(cudaMemcpyAsync(S.pos.p, m.positions.data(), nv * 12, cudaMemcpyHostToDevice, s));
    const bool normals = !m.normals.empty();
    if (normals) MCK(cudaMemcpyAsync(S.nrm.p, m.normals.data(), nv * 12, cudaMemcpyHostToDevice, s));
    MCK(cudaMemcpyAsync(S.tris.p, m.triangles.data(), nt * 12, cudaMemcpyHostToDevice, s));
    m.vertex_component.resize(nv);
    return measure_core(d, S.pos.as<float>(), normals ? S.nrm.as<float>() : nullptr, S.tris.as<uint32_t>(), nv, nt,
                        comps, bad, S, msg, m.vertex_component.data(), reinterpret_cast<uint32_t*>(m.triangles.data()));
}

void* MeasureScratch::staging(size_t bytes) {
    if (bytes <= host_cap) return host;
    pinned_free(host);
    host_cap = 0;
    const size_t want = bytes + bytes / 4;
    host = pinned_alloc(want);
    if (host) host_cap = want;
    return host;
}

int finish_on_device(smb_device* d, const DeviceMesh& in, smbh::MeshRef* out, void** block,
                     std::vector<smbh::Component>& comps, size_t* bad, MeasureScratch& S, std::string* msg,
                     double* ms_assemble) {
    *block = nullptr;
    cudaStream_t s = d->stream;
    const size_t nv = in.n_edges, nt = in.n_tris;
    if (nv >= (size_t(1) << 31) || nt >= (size_t(1) << 31) || in.n_bricks == 0) {
        if (msg) *msg = "mesh too large (or empty) for the device path";
        return 1;
    }
    char e[256];
    auto R = [&](DBuf& b, size_t bytes) { return b.reserve(std::max<size_t>(bytes, 16), e, sizeof e) == 0; };
    if (!R(S.packed, size_t(in.n_bricks) * 8) || !R(S.tris, nt * 12) || !R(S.err, 16)) {
        if (msg) *msg = std::string("device memory for the assembly: ") + e;
        return 1;
    }
    const size_t stage = nv * 33 + nt * 12;
    unsigned char* H = static_cast<unsigned char*>(S.staging(stage));
    if (!H) {
        if (msg) *msg = "page-locked staging memory";
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    auto blocks = [](uint64_t n) { return unsigned((n + 255) / 256); };
    unsigned long long* err = S.err.as<unsigned long long>();
    if (cudaMemsetAsync(err, 0, 8, s) != cudaSuccess) return 1;
    k_packed_keys<<<blocks(in.n_bricks), 256, 0, s>>>(in.keys, uint32_t(in.n_bricks), S.packed.as<unsigned long long>(),
                                                      err);
    if (nt)
        k_assemble<<<blocks(nt), 256, 0, s>>>(S.packed.as<unsigned long long>(), in.keys, uint32_t(in.n_bricks),
                                              in.edge_off, in.edges, in.tri_off, in.tri_refs, uint32_t(nt),
                                              S.tris.as<uint32_t>(), err);
    count_launches(nt ? 2 : 1);
    unsigned long long ferr = 0;
    if (cudaMemcpyAsync(&ferr, err, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        if (msg) *msg = "device assembly failed";
        return 1;
    }
    if (ms_assemble) *ms_assemble = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (ferr) {
        if (msg)
            *msg = (ferr & 4) ? "bricks are not in packed-key order"
                   : (ferr & 1) ? "triangle references an edge of a missing brick"
                                : "triangle references an edge without vertex";
        return 2;
    }
    // Staging layout: positions, normals (12 B each), atoms, components
    // (4 B), patches (1 B) per vertex, then the triangles.
    unsigned char* h_pos = H;
    unsigned char* h_nrm = h_pos + nv * 12;
    unsigned char* h_atom = h_nrm + nv * 12;
    unsigned char* h_comp = h_atom + nv * 4;
    unsigned char* h_patch = h_comp + nv * 4;
    unsigned char* h_tris = h_patch + nv;
    // The vertex arrays go back on the copy stream while the measure's
    // kernels run on the main one (the copies wait for everything the main
    // stream has queued so far); every return below waits for them.
    cudaStream_t cs = d->copy ? d->copy : s;
    struct Join {
        cudaStream_t c;
        ~Join() {
            if (c) cudaStreamSynchronize(c);
        }
    } join{cs != s ? cs : nullptr};
    if (cs != s) {
        cudaEvent_t ready;
        if (cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess) {
            if (msg) *msg = "copy event";
            return 1;
        }
        const bool ok = cudaEventRecord(ready, s) == cudaSuccess && cudaStreamWaitEvent(cs, ready, 0) == cudaSuccess;
        cudaEventDestroy(ready);
        if (!ok) {
            if (msg) *msg = "copy event";
            return 1;
        }
    }
    auto d2h = [&](void* dst, const void* src, size_t bytes) {
        return !bytes || cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, cs) == cudaSuccess;
    };
    if (!d2h(h_pos, in.pos, nv * 12) || !d2h(h_nrm, in.nrm, nv * 12) || !d2h(h_atom, in.atoms, nv * 4) ||
        !d2h(h_patch, in.patches, nv)) {
        if (msg) *msg = "vertex copy";
        return 1;
    }
    if (!measure_core(d, in.pos, in.nrm, S.tris.as<uint32_t>(), nv, nt, comps, bad, S, msg,
                      reinterpret_cast<uint32_t*>(h_comp), reinterpret_cast<uint32_t*>(h_tris)))
        return 1;
    if (*bad) return 0;
    // The staging block becomes the mesh's storage.
    out->pos = reinterpret_cast<const float*>(h_pos);
    out->nrm = reinterpret_cast<const float*>(h_nrm);
    out->atom = reinterpret_cast<const uint32_t*>(h_atom);
    out->comp = reinterpret_cast<const uint32_t*>(h_comp);
    out->patch = reinterpret_cast<const uint8_t*>(h_patch);
    out->tris = reinterpret_cast<const uint32_t*>(h_tris);
    out->nv = nv, out->nt = nt;
    *block = S.host;
    S.host = nullptr, S.host_cap = 0;
    return 0;
}

}  // namespace smb
