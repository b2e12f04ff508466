// sm_100a kernels of the SES mesh stage: brick classification (a), ordered
// candidate gather (b), exact field sampling with TMA-staged candidates (c),
// marching-cubes edge/cell compaction (d).  Host launchers at the end.
//
// Numerics: built with -fmad=false -prec-div=true -prec-sqrt=true
// -ftz=false.  f64 decisions (classification, list membership, list order)
// and f32 sample values follow the CPU back end of sesmesh 1.3.2
// operation by operation, so every output is bit-identical to it.
#include <atomic>
#include <type_traits>
#include <cstdio>

#include "common.cuh"
#include <cstddef>

#include "kernels.hpp"
#include "mlp.cuh"
#include "scan.cuh"
// Global memory (read through the L1), not __constant__: threads of a warp
// read different entries.
#define SMB_MC_QUAL __device__
#include "../mc_table.inc"

namespace smb {

// Feature words (the reference's DeviceEdges encoding, field/gpu.rs:155-179):
// kind << 29 | id.
constexpr uint32_t FEAT_SHIFT_D = 29;

// ---------------------------------------------------------------------------
// Arithmetic self-test: IEEE f32 and f64 operations whose results the host
// recomputes; a build with contracted multiply-adds or approximate division
// or square root fails it.  Eight f32 and four f64 results per pair.
__global__ void k_selftest(const float* a, const float* b, uint32_t* out, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x = a[i], y = b[i];
    float dx = x - y, dy = y * 0.75f - x, dz = x * y - 1.0f;
    float d = sqrtf(dx * dx + dy * dy + dz * dz);
    float r[8] = {x + y, x * y, x / y, sqrtf(fabsf(x)), d, (d - y) / d, fminf(x, y), fabsf(d - fabsf(y))};
    for (int k = 0; k < 8; k++) out[12 * i + k] = __float_as_uint(r[k]);
    double X = double(x) * 1.0000001, Y = double(y) - 0.3;
    double D = X * Y + X, E = sqrt(fabs(X * X + Y * Y - X)), F = X / (Y + 2.5), G = floor(X * 3.7);
    double rr[4] = {D, E, F, G};
    for (int k = 0; k < 4; k++) {
        unsigned long long u = __double_as_longlong(rr[k]);
        out[12 * i + 8 + k] = uint32_t(u ^ (u >> 32));
    }
}

// ---------------------------------------------------------------------------
// Device-wide exclusive scan of u32 values (three passes over tiles).
__global__ void k_scan_tiles(const uint32_t* in, uint32_t n, unsigned long long* tile_sums) {
    __shared__ unsigned long long sh[SCAN_THREADS / 32];
    uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE;
    unsigned long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
        uint64_t i = base + uint64_t(k) * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
    }
    unsigned long long total;
    block_exclusive_scan<SCAN_THREADS>(s, sh, &total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_scan_tile_sums(unsigned long long* tile_sums, uint32_t n_tiles, unsigned long long* total) {
    __shared__ unsigned long long sh[SCAN_THREADS / 32];
    unsigned long long carry = 0;
    for (uint32_t b0 = 0; b0 < n_tiles; b0 += SCAN_THREADS) {
        uint32_t i = b0 + threadIdx.x;
        unsigned long long v = i < n_tiles ? tile_sums[i] : 0, t;
        unsigned long long e = block_exclusive_scan<SCAN_THREADS>(v, sh, &t);
        if (i < n_tiles) tile_sums[i] = carry + e;
        carry += t;
    }
    if (threadIdx.x == 0) *total = carry;
}

// out[i] = exclusive prefix of in; with keep != null, also writes the
// indices i with in[i] != 0 to keep[prefix] (order-preserving compaction).
__global__ void k_scan_apply(const uint32_t* in, uint32_t n, const unsigned long long* tile_sums, uint32_t* out,
                             uint32_t* keep) {
    __shared__ unsigned long long sh[SCAN_THREADS / 32];
    uint64_t base = uint64_t(blockIdx.x) * SCAN_TILE + uint64_t(threadIdx.x) * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    unsigned long long s = 0;
    for (int k = 0; k < SCAN_ITEMS; k++) {
        uint64_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        s += v[k];
    }
    unsigned long long t;
    unsigned long long run = tile_sums[blockIdx.x] + block_exclusive_scan<SCAN_THREADS>(s, sh, &t);
    for (int k = 0; k < SCAN_ITEMS; k++) {
        uint64_t i = base + k;
        if (i < n) {
            if (out) out[i] = uint32_t(run);
            if (keep && v[k]) keep[run] = uint32_t(i);
        }
        run += v[k];
    }
}

// ---------------------------------------------------------------------------
// (a) Classification.
__device__ __forceinline__ long long sat_floor(double v) {
    double f = floor(v);
    if (isnan(f)) return 0;
    if (f <= -9.2e18) return LLONG_MIN;
    if (f >= 9.2e18) return LLONG_MAX;
    return (long long)f;
}

// The structure whose range [off[s], off[s + 1]) holds v (off ascending,
// n + 1 entries).
template <class T>
__device__ __forceinline__ uint32_t structure_of(const T* off, uint32_t n, T v) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (off[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

// lattice::touched_bricks (field/lattice.rs:105-163): every non-contained
// sphere marks the bricks its ball of radius R + CLASSIFY_EPS overlaps, in a
// dense flag grid over the bricks' bounding box.
template <bool MANY>
__global__ void k_mark_touched(DArr A0, DLat L0, BrickBox box0, uint32_t* flags0, int* err0, Scene S,
                               uint32_t n_total) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t st = 0;
    if constexpr (MANY) {
        if (i >= n_total) return;
        st = structure_of(S.sph_off, S.n_struct, i);
        i -= S.sph_off[st];
    }
    const DArr& A = MANY ? S.arr[st] : A0;
    const DLat& L = MANY ? S.lat[st] : L0;
    const BrickBox& box = MANY ? S.box[st] : box0;
    uint32_t* flags = MANY ? flags0 + S.flag_off[st] : flags0;
    int* err = MANY ? S.err + st : err0;
    if (i >= A.n || A.status[i] == STATUS_CONTAINED) return;
    double4 c = A.sph[i];
    double r = c.w + CLASSIFY_EPS;
    double bh = double(L.b) * L.h;
    long long lo[3] = {sat_floor((c.x - r) / bh), sat_floor((c.y - r) / bh), sat_floor((c.z - r) / bh)};
    long long hi[3] = {sat_floor((c.x + r) / bh), sat_floor((c.y + r) / bh), sat_floor((c.z + r) / bh)};
    for (int a = 0; a < 3; a++) {
        if (llabs(lo[a]) >= KEY_BIAS - 1 || llabs(hi[a]) >= KEY_BIAS - 1) {
            atomicExch(err, ERR_KEY_RANGE);
            return;
        }
        if (lo[a] < box.lo[a] || hi[a] > box.lo[a] + (long long)box.n[a] - 1) {
            atomicExch(err, ERR_BOX);
            return;
        }
    }
    for (long long z = lo[2]; z <= hi[2]; z++)
        for (long long y = lo[1]; y <= hi[1]; y++)
            for (long long x = lo[0]; x <= hi[0]; x++)
                flags[((uint64_t(z - box.lo[2]) * box.n[1]) + uint64_t(y - box.lo[1])) * box.n[0] + uint64_t(x - box.lo[0])] = 1;
}

__device__ __forceinline__ void cell_key(const BrickBox& box, uint32_t cell, int k[3]) {
    k[0] = int(box.lo[0] + cell % box.n[0]);
    k[1] = int(box.lo[1] + (cell / box.n[0]) % box.n[1]);
    k[2] = int(box.lo[2] + cell / (box.n[0] * box.n[1]));
}

// lattice::surface_bricks (field/lattice.rs:168-181): the exact f64 test at
// each touched brick's centre, one warp per brick.
template <bool MANY>
__global__ void k_classify_bricks(DArr A0, DLat L0, BrickBox box0, const uint32_t* touched, uint32_t n_touched,
                                  uint32_t* surface, Scene S) {
    uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (w >= n_touched) return;
    const uint32_t flag = touched[w];
    uint32_t st = 0, cell = flag;
    if constexpr (MANY) {
        st = structure_of(S.flag_off, S.n_struct, (unsigned long long)flag);
        cell = uint32_t(flag - S.flag_off[st]);
    }
    const DArr& A = MANY ? S.arr[st] : A0;
    const DLat& L = MANY ? S.lat[st] : L0;
    const BrickBox& box = MANY ? S.box[st] : box0;
    int k[3];
    cell_key(box, cell, k);
    double bh = double(L.b);
    double cx = (double(k[0]) + 0.5) * bh * L.h, cy = (double(k[1]) + 0.5) * bh * L.h, cz = (double(k[2]) + 0.5) * bh * L.h;
    int s = uniform_sign_warp(A, cx, cy, cz, L.rho_brick, lane);
    if (lane == 0) surface[flag] = s < 0 ? 1u : 0u;
}

template <bool MANY>
__global__ void k_cells_to_keys(BrickBox box0, const uint32_t* cells, uint32_t n, int4* keys, Scene S) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t st = 0, cell = cells[i];
    if constexpr (MANY) {
        st = structure_of(S.flag_off, S.n_struct, (unsigned long long)cell);
        cell = uint32_t(cell - S.flag_off[st]);
    }
    int k[3];
    cell_key(MANY ? S.box[st] : box0, cell, k);
    keys[i] = make_int4(k[0], k[1], k[2], int(st));
}

// Owner of a brick sample (Engine::assign, field/kernel.rs:489-546): the
// first sub-block in (z, y, x) order that contains the sample and is not
// uniform; -1 if all containing sub-blocks are uniform, then *positive is
// the sign of the last one visited.
__device__ __forceinline__ int sample_owner(int x, int y, int z, int sub, const uint32_t st[8], bool* positive) {
    auto range = [&](int v, int& lo, int& hi) {
        hi = min(v / sub, 1);
        lo = (v > 0 && v % sub == 0) ? min(v / sub - 1, 1) : hi;
    };
    int x0, x1, y0, y1, z0, z1;
    range(x, x0, x1);
    range(y, y0, y1);
    range(z, z0, z1);
    bool pos = true;
    for (int sz = z0; sz <= z1; sz++)
        for (int sy = y0; sy <= y1; sy++)
            for (int sx = x0; sx <= x1; sx++) {
                int sb = sx + 2 * sy + 4 * sz;
                if (st[sb] == ST_SAMPLE) return sb;
                pos = st[sb] == ST_OUT;
            }
    *positive = pos;
    return -1;
}

// The sub-blocks whose closed box holds lattice coordinate v on one axis, as
// a two-bit mask (bit 0 the lower half, bit 1 the upper): the index ranges
// sample_owner scans.
__device__ __forceinline__ uint32_t axis_halves(int v, int sub) {
    const int hi = min(v / sub, 1);
    const int lo = (v > 0 && v % sub == 0) ? min(v / sub - 1, 1) : hi;
    return (2u << hi) - (1u << lo);
}

// sample_owner on state masks (bit q of sampled / out: sub-block q is
// ST_SAMPLE / ST_OUT): the containing sub-blocks in sample_owner's scan order
// are the set bits of `held` in ascending order (sb = sx + 2 sy + 4 sz), so
// the owner is the lowest held sampled sub-block, and without one the sign
// is the state of the highest held sub-block, the last one the scan visits.
__device__ __forceinline__ int owner_of_masks(uint32_t xm, uint32_t ym, uint32_t zm, uint32_t sampled, uint32_t out,
                                              bool* positive) {
    const uint32_t row = ((ym & 1u) ? xm : 0u) | ((ym & 2u) ? xm << 2 : 0u);
    const uint32_t held = ((zm & 1u) ? row : 0u) | ((zm & 2u) ? row << 4 : 0u);
    const uint32_t m = held & sampled;
    if (m) return __ffs(int(m)) - 1;
    *positive = (out >> (31 - __clz(int(held)))) & 1u;
    return -1;
}

// Engine::sub_states (field/kernel.rs:467-482): one warp per sub-block,
// independent of the brick's other sub-blocks (the +-band values of samples
// no sampled sub-block owns are written by the marching-cubes count pass).
template <bool MANY>
__global__ void __launch_bounds__(256, 5) k_substates(DArr A0, DLat L0, const int4* keys, uint32_t n_bricks, uint32_t* rec,
                                                   uint32_t* sampled, Scene S) {
    const uint32_t j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= n_bricks * 8) return;
    const uint32_t brick = j >> 3, w = j & 7;
    int4 key = keys[brick];
    const DArr& A = MANY ? S.arr[key.w] : A0;
    const DLat& L = MANY ? S.lat[key.w] : L0;
    double h = L.h, sub = double(L.sub), half = double(L.sub) * 0.5;
    double bx = double((long long)key.x * L.b) * h, by = double((long long)key.y * L.b) * h,
           bz = double((long long)key.z * L.b) * h;
    double ox = double(w & 1) * sub + half, oy = double((w >> 1) & 1) * sub + half, oz = double((w >> 2) & 1) * sub + half;
    int s = uniform_sign_warp(A, bx + ox * h, by + oy * h, bz + oz * h, L.rho_sub, lane);
    uint32_t state = s < 0 ? ST_SAMPLE : (s == 1 ? ST_OUT : ST_IN);
    uint32_t* r = rec + size_t(j) * REC_WORDS;
    if (lane < REC_WORDS) r[lane] = lane == R_STATE ? state : 0u;
    if (lane == 0) sampled[j] = state == ST_SAMPLE ? 1u : 0u;
}

// ---------------------------------------------------------------------------
// (b) Candidate gather, one warp per sampled sub-block (Engine::gather_ses,
// field/kernel.rs:671-752, with gather_near :614-651).  Lists keep the CPU's
// order: near spheres in cell-scan order, those that can contain a sample
// first; S by (lb, index) and C by (distance, index), both f64; V in
// cell-scan order.  Blockers are near-list positions.

__device__ __forceinline__ int warp_append(bool p, int& count) {
    unsigned m = __ballot_sync(0xffffffffu, p);
    int lane = threadIdx.x & 31;
    int pos = count + __popc(m & ((1u << lane) - 1u));
    count += __popc(m);
    return p ? pos : -1;
}

// All lanes run the same iterations (item valid or not), so warp_append
// sees the items in scan order.
template <class F>
__device__ __forceinline__ void warp_scan_box(const DGrid& g, double x, double y, double z, double r, int lane, F&& f) {
    warp_box_items(g, cell_box(g, x, y, z, r), lane, f);
}

// Open-addressing table of a sub-block's near spheres: 2^bits 16-bit slots
// holding near-list positions (0xFFFF empty), at most half of them used, so
// a lookup ends at the sphere's slot or at an empty one.
__device__ __forceinline__ uint32_t near_hash(uint32_t id, uint32_t bits) { return (id * 0x9E3779B1u) >> (32 - bits); }

__device__ __forceinline__ int lookup_near(const uint16_t* tab, uint32_t bits, const uint32_t* near_ids, uint32_t id) {
    const uint32_t mask = (1u << bits) - 1;
    for (uint32_t h = near_hash(id, bits);; h = (h + 1) & mask) {
        const uint32_t l = tab[h];
        if (l == 0xFFFFu) return -1;
        if (near_ids[l] == id) return int(l);
    }
}

// One candidate's blocker row: the near-list members among items[p .. e)
// (lookup_near on each), counted, and with w their near-list positions
// written in order to w[0 ..] and pk[0 ..].  Four ids at a time: their
// loads and first probes are issued together, so a lane has four lookups in
// flight instead of one dependent chain per id; a probe that meets another
// sphere goes on probing.  Not inlined: the four rows of a sub-block (S and
// C, counted and written) share one copy, which keeps the gather within the
// instruction cache.
__device__ __noinline__ uint32_t near_members(const uint16_t* tab, uint32_t bits, const uint32_t* near_ids,
                                              const uint32_t* items, uint32_t p, uint32_t e, uint32_t* w,
                                              uint32_t* pk) {
    const uint32_t mask = (1u << bits) - 1;
    uint32_t n = 0;
    auto take = [&](uint32_t l) {
        if (w) w[n] = l, pk[n] = l;
        n++;
    };
    constexpr int W = 4;
    for (; p + W <= e; p += W) {
        uint32_t id[W], h[W], slot[W], at[W];
#pragma unroll
        for (int u = 0; u < W; u++) id[u] = items[p + u];
#pragma unroll
        for (int u = 0; u < W; u++) h[u] = near_hash(id[u], bits), slot[u] = tab[h[u]];
        // An empty slot reads near_ids[0] (in the scratch, unused).
#pragma unroll
        for (int u = 0; u < W; u++) at[u] = near_ids[slot[u] == 0xFFFFu ? 0u : slot[u]];
#pragma unroll
        for (int u = 0; u < W; u++) {
            if (slot[u] == 0xFFFFu) continue;
            if (at[u] == id[u]) {
                take(slot[u]);
                continue;
            }
            for (uint32_t q = (h[u] + 1) & mask;; q = (q + 1) & mask) {
                const uint32_t l = tab[q];
                if (l == 0xFFFFu) break;
                if (near_ids[l] == id[u]) {
                    take(l);
                    break;
                }
            }
        }
    }
    for (; p < e; p++) {
        const int l = lookup_near(tab, bits, near_ids, items[p]);
        if (l >= 0) take(uint32_t(l));
    }
    return n;
}

__device__ __forceinline__ unsigned warp_inclusive_scan(unsigned v) {
    int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        unsigned y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    return v;
}


// One warp: the lists of work item `item` (a sampled sub-block).
// WIDE: blocker rows through near_members (four lookups in flight), which
// pays where a sub-block's lists fill several rounds of the warp's lanes
// (a 2.4 M-sphere shell at 1 A, 141 near spheres per sub-block: 291 -> 256
// ms; a 58,800-sphere assembly at 0.25 A, 30: 12.1 -> 13.2 ms); otherwise a
// lane walks its row one lookup at a time.
template <bool MANY, bool WIDE>
__device__ __forceinline__ void gather_item(uint32_t item, const DArr& A0, const DLat& L0, const int4* keys,
                                            const uint32_t* work, const GatherOut& O, const GatherCaps& caps,
                                            const Scene& S, unsigned char* smem_raw) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char* base = smem_raw + size_t(wib) * gather_smem_bytes(caps);
    double* s_key = reinterpret_cast<double*>(base);
    double* c_key = s_key + caps.s;
    uint32_t* near_ids = reinterpret_cast<uint32_t*>(c_key + caps.c);
    // The near table takes the 2 caps.near words after the near ids: 2^bits
    // >= 2 caps.near 16-bit slots.
    uint16_t* near_tab = reinterpret_cast<uint16_t*>(near_ids + caps.near);
    const uint32_t tab_bits = 31u - uint32_t(__clz(4 * caps.near));
    uint32_t* s_id = near_ids + 3 * caps.near;
    uint32_t* s_loc = s_id + caps.s;
    uint32_t* s_perm = s_loc + caps.s;
    uint32_t* s_off = s_perm + caps.s;
    uint32_t* c_id = s_off + caps.s + 1;
    uint32_t* c_perm = c_id + caps.c;
    uint32_t* c_off = c_perm + caps.c;
    uint32_t* v_id = c_off + caps.c + 1;

    const uint32_t j = work[item];
    const uint32_t brick = j >> 3, sb = j & 7;
    uint32_t* rec = O.rec + size_t(j) * REC_WORDS;
    const int4 key = keys[brick];
    const DArr& A = MANY ? S.arr[key.w] : A0;
    const DLat& L = MANY ? S.lat[key.w] : L0;
    // Sub-block centre as Engine::prepare_sub computes it (kernel.rs:575-583).
    const double h = L.h, sub = double(L.sub), half = double(L.sub) * 0.5;
    const double px = double((long long)key.x * L.b) * h, py = double((long long)key.y * L.b) * h,
                 pz = double((long long)key.z * L.b) * h;
    const double bx = px + (double(sb & 1) * sub + half) * h, by = py + (double((sb >> 1) & 1) * sub + half) * h,
                 bz = pz + (double((sb >> 2) & 1) * sub + half) * h;
    const double rho = L.rho_sub;
    // A sphere field gathers the near spheres alone, within band + rho
    // (gather_spheres, field/kernel.rs:651-654).
    const bool spheres = A.flags & DARR_SPHERES;
    const double reach_probe = spheres ? 0.0 : A.probe;
    const double reach = reach_probe + L.band + rho;
    // The exact refinement's ball (exact.cu x_ball: rho with a relative and
    // an absolute 1e-9 margin).  With O.window the scans cover its larger
    // boxes (the extra cells hold nothing this ball keeps, so the lists and
    // their order do not change) and each candidate is also tested against
    // it; a disagreement marks the sub-block.
    const bool win = O.window != nullptr;
    const double rho_x = 0.5 * sqrt(3.0) * sub * h * (1.0 + 1e-9) + 1e-9;
    const double reach_x = reach_probe + L.band + rho_x;
    const double r_sph = win ? reach_x + A.max_expanded : reach + A.max_expanded;
    const double r_circ = win ? reach_x + A.rho_max : reach + A.rho_max, r_vert = win ? reach_x : reach;
    bool differ = false;

    if (lane == 0) rec[R_FLAGS] = 0;
    auto overflow = [&](uint32_t bit) {
        if (lane == 0) {
            rec[R_FLAGS] |= bit;
            unsigned long long q = atomicAdd(&O.counters[bit == REC_OVERFLOW ? CNT_OVERFLOW : CNT_NOMEM], 1ull);
            if (bit == REC_OVERFLOW && O.retry) O.retry[q] = j;
            // Many structures: a structure is flagged unless a retry with
            // larger caps follows.
            if (O.fail && !(bit == REC_OVERFLOW && O.retry)) O.fail[key.w] = 1;
        }
    };

    // Near spheres (gather_near: those that can contain a sample first, each
    // class in scan order), in one scan: the kept ids, bit 31 marking the
    // first class, go in scan order to the near table's space, and a stable
    // partition puts them in place.  A sphere whose squared distance is
    // clear of (R + the largest reach)^2 by 2^-38 is beyond every threshold
    // below (its rounded distance exceeds each of them), so it is neither
    // kept nor a disagreement, and its square root is not taken.
    uint32_t* scan_buf = reinterpret_cast<uint32_t*>(near_tab);
    int nn = 0;
    warp_scan_box(A.gs, bx, by, bz, r_sph, lane, [&](bool valid, uint32_t k) {
        bool keep = false, contains = false;
        if (valid && A.status[k] != STATUS_CONTAINED) {
            double4 c = A.sph[k];
            const double d2 = sq3(bx, by, bz, c.x, c.y, c.z);
            const double T = c.w + (win ? reach_x : reach);
            if (d2 < T * T * (1.0 + 0x1p-38)) {
                const double d = sqrt(d2);
                contains = d < c.w + rho;
                const bool near = !(d >= c.w + reach);
                keep = near;
                if (win) {
                    const bool exposed = !spheres && A.status[k] == STATUS_EXPOSED;
                    const double lb = fabs(d - c.w);
                    differ |= (d < c.w + reach_x) != near || (d < c.w + rho_x) != contains ||
                              (exposed && lb <= reach_x) != (exposed && near && lb <= reach);
                }
            }
        }
        int pos = warp_append(keep, nn);
        if (pos >= 0 && pos < caps.near) scan_buf[pos] = k | (contains ? 0x80000000u : 0u);
    });
    if (lane == 0) atomicMax(&O.counters[CNT_MAXNN], (unsigned long long)nn);
    if (nn > caps.near) return overflow(REC_OVERFLOW);
    __syncwarp();
    int n_in = 0;
    for (int b0 = 0; b0 < nn; b0 += 32) {
        const int i = b0 + lane;
        n_in += __popc(__ballot_sync(0xffffffffu, i < nn && (scan_buf[i] >> 31)));
    }
    {
        const uint32_t below = (1u << lane) - 1u;
        int at_in = 0, at_out = n_in;
        for (int b0 = 0; b0 < nn; b0 += 32) {
            const int i = b0 + lane;
            const uint32_t w = i < nn ? scan_buf[i] : 0u;
            const bool f = i < nn && (w >> 31), g = i < nn && !(w >> 31);
            const uint32_t mf = __ballot_sync(0xffffffffu, f), mg = __ballot_sync(0xffffffffu, g);
            if (f) near_ids[at_in + __popc(mf & below)] = w & 0x7FFFFFFFu;
            if (g) near_ids[at_out + __popc(mg & below)] = w;
            at_in += __popc(mf), at_out += __popc(mg);
        }
    }
    __syncwarp();
    // The near table for blocker lookups (positions in the near list).
    for (uint32_t i = lane; i < (1u << tab_bits); i += 32) near_tab[i] = 0xFFFFu;
    __syncwarp();
    for (int i = lane; i < nn; i += 32) {
        const uint32_t mask = (1u << tab_bits) - 1;
        uint32_t h = near_hash(near_ids[i], tab_bits);
        while (atomicCAS(&near_tab[h], (unsigned short)0xFFFFu, (unsigned short)i) != (unsigned short)0xFFFFu)
            h = (h + 1) & mask;  // ends: at most half of the slots are taken
    }
    __syncwarp();
    // Class S candidates among the near spheres.
    int ns = 0;
    for (int b0 = 0; b0 < nn; b0 += 32) {
        int i = b0 + lane;
        bool p = false;
        double lb = 0;
        uint32_t k = 0;
        if (i < nn && !spheres) {
            k = near_ids[i];
            if (A.status[k] == STATUS_EXPOSED) {
                double4 c = A.sph[k];
                lb = fabs(dist3(bx, by, bz, c.x, c.y, c.z) - c.w);
                p = lb <= reach;
            }
        }
        int pos = warp_append(p, ns);
        if (pos >= 0 && pos < caps.s) s_key[pos] = lb, s_id[pos] = k, s_loc[pos] = uint32_t(i);
    }
    // Class C candidates.
    int nc = 0;
    warp_scan_box(A.gc, bx, by, bz, r_circ, lane, [&](bool valid, uint32_t ci) {
        double d = valid ? circle_reach_dist_above(A, bx, by, bz, ci, win ? reach_x : reach) : 0.0;
        bool p = valid && d <= reach;
        if (win && valid) differ |= (d <= reach_x) != p;
        int pos = warp_append(p, nc);
        if (pos >= 0 && pos < caps.c) c_key[pos] = d, c_id[pos] = ci;
    });
    // Class V, cell-scan order.
    int nv = 0;
    warp_scan_box(A.gv, bx, by, bz, r_vert, lane, [&](bool valid, uint32_t vi) {
        bool p = false;
        if (valid) {
            double4 q = A.vert[vi];
            const double d = dist3(bx, by, bz, q.x, q.y, q.z);
            p = d <= reach;
            if (win) differ |= (d <= reach_x) != p;
        }
        int pos = warp_append(p, nv);
        if (pos >= 0 && pos < caps.v) v_id[pos] = vi;
    });
    if (lane == 0) {
        atomicMax(&O.counters[CNT_MAXNS], (unsigned long long)ns);
        atomicMax(&O.counters[CNT_MAXNC], (unsigned long long)nc);
        atomicMax(&O.counters[CNT_MAXNV], (unsigned long long)nv);
    }
    if (ns > caps.s || nc > caps.c || nv > caps.v) return overflow(REC_OVERFLOW);
    __syncwarp();
    // Rank sorts: (key, index) pairs are distinct, so ranks are a permutation.
    for (int i = lane; i < ns; i += 32) {
        double kv = s_key[i];
        uint32_t id = s_id[i];
        int rank = 0;
        for (int q = 0; q < ns; q++) rank += (s_key[q] < kv) || (s_key[q] == kv && s_id[q] < id);
        s_perm[rank] = uint32_t(i);
    }
    for (int i = lane; i < nc; i += 32) {
        double kv = c_key[i];
        uint32_t id = c_id[i];
        int rank = 0;
        for (int q = 0; q < nc; q++) rank += (c_key[q] < kv) || (c_key[q] == kv && c_id[q] < id);
        c_perm[rank] = uint32_t(i);
    }
    __syncwarp();
    // Blocker counts and offsets, in sorted order.
    unsigned run = 0;
    if (lane == 0) s_off[0] = 0;
    for (int b0 = 0; b0 < ns; b0 += 32) {
        int r = b0 + lane;
        unsigned cnt = 0;
        if (r < ns) {
            uint32_t k = s_id[s_perm[r]];
            if constexpr (WIDE)
                cnt = near_members(near_tab, tab_bits, near_ids, A.nb_items, A.nb_off[k], A.nb_off[k + 1], nullptr,
                                   nullptr);
            else
                for (uint32_t p = A.nb_off[k], e = A.nb_off[k + 1]; p < e; p++)
                    cnt += lookup_near(near_tab, tab_bits, near_ids, A.nb_items[p]) >= 0;
        }
        unsigned inc = warp_inclusive_scan(cnt);
        if (r < ns) s_off[r + 1] = run + inc;
        run += __shfl_sync(0xffffffffu, inc, 31);
    }
    const unsigned nsb = run;
    run = 0;
    if (lane == 0) c_off[0] = 0;
    for (int b0 = 0; b0 < nc; b0 += 32) {
        int r = b0 + lane;
        unsigned cnt = 0;
        if (r < nc) {
            uint32_t ci = c_id[c_perm[r]];
            if constexpr (WIDE)
                cnt = near_members(near_tab, tab_bits, near_ids, A.cb_items, A.cb_off[ci], A.cb_off[ci + 1], nullptr,
                                   nullptr);
            else
                for (uint32_t p = A.cb_off[ci], e = A.cb_off[ci + 1]; p < e; p++)
                    cnt += lookup_near(near_tab, tab_bits, near_ids, A.cb_items[p]) >= 0;
        }
        unsigned inc = warp_inclusive_scan(cnt);
        if (r < nc) c_off[r + 1] = run + inc;
        run += __shfl_sync(0xffffffffu, inc, 31);
    }
    const unsigned ncb = run;
    __syncwarp();

    // Space: ids (CSR words) and the packed f32 block the sampler stages.
    const unsigned long long ids_words =
        (unsigned long long)nn + 2ull * ns + 1 + nsb + 2ull * nc + 1 + ncb + nv;
    const unsigned long long tail_words = 2ull * ns + 1 + nsb + 2ull * nc + 1 + ncb;
    const unsigned long long units = 2ull * nn + ns + 3ull * nc + nv + (tail_words + 3) / 4;
    unsigned long long ids_base = 0, pack_base = 0;
    if (lane == 0) {
        ids_base = atomicAdd(&O.counters[CNT_IDS], ids_words);
        pack_base = atomicAdd(&O.counters[CNT_PACK], units);
        atomicMax(&O.counters[CNT_MAXPACK], units);
    }
    ids_base = __shfl_sync(0xffffffffu, ids_base, 0);
    pack_base = __shfl_sync(0xffffffffu, pack_base, 0);
    if (ids_base + ids_words > O.ids_cap || pack_base + units > O.pack_cap || units > O.unit_cap)
        return overflow(REC_NOMEM);

    // CSR ids: near, S, s_off, s_blk, C, c_off, c_blk, V.
    uint32_t* ids = O.ids + ids_base;
    uint32_t* w_near = ids;
    uint32_t* w_s = w_near + nn;
    uint32_t* w_soff = w_s + ns;
    uint32_t* w_sblk = w_soff + ns + 1;
    uint32_t* w_c = w_sblk + nsb;
    uint32_t* w_coff = w_c + nc;
    uint32_t* w_cblk = w_coff + nc + 1;
    uint32_t* w_v = w_cblk + ncb;
    // Packed block: nearA (x,y,z,R^2), nearT (x,y,z,(R-tol)^2), S (x,y,z,R),
    // C (3 x float4), V (x,y,z,0), then the S and C pruning keys (f32) and
    // the s_off, s_blk, c_off, c_blk words.
    float4* pk = reinterpret_cast<float4*>(O.pack + pack_base);
    float4* p_nearA = pk;
    float4* p_nearT = p_nearA + nn;
    float4* p_s = p_nearT + nn;
    float4* p_c = p_s + ns;
    float4* p_v = p_c + 3 * nc;
    float* p_skey = reinterpret_cast<float*>(p_v + nv);
    float* p_ckey = p_skey + ns;
    uint32_t* p_soff = reinterpret_cast<uint32_t*>(p_ckey + nc);
    uint32_t* p_sblk = p_soff + ns + 1;
    uint32_t* p_coff = p_sblk + nsb;
    uint32_t* p_cblk = p_coff + nc + 1;

    for (int i = lane; i < nn; i += 32) {
        uint32_t k = near_ids[i];
        w_near[i] = k;
        double4 c = A.sph[k];
        float x = float(c.x - L.fx), y = float(c.y - L.fy), z = float(c.z - L.fz);
        float r32 = float(c.w);
        float rt = fmaxf(r32 - INSIDE_TOL, 0.0f);
        p_nearA[i] = make_float4(x, y, z, r32 * r32);
        // A sphere field has no blockers: its samples take R itself.
        p_nearT[i] = make_float4(x, y, z, spheres ? r32 : rt * rt);
    }
    for (int r = lane; r <= ns; r += 32) w_soff[r] = s_off[r], p_soff[r] = s_off[r];
    // Pruning keys: every sample the sub-block evaluates lies within rho of
    // its centre, and |d - R| and the circle distance are 1-Lipschitz, so a
    // candidate whose centre value minus rho exceeds the sample's current best
    // cannot improve it; PRUNE_MARGIN (1e-3 A) covers f32 rounding, so the
    // skipped candidates are exactly those whose test would fail.
    for (int r = lane; r < ns; r += 32)
        p_skey[r] = __double2float_rd(s_key[s_perm[r]] - rho - PRUNE_MARGIN);
    for (int r = lane; r < nc; r += 32)
        p_ckey[r] = __double2float_rd(c_key[c_perm[r]] - rho - PRUNE_MARGIN);
    for (int r = lane; r < ns; r += 32) {
        uint32_t i = s_perm[r], k = s_id[i];
        w_s[r] = k;
        double4 c = A.sph[k];
        p_s[r] = make_float4(float(c.x - L.fx), float(c.y - L.fy), float(c.z - L.fz), float(c.w));
        uint32_t o = s_off[r];
        if constexpr (WIDE) {
            near_members(near_tab, tab_bits, near_ids, A.nb_items, A.nb_off[k], A.nb_off[k + 1], w_sblk + o,
                         p_sblk + o);
        } else {
            for (uint32_t p = A.nb_off[k], e = A.nb_off[k + 1]; p < e; p++) {
                int l = lookup_near(near_tab, tab_bits, near_ids, A.nb_items[p]);
                if (l >= 0) w_sblk[o] = uint32_t(l), p_sblk[o] = uint32_t(l), o++;
            }
        }
    }
    for (int r = lane; r <= nc; r += 32) w_coff[r] = c_off[r], p_coff[r] = c_off[r];
    for (int r = lane; r < nc; r += 32) {
        uint32_t ci = c_id[c_perm[r]];
        w_c[r] = ci;
        const double* c = A.circ + 12 * size_t(ci);
        p_c[3 * r] = make_float4(float(c[0] - L.fx), float(c[1] - L.fy), float(c[2] - L.fz), float(c[9]));
        p_c[3 * r + 1] = make_float4(float(c[3]), float(c[4]), float(c[5]), float(c[6]));
        p_c[3 * r + 2] = make_float4(float(c[7]), float(c[8]), 0.0f, 0.0f);
        uint32_t o = c_off[r];
        if constexpr (WIDE) {
            near_members(near_tab, tab_bits, near_ids, A.cb_items, A.cb_off[ci], A.cb_off[ci + 1], w_cblk + o,
                         p_cblk + o);
        } else {
            for (uint32_t p = A.cb_off[ci], e = A.cb_off[ci + 1]; p < e; p++) {
                int l = lookup_near(near_tab, tab_bits, near_ids, A.cb_items[p]);
                if (l >= 0) w_cblk[o] = uint32_t(l), p_cblk[o] = uint32_t(l), o++;
            }
        }
    }
    for (int i = lane; i < nv; i += 32) {
        uint32_t vi = v_id[i];
        w_v[i] = vi;
        double4 q = A.vert[vi];
        p_v[i] = make_float4(float(q.x - L.fx), float(q.y - L.fy), float(q.z - L.fz), 0.0f);
    }
    const bool any_differ = __any_sync(0xffffffffu, differ);
    if (lane == 0) {
        if (win) O.window[j] = any_differ ? 1 : 0;
        rec[R_IDS] = uint32_t(ids_base);
        rec[R_INSIDE] = uint32_t(n_in);
        rec[R_NEAR] = uint32_t(nn);
        rec[R_S] = uint32_t(ns);
        rec[R_C] = uint32_t(nc);
        rec[R_V] = uint32_t(nv);
        rec[R_SBLK] = nsb;
        rec[R_CBLK] = ncb;
        rec[R_PACK] = uint32_t(pack_base);
        rec[R_PACKLEN] = uint32_t(units);
    }
}

// Warp per work item, the grid striding over the items (many structures:
// the item count is read on the device).
template <bool MANY, bool WIDE>
__global__ void __launch_bounds__(256, MANY ? 2 : 4) k_gather(DArr A0, DLat L0, const int4* keys, const uint32_t* work, uint32_t n_work, GatherOut O,
                         GatherCaps caps, Scene S) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t n = MANY ? uint32_t(*S.n_work) : n_work;
    const uint32_t wpb = blockDim.x >> 5;
    for (uint32_t item = blockIdx.x * wpb + (threadIdx.x >> 5); item < n; item += gridDim.x * wpb)
        gather_item<MANY, WIDE>(item, A0, L0, keys, work, O, caps, S, smem_raw);
}

// ---------------------------------------------------------------------------
// (c) Sampling: one CTA per sampled sub-block.  Its packed candidate block
// is one contiguous, 16-byte aligned run of global memory, staged in shared
// memory by the TMA bulk-copy engine (cp.async.bulk, mbarrier completion);
// each thread then evaluates owned samples against it with broadcast
// shared-memory reads.  ses_kernel (field/kernel.rs:837-952) per lane.

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

constexpr uint32_t BULK_CHUNK = 32768;            // bytes per bulk copy
constexpr int SAMPLE_CHUNK = 512;                 // samples per ownership compaction
constexpr uint32_t MBAR_SPIN_LIMIT = 1u << 24;     // bounded wait

// list (single structure): blocks whose packed block exceeds limit_units
// append their index to list (list[0] = count) and return; LIST: block b
// samples the list's b-th entry (none past the count).  FEAT: each owned
// sample's nearest feature also goes to feats (same layout as values), in
// the refinement's encoding kind << 29 | id (0 solvent, 1 beyond, 2 sphere,
// 3 circle, 4 SAS vertex; ids of the structure's arrangement): the candidate
// that set the sample's least distance, the first of equal ones.  Values are
// the same with and without it.
template <bool TMA, bool COUNT, bool MANY, bool LIST = false, bool FEAT = false>
__global__ void __launch_bounds__(128) k_sample(DLat L0, const int4* keys, const uint32_t* work, uint32_t n_work,
                                                const uint32_t* rec, const uint4* pack, float* values,
                                                unsigned long long* counters, Scene SC, uint32_t limit_units,
                                                uint32_t* list, const uint32_t* ids, uint32_t* feats) {
    extern __shared__ __align__(16) uint4 sm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t sts[8];
    __shared__ uint32_t own_mask[SAMPLE_CHUNK / 32];
    __shared__ uint16_t own_list[SAMPLE_CHUNK];
    if (MANY && blockIdx.x >= uint32_t(*SC.n_work)) return;
    if (LIST && blockIdx.x >= list[0]) return;
    const uint32_t slot = LIST ? list[1 + blockIdx.x] : blockIdx.x;
    const uint32_t j = work[slot];
    const uint32_t brick = j >> 3, sb = j & 7;
    const DLat& L = MANY ? SC.lat[keys[brick].w] : L0;
    const uint32_t* R = rec + size_t(j) * REC_WORDS;
    if (R[R_FLAGS] != 0) return;
    const int nn = int(R[R_NEAR]), n_in = int(R[R_INSIDE]), ns = int(R[R_S]), nc = int(R[R_C]), nv = int(R[R_V]);
    const int nsb = int(R[R_SBLK]);
    const uint32_t units = R[R_PACKLEN];
    if (!LIST && list && units > limit_units) {
        if (threadIdx.x == 0) list[1 + atomicAdd(list, 1u)] = slot;
        return;
    }
    const uint4* src = pack + R[R_PACK];
    if (threadIdx.x < 8) sts[threadIdx.x] = rec[(size_t(brick) * 8 + threadIdx.x) * REC_WORDS + R_STATE];
    if (TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            uint32_t bytes = units * 16u;
            mbar_expect_tx(&bar, bytes);
            for (uint32_t o = 0; o < bytes; o += BULK_CHUNK)
                bulk_g2s(reinterpret_cast<unsigned char*>(sm) + o, reinterpret_cast<const unsigned char*>(src) + o,
                         min(BULK_CHUNK, bytes - o), &bar);
        }
        __syncthreads();
        uint32_t spins = 0;
        while (!mbar_try_wait(&bar, 0)) {
            if (++spins >= MBAR_SPIN_LIMIT) {
                if (threadIdx.x == 0) atomicAdd(&counters[CNT_TIMEOUT], 1ull);
                return;
            }
        }
    } else {
        for (uint32_t u = threadIdx.x; u < units; u += blockDim.x) sm[u] = src[u];
        __syncthreads();
    }
    const float4* nearA = reinterpret_cast<const float4*>(sm);
    const float4* nearT = nearA + nn;
    const float4* S = nearT + nn;
    const float4* C = S + ns;
    const float4* V = C + 3 * nc;
    const float* s_key = reinterpret_cast<const float*>(V + nv);
    const float* c_key = s_key + ns;
    const uint32_t* s_off = reinterpret_cast<const uint32_t*>(c_key + nc);
    const uint32_t* s_blk = s_off + ns + 1;
    const uint32_t* c_off = s_blk + nsb;
    const uint32_t* c_blk = c_off + nc + 1;
    uint32_t st[8];
    for (int q = 0; q < 8; q++) st[q] = sts[q];

    const int sub = L.sub, side = L.b + 1, sp = sub + 1;
    const int ox = int(sb & 1) * sub, oy = int((sb >> 1) & 1) * sub, oz = int((sb >> 2) & 1) * sub;
    // The sub-block's owned samples (sample_owner), compacted in sample
    // order a chunk of SAMPLE_CHUNK at a time, so that the threads take
    // owned samples only: the samples of a face that a neighbouring
    // sub-block owns cost no masked-off lanes.  f(x, y, z) per owned sample.
    const int n_samples = sp * sp * sp;
    auto for_owned = [&](auto&& f) {
        const int lane = int(threadIdx.x & 31), warp = int(threadIdx.x >> 5), nw = int(blockDim.x >> 5);
        for (int c0 = 0; c0 < n_samples; c0 += SAMPLE_CHUNK) {
            for (int q = warp; q < SAMPLE_CHUNK / 32; q += nw) {
                const int t = c0 + q * 32 + lane;
                bool own = false;
                if (t < n_samples) {
                    const int x = ox + t % sp, y = oy + (t / sp) % sp, z = oz + t / (sp * sp);
                    bool positive;
                    own = sample_owner(x, y, z, sub, st, &positive) == int(sb);
                }
                const uint32_t m = __ballot_sync(0xffffffffu, own);
                if (lane == 0) own_mask[q] = m;
            }
            __syncthreads();
            int total = 0;
            for (int q = 0; q < SAMPLE_CHUNK / 32; q++) total += __popc(own_mask[q]);
            for (int q = warp; q < SAMPLE_CHUNK / 32; q += nw) {
                const uint32_t m = own_mask[q];
                if ((m >> lane) & 1u) {
                    int before = 0;
                    for (int p = 0; p < q; p++) before += __popc(own_mask[p]);
                    own_list[before + __popc(m & ((1u << lane) - 1u))] = uint16_t(q * 32 + lane);
                }
            }
            __syncthreads();
            for (int i = int(threadIdx.x); i < total; i += int(blockDim.x)) {
                const int t = c0 + int(own_list[i]);
                f(ox + t % sp, oy + (t / sp) % sp, oz + t / (sp * sp));
            }
            __syncthreads();
        }
    };
    const int4 key = keys[brick];
    const long long gx = (long long)key.x * L.b - L.frame[0], gy = (long long)key.y * L.b - L.frame[1],
                    gz = (long long)key.z * L.b - L.frame[2];
    const float probe = L.probe32, cutoff2 = L.cutoff2;
    float* out = values + size_t(brick) * L.spb;
    // COUNT: arithmetic operations as executed (the algorithmic count of the
    // roofline; compares and selects are not counted).
    unsigned long long ops = 0, owned = 0;
    if (L.kind) {
        // A sphere field (sphere_kernel, field/kernel.rs:957-981): the least
        // |x - c| - R over every near sphere, clamped at band; nearT holds
        // (x, y, z, R).  COUNT: 9 per sphere.
        const float band = L.band32;
        for_owned([&](int x, int y, int z) {
            const float px = float(gx + x) * L.h32, py = float(gy + y) * L.h32, pz = float(gz + z) * L.h32;
            if (COUNT) owned++, ops += 9ull * nn;
            float best = band;
            uint32_t fi = 0xFFFFFFFFu;
            for (int k = 0; k < nn; k++) {
                const float4 a = nearT[k];
                const float dx = px - a.x, dy = py - a.y, dz = pz - a.z;
                const float v = sqrtf(dx * dx + dy * dy + dz * dz) - a.w;
                if (FEAT) {
                    if (v < best) best = v, fi = uint32_t(k);
                } else {
                    best = fminf(best, v);
                }
            }
            out[(z * side + y) * side + x] = best;
            if (FEAT)
                feats[size_t(brick) * L.spb + (z * side + y) * side + x] =
                    fi == 0xFFFFFFFFu ? (1u << FEAT_SHIFT_D) : ((2u << FEAT_SHIFT_D) | ids[R[R_IDS] + fi]);
        });
        if (COUNT) {
            atomicAdd(&counters[CNT_OPS], ops);
            atomicAdd(&counters[CNT_OWNED], owned);
        }
        return;
    }
    for_owned([&](int x, int y, int z) {
        // Lattice::local (field/lattice.rs:69): from integers only.
        const float px = float(gx + x) * L.h32, py = float(gy + y) * L.h32, pz = float(gz + z) * L.h32;
        if (COUNT) owned++, ops += 8ull * n_in;
        bool inside = false;
        for (int k = 0; k < n_in; k++) {
            float4 a = nearA[k];
            float dx = px - a.x, dy = py - a.y, dz = pz - a.z;
            inside |= (dx * dx + dy * dy + dz * dz) < a.w;
        }
        float value = probe;
        uint32_t fk = 0, fi = 0;  // FEAT: kind and list position of the nearest feature
        if (inside) {
            if (COUNT) ops += 9ull * nv + 2;
            float best2 = cutoff2;
            fk = 1;
            for (int v = 0; v < nv; v++) {
                float4 q = V[v];
                float dx = px - q.x, dy = py - q.y, dz = pz - q.z;
                const float d2 = dx * dx + dy * dy + dz * dz;
                if (FEAT) {
                    if (d2 < best2) best2 = d2, fk = 4, fi = uint32_t(v);
                } else {
                    best2 = fminf(best2, d2);
                }
            }
            for (int si = 0; si < ns; si++) {
                const float kk = s_key[si];
                if (kk > 0.0f && kk * kk >= best2) break;
                if (COUNT) ops += 12;
                float4 c = S[si];
                float dx = px - c.x, dy = py - c.y, dz = pz - c.z;
                float dist = sqrtf(dx * dx + dy * dy + dz * dz);
                float lb = fabsf(dist - c.w);
                float lb2 = lb * lb;
                bool valid = lb2 < best2 && 1e-6f < dist;
                if (!valid) continue;
                if (COUNT) ops += 7;
                float scale = c.w / dist;
                float qx = c.x + dx * scale, qy = c.y + dy * scale, qz = c.z + dz * scale;
                for (uint32_t p = s_off[si], e = s_off[si + 1]; p < e; p++) {
                    if (COUNT) ops += 8;
                    float4 b = nearT[s_blk[p]];
                    float ex = qx - b.x, ey = qy - b.y, ez = qz - b.z;
                    if (!((ex * ex + ey * ey + ez * ez) >= b.w)) {
                        valid = false;
                        break;
                    }
                }
                if (valid) {
                    best2 = lb2;
                    if (FEAT) fk = 2, fi = uint32_t(si);
                }
            }
            for (int ci = 0; ci < nc; ci++) {
                const float kk = c_key[ci];
                if (kk > 0.0f && kk * kk >= best2) break;
                if (COUNT) ops += 9;
                float4 m = C[3 * ci], u = C[3 * ci + 1], e2 = C[3 * ci + 2];
                float yx = px - m.x, yy = py - m.y, yz = pz - m.z;
                float along = yx * u.x + yy * u.y + yz * u.z;
                // d2 = fl(a2 + tt tt) >= a2 (rounding is monotone): where the
                // plane distance alone fails the test, d2 fails it too.
                const float a2 = along * along;
                if (!(a2 < best2)) continue;
                if (COUNT) ops += 17;
                float wx = yx - u.x * along, wy = yy - u.y * along, wz = yz - u.z * along;
                float wl = sqrtf(wx * wx + wy * wy + wz * wz);
                float tt = wl - m.w;
                float d2 = a2 + tt * tt;
                if (!(d2 < best2)) continue;
                if (COUNT) ops += 7;
                bool degenerate = wl < 1e-6f;
                float s = m.w / wl;
                float qx = degenerate ? m.x + u.w * m.w : m.x + wx * s;
                float qy = degenerate ? m.y + e2.x * m.w : m.y + wy * s;
                float qz = degenerate ? m.z + e2.y * m.w : m.z + wz * s;
                bool valid = true;
                for (uint32_t p = c_off[ci], e = c_off[ci + 1]; p < e; p++) {
                    if (COUNT) ops += 8;
                    float4 b = nearT[c_blk[p]];
                    float ex = qx - b.x, ey = qy - b.y, ez = qz - b.z;
                    if (!((ex * ex + ey * ey + ez * ez) >= b.w)) {
                        valid = false;
                        break;
                    }
                }
                if (valid) {
                    best2 = d2;
                    if (FEAT) fk = 3, fi = uint32_t(ci);
                }
            }
            value = probe - sqrtf(best2);
        }
        out[(z * side + y) * side + x] = value;
        if (FEAT) {
            // List position to the arrangement's id: the sub-block's id words
            // are near, S, S offsets, S blockers, C, C offsets, C blockers, V.
            const uint32_t* l = ids + R[R_IDS];
            uint32_t id = 0;
            if (fk == 2) id = l[nn + fi];
            else if (fk == 3) id = l[nn + 2 * ns + 1 + nsb + fi];
            else if (fk == 4) id = l[nn + 2 * ns + 1 + nsb + 2 * nc + 1 + R[R_CBLK] + fi];
            feats[size_t(brick) * L.spb + (z * side + y) * side + x] = (fk << FEAT_SHIFT_D) | id;
        }
    });
    if (COUNT) {
        atomicAdd(&counters[CNT_OPS], ops);
        atomicAdd(&counters[CNT_OWNED], owned);
    }
}

// ---------------------------------------------------------------------------
// (d) Marching cubes per brick (mesh_brick edge scan and cells(),
// mesh/extract.rs:146-265): owned crossing edges in (z, y, x, axis) order
// and triangle references (code << 28 | local edge id) in cell order, both
// compacted with a block scan over contiguous cell ranges per thread.
constexpr int MC_THREADS = 256;

// Lower corner of cube edge e (edges 0-3 along x, 4-7 along y, 8-11 along
// z), corner bits x | y << 1 | z << 2, one nibble per edge:
// {0, 2, 4, 6, 0, 1, 4, 5, 0, 1, 2, 3}.
constexpr unsigned long long MC_EDGE_LOWER = 0x321054106420ull;

// BC: the brick edge when it is known at compile time (constant divisors),
// 0 to read it from the lattice; the outputs do not depend on it.
template <bool FILL, bool MANY, int BC>
__global__ void __launch_bounds__(MC_THREADS) k_mc(DLat L0, uint32_t n_bricks, float* values, const uint32_t* rec, uint32_t* counts,
                                                   const uint32_t* edge_off, const uint32_t* tri_off, uint32_t* edges,
                                                   float2* edge_vals, uint32_t* tris, const int4* keys,
                                                   unsigned long long edge_cap, unsigned long long tri_cap, Scene S) {
    extern __shared__ float v[];
    __shared__ uint16_t t_off[257];
    __shared__ uint8_t t_edges[FILL ? SMB_MC_TRIANGLES * 3 : 1];
    __shared__ unsigned long long sh[MC_THREADS / 32];
    __shared__ uint32_t masks[2];
    const uint32_t brick = blockIdx.x;
    if (brick >= n_bricks) return;
    const DLat& L = MANY ? S.lat[keys[brick].w] : L0;
    if (FILL && (edge_off[brick + 1] > edge_cap || tri_off[brick + 1] > tri_cap)) {
        if (MANY && threadIdx.x == 0) S.fail[keys[brick].w] = 1;
        return;
    }
    const int b = BC ? BC : L.b, s = b + 1, spb = s * s * s;
    float* src = values + size_t(brick) * spb;
    if (!FILL) {
        // Samples that no sampled sub-block owns get +-band here (Engine::
        // assign, field/kernel.rs:489-546): the sign of the last containing
        // uniform sub-block.
        const int sub = BC ? BC / 2 : L.sub;
        if (threadIdx.x < 32) {
            const uint32_t q = threadIdx.x & 7;
            const uint32_t st = rec[(size_t(brick) * 8 + q) * REC_WORDS + R_STATE];
            const uint32_t ms = __ballot_sync(0xffffffffu, threadIdx.x < 8 && st == ST_SAMPLE);
            const uint32_t mo = __ballot_sync(0xffffffffu, threadIdx.x < 8 && st == ST_OUT);
            if (threadIdx.x == 0) masks[0] = ms, masks[1] = mo;
        }
        __syncthreads();
        const uint32_t ms = masks[0], mo = masks[1];
        const float band = L.band32;
        for (int i = threadIdx.x; i < spb; i += blockDim.x) {
            const int x = i % s, y = (i / s) % s, z = i / (s * s);
            bool positive;
            if (owner_of_masks(axis_halves(x, sub), axis_halves(y, sub), axis_halves(z, sub), ms, mo, &positive) < 0) {
                const float bv = positive ? band : -band;
                src[i] = bv;
                v[i] = bv;
            } else {
                v[i] = src[i];
            }
        }
    } else {
        for (int i = threadIdx.x; i < spb; i += blockDim.x) v[i] = src[i];
        const uint8_t* te = &SMB_TRI_EDGES[0][0];
        for (int i = threadIdx.x; i < SMB_MC_TRIANGLES * 3; i += blockDim.x) t_edges[i] = te[i];
    }
    for (int i = threadIdx.x; i < 257; i += blockDim.x) t_off[i] = SMB_TRI_OFFSET[i];
    __syncthreads();
    const int cells = b * b * b;
    const int per = (cells + MC_THREADS - 1) / MC_THREADS;
    const int c0 = min(int(threadIdx.x) * per, cells), c1 = min(c0 + per, cells);
    const int ss = s * s;
    unsigned ne = 0, nt = 0;
    for (int c = c0; c < c1; c++) {
        const int x = c % b, y = (c / b) % b, z = c / (b * b);
        const int i = (z * s + y) * s + x;
        const bool a = v[i] < 0.0f;
        ne += (a != (v[i + 1] < 0.0f)) + (a != (v[i + s] < 0.0f)) + (a != (v[i + ss] < 0.0f));
        int cs = 0;
        cs |= int(a);
        cs |= int(v[i + 1] < 0.0f) << 1;
        cs |= int(v[i + s] < 0.0f) << 2;
        cs |= int(v[i + s + 1] < 0.0f) << 3;
        cs |= int(v[i + ss] < 0.0f) << 4;
        cs |= int(v[i + ss + 1] < 0.0f) << 5;
        cs |= int(v[i + ss + s] < 0.0f) << 6;
        cs |= int(v[i + ss + s + 1] < 0.0f) << 7;
        nt += t_off[cs + 1] - t_off[cs];
    }
    unsigned long long te, tt;
    unsigned long long pe = block_exclusive_scan<MC_THREADS>(ne, sh, &te);
    unsigned long long pt = block_exclusive_scan<MC_THREADS>(nt, sh, &tt);
    if (!FILL) {
        if (threadIdx.x == 0) counts[brick] = uint32_t(te), counts[n_bricks + brick] = uint32_t(tt);
        return;
    }
    uint32_t eo = edge_off[brick] + uint32_t(pe), to = tri_off[brick] + uint32_t(pt);
    for (int c = c0; c < c1; c++) {
        const int x = c % b, y = (c / b) % b, z = c / (b * b);
        const int i = (z * s + y) * s + x;
        const float va = v[i];
        const float vn[3] = {v[i + 1], v[i + s], v[i + ss]};
        for (int ax = 0; ax < 3; ax++) {
            if ((va < 0.0f) != (vn[ax] < 0.0f)) {
                edges[eo] = uint32_t(c * 3 + ax);
                edge_vals[eo] = make_float2(va, vn[ax]);
                eo++;
            }
        }
        int cs = 0;
        cs |= int(va < 0.0f);
        cs |= int(vn[0] < 0.0f) << 1;
        cs |= int(vn[1] < 0.0f) << 2;
        cs |= int(v[i + s + 1] < 0.0f) << 3;
        cs |= int(vn[2] < 0.0f) << 4;
        cs |= int(v[i + ss + 1] < 0.0f) << 5;
        cs |= int(v[i + ss + s] < 0.0f) << 6;
        cs |= int(v[i + ss + s + 1] < 0.0f) << 7;
        for (int t = t_off[cs]; t < t_off[cs + 1]; t++) {
            for (int k = 0; k < 3; k++) {
                const int e = t_edges[3 * t + k];
                const int axis = e >> 2, lo = int((MC_EDGE_LOWER >> (4 * e)) & 0xFu);
                const int lx = x + (lo & 1), ly = y + ((lo >> 1) & 1), lz = z + (lo >> 2);
                // A vertex on the brick's upper face belongs to the next
                // brick: its code bit is set and its coordinate is 0 there.
                const uint32_t code = uint32_t(lx == b) | uint32_t(ly == b) << 1 | uint32_t(lz == b) << 2;
                const int cx = lx == b ? 0 : lx, cy = ly == b ? 0 : ly, cz = lz == b ? 0 : lz;
                tris[3 * size_t(to) + k] = (code << 28) | uint32_t(((cz * b + cy) * b + cx) * 3 + axis);
            }
            to++;
        }
    }
}


// ---------------------------------------------------------------------------
// (e) Fast mode: f32 root refinement of the crossing edges on the device,
// the reference's definition of plain f32 refinement (sesmesh-gpu
// kernels/sesmesh.cuh:445-750): brick-local coordinates from double-float
// pairs (frame-local f32 value + f32 residual, minus the brick origin as an
// exact product pair), safeguarded Newton / Illinois (at most max_iter
// evaluations) then bisection.  One CTA per sampled sub-block: its candidate
// lists (the gather's, bit-identical to the CPU's) are turned into
// brick-local coordinates once, in shared memory; each thread refines the
// brick's crossing edges whose lower sample lies in the sub-block.

__device__ __forceinline__ void split_df(double v, float& hi, float& lo) {
    hi = float(v);
    lo = float(v - double(hi));
}

// O * h as a pair (hi, lo): hi = O h_hi rounded, lo = its error + O h_lo.
__device__ __forceinline__ void origin_pair(long long o, float h_hi, float h_lo, float& hi, float& lo) {
    float of = float(o);
    hi = of * h_hi;
    lo = fmaf(of, h_hi, -hi) + of * h_lo;
}

struct RefOut {
    float* t;
    uint32_t* feat;
    float* q;
    uint32_t* evals;
};


// Sub-block edge lists for refinement: per work item (a sampled sub-block;
// without flags unless any_flags: the f32 refinement stages the sampler's
// lists, which a flagged sub-block lacks), its brick's crossing edges whose
// lower sample lies in the sub-block, in the brick's (ascending) order.  Warp per item; FILL = false
// counts (and records the largest count), FILL = true writes at item_off[i]
// and the list's tail item_off[n] = *total.
template <bool FILL, bool MANY>
__global__ void __launch_bounds__(256) k_item_edges(const DLat L, const uint32_t* work, uint32_t n_host,
                                                    const uint32_t* rec, const uint32_t* edge_off,
                                                    const uint32_t* edges, uint32_t* counts, uint32_t* item_off,
                                                    uint32_t* item_edges, const unsigned long long* total,
                                                    unsigned long long* counters, const int4* keys, Scene S,
                                                    const uint8_t* mask, bool any_flags) {
    const uint32_t lane = threadIdx.x & 31, i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t n = MANY ? uint32_t(*S.n_work) : n_host;
    if (FILL && blockIdx.x == 0 && threadIdx.x == 0) item_off[n] = uint32_t(*total);
    if (i >= n) {
        if (!FILL && MANY && lane == 0 && i < n_host) counts[i] = 0;  // the scan runs over n_host entries
        return;
    }
    const uint32_t j = work[i], brick = j >> 3, sb = j & 7;
    const uint32_t* R = rec + size_t(j) * REC_WORDS;
    // Many structures: a structure over a list or buffer limit is redone on
    // its own, and its marching-cubes output may be incomplete.
    if (R[R_STATE] != ST_SAMPLE || (R[R_FLAGS] != 0 && !any_flags) || (MANY && S.fail[keys[brick].w])) {
        if (!FILL && lane == 0) counts[i] = 0;
        return;
    }
    const int b = L.b, sub = L.sub;
    const uint32_t e0 = edge_off[brick], e1 = edge_off[brick + 1];
    uint32_t at = FILL ? item_off[i] : 0u;
    for (uint32_t base = e0; base < e1; base += 32) {
        const uint32_t k = base + lane;
        bool mine = false;
        if (k < e1) {
            const uint32_t cell = edges[k] / 3;
            const int ex = int(cell % b), ey = int((cell / b) % b), ez = int(cell / (b * b));
            mine = uint32_t(min(ex / sub, 1) + 2 * min(ey / sub, 1) + 4 * min(ez / sub, 1)) == sb && (!mask || mask[k]);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, mine);
        if (FILL && mine) item_edges[at + __popc(m & ((1u << lane) - 1u))] = k;
        at += __popc(m);
    }
    if (!FILL && lane == 0) {
        counts[i] = at;
        atomicMax(reinterpret_cast<unsigned int*>(&counters[CNT_MAXITEM]), at);
    }
}

// *dst = *src (a device count kept before the kernel that reads it grows it).
__global__ void k_copy_count(unsigned long long* dst, const unsigned long long* src) {
    if (threadIdx.x == 0) *dst = *src;
}

// dst = the low 32 bits of a device total (the tail of an offset list).
__global__ void k_put_total(uint32_t* dst, const unsigned long long* total) {
    if (threadIdx.x == 0) *dst = uint32_t(*total);
}

// Brick-local frame of one brick: the origin (key * b - frame) * h as an f32
// pair, and the f64 -> brick-local f32 transform of the refinement.
struct BrickFrame {
    float ohx, olx, ohy, oly, ohz, olz;
};

__device__ __forceinline__ BrickFrame brick_frame(const DLat& L, const RefineConsts& RC, int4 key) {
    BrickFrame F;
    origin_pair((long long)key.x * L.b - L.frame[0], RC.h_hi, RC.h_lo, F.ohx, F.olx);
    origin_pair((long long)key.y * L.b - L.frame[1], RC.h_hi, RC.h_lo, F.ohy, F.oly);
    origin_pair((long long)key.z * L.b - L.frame[2], RC.h_hi, RC.h_lo, F.ohz, F.olz);
    return F;
}

__device__ __forceinline__ void to_local(const DLat& L, const BrickFrame& F, double x, double y, double z, float& lx,
                                         float& ly, float& lz) {
    float hx, lo_x, hy, lo_y, hz, lo_z;
    split_df(x - L.fx, hx, lo_x);
    split_df(y - L.fy, hy, lo_y);
    split_df(z - L.fz, hz, lo_z);
    lx = (hx - F.ohx) + (lo_x - F.olx);
    ly = (hy - F.ohy) + (lo_y - F.oly);
    lz = (hz - F.ohz) + (lo_z - F.olz);
}

// One sub-block's candidates staged in shared memory, brick-local f32:
// near (x, y, z, R) and (x, y, z, (R - tol)^2), S (x, y, z, R), C 3 x float4,
// V (x, y, z, id); then S ids, s_off, s_blk, c_off, c_blk words.
struct RefStage {
    const float4 *nearA, *nearT, *S, *C, *V;
    const uint32_t *s_id, *s_off, *s_blk, *c_off, *c_blk;
    int n_in, ns, nc, nv;
    // Pruning keys (each candidate's value at the sub-block's centre, less
    // rho and a 1e-3 A margin; C keys in C[3 i + 2].w): s_key null when the
    // region has no room for the S keys (then neither list is pruned).
    const float* s_key;
    float cx, cy, cz, rho;
    // A sphere field: every near sphere is a candidate (eval_point's
    // non-SES branch, sesmesh.cuh:486-503); near_id their ids.
    int nn;
    const uint32_t* near_id;
    bool spheres;
};

// One warp (BLOCK = false) or the whole block: stages work item j's
// candidates at `base` and returns the view (ends with a warp / block barrier).
template <bool BLOCK>
__device__ RefStage stage_candidates(const DArr& A, const DLat& L, const BrickFrame& F, const uint32_t* R,
                                     const uint32_t* ids, unsigned char* base, size_t cap, float cx, float cy,
                                     float cz, float rho) {
    const int lane = BLOCK ? int(threadIdx.x) : int(threadIdx.x & 31), step = BLOCK ? int(blockDim.x) : 32;
    const int nn = int(R[R_NEAR]), n_in = int(R[R_INSIDE]), ns = int(R[R_S]), nc = int(R[R_C]), nv = int(R[R_V]);
    const int nsb = int(R[R_SBLK]), ncb = int(R[R_CBLK]);
    const uint32_t* l_near = ids + R[R_IDS];
    const uint32_t* l_s = l_near + nn;
    const uint32_t* l_soff = l_s + ns;
    const uint32_t* l_sblk = l_soff + ns + 1;
    const uint32_t* l_c = l_sblk + nsb;
    const uint32_t* l_coff = l_c + nc;
    const uint32_t* l_cblk = l_coff + nc + 1;
    const uint32_t* l_v = l_cblk + ncb;
    float4* nearA = reinterpret_cast<float4*>(base);
    float4* nearT = nearA + nn;
    float4* S = nearT + nn;
    float4* C = S + ns;
    float4* V = C + 3 * nc;
    uint32_t* s_id = reinterpret_cast<uint32_t*>(V + nv);
    uint32_t* s_off = s_id + ns;
    uint32_t* s_blk = s_off + ns + 1;
    uint32_t* c_off = s_blk + nsb;
    uint32_t* c_blk = c_off + nc + 1;
    float* s_key = reinterpret_cast<float*>(c_blk + ncb);
    const bool keyed = size_t(reinterpret_cast<unsigned char*>(s_key + ns) - base) <= cap;
    for (int i = lane; i < nn; i += step) {
        double4 c = A.sph[l_near[i]];
        float x, y, z;
        to_local(L, F, c.x, c.y, c.z, x, y, z);
        float r32 = float(c.w), rt = fmaxf(r32 - INSIDE_TOL, 0.0f);
        nearA[i] = make_float4(x, y, z, r32);
        nearT[i] = make_float4(x, y, z, rt * rt);
    }
    if (BLOCK) __syncthreads();
    else __syncwarp();
    for (int i = lane; i <= ns; i += step) s_off[i] = l_soff[i];
    for (int i = lane; i < nsb; i += step) s_blk[i] = l_sblk[i];
    for (int i = lane; i <= nc; i += step) c_off[i] = l_coff[i];
    for (int i = lane; i < ncb; i += step) c_blk[i] = l_cblk[i];
    for (int i = lane; i < ns; i += step) {
        // S candidates are near spheres: find the position (lists are short).
        uint32_t k = l_s[i];
        int pos = 0;
        for (int q = 0; q < nn; q++)
            if (l_near[q] == k) {
                pos = q;
                break;
            }
        S[i] = nearA[pos];
        s_id[i] = k;
        if (keyed) {
            const float4 c = nearA[pos];
            const float dx = cx - c.x, dy = cy - c.y, dz = cz - c.z;
            s_key[i] = fabsf(sqrtf(dx * dx + dy * dy + dz * dz) - c.w) - rho - 1e-3f;
        }
    }
    for (int i = lane; i < nc; i += step) {
        const double* c = A.circ + 12 * size_t(l_c[i]);
        float x, y, z;
        to_local(L, F, c[0], c[1], c[2], x, y, z);
        C[3 * i] = make_float4(x, y, z, float(c[9]));
        C[3 * i + 1] = make_float4(float(c[3]), float(c[4]), float(c[5]), float(c[6]));
        float key = 0.0f;
        {
            const float ux = float(c[3]), uy = float(c[4]), uz = float(c[5]);
            const float yx = cx - x, yy = cy - y, yz = cz - z;
            const float along = yx * ux + yy * uy + yz * uz;
            const float wx = yx - ux * along, wy = yy - uy * along, wz = yz - uz * along;
            const float wl = sqrtf(wx * wx + wy * wy + wz * wz), tt = wl - float(c[9]);
            key = sqrtf(along * along + tt * tt) - rho - 1e-3f;
        }
        C[3 * i + 2] = make_float4(float(c[7]), float(c[8]), __int_as_float(int(l_c[i])), key);
    }
    for (int i = lane; i < nv; i += step) {
        double4 p = A.vert[l_v[i]];
        float x, y, z;
        to_local(L, F, p.x, p.y, p.z, x, y, z);
        V[i] = make_float4(x, y, z, __int_as_float(int(l_v[i])));
    }
    if (BLOCK) __syncthreads();
    else __syncwarp();
    return RefStage{nearA, nearT, S,  C,  V,  s_id, s_off, s_blk, c_off, c_blk, n_in, ns, nc, nv,
                    keyed ? s_key : nullptr, cx, cy, cz, rho, nn, l_near, (A.flags & DARR_SPHERES) != 0};
}

struct Eval {
    float value, qx, qy, qz;
    uint32_t feat;
};

// eval_local in f32, brick-local (sesmesh.cuh eval_point semantics), by a
// group of RG lanes that all hold the same point: the lanes take RG
// candidates of a list at a time and the group keeps the least value, the
// earliest candidate on ties (a candidate replaces the best only when
// strictly smaller, in list order, as one lane walking the list would), so
// the result does not depend on RG.  gl: the lane's place in the group, gm:
// the group's lanes.  RG = 1 is one lane per point.

// The group's least (v, i), lexicographic.
template <int RG>
__device__ __forceinline__ void group_argmin(uint32_t gm, float& v, int& i) {
#pragma unroll
    for (int o = RG / 2; o; o >>= 1) {
        const float v2 = __shfl_xor_sync(gm, v, o);
        const int i2 = __shfl_xor_sync(gm, i, o);
        if (v2 < v || (v2 == v && i2 < i)) v = v2, i = i2;
    }
}

template <int RG, bool COUNT = false>
__device__ __forceinline__ Eval eval_f32(const RefStage& st, float probe, float band, float x, float y, float z,
                                         int gl, uint32_t gm, unsigned long long* ops = nullptr) {
    static_assert(RG == 1 || RG == 8 || RG == 32, "groups of 1, 8 or 32 lanes");
    Eval e;
    e.qx = x, e.qy = y, e.qz = z;
    if (st.spheres) {
        // min(band, min |x - c| - R) over the near spheres; q carries the
        // minimising sphere's centre for the slope (the refinement writes x).
        float best = band;
        e.feat = 1u << FEAT_SHIFT_D;
        for (int k0 = 0; k0 < st.nn; k0 += RG) {
            const int k = k0 + gl;
            float v = INFINITY;
            if (k < st.nn) {
                const float4 a = st.nearA[k];
                const float dx = x - a.x, dy = y - a.y, dz = z - a.z;
                v = sqrtf(dx * dx + dy * dy + dz * dz) - a.w;
                if (COUNT) *ops += 9;
            }
            int w = k;
            group_argmin<RG>(gm, v, w);
            if (v < best) {
                const float4 a = st.nearA[w];
                best = v, e.feat = (2u << FEAT_SHIFT_D) | st.near_id[w], e.qx = a.x, e.qy = a.y, e.qz = a.z;
            }
        }
        e.value = best;
        return e;
    }
    bool inside = false;
    for (int k0 = 0; k0 < st.n_in; k0 += RG) {
        const int k = k0 + gl;
        bool in = false;
        if (k < st.n_in) {
            float4 a = st.nearA[k];
            float dx = x - a.x, dy = y - a.y, dz = z - a.z;
            in = sqrtf(dx * dx + dy * dy + dz * dz) < a.w;
            if (COUNT) *ops += 9;
        }
        if (__any_sync(gm, in)) {
            inside = true;
            break;
        }
    }
    if (!inside) {
        e.value = probe;
        e.feat = 0u << FEAT_SHIFT_D;
        return e;
    }
    float best = probe + band;
    e.feat = 1u << FEAT_SHIFT_D;
    // Pruning: a candidate's value here is at least its value at the centre
    // minus |x - centre| (1-Lipschitz), the lists ascend in that centre value
    // (the gather's order), and the keys hold it less rho and a 1e-3 A margin
    // (far above f32 rounding): a loop stops once a key reaches best - slack,
    // slack = rho - |x - centre|, since no later candidate can go below best;
    // a lane skips a candidate whose key does.
    const bool pruned = st.s_key != nullptr;
    float slack = 0.0f;
    if (pruned) {
        const float qx = x - st.cx, qy = y - st.cy, qz = z - st.cz;
        slack = fmaxf(st.rho - sqrtf(qx * qx + qy * qy + qz * qz) - 1e-5f, 0.0f);
        if (COUNT && gl == 0) *ops += 11;
    }
    const int g0 = int(threadIdx.x & 31) & ~(RG - 1);  // the group's first lane
    for (int i0 = 0; i0 < st.ns; i0 += RG) {
        if (pruned && st.s_key[i0] >= best - slack) break;
        const int i = i0 + gl;
        float v = INFINITY, qx = 0.0f, qy = 0.0f, qz = 0.0f;
        if (i < st.ns && !(pruned && st.s_key[i] >= best - slack)) {
            float4 c = st.S[i];
            const float cx = c.x, cy = c.y, cz = c.z, rr = c.w;
            float dx = x - cx, dy = y - cy, dz = z - cz;
            float len = sqrtf(dx * dx + dy * dy + dz * dz);
            float lb = fabsf(len - rr);
            if (COUNT) *ops += 10;
            if (!(lb >= best || len < 1e-12f)) {
                float sc = rr / len;
                qx = cx + dx * sc, qy = cy + dy * sc, qz = cz + dz * sc;
                if (COUNT) *ops += 7;
                bool free = true;
                for (uint32_t p = st.s_off[i], e2 = st.s_off[i + 1]; p < e2 && free; p++) {
                    if (COUNT) *ops += 8;
                    float4 t = st.nearT[st.s_blk[p]];
                    float ex = qx - t.x, ey = qy - t.y, ez = qz - t.z;
                    free = ex * ex + ey * ey + ez * ez >= t.w;
                }
                if (free) v = lb;
            }
        }
        int w = i;
        group_argmin<RG>(gm, v, w);
        if (v < best) {
            const int src = g0 + (w - i0);
            best = v;
            e.feat = (2u << FEAT_SHIFT_D) | st.s_id[w];
            e.qx = __shfl_sync(gm, qx, src), e.qy = __shfl_sync(gm, qy, src), e.qz = __shfl_sync(gm, qz, src);
        }
    }
    for (int i0 = 0; i0 < st.nc; i0 += RG) {
        if (pruned && st.C[3 * i0 + 2].w >= best - slack) break;
        const int i = i0 + gl;
        float v = INFINITY, qx = 0.0f, qy = 0.0f, qz = 0.0f;
        if (i < st.nc) {
            float4 m = st.C[3 * i], u = st.C[3 * i + 1], w2 = st.C[3 * i + 2];
            if (!(pruned && w2.w >= best - slack)) {
                float yx = x - m.x, yy = y - m.y, yz = z - m.z;
                float along = yx * u.x + yy * u.y + yz * u.z;
                float wx = yx - u.x * along, wy = yy - u.y * along, wz = yz - u.z * along;
                float wl = sqrtf(wx * wx + wy * wy + wz * wz);
                float tt = wl - m.w;
                float dist = sqrtf(along * along + tt * tt);
                if (COUNT) *ops += 26;
                if (!(dist >= best)) {
                    if (COUNT) *ops += 9;
                    if (wl > 1e-12f) {
                        qx = m.x + (wx / wl) * m.w, qy = m.y + (wy / wl) * m.w, qz = m.z + (wz / wl) * m.w;
                    } else {
                        qx = m.x + u.w * m.w, qy = m.y + w2.x * m.w, qz = m.z + w2.y * m.w;
                    }
                    bool free = true;
                    for (uint32_t p = st.c_off[i], e2 = st.c_off[i + 1]; p < e2 && free; p++) {
                        if (COUNT) *ops += 8;
                        float4 t = st.nearT[st.c_blk[p]];
                        float ex = qx - t.x, ey = qy - t.y, ez = qz - t.z;
                        free = ex * ex + ey * ey + ez * ez >= t.w;
                    }
                    if (free) v = dist;
                }
            }
        }
        int w = i;
        group_argmin<RG>(gm, v, w);
        if (v < best) {
            const int src = g0 + (w - i0);
            best = v;
            e.feat = (3u << FEAT_SHIFT_D) | uint32_t(__float_as_int(st.C[3 * w + 2].z));
            e.qx = __shfl_sync(gm, qx, src), e.qy = __shfl_sync(gm, qy, src), e.qz = __shfl_sync(gm, qz, src);
        }
    }
    for (int i0 = 0; i0 < st.nv; i0 += RG) {
        const int i = i0 + gl;
        float v = INFINITY;
        if (i < st.nv) {
            float4 p = st.V[i];
            float dx = x - p.x, dy = y - p.y, dz = z - p.z;
            v = sqrtf(dx * dx + dy * dy + dz * dz);
            if (COUNT) *ops += 9;
        }
        int w = i;
        group_argmin<RG>(gm, v, w);
        if (v < best) {
            const float4 p = st.V[w];
            best = v, e.feat = (4u << FEAT_SHIFT_D) | uint32_t(__float_as_int(p.w)), e.qx = p.x, e.qy = p.y, e.qz = p.z;
        }
    }
    if (COUNT && gl == 0) *ops += 1;
    e.value = probe - best;
    return e;
}

// The f32 root search of one crossing edge (extract.rs:425-535 iteration:
// Newton with the Illinois bracket for MAX_ITER evaluations, then
// bisection), from t_start; writes edge k's outputs.
// expect (the warm start's candidate, 0 for none): the first evaluation is
// at t_start and is accepted only within the tolerance and on that
// candidate; otherwise the iteration starts over from the linear guess, as
// from t_start = t_lin with expect = 0 (the reference's fast mode).
template <int RG, bool COUNT = false>
__device__ __forceinline__ void refine_edge_f32(const RefStage& st, const RefineConsts& RC, float probe, float band,
                                                float ax, float ay, float az, uint32_t axis, float fa, float fb,
                                                float t_start, uint32_t expect, uint32_t k, const RefOut& out, int gl,
                                                uint32_t gm, unsigned long long* ops = nullptr) {
    const float h = RC.h_hi, hd = RC.h_hi + RC.h_lo;
    float t = t_start;
    float t0 = 0.0f, g0 = fa, t1 = 1.0f, g1 = fb;
    int side_ = 0;
    bool converged = false;
    uint32_t evals = 0;
    Eval last;
    last.feat = 1u << FEAT_SHIFT_D, last.qx = last.qy = last.qz = 0.0f, last.value = 0.0f;
    if (expect) {
        const float x = ax + (axis == 0 ? hd * t : 0.0f), y = ay + (axis == 1 ? hd * t : 0.0f),
                    z = az + (axis == 2 ? hd * t : 0.0f);
        const Eval e = eval_f32<RG, COUNT>(st, probe, band, x, y, z, gl, gm, ops);
        evals++;
        last = e;
        if (fabsf(e.value) <= RC.tol && e.feat == expect) converged = true;
        else t = fminf(fmaxf(fa / (fa - fb), 0.0f), 1.0f);
    }
    for (uint32_t it = 0; it < RC.max_iter && !converged; it++) {
        float x = ax + (axis == 0 ? hd * t : 0.0f), y = ay + (axis == 1 ? hd * t : 0.0f), z = az + (axis == 2 ? hd * t : 0.0f);
        Eval e = eval_f32<RG, COUNT>(st, probe, band, x, y, z, gl, gm, ops);
        evals++;
        last = e;
        float gv = e.value;
        if (fabsf(gv) <= RC.tol) {
            converged = true;
            break;
        }
        if ((gv < 0.0f) == (g0 < 0.0f)) {
            t0 = t, g0 = gv;
            if (side_ == -1) g1 *= 0.5f;
            side_ = -1;
        } else {
            t1 = t, g1 = gv;
            if (side_ == 1) g0 *= 0.5f;
            side_ = 1;
        }
        float slope = 0.0f;
        uint32_t kind = e.feat >> FEAT_SHIFT_D;
        if (kind != 0 && kind != 1) {
            // slope_of (sesmesh.cuh:599-618): towards the closest point (SES),
            // away from the sphere's centre (a sphere field).
            float wx = e.qx - x, wy = e.qy - y, wz = e.qz - z;
            if (st.spheres) wx = -wx, wy = -wy, wz = -wz;
            float len = sqrtf(wx * wx + wy * wy + wz * wz);
            if (len > 1e-12f) slope = ((axis == 0 ? wx : (axis == 1 ? wy : wz)) / len) * h;
        }
        float newton = t - gv / slope;
        if (fabsf(slope) > 1e-3f * hd && newton > t0 && newton < t1) {
            t = newton;
        } else {
            float s = (t0 * g1 - t1 * g0) / (g1 - g0);
            t = (isfinite(s) && s > t0 && s < t1) ? s : 0.5f * (t0 + t1);
        }
    }
    if (!converged) {
        bool neg0 = g0 < 0.0f;
        for (uint32_t it = 0; it < RC.max_bisect; it++) {
            t = 0.5f * (t0 + t1);
            float x = ax + (axis == 0 ? hd * t : 0.0f), y = ay + (axis == 1 ? hd * t : 0.0f), z = az + (axis == 2 ? hd * t : 0.0f);
            Eval e = eval_f32<RG, COUNT>(st, probe, band, x, y, z, gl, gm, ops);
            evals++;
            last = e;
            if (fabsf(e.value) <= RC.tol || (t1 - t0) * hd <= 2.0f * RC.tol) break;
            if ((e.value < 0.0f) == neg0) t0 = t;
            else t1 = t;
        }
    }
    if (gl) return;
    if (st.spheres) {  // a sphere field's closest point is the evaluated point (sesmesh.cuh:499-501)
        last.qx = ax + (axis == 0 ? hd * t : 0.0f), last.qy = ay + (axis == 1 ? hd * t : 0.0f),
        last.qz = az + (axis == 2 ? hd * t : 0.0f);
    }
    out.t[k] = t;
    out.feat[k] = last.feat;
    out.q[3 * size_t(k)] = last.qx, out.q[3 * size_t(k) + 1] = last.qy, out.q[3 * size_t(k) + 2] = last.qz;
    out.evals[k] = evals | (converged ? 0x80000000u : 0u);
}

// ---------------------------------------------------------------------------
// Learned warm start of the f32 refinement.  Per listed edge (row e of the
// items' edge lists): the nearest feature the sampler recorded at the edge's
// two samples (k_sample<.., FEAT>) names one candidate, a sphere, a circle or
// a SAS vertex of the structure; refine_edge_f32's own iteration (its Newton
// / Illinois steps, the same f32 operations) run on that candidate alone
// gives t_c with no field evaluation.  Where the candidate is the surface's
// nearest feature at the iterates, t_c is where the refinement would stop.
// The edge's features then go through the MLP (k_mlp_forward), whose output
// picks each edge's start: t_c or the linear guess (or, with the root head,
// is the start itself).  The refinement (k_refine<REFINE_WARM>) is the plain
// one from those starts: a start at which the field is within the tolerance is
// accepted after one evaluation, any other falls back to the bracketed
// iteration.

// One candidate in the refinement's brick-local f32 form (stage_candidates):
// S a = (x, y, z, R); C a = (centre, radius), b = (axis, e1.x), c = (e1.y,
// e1.z, -, -); V a = (x, y, z, -).
struct WarmCand {
    float4 a, b, c;
    uint32_t kind;
};

__device__ __forceinline__ WarmCand warm_cand(const DArr& A, const DLat& L, const BrickFrame& F, uint32_t word) {
    WarmCand w;
    w.kind = word >> FEAT_SHIFT_D;
    const uint32_t id = word & ((1u << FEAT_SHIFT_D) - 1);
    w.a = w.b = w.c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    // A word outside the arrangement's tables (none the sampler writes) is
    // no candidate.
    if ((w.kind == 2 && id >= A.n) || (w.kind == 3 && id >= A.nc) || (w.kind == 4 && id >= A.nv)) w.kind = 1;
    float x, y, z;
    if (w.kind == 2) {
        const double4 c = A.sph[id];
        to_local(L, F, c.x, c.y, c.z, x, y, z);
        w.a = make_float4(x, y, z, float(c.w));
    } else if (w.kind == 3) {
        const double* c = A.circ + 12 * size_t(id);
        to_local(L, F, c[0], c[1], c[2], x, y, z);
        w.a = make_float4(x, y, z, float(c[9]));
        w.b = make_float4(float(c[3]), float(c[4]), float(c[5]), float(c[6]));
        w.c = make_float4(float(c[7]), float(c[8]), 0.0f, 0.0f);
    } else if (w.kind == 4) {
        const double4 p = A.vert[id];
        to_local(L, F, p.x, p.y, p.z, x, y, z);
        w.a = make_float4(x, y, z, 0.0f);
    } else {
        w.kind = 1;
    }
    return w;
}

// The candidate's part of eval_f32 at (x, y, z): probe less its distance
// when that is below probe + band (found), else -band; q its closest point.
// The inside test and the blockers are not applied: the field decides the
// result.
__device__ __forceinline__ float cand_eval(const WarmCand& w, float probe, float band, float x, float y, float z,
                                           float& qx, float& qy, float& qz, bool& found) {
    float best = probe + band;
    found = false;
    qx = x, qy = y, qz = z;
    if (w.kind == 2) {
        const float dx = x - w.a.x, dy = y - w.a.y, dz = z - w.a.z;
        const float len = sqrtf(dx * dx + dy * dy + dz * dz);
        const float lb = fabsf(len - w.a.w);
        if (!(lb >= best || len < 1e-12f)) {
            const float sc = w.a.w / len;
            qx = w.a.x + dx * sc, qy = w.a.y + dy * sc, qz = w.a.z + dz * sc;
            best = lb, found = true;
        }
    } else if (w.kind == 3) {
        const float4 m = w.a, u = w.b;
        const float yx = x - m.x, yy = y - m.y, yz = z - m.z;
        const float along = yx * u.x + yy * u.y + yz * u.z;
        const float wx = yx - u.x * along, wy = yy - u.y * along, wz = yz - u.z * along;
        const float wl = sqrtf(wx * wx + wy * wy + wz * wz);
        const float tt = wl - m.w;
        const float dist = sqrtf(along * along + tt * tt);
        if (!(dist >= best)) {
            if (wl > 1e-12f) {
                qx = m.x + (wx / wl) * m.w, qy = m.y + (wy / wl) * m.w, qz = m.z + (wz / wl) * m.w;
            } else {
                qx = m.x + u.w * m.w, qy = m.y + w.c.x * m.w, qz = m.z + w.c.y * m.w;
            }
            best = dist, found = true;
        }
    } else if (w.kind == 4) {
        const float dx = x - w.a.x, dy = y - w.a.y, dz = z - w.a.z;
        const float v = sqrtf(dx * dx + dy * dy + dz * dz);
        if (v < best) qx = w.a.x, qy = w.a.y, qz = w.a.z, best = v, found = true;
    }
    return probe - best;
}

// refine_edge_f32's Newton / Illinois steps on the candidate alone (no
// bisection): t_c where |g| <= tol within MAX_ITER steps (*conv), the
// steps taken and the last |g|.
__device__ __forceinline__ float cand_iteration(const WarmCand& w, const RefineConsts& RC, float probe, float band,
                                                float ax, float ay, float az, uint32_t axis, float fa, float fb,
                                                int* iters, float* last_g, bool* conv) {
    const float h = RC.h_hi, hd = RC.h_hi + RC.h_lo;
    float t = fminf(fmaxf(fa / (fa - fb), 0.0f), 1.0f);
    float t0 = 0.0f, g0 = fa, t1 = 1.0f, g1 = fb;
    int side_ = 0, it = 0;
    *conv = false;
    float gv = fa;
    for (; it < int(RC.max_iter); it++) {
        const float x = ax + (axis == 0 ? hd * t : 0.0f), y = ay + (axis == 1 ? hd * t : 0.0f),
                    z = az + (axis == 2 ? hd * t : 0.0f);
        float qx, qy, qz;
        bool found;
        gv = cand_eval(w, probe, band, x, y, z, qx, qy, qz, found);
        if (fabsf(gv) <= RC.tol) {
            *conv = true;
            it++;
            break;
        }
        if ((gv < 0.0f) == (g0 < 0.0f)) {
            t0 = t, g0 = gv;
            if (side_ == -1) g1 *= 0.5f;
            side_ = -1;
        } else {
            t1 = t, g1 = gv;
            if (side_ == 1) g0 *= 0.5f;
            side_ = 1;
        }
        float slope = 0.0f;
        if (found) {
            const float wx = qx - x, wy = qy - y, wz = qz - z;
            const float len = sqrtf(wx * wx + wy * wy + wz * wz);
            if (len > 1e-12f) slope = ((axis == 0 ? wx : (axis == 1 ? wy : wz)) / len) * h;
        }
        const float newton = t - gv / slope;
        if (fabsf(slope) > 1e-3f * hd && newton > t0 && newton < t1) {
            t = newton;
        } else {
            const float sv = (t0 * g1 - t1 * g0) / (g1 - g0);
            t = (isfinite(sv) && sv > t0 && sv < t1) ? sv : 0.5f * (t0 + t1);
        }
    }
    *iters = it;
    *last_g = fabsf(gv);
    return t;
}

__device__ __forceinline__ float log_mismatch(float m) { return log10f(fmaxf(m, 1e-9f)) / 9.0f + 1.0f; }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// Features of row e (SMB_MLP_FEATURES = 32 f32):
//   0-1   fa / h, fb / h
//   2-7   finite-difference gradients of the samples at both ends (central
//         inside the brick, else one-sided)
//   8     t_lin = fa / (fa - fb)
//   9-11  the candidate's kind, one-hot (sphere, circle, SAS vertex; zeros
//         without one)
//   12    1 where both samples name the same feature
//   13    1 where they name two different candidates
//   14    1 where the candidate's iteration converged
//   15    its steps / 8
//   16    (t_c - t_lin) * 8, clamped to [-4, 4]
//   17    t_c (t_lin without a converged candidate)
//   18    log10(max(m, 1e-9)) / 9 + 1 of its last |g|
//   19-20 the same of the candidate's mismatch at the two samples,
//         |g(end) - f(end)|
//   21-23 the candidate's centre (sphere, circle) or position (vertex)
//         less the edge midpoint, / 4 A
//   24    its size / 4 A: the atom radius R - probe (sphere), the circle's
//         radius, 0 (vertex)
//   25-26 spacing h and probe radius (A)
//   27-28 both gradients along the edge times h / (fb - fa), clamped to
//         [-10, 10]
//   29-30 |gradient| - 1 at both ends, clamped to [-4, 4]
//   31    the other sample's feature kind / 4
// starts[e] = (t_c, or -1 without a converged candidate; t_lin).
// Row e's features into f and its starts (t_c or -1, t_lin); *cand gets the
// candidate's feature word (0 without one).
template <bool MANY>
__device__ __forceinline__ float2 warm_row(const DArr& A0, const DLat& L0, const RefineConsts& RC0, const int4* keys,
                                           const uint32_t* work, uint32_t n_items, const uint32_t* rec,
                                           const uint32_t* edges, const float2* edge_vals, const uint32_t* item_off,
                                           const uint32_t* item_edges, const float* values, const uint32_t* feats,
                                           const Scene& S, uint32_t e, float* f, uint32_t* cand,
                                           uint32_t item = 0xFFFFFFFFu) {
    // The item holding row e: the last lo with item_off[lo] <= e (items
    // without rows repeat an offset); `item` when the caller found it.
    uint32_t lo = item;
    if (lo == 0xFFFFFFFFu) {
        lo = 0;
        uint32_t hi = n_items;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (item_off[mid] <= e) lo = mid;
            else hi = mid;
        }
    }
    const uint32_t brick = work[lo] >> 3;
    const int4 key = keys[brick];
    const DArr& A = MANY ? S.arr[key.w] : A0;
    const DLat& L = MANY ? S.lat[key.w] : L0;
    const RefineConsts& RC = MANY ? S.rc[key.w] : RC0;
    const uint32_t k = item_edges[e];
    const int b = L.b, side = b + 1;
    const float h = RC.h_hi, hd = RC.h_hi + RC.h_lo, probe = L.probe32, band = L.band32;
    const uint32_t code = edges[k], cell = code / 3, axis = code % 3;
    const int ex = int(cell % b), ey = int((cell / b) % b), ez = int(cell / (b * b));
    const float ax = float(ex) * h + float(ex) * RC.h_lo, ay = float(ey) * h + float(ey) * RC.h_lo,
                az = float(ez) * h + float(ez) * RC.h_lo;
    const float2 fv = edge_vals[k];
    const float fa = fv.x, fb = fv.y;
    const float t_lin = fminf(fmaxf(fa / (fa - fb), 0.0f), 1.0f);
    const float* val = values + size_t(brick) * L.spb;
    uint32_t st[8];
    for (int q = 0; q < 8; q++) st[q] = rec[(size_t(brick) * 8 + q) * REC_WORDS + R_STATE];
    // The recorded feature of a sample its sampled, unflagged owner wrote.
    auto word = [&](int x, int y, int z) -> uint32_t {
        bool positive;
        const int o = sample_owner(x, y, z, L.sub, st, &positive);
        if (o < 0 || rec[(size_t(brick) * 8 + o) * REC_WORDS + R_FLAGS] != 0) return 1u << FEAT_SHIFT_D;
        return feats[size_t(brick) * L.spb + (z * side + y) * side + x];
    };
    const int bx = ex + (axis == 0), by = ey + (axis == 1), bz = ez + (axis == 2);
    const uint32_t wa = word(ex, ey, ez), wb = word(bx, by, bz);
    const uint32_t ka = wa >> FEAT_SHIFT_D, kb = wb >> FEAT_SHIFT_D;
    const uint32_t primary = ka >= 2 ? wa : (kb >= 2 ? wb : (1u << FEAT_SHIFT_D));
    const BrickFrame F = brick_frame(L, RC, key);
    const WarmCand w = warm_cand(A, L, F, primary);
    *cand = w.kind >= 2 ? primary : 0u;
    auto V = [&](int x, int y, int z) { return val[(z * side + y) * side + x]; };
    auto grad = [&](int x, int y, int z, float* g) {
        const int c[3] = {x, y, z};
        for (int d = 0; d < 3; d++) {
            int lo3[3] = {c[0], c[1], c[2]}, hi3[3] = {c[0], c[1], c[2]};
            lo3[d]--, hi3[d]++;
            if (lo3[d] >= 0 && hi3[d] <= b) g[d] = (V(hi3[0], hi3[1], hi3[2]) - V(lo3[0], lo3[1], lo3[2])) / (2.0f * h);
            else if (hi3[d] <= b) g[d] = (V(hi3[0], hi3[1], hi3[2]) - V(x, y, z)) / h;
            else g[d] = (V(x, y, z) - V(lo3[0], lo3[1], lo3[2])) / h;
        }
    };
    f[0] = fa / h, f[1] = fb / h;
    grad(ex, ey, ez, f + 2);
    grad(bx, by, bz, f + 5);
    f[8] = t_lin;
    f[9] = w.kind == 2, f[10] = w.kind == 3, f[11] = w.kind == 4;
    f[12] = wa == wb;
    f[13] = ka >= 2 && kb >= 2 && wa != wb;
    float t_c = -1.0f;
    if (w.kind >= 2) {
        int iters = 0;
        float last_g = 0.0f;
        bool conv = false;
        const float tc = cand_iteration(w, RC, probe, band, ax, ay, az, axis, fa, fb, &iters, &last_g, &conv);
        if (conv) t_c = tc;
        f[14] = conv, f[15] = float(iters) * 0.125f;
        f[16] = clampf(tc - t_lin, -0.5f, 0.5f) * 8.0f;
        f[17] = conv ? tc : t_lin;
        f[18] = log_mismatch(last_g);
        float qx, qy, qz;
        bool found;
        const float bxf = ax + (axis == 0 ? hd : 0.0f), byf = ay + (axis == 1 ? hd : 0.0f),
                    bzf = az + (axis == 2 ? hd : 0.0f);
        f[19] = log_mismatch(fabsf(cand_eval(w, probe, band, ax, ay, az, qx, qy, qz, found) - fa));
        f[20] = log_mismatch(fabsf(cand_eval(w, probe, band, bxf, byf, bzf, qx, qy, qz, found) - fb));
        const float mx = ax + (axis == 0 ? 0.5f * hd : 0.0f), my = ay + (axis == 1 ? 0.5f * hd : 0.0f),
                    mz = az + (axis == 2 ? 0.5f * hd : 0.0f);
        f[21] = (w.a.x - mx) * 0.25f, f[22] = (w.a.y - my) * 0.25f, f[23] = (w.a.z - mz) * 0.25f;
        f[24] = (w.kind == 2 ? w.a.w - probe : (w.kind == 3 ? w.a.w : 0.0f)) * 0.25f;
    } else {
        f[14] = 0.0f, f[15] = 0.0f, f[16] = 0.0f, f[17] = t_lin, f[18] = 1.0f, f[19] = 1.0f, f[20] = 1.0f;
        f[21] = f[22] = f[23] = f[24] = 0.0f;
    }
    f[25] = h, f[26] = probe;
    const float inv = h / (fb - fa);
    f[27] = clampf(f[2 + axis] * inv, -10.0f, 10.0f);
    f[28] = clampf(f[5 + axis] * inv, -10.0f, 10.0f);
    f[29] = clampf(sqrtf(f[2] * f[2] + f[3] * f[3] + f[4] * f[4]) - 1.0f, -4.0f, 4.0f);
    f[30] = clampf(sqrtf(f[5] * f[5] + f[6] * f[6] + f[7] * f[7]) - 1.0f, -4.0f, 4.0f);
    f[31] = float(primary == wa ? kb : ka) * 0.25f;
    return make_float2(t_c, t_lin);
}

// The item holding row e (the last lo with item_off[lo] <= e), found by a
// warp for its 32 consecutive rows e0 .. e0 + 31 (e0 < E = item_off[n]):
// each step probes 32 points that split (lo, hi) 33 ways, keeping
// item_off[lo] <= e0 < item_off[hi], so a few steps replace the 19 of a
// lane's own binary search over 384 K items; each lane then walks from the
// warp's item to its own row's.  All 32 lanes take part.
__device__ __forceinline__ uint32_t warp_item_of(const uint32_t* item_off, uint32_t n_items, uint32_t e0, uint32_t e,
                                                 uint32_t E) {
    const int lane = int(threadIdx.x & 31);
    uint32_t lo = 0, hi = n_items;
    while (hi - lo > 1) {
        const uint32_t span = hi - lo;
        const uint32_t p = span <= 32 ? lo + 1 + uint32_t(lane)
                                      : lo + uint32_t((unsigned long long)span * uint32_t(lane + 1) / 33ull);
        const bool valid = p > lo && p < hi;
        const bool le = valid && item_off[p] <= e0;
        const uint32_t m_le = __ballot_sync(0xffffffffu, le), m_gt = __ballot_sync(0xffffffffu, valid && !le);
        const uint32_t nlo = m_le ? __shfl_sync(0xffffffffu, p, 31 - __clz(int(m_le))) : lo;
        const uint32_t nhi = m_gt ? __shfl_sync(0xffffffffu, p, __ffs(int(m_gt)) - 1) : hi;
        lo = nlo, hi = nhi;
    }
    if (e < E)
        while (item_off[lo + 1] <= e) lo++;
    return lo;
}

// Features of every row (export for training: smb_batch_edge_features).
template <bool MANY>
__global__ void __launch_bounds__(256) k_warm_features(DArr A0, DLat L0, RefineConsts RC0, const int4* keys,
                                                       const uint32_t* work, uint32_t n_host, const uint32_t* rec,
                                                       const uint32_t* edges, const float2* edge_vals,
                                                       const uint32_t* item_off, const uint32_t* item_edges,
                                                       const float* values, const uint32_t* feats, float* x_out,
                                                       Scene S) {
    const uint32_t n_items = MANY ? uint32_t(*S.n_work) : n_host;
    const uint32_t E = item_off[n_items];
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < E; e += gridDim.x * blockDim.x) {
        float f[MLP_IN];
        uint32_t cand;
        warm_row<MANY>(A0, L0, RC0, keys, work, n_items, rec, edges, edge_vals, item_off, item_edges, values, feats, S,
                       e, f, &cand);
        float4* xo = reinterpret_cast<float4*>(x_out + size_t(e) * MLP_IN);
        for (int c = 0; c < MLP_IN / 4; c++) xo[c] = make_float4(f[4 * c], f[4 * c + 1], f[4 * c + 2], f[4 * c + 3]);
    }
}

// The warm start's choice per row, features and MLP fused: a persistent CTA
// of 128 threads per 128-row tile at a time (thread r computes row r's
// features into the tile, one tensor-core forward pass per tile, weights
// and TMEM set up once per CTA).  start[e] = (t_c, the candidate's feature
// word) where the gate answers >= 0.5, the candidate's iteration converged
// and both samples name that candidate (feature 12: where they name two,
// the edge can hold a root of each, and t_c may be the one the iteration
// from t_lin does not reach), else (t_lin, 0) (use 0); or (the output
// itself, a root parameter in [0, 1], 0) (use 1).  The word travels as
// float bits.
template <bool MANY>
__global__ void __launch_bounds__(128) k_warm_starts(DArr A0, DLat L0, RefineConsts RC0, const int4* keys,
                                                     const uint32_t* work, uint32_t n_host, const uint32_t* rec,
                                                     const uint32_t* edges, const float2* edge_vals,
                                                     const uint32_t* item_off, const uint32_t* item_edges,
                                                     const float* values, const uint32_t* feats, MlpDev P, int use,
                                                     float2* start, unsigned long long* counters, Scene S) {
    const uint32_t n_items = MANY ? uint32_t(*S.n_work) : n_host;
    const uint32_t E = item_off[n_items];
    const uint32_t tiles = (E + MLP_ROWS - 1) / MLP_ROWS;
    if (blockIdx.x >= tiles) return;  // the whole CTA, before any TMEM is taken
    extern __shared__ __align__(128) unsigned char wsm[];
    MlpSmem& M = *reinterpret_cast<MlpSmem*>(wsm);
    mlp_setup(M, P);
    uint32_t phase = 0;
    for (uint32_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const uint32_t e = tile * MLP_ROWS + threadIdx.x;
        const uint32_t e0 = e & ~31u;  // the warp's first row (warp-uniform)
        const uint32_t item = e0 < E ? warp_item_of(item_off, n_items, e0, e, E) : 0u;
        float f[MLP_IN];
        float2 sc = make_float2(-1.0f, 0.0f);
        uint32_t cand = 0;
        if (e < E) {
            sc = warm_row<MANY>(A0, L0, RC0, keys, work, n_items, rec, edges, edge_vals, item_off, item_edges, values,
                                feats, S, e, f, &cand, item);
        } else {
            for (int c = 0; c < MLP_IN; c++) f[c] = 0.0f;
        }
        mlp_put_row(M, f);
        float p = 0.0f;
        const bool ok = mlp_forward(M, phase, &p, nullptr, nullptr, nullptr);
        if (!ok && threadIdx.x == 0) atomicAdd(&counters[CNT_TIMEOUT], 1ull);
        if (e < E) {
            float2 w = make_float2(sc.y, 0.0f);
            if (ok && use == 1) w.x = p;
            else if (ok && p >= 0.5f && sc.x >= 0.0f && f[12] > 0.5f) w = make_float2(sc.x, __uint_as_float(cand));
            start[e] = w;
        }
    }
    mlp_teardown(M);
}

// Fast-mode refinement over the work items' edge lists (k_item_edges).
// Work is claimed from a queue (counters[CNT_QUEUE]) by persistent CTAs:
// each warp claims items and refines the item's edges, a group of RG lanes
// per edge, candidates staged in the warp's shared region; REFINE_PLAIN
// starts each edge at the linear guess (the reference's fast mode),
// REFINE_WARM at start[e] (row e of the edge lists: the warm start's
// choice).  WIDE: candidates too large for a region per warp; the CTA
// refines one item at a time with all its threads.
constexpr int REFINE_WARPS = 4;
// Warps of a block in the plain pass over the listed sub-blocks (those over
// a warp's region): the block's warps take one sub-block's edges.
#ifndef WIDE_LIST_WARPS
#define WIDE_LIST_WARPS 16
#endif

// Largest staging region for the two-warp blocks of the single-structure
// refinement (ten or more blocks to an SM; at most 80 registers, so twelve
// blocks where the regions allow).
constexpr size_t PAIR_REGION_MAX = 20480;

struct RefinePlan {
    uint32_t cand_bytes;  // one staging region
};

// OVF: a block-wide pass (WIDE) that lists the sub-blocks over its region
// (the split pass); per-warp passes always can.
template <int MODE, bool WIDE, bool MANY, int RG, int NT = 32 * REFINE_WARPS, bool COUNT = false, bool OVF = false>
__global__ void __launch_bounds__(NT, NT == 64 ? 12 : (NT > 32 * REFINE_WARPS ? 2 : 1)) k_refine(
    DArr A0, DLat L0, RefineConsts RC0, const int4* keys, const uint32_t* work, const uint32_t* rec, const uint32_t* ids,
    const uint32_t* edges, const float2* edge_vals, const uint32_t* item_off, const uint32_t* item_edges,
    uint32_t n_host, RefOut out, const float2* start, RefinePlan P, unsigned long long* counters, Scene S,
    uint32_t* ovf, const uint32_t* list) {
    const uint32_t n_items = MANY ? uint32_t(*S.n_work) : n_host;
    extern __shared__ __align__(128) float4 rs[];
    __shared__ uint32_t sh_q, sh_edge, sh_wedge[REFINE_WARPS];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = reinterpret_cast<unsigned char*>(rs) + (WIDE ? 0 : size_t(warp) * P.cand_bytes);
    unsigned int* queue = reinterpret_cast<unsigned int*>(&counters[CNT_QUEUE]);
    auto edge_geom = [&](const DLat& L, const RefineConsts& RC, uint32_t k, uint32_t& axis, float& ax, float& ay,
                         float& az) {
        const int b = L.b;
        const float h = RC.h_hi;
        const uint32_t code = edges[k], cell = code / 3;
        axis = code % 3;
        const int ex = int(cell % b), ey = int((cell / b) % b), ez = int(cell / (b * b));
        ax = float(ex) * h + float(ex) * RC.h_lo, ay = float(ey) * h + float(ey) * RC.h_lo,
        az = float(ez) * h + float(ez) * RC.h_lo;
    };
    // Refines item i's edges with the lanes of one warp (WIDE: the block).
    auto refine_item = [&](uint32_t i) {
        const uint32_t a0 = item_off[i], a1 = item_off[i + 1];
        if (a0 == a1) return;
        const uint32_t j = work[i], brick = j >> 3;
        const int4 key = keys[brick];
        const DArr& A = MANY ? S.arr[key.w] : A0;
        const DLat& L = MANY ? S.lat[key.w] : L0;
        const RefineConsts& RC = MANY ? S.rc[key.w] : RC0;
        const float probe = L.probe32, band = L.band32;
        const BrickFrame F = brick_frame(L, RC, key);
        const uint32_t* R = rec + size_t(j) * REC_WORDS;
        if ((!WIDE || OVF) && ovf) {
            // A sub-block whose candidates outgrow this warp's (block's)
            // region goes to the list the whole-block pass takes after this
            // one.
            const size_t nn = R[R_NEAR], ns = R[R_S], nc = R[R_C], nv = R[R_V];
            const size_t need = (2 * nn + ns + 3 * nc + nv) * 16 + (2 * ns + 1 + R[R_SBLK] + nc + 1 + R[R_CBLK]) * 4;
            if (need > P.cand_bytes) {
                if (WIDE ? threadIdx.x == 0 : lane == 0) ovf[1 + atomicAdd(ovf, 1u)] = i;
                return;
            }
        }
        if (WIDE) {
            __syncthreads();
            if (threadIdx.x == 0) sh_edge = a0;  // read after the staging's barrier
        } else {
            __syncwarp();
            if (lane == 0) sh_wedge[warp] = a0;
        }
        const int sb = int(j & 7), sub = L.sub;
        const float h32 = float(L.h), half = 0.5f * float(sub);
        const float ccx = (float((sb & 1) * sub) + half) * h32, ccy = (float(((sb >> 1) & 1) * sub) + half) * h32,
                    ccz = (float((sb >> 2) * sub) + half) * h32;
        const float crho = float(L.rho_sub) * 1.000001f + 1e-6f;
        const RefStage st = WIDE ? stage_candidates<true>(A, L, F, R, ids, mine, P.cand_bytes, ccx, ccy, ccz, crho)
                                 : stage_candidates<false>(A, L, F, R, ids, mine, P.cand_bytes, ccx, ccy, ccz, crho);
        // A group of RG lanes per edge.
        const uint32_t step = (WIDE ? blockDim.x : 32u) / RG, gl = lane % RG;
        const uint32_t gm = (0xffffffffu >> (32 - RG)) << (lane & ~uint32_t(RG - 1));
        auto edge = [&](uint32_t e) {
            const uint32_t k = item_edges[e];
            uint32_t axis;
            float ax, ay, az;
            edge_geom(L, RC, k, axis, ax, ay, az);
            const float2 fv = edge_vals[k];
            float t0 = fminf(fmaxf(fv.x / (fv.x - fv.y), 0.0f), 1.0f);
            uint32_t expect = 0;
            if (MODE == REFINE_WARM) {
                const float2 w = start[e];
                t0 = w.x, expect = __float_as_uint(w.y);
            }
            unsigned long long ops = 0;
            refine_edge_f32<RG, COUNT>(st, RC, probe, band, ax, ay, az, axis, fv.x, fv.y, t0, expect, k, out, int(gl),
                                       gm, COUNT ? &ops : nullptr);
            if (COUNT) {
                for (int o = RG / 2; o; o >>= 1) ops += __shfl_xor_sync(gm, ops, o);
                if (gl == 0 && ops) atomicAdd(&counters[CNT_OPS], ops);
            }
        };
        if (WIDE || RG < 32) {
            // The block's (warp's) groups claim the edges one at a time
            // (their evaluation counts differ).
            uint32_t* next = WIDE ? &sh_edge : &sh_wedge[warp];
            const uint32_t leader = lane & ~uint32_t(RG - 1);
            for (;;) {
                uint32_t e = 0;
                if (gl == 0) e = atomicAdd(next, 1u);
                e = __shfl_sync(gm, e, leader);
                if (e >= a1) break;
                edge(e);
            }
        } else {
            for (uint32_t e = a0 + lane / RG; e < a1; e += step) edge(e);
        }
    };
    if constexpr (WIDE) {
        if (list) {
            // The sub-blocks the per-warp pass listed, one per block at a time.
            const uint32_t n = *list;
            for (;;) {
                __syncthreads();
                if (threadIdx.x == 0) sh_q = atomicAdd(queue, 1u);
                __syncthreads();
                const uint32_t q = sh_q;
                if (q >= n) break;
                refine_item(list[1 + q]);
            }
            return;
        }
        // Items in queue order, one per block at a time.
        for (;;) {
            __syncthreads();
            if (threadIdx.x == 0) sh_q = atomicAdd(queue, 1u);
            __syncthreads();
            const uint32_t q = sh_q;
            if (q >= n_items) break;
            refine_item(q);
        }
        return;
    } else {
        for (;;) {
            uint32_t i = 0;
            if (lane == 0) i = atomicAdd(queue, 1u);
            i = __shfl_sync(0xffffffffu, i, 0);
            if (i >= n_items) break;
            refine_item(i);
        }
    }
}

// ---------------------------------------------------------------------------
// Host launchers.  Each counts the kernels it launches.
static std::atomic<unsigned long long> g_launches{0};
unsigned long long kernel_launches() { return g_launches.load(); }
void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
#define COUNT(n) g_launches.fetch_add(n, std::memory_order_relaxed)

void launch_selftest(const float* a, const float* b, uint32_t* out, uint32_t n, cudaStream_t s) {
    COUNT(1);
    k_selftest<<<(n + 255) / 256, 256, 0, s>>>(a, b, out, n);
}

void launch_scan(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* keep, unsigned long long* tiles,
                 unsigned long long* total, cudaStream_t s) {
    uint32_t n_tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (n_tiles == 0) {
        cudaMemsetAsync(total, 0, sizeof(unsigned long long), s);
        return;
    }
    COUNT(3);
    k_scan_tiles<<<n_tiles, SCAN_THREADS, 0, s>>>(in, n, tiles);
    k_scan_tile_sums<<<1, SCAN_THREADS, 0, s>>>(tiles, n_tiles, total);
    k_scan_apply<<<n_tiles, SCAN_THREADS, 0, s>>>(in, n, tiles, out, keep);
}

uint32_t scan_tiles_needed(uint32_t n) { return (n + SCAN_TILE - 1) / SCAN_TILE + 1; }

void launch_mark_touched(const DArr& A, const DLat& L, const BrickBox& box, uint32_t* flags, int* err, cudaStream_t s,
                         const Scene* many, uint32_t n_total) {
    if (many) {
        if (n_total) COUNT(1), k_mark_touched<true><<<(n_total + 127) / 128, 128, 0, s>>>(A, L, box, flags, err, *many,
                                                                                          n_total);
        return;
    }
    if (A.n) COUNT(1), k_mark_touched<false><<<(A.n + 127) / 128, 128, 0, s>>>(A, L, box, flags, err, Scene{}, 0);
}

void launch_classify_bricks(const DArr& A, const DLat& L, const BrickBox& box, const uint32_t* touched, uint32_t n,
                            uint32_t* surface, cudaStream_t s, const Scene* many) {
    if (!n) return;
    COUNT(1);
    if (many) k_classify_bricks<true><<<(n + 7) / 8, 256, 0, s>>>(A, L, box, touched, n, surface, *many);
    else k_classify_bricks<false><<<(n + 7) / 8, 256, 0, s>>>(A, L, box, touched, n, surface, Scene{});
}

void launch_cells_to_keys(const BrickBox& box, const uint32_t* cells, uint32_t n, int4* keys, cudaStream_t s,
                          const Scene* many) {
    if (!n) return;
    COUNT(1);
    if (many) k_cells_to_keys<true><<<(n + 255) / 256, 256, 0, s>>>(box, cells, n, keys, *many);
    else k_cells_to_keys<false><<<(n + 255) / 256, 256, 0, s>>>(box, cells, n, keys, Scene{});
}

void launch_substates(const DArr& A, const DLat& L, const int4* keys, uint32_t n, uint32_t* rec, uint32_t* sampled,
                      cudaStream_t s, const Scene* many) {
    if (!n) return;
    COUNT(1);
    if (many) k_substates<true><<<n, 256, 0, s>>>(A, L, keys, n, rec, sampled, *many);
    else k_substates<false><<<n, 256, 0, s>>>(A, L, keys, n, rec, sampled, Scene{});
}

cudaError_t launch_gather(const DArr& A, const DLat& L, const int4* keys, const uint32_t* work, uint32_t n,
                          const GatherOut& O, const GatherCaps& caps, int warps, cudaStream_t s, const Scene* many) {
    if (!n) return cudaSuccess;
    size_t smem = gather_smem_bytes(caps) * size_t(warps);
    // Lists of several warp rounds (the caps come from the largest lists
    // seen): blocker rows with four lookups in flight.
    auto kern = many ? k_gather<true, false> : caps.near >= 128 ? k_gather<false, true> : k_gather<false, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    COUNT(1);
    // Many structures: n is an upper bound of the device count; the grid
    // strides (a few waves of blocks, not one per possible item).
    uint32_t blocks = (n + warps - 1) / warps;
    if (many) blocks = std::min<uint32_t>(blocks, 148u * 32u);
    kern<<<blocks, 32 * warps, smem, s>>>(A, L, keys, work, n, O, caps, many ? *many : Scene{});
    return cudaGetLastError();
}

cudaError_t launch_sample(const DLat& L, const int4* keys, const uint32_t* work, uint32_t n, const uint32_t* rec,
                          const uint4* pack, uint32_t max_units, float* values, unsigned long long* counters, bool tma,
                          bool count, cudaStream_t s, const Scene* many, uint32_t* list, size_t small,
                          const uint32_t* ids, uint32_t* feats) {
    if (!n) return cudaSuccess;
    size_t smem = size_t(max_units) * 16;
    const bool feat = feats != nullptr && !count;
    auto kern = feat ? (many ? k_sample<true, false, true, false, true>
                             : (tma ? k_sample<true, false, false, false, true>
                                    : k_sample<false, false, false, false, true>))
                     : many ? k_sample<true, false, true>
                     : (count ? k_sample<true, true, false>
                              : (tma ? k_sample<true, false, false> : k_sample<false, false, false>));
    // Shared memory for the largest block on every CTA can leave an SM a
    // few CTAs: the blocks up to `small` bytes run first with that much,
    // the rest after them with all of it.
    const bool split = list && !many && !count && tma && small >= 16 && smem > small;
    const size_t first = split ? small / 16 * 16 : smem;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(first));
    if (e != cudaSuccess) return e;
    if (split && (e = cudaMemsetAsync(list, 0, 4, s)) != cudaSuccess) return e;
    COUNT(1);
    kern<<<n, 128, first, s>>>(L, keys, work, n, rec, pack, values, counters, many ? *many : Scene{},
                               uint32_t(first / 16), split ? list : nullptr, ids, feats);
    if (!split) return cudaGetLastError();
    auto rest = feat ? k_sample<true, false, false, true, true> : k_sample<true, false, false, true>;
    if ((e = cudaFuncSetAttribute(rest, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) != cudaSuccess)
        return e;
    COUNT(1);
    rest<<<n, 128, smem, s>>>(L, keys, work, n, rec, pack, values, counters, Scene{}, 0, list, ids, feats);
    return cudaGetLastError();
}

cudaError_t launch_mc(const DLat& L, uint32_t n, float* values, const uint32_t* rec, uint32_t* counts, const uint32_t* edge_off,
                      const uint32_t* tri_off, uint32_t* edges, float2* edge_vals, uint32_t* tris, bool fill,
                      cudaStream_t s, const int4* keys, unsigned long long edge_cap, unsigned long long tri_cap,
                      const Scene* many) {
    if (!n) return cudaSuccess;
    size_t smem = size_t(L.spb) * 4;
    // Brick edges 10 (the default) and 8 and 16 (those the many-structure
    // tuning tries) with constant divisors.
    auto pick = [&](auto bc) {
        constexpr int BC = decltype(bc)::value;
        return many ? (fill ? k_mc<true, true, BC> : k_mc<false, true, BC>)
                    : (fill ? k_mc<true, false, BC> : k_mc<false, false, BC>);
    };
    auto kern = L.b == 10  ? pick(std::integral_constant<int, 10>{})
                : L.b == 8  ? pick(std::integral_constant<int, 8>{})
                : L.b == 16 ? pick(std::integral_constant<int, 16>{})
                            : pick(std::integral_constant<int, 0>{});
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    COUNT(1);
    kern<<<n, MC_THREADS, smem, s>>>(L, n, values, rec, counts, edge_off, tri_off, edges, edge_vals, tris, keys, edge_cap,
                                     tri_cap, many ? *many : Scene{});
    return cudaGetLastError();
}

void launch_copy_count(unsigned long long* dst, const unsigned long long* src, cudaStream_t s) {
    COUNT(1);
    k_copy_count<<<1, 32, 0, s>>>(dst, src);
}

void launch_put_total(uint32_t* dst, const unsigned long long* total, cudaStream_t s) {
    COUNT(1);
    k_put_total<<<1, 32, 0, s>>>(dst, total);
}

size_t refine_smem_bytes(uint32_t nn, uint32_t ns, uint32_t nc, uint32_t nv, uint32_t nsb, uint32_t ncb) {
    return (size_t(2) * nn + ns + 3 * size_t(nc) + nv) * 16 + (size_t(ns) * 2 + 1 + nsb + nc + 1 + ncb) * 4;
}

void launch_item_edges(const DLat& L, const uint32_t* work, uint32_t n, const uint32_t* rec, const uint32_t* edge_off,
                       const uint32_t* edges, uint32_t* counts, uint32_t* item_off, uint32_t* item_edges,
                       unsigned long long* tiles, unsigned long long* total, unsigned long long* counters,
                       cudaStream_t s, const Scene* many, const int4* keys, const uint8_t* mask, bool all_items) {
    const uint32_t blocks = (n * 32 + 255) / 256;
    const Scene sc = many ? *many : Scene{};
    if (n) {
        COUNT(1);
        if (many) k_item_edges<false, true><<<blocks, 256, 0, s>>>(L, work, n, rec, edge_off, edges, counts, item_off,
                                                                 item_edges, total, counters, keys, sc, mask, mask != nullptr || all_items);
        else k_item_edges<false, false><<<blocks, 256, 0, s>>>(L, work, n, rec, edge_off, edges, counts, item_off,
                                                              item_edges, total, counters, keys, sc, mask, mask != nullptr || all_items);
    }
    launch_scan(counts, n, item_off, nullptr, tiles, total, s);
    COUNT(1);
    if (many) k_item_edges<true, true><<<max(blocks, 1u), 256, 0, s>>>(L, work, n, rec, edge_off, edges, counts, item_off,
                                                                     item_edges, total, counters, keys, sc, mask, mask != nullptr || all_items);
    else k_item_edges<true, false><<<max(blocks, 1u), 256, 0, s>>>(L, work, n, rec, edge_off, edges, counts, item_off,
                                                                  item_edges, total, counters, keys, sc, mask, mask != nullptr || all_items);
}

cudaError_t launch_refine(const DArr& A, const DLat& L, const RefineConsts& RC, const int4* keys, const uint32_t* work,
                          const uint32_t* rec, const uint32_t* ids, const uint32_t* edges, const float2* edge_vals,
                          const uint32_t* item_off, const uint32_t* item_edges, uint32_t n_items, float* t,
                          uint32_t* feat, float* q, uint32_t* evals, size_t cand_bytes, int mode, const float2* start,
                          unsigned long long* counters, int sms, size_t smem_limit, cudaStream_t s, size_t* smem_out,
                          const Scene* many, uint32_t* ovf, size_t region, int group, bool count) {
    auto al = [](size_t v) { return (v + 127) / 128 * 128; };
    RefinePlan P;
    P.cand_bytes = uint32_t(al(cand_bytes));
    const size_t narrow = size_t(REFINE_WARPS) * P.cand_bytes;
    const size_t wide = P.cand_bytes;
    // One staging region per warp (an item per warp in flight, as many items
    // per SM as regions fit) while four fit in a block, else one per block.
    // The single-structure pass instead gives blocks of two warps one region
    // each: of the largest sub-block's size where that is at most
    // PAIR_REGION_MAX, else of the size asked for (default: an eighth of the
    // SM's shared memory), handing the sub-blocks that outgrow it to a
    // whole-block pass over a list.
    const bool use_wide = narrow > smem_limit;
    size_t small = region ? region / 128 * 128 : (smem_limit / 2 - 1024) / REFINE_WARPS / 128 * 128;
    small = std::max<size_t>(std::min(small, size_t(P.cand_bytes)), 128);
    const bool split = !many && ovf && (use_wide || small < P.cand_bytes);
    const size_t smem = use_wide ? wide : narrow;
    if (smem_out) *smem_out = smem;
    if (!n_items) return cudaSuccess;
    // Launches kern with `bytes` of shared memory on as many CTAs as stay
    // resident.
    auto run = [&](auto kern, const RefinePlan& PL, size_t bytes, uint32_t* o, const uint32_t* list, uint32_t units,
                   int threads = 32 * REFINE_WARPS) -> cudaError_t {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        if (e != cudaSuccess) return e;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, bytes);
        if (e != cudaSuccess) return e;
        const uint32_t grid = std::min<uint32_t>(units, uint32_t(std::max(1, sms * std::max(per_sm, 1))));
        cudaMemsetAsync(&counters[CNT_QUEUE], 0, sizeof(unsigned long long), s);
        COUNT(1);
        kern<<<grid, threads, bytes, s>>>(A, L, RC, keys, work, rec, ids, edges, edge_vals, item_off, item_edges,
                                          n_items, RefOut{t, feat, q, evals}, start, PL, counters,
                                          many ? *many : Scene{}, o, list);
        return cudaGetLastError();
    };
    const uint32_t quads = (n_items + REFINE_WARPS - 1) / REFINE_WARPS;
    const bool g32 = group == 32, warm = mode == REFINE_WARM;
    auto pick = [&](auto narrow_k, auto wide_k) { return use_wide ? wide_k : narrow_k; };
    if (count && !many) {
        // The counting pass: groups of 8, every sub-block in one pass.
        constexpr int NW = 32 * REFINE_WARPS;
        auto kern = warm ? pick(k_refine<REFINE_WARM, false, false, 8, NW, true>,
                                k_refine<REFINE_WARM, true, false, 8, NW, true>)
                         : pick(k_refine<REFINE_PLAIN, false, false, 8, NW, true>,
                                k_refine<REFINE_PLAIN, true, false, 8, NW, true>);
        return run(kern, P, smem, nullptr, nullptr, use_wide ? n_items : quads);
    }
    // Lists of up to PAIR_REGION_MAX bytes (single structure, groups of 8,
    // no region asked for): blocks of two warps that share one staging
    // region per sub-block.  A region then costs a warp half of what a region
    // of its own does, so the registers, not the shared memory, set the warps
    // per SM (24 instead of 12 with 16 KiB lists) and more warps
    // hide the evaluations' dependent latency; the edges and their outputs
    // are the same.
    if (!many && !g32 && region == 0 && P.cand_bytes <= PAIR_REGION_MAX) {
        auto kp = warm ? k_refine<REFINE_WARM, true, false, 8, 64> : k_refine<REFINE_PLAIN, true, false, 8, 64>;
        return run(kp, P, wide, nullptr, nullptr, n_items, 64);
    }
    if (split) {
        RefinePlan PS = P;
        PS.cand_bytes = uint32_t(small);
        cudaError_t e = cudaMemsetAsync(ovf, 0, 4, s);
        if (e != cudaSuccess) return e;
        // The list pass: WIDE_LIST_WARPS warps share each sub-block's lists.
        auto kw = warm ? (g32 ? k_refine<REFINE_WARM, true, false, 32, 32 * WIDE_LIST_WARPS>
                              : k_refine<REFINE_WARM, true, false, 8, 32 * WIDE_LIST_WARPS>)
                       : (g32 ? k_refine<REFINE_PLAIN, true, false, 32, 32 * WIDE_LIST_WARPS>
                              : k_refine<REFINE_PLAIN, true, false, 8, 32 * WIDE_LIST_WARPS>);
        // Two-warp blocks sharing a region of the same size over the
        // sub-blocks that fit it (twice the warps per SM of per-warp regions).
        auto kp = warm ? (g32 ? k_refine<REFINE_WARM, true, false, 32, 64, false, true>
                              : k_refine<REFINE_WARM, true, false, 8, 64, false, true>)
                       : (g32 ? k_refine<REFINE_PLAIN, true, false, 32, 64, false, true>
                              : k_refine<REFINE_PLAIN, true, false, 8, 64, false, true>);
        e = run(kp, PS, small, ovf, nullptr, n_items, 64);
        if (e != cudaSuccess) return e;
        return run(kw, P, wide, nullptr, ovf, n_items, 32 * WIDE_LIST_WARPS);
    }
    // Groups of lanes per edge: one lane in the many-structure pass (short
    // lists, few evaluations after the warm start), else 8 or 32 as asked.
    auto kern =
        many ? (warm ? pick(k_refine<REFINE_WARM, false, true, 1>, k_refine<REFINE_WARM, true, true, 1>)
                     : pick(k_refine<REFINE_PLAIN, false, true, 1>, k_refine<REFINE_PLAIN, true, true, 1>))
        : warm ? (g32 ? pick(k_refine<REFINE_WARM, false, false, 32>, k_refine<REFINE_WARM, true, false, 32>)
                      : pick(k_refine<REFINE_WARM, false, false, 8>, k_refine<REFINE_WARM, true, false, 8>))
               : (g32 ? pick(k_refine<REFINE_PLAIN, false, false, 32>, k_refine<REFINE_PLAIN, true, false, 32>)
                      : pick(k_refine<REFINE_PLAIN, false, false, 8>, k_refine<REFINE_PLAIN, true, false, 8>));
    return run(kern, P, smem, nullptr, nullptr, use_wide ? n_items : quads);
}

void launch_warm_features(const DArr& A, const DLat& L, const RefineConsts& RC, const int4* keys, const uint32_t* work,
                          uint32_t n_items, const uint32_t* rec, const uint32_t* edges, const float2* edge_vals,
                          const uint32_t* item_off, const uint32_t* item_edges, const float* values,
                          const uint32_t* feats, float* x_out, size_t max_rows, int sms, cudaStream_t s,
                          const Scene* many) {
    if (!many && !n_items) return;
    const uint32_t grid = uint32_t(std::max<size_t>(1, std::min<size_t>((max_rows + 255) / 256, size_t(sms) * 16)));
    COUNT(1);
    if (many)
        k_warm_features<true><<<grid, 256, 0, s>>>(A, L, RC, keys, work, n_items, rec, edges, edge_vals, item_off,
                                                   item_edges, values, feats, x_out, *many);
    else
        k_warm_features<false><<<grid, 256, 0, s>>>(A, L, RC, keys, work, n_items, rec, edges, edge_vals, item_off,
                                                    item_edges, values, feats, x_out, Scene{});
}

cudaError_t launch_warm_starts(const DArr& A, const DLat& L, const RefineConsts& RC, const int4* keys,
                               const uint32_t* work, uint32_t n_items, const uint32_t* rec, const uint32_t* edges,
                               const float2* edge_vals, const uint32_t* item_off, const uint32_t* item_edges,
                               const float* values, const uint32_t* feats, const MlpDev& P, int use, float2* start,
                               unsigned long long* counters, size_t max_rows, int sms, cudaStream_t s,
                               const Scene* many) {
    if ((!many && !n_items) || !max_rows) return cudaSuccess;
    const size_t smem = sizeof(MlpSmem) + 128;
    auto kern = many ? k_warm_starts<true> : k_warm_starts<false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    // Four CTAs per SM: 128 TMEM columns each of the SM's 512.
    const size_t tiles = (max_rows + MLP_ROWS - 1) / MLP_ROWS;
    const uint32_t grid = uint32_t(std::max<size_t>(1, std::min<size_t>(tiles, size_t(sms) * 4)));
    COUNT(1);
    kern<<<grid, MLP_ROWS, smem, s>>>(A, L, RC, keys, work, n_items, rec, edges, edge_vals, item_off, item_edges,
                                      values, feats, P, use, start, counters, many ? *many : Scene{});
    return cudaGetLastError();
}

}  // namespace smb
