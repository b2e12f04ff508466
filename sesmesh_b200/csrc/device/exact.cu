// Exact mode's vertex refinement on the device, in f64.  Per sampled
// sub-block: the candidates of its ball (SesField::gather_local,
// crates/sesmesh/src/field/point.rs:496-582, with the pruning keys of the
// host restatement), then per crossing edge whose lower sample lies in the
// sub-block the root search (extract::vertex, crates/sesmesh/src/mesh/
// extract.rs:425-535, eval_local point.rs:686-738, gradient extract.rs:
// 539-549) and the vertex attributes (attributes, extract.rs:553-597).
//
// Every f64 expression keeps the CPU's operation order (the library is
// built without FMA contraction; f64 division and square root are IEEE), so
// positions, normals, atoms, patches, root parameters and evaluation counts
// equal host/mesher.cpp refine_edge's bit for bit.  The candidate lists
// are sets sorted by unique keys (near by index, S by (lb, index), C by
// (distance, index), V by (distance, index)) and the inside test is an
// any-of, so collecting them in a different order gives the same lists.
//
// Edges stay with the host (marked evals = 0) only when their sub-block's
// lists exceed a warp's 256 KiB global slab.
#include <algorithm>

#include "common.cuh"
#include "kernels.hpp"

namespace smb {

namespace {

constexpr double X_EPS = 1e-9;    // blocker tolerance (point.rs:422-476)
constexpr double X_TOL = 1e-5;    // extract.rs:35
constexpr int X_MAX_ITER = 8;     // extract.rs:29
constexpr int X_MAX_BISECT = 64;  // extract.rs:33
constexpr double X_PRUNE = 1e-9;  // margin of the candidates' pruning keys
constexpr uint32_t XF_SOLVENT = 0, XF_BEYOND = 1, XF_SPHERE = 2, XF_CIRCLE = 3, XF_VERTEX = 4;
constexpr int X_WARPS = 4;
constexpr size_t EXACT_SLAB = size_t(256) << 10;  // bytes of a warp's global list region

// List sizes of one ball.
struct XCounts {
    uint32_t nn, ni, ns, nc, nv;
};

// One ball's lists in shared memory.  near: ascending sphere index, with
// (centre, R); blockers are positions in it.  t_key / t_id: unsorted
// scratch of the list being built; the blocker lists take its place once
// the lists are sorted.
struct XView {
    uint32_t* near_id;
    double4* near_c;
    double4* in_c;
    double4* s_c;
    double* s_key;
    uint32_t *s_id, *s_off, *s_blk;
    double4 *c_m, *c_u;  // (centre, radius), (axis, e1.x)
    double* c_key;
    uint32_t *c_id, *c_off, *c_blk;
    double4* v_p;
    double* v_key;
    uint32_t* v_id;
    double* t_key;
    uint32_t* t_id;
    uint32_t nn, ni, ns, nc, nv;
    double cx, cy, cz, rho;  // the ball
};

__device__ __forceinline__ size_t xal(size_t v) { return (v + 15) & ~size_t(15); }

// Lays one ball's lists out from `base`; *tail gets the offset where the
// scratch (and later the blocker lists) start.  Returns the bytes the lists
// and the scratch take.
__device__ __forceinline__ size_t x_layout(const XCounts& c, unsigned char* base, XView& v, size_t* tail) {
    size_t o = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base + o;
        o = xal(o + bytes);
        return p;
    };
    v.near_c = reinterpret_cast<double4*>(take(size_t(c.nn) * 32));
    v.in_c = reinterpret_cast<double4*>(take(size_t(c.ni) * 32));
    v.s_c = reinterpret_cast<double4*>(take(size_t(c.ns) * 32));
    v.c_m = reinterpret_cast<double4*>(take(size_t(c.nc) * 32));
    v.c_u = reinterpret_cast<double4*>(take(size_t(c.nc) * 32));
    v.v_p = reinterpret_cast<double4*>(take(size_t(c.nv) * 32));
    v.s_key = reinterpret_cast<double*>(take(size_t(c.ns) * 8));
    v.c_key = reinterpret_cast<double*>(take(size_t(c.nc) * 8));
    v.v_key = reinterpret_cast<double*>(take(size_t(c.nv) * 8));
    v.near_id = reinterpret_cast<uint32_t*>(take(size_t(c.nn) * 4));
    v.s_id = reinterpret_cast<uint32_t*>(take(size_t(c.ns) * 4));
    v.s_off = reinterpret_cast<uint32_t*>(take(size_t(c.ns + 1) * 4));
    v.c_id = reinterpret_cast<uint32_t*>(take(size_t(c.nc) * 4));
    v.c_off = reinterpret_cast<uint32_t*>(take(size_t(c.nc + 1) * 4));
    v.v_id = reinterpret_cast<uint32_t*>(take(size_t(c.nv) * 4));
    *tail = o;
    const uint32_t tk = max(c.ns, max(c.nc, c.nv)), ti = max(c.nn + c.ns, max(c.nc, c.nv));
    v.t_key = reinterpret_cast<double*>(take(size_t(tk) * 8));
    v.t_id = reinterpret_cast<uint32_t*>(take(size_t(ti) * 4));
    v.nn = c.nn, v.ni = c.ni, v.ns = c.ns, v.nc = c.nc, v.nv = c.nv;
    return o;
}

template <bool WIDE>
__device__ __forceinline__ void x_sync() {
    if (WIDE) __syncthreads();
    else __syncwarp();
}

// Threads tid, tid + T, ... visit the items of the cells overlapping the
// cube of half-size r around (x, y, z) (geom/cells.rs:113-130).
template <class F>
__device__ __forceinline__ void x_for_near(const DGrid& g, double x, double y, double z, double r, uint32_t tid,
                                           uint32_t T, F&& f) {
    CellBox bx = cell_box(g, x, y, z, r);
    if (T == 32) {  // a warp: the rows flattened (warp_box_items)
        warp_box_items(g, bx, int(tid), [&](bool valid, uint32_t k) {
            if (valid) f(k);
        });
        return;
    }
    for (uint32_t zc = bx.z0; zc <= bx.z1; zc++)
        for (uint32_t yc = bx.y0; yc <= bx.y1; yc++) {
            size_t row = (size_t(zc) * g.dy + yc) * g.dx;
            uint32_t a = g.starts[row + bx.x0], e = g.starts[row + bx.x1 + 1];
            for (uint32_t i = a + tid; i < e; i += T) f(g.items[i]);
        }
}

// Position of id in the ascending near list, or -1.
__device__ __forceinline__ int x_find(const uint32_t* ids, uint32_t n, uint32_t id) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (ids[mid] < id) lo = mid + 1;
        else hi = mid;
    }
    return (lo < n && ids[lo] == id) ? int(lo) : -1;
}

// Blocker rows of the n sorted candidates kept to near spheres: counts
// into off[1..n] ...  Rows that ascend (sorted: the arrangement's rows and
// circle-blocker lists do) are merged with the ascending near list; other
// rows are searched entry by entry.  Either way the kept entries keep their
// row order.
__device__ __forceinline__ void x_blocker_counts(const XView& v, const uint32_t* ids, uint32_t n,
                                                 const uint32_t* row_off, const uint32_t* row_items, uint32_t* off,
                                                 bool sorted, uint32_t tid, uint32_t T) {
    for (uint32_t i = tid; i < n; i += T) {
        const uint32_t k = ids[i];
        uint32_t c = 0;
        if (sorted) {
            uint32_t p = row_off[k], pe = row_off[k + 1], q = 0;
            while (p < pe && q < v.nn) {
                const uint32_t x = row_items[p], y = v.near_id[q];
                c += x == y;
                p += x <= y;
                q += y <= x;
            }
        } else {
            for (uint32_t p = row_off[k], e = row_off[k + 1]; p < e; p++)
                c += x_find(v.near_id, v.nn, row_items[p]) >= 0;
        }
        off[i + 1] = c;
    }
}

// ... then, with off scanned, the near-list positions into blk.
__device__ __forceinline__ void x_blocker_fill(const XView& v, const uint32_t* ids, uint32_t n,
                                               const uint32_t* row_off, const uint32_t* row_items,
                                               const uint32_t* off, uint32_t* blk, bool sorted, uint32_t tid,
                                               uint32_t T) {
    for (uint32_t i = tid; i < n; i += T) {
        const uint32_t k = ids[i];
        uint32_t at = off[i];
        if (sorted) {
            uint32_t p = row_off[k], pe = row_off[k + 1], q = 0;
            while (p < pe && q < v.nn) {
                const uint32_t x = row_items[p], y = v.near_id[q];
                if (x == y) blk[at++] = q;
                p += x <= y;
                q += y <= x;
            }
        } else {
            for (uint32_t p = row_off[k], e = row_off[k + 1]; p < e; p++) {
                int pos = x_find(v.near_id, v.nn, row_items[p]);
                if (pos >= 0) blk[at++] = uint32_t(pos);
            }
        }
    }
}

// off[0] = 0 and off[1..n] turned into their inclusive prefix sums, by the
// warp (lanes over chunks of 32) or, in a block, by one thread.
template <bool WIDE>
__device__ __forceinline__ void x_offsets(uint32_t* off, uint32_t n, uint32_t tid) {
    if (WIDE) {
        if (tid == 0) {
            off[0] = 0;
            for (uint32_t i = 1; i <= n; i++) off[i] += off[i - 1];
        }
        return;
    }
    uint32_t carry = 0;
    for (uint32_t b = 0; b < n; b += 32) {
        const uint32_t i = b + tid + 1;
        uint32_t x = i <= n ? off[i] : 0u;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (int(tid) >= o) x += y;
        }
        if (i <= n) off[i] = carry + x;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (tid == 0) off[0] = 0;
}

// Rank of (key, id) among n scratch pairs in (key, id) order.
__device__ __forceinline__ uint32_t x_rank(const double* keys, const uint32_t* ids, uint32_t n, double key,
                                           uint32_t id) {
    uint32_t r = 0;
    for (uint32_t q = 0; q < n; q++) {
        const double kq = keys[q];
        r += (kq < key || (kq == key && ids[q] < id)) ? 1u : 0u;
    }
    return r;
}

// gather_local of sub-block j's ball into `base` (cap bytes) with threads
// tid of T; false when the lists do not fit.  cnt: 8 shared counters.
// hint: the gather's record of the sub-block, or null.  Its list sizes are
// those of a ball a hair smaller (the gather's rho has no margins), so with
// a few entries more they bound this ball's sizes and the counting pass is
// skipped; a list that outgrows them after all sends the ball back to the
// counting pass.
// slack: entries added to each hinted size (X_HINT_SLACK; 0 with the
// bounds one short, which sends every ball through the counted layout).
constexpr int X_HINT_SLACK = 4;

// Blocker rows of the ball's S and C candidates kept to its near spheres,
// laid out from `tail`; false when they do not fit in cap.
template <bool WIDE>
__device__ bool x_blockers(const DArr& A, unsigned char* base, size_t cap, size_t tail, uint32_t tid, uint32_t T,
                           XView& v) {
    const bool sorted = A.flags & DARR_ROWS_SORTED;
    x_blocker_counts(v, v.s_id, v.ns, A.nb_off, A.nb_items, v.s_off, sorted, tid, T);
    x_blocker_counts(v, v.c_id, v.nc, A.cb_off, A.cb_items, v.c_off, sorted, tid, T);
    x_sync<WIDE>();
    x_offsets<WIDE>(v.s_off, v.ns, tid);
    x_offsets<WIDE>(v.c_off, v.nc, tid);
    x_sync<WIDE>();
    const size_t nsb = v.s_off[v.ns], ncb = v.c_off[v.nc];
    v.s_blk = reinterpret_cast<uint32_t*>(base + tail);
    v.c_blk = reinterpret_cast<uint32_t*>(base + xal(tail + nsb * 4));
    if (xal(tail + nsb * 4) + ncb * 4 > cap) return false;
    x_blocker_fill(v, v.s_id, v.ns, A.nb_off, A.nb_items, v.s_off, v.s_blk, sorted, tid, T);
    x_blocker_fill(v, v.c_id, v.nc, A.cb_off, A.cb_items, v.c_off, v.c_blk, sorted, tid, T);
    x_sync<WIDE>();
    return true;
}

// The ball's lists straight from the gather's candidate ids (ids: the
// sub-block's CSR words, hint its record), for a sub-block whose gather
// found no candidate on which the two balls disagree: the sets are then
// equal, S and C come in the same (key, index) order, the near list's
// first R_INSIDE entries are the inside spheres, and the gather's blocker
// lists (the rows kept to near spheres, in row order) are this ball's.
// The near list keeps the gather's order, so the blocker positions carry
// over as they are: near order reaches the results only through the
// blocker tests, whose outcome (any blocker contains the point) and count
// do not depend on it.  V is re-sorted by (distance, index).  False when
// the lists do not fit in cap.
template <bool WIDE>
__device__ bool x_ball_from_ids(const DArr& A, double cx, double cy, double cz, double rho, unsigned char* base,
                                size_t cap, uint32_t tid, uint32_t T, XView& v, const uint32_t* hint,
                                const uint32_t* ids) {
    const XCounts c{hint[R_NEAR], hint[R_INSIDE], hint[R_S], hint[R_C], hint[R_V]};
    size_t tail = 0;
    const size_t need = x_layout(c, base, v, &tail);
    x_sync<WIDE>();
    const size_t nsb = hint[R_SBLK], ncb = hint[R_CBLK];
    if (need > cap || xal(tail + nsb * 4) + ncb * 4 > cap) return false;
    const uint32_t* l_near = ids;
    const uint32_t* l_s = l_near + c.nn;
    const uint32_t* l_soff = l_s + c.ns;
    const uint32_t* l_sblk = l_soff + c.ns + 1;
    const uint32_t* l_c = l_sblk + nsb;
    const uint32_t* l_coff = l_c + c.nc;
    const uint32_t* l_cblk = l_coff + c.nc + 1;
    const uint32_t* l_v = l_cblk + ncb;
    for (uint32_t i = tid; i < c.nn; i += T) {
        const uint32_t k = l_near[i];
        const double4 sp = A.sph[k];
        v.near_id[i] = k;
        v.near_c[i] = sp;
        if (i < c.ni) v.in_c[i] = sp;
    }
    for (uint32_t i = tid; i < c.ns; i += T) {
        const uint32_t k = l_s[i];
        const double4 s = A.sph[k];
        v.s_id[i] = k;
        v.s_key[i] = fabs(dist3(cx, cy, cz, s.x, s.y, s.z) - s.w) - rho - X_PRUNE;
        v.s_c[i] = s;
    }
    for (uint32_t i = tid; i < c.nc; i += T) {
        const uint32_t ci = l_c[i];
        const double* C = A.circ + 12 * size_t(ci);
        v.c_id[i] = ci;
        v.c_key[i] = circle_reach_dist(A, cx, cy, cz, ci) - rho - X_PRUNE;
        v.c_m[i] = make_double4(C[0], C[1], C[2], C[9]);
        v.c_u[i] = make_double4(C[3], C[4], C[5], C[6]);
    }
    for (uint32_t i = tid; i <= c.ns; i += T) v.s_off[i] = l_soff[i];
    for (uint32_t i = tid; i <= c.nc; i += T) v.c_off[i] = l_coff[i];
    // V: (distance, index) pairs in the scratch.
    for (uint32_t i = tid; i < c.nv; i += T) {
        const uint32_t vi = l_v[i];
        const double4 p = A.vert[vi];
        v.t_key[i] = dist3(cx, cy, cz, p.x, p.y, p.z);
        v.t_id[i] = vi;
    }
    x_sync<WIDE>();
    for (uint32_t i = tid; i < c.nv; i += T) {
        const double d = v.t_key[i];
        const uint32_t vi = v.t_id[i];
        const uint32_t r = x_rank(v.t_key, v.t_id, c.nv, d, vi);
        v.v_id[r] = vi;
        v.v_key[r] = d - rho - X_PRUNE;
        v.v_p[r] = A.vert[vi];
    }
    x_sync<WIDE>();
    // The blocker lists take the scratch's place.
    v.s_blk = reinterpret_cast<uint32_t*>(base + tail);
    v.c_blk = reinterpret_cast<uint32_t*>(base + xal(tail + nsb * 4));
    for (uint32_t p = tid; p < nsb; p += T) v.s_blk[p] = l_sblk[p];
    for (uint32_t p = tid; p < ncb; p += T) v.c_blk[p] = l_cblk[p];
    x_sync<WIDE>();
    return true;
}

// gather_local of a sphere field (point.rs:566-579): the spheres not
// contained with |b - c| - R < band + rho, by (that value, index), into
// in_c (centre, R), s_id and s_key; ni = ns = their count.
template <bool WIDE>
__device__ bool x_ball_spheres(const DArr& A, const DLat& L, double cx, double cy, double cz, double rho,
                               unsigned char* base, size_t cap, uint32_t* cnt, uint32_t tid, uint32_t T, XView& v) {
    const double reach = L.band + rho;
    x_sync<WIDE>();
    if (tid < 8) cnt[tid] = 0;
    x_sync<WIDE>();
    x_for_near(A.gs, cx, cy, cz, reach + A.max_expanded, tid, T, [&](uint32_t k) {
        if (A.status[k] == STATUS_CONTAINED) return;
        const double4 c = A.sph[k];
        if (dist3(cx, cy, cz, c.x, c.y, c.z) - c.w < reach) atomicAdd(&cnt[0], 1u);
    });
    x_sync<WIDE>();
    const uint32_t n = cnt[0];
    size_t tail = 0;
    const size_t need = x_layout(XCounts{0, n, n, 0, 0}, base, v, &tail);
    x_sync<WIDE>();
    if (need > cap) return false;
    if (tid < 8) cnt[tid] = 0;
    x_sync<WIDE>();
    x_for_near(A.gs, cx, cy, cz, reach + A.max_expanded, tid, T, [&](uint32_t k) {
        if (A.status[k] == STATUS_CONTAINED) return;
        const double4 c = A.sph[k];
        const double key = dist3(cx, cy, cz, c.x, c.y, c.z) - c.w;
        if (key < reach) {
            const uint32_t p = atomicAdd(&cnt[0], 1u);
            if (p < n) v.t_key[p] = key, v.t_id[p] = k;
        }
    });
    x_sync<WIDE>();
    for (uint32_t i = tid; i < n; i += T) {
        const double key = v.t_key[i];
        const uint32_t id = v.t_id[i];
        uint32_t r = 0;
        for (uint32_t q = 0; q < n; q++) r += (v.t_key[q] < key || (v.t_key[q] == key && v.t_id[q] < id)) ? 1u : 0u;
        v.in_c[r] = A.sph[id];
        v.s_id[r] = id;
        v.s_key[r] = key;
    }
    x_sync<WIDE>();
    return true;
}

template <bool WIDE>
__device__ bool x_ball(const DArr& A, const DLat& L, int4 key, uint32_t j, unsigned char* base, size_t cap,
                       uint32_t* cnt, uint32_t tid, uint32_t T, XView& v, const uint32_t* hint = nullptr,
                       int slack = X_HINT_SLACK, const uint32_t* ids = nullptr, const uint8_t* window = nullptr) {
    const int b = L.b, sub = L.sub, sb = int(j & 7);
    const double h = L.h, subd = double(sub);
    // local_of (extract.rs:165-177, 195-206): ball centre and radius.
    const double bx = double((long long)key.x * b) * h, by = double((long long)key.y * b) * h,
                 bz = double((long long)key.z * b) * h;
    const double cx = bx + (double((sb & 1) * sub) + 0.5 * subd) * h;
    const double cy = by + (double(((sb >> 1) & 1) * sub) + 0.5 * subd) * h;
    const double cz = bz + (double((sb >> 2) * sub) + 0.5 * subd) * h;
    const double rho = 0.5 * sqrt(3.0) * subd * h * (1.0 + 1e-9) + 1e-9;
    const double reach = A.probe + L.band + rho;
    v.cx = cx, v.cy = cy, v.cz = cz, v.rho = rho;
    if (A.flags & DARR_SPHERES) return x_ball_spheres<WIDE>(A, L, cx, cy, cz, rho, base, cap, cnt, tid, T, v);
    bool hinted = hint && hint[R_FLAGS] == 0;
    if (hinted && ids && window && window[j] == 0 && slack > 0)
        return x_ball_from_ids<WIDE>(A, cx, cy, cz, rho, base, cap, tid, T, v, hint, ids + hint[R_IDS]);
    // Two attempts at most: hinted (when there is a hint), then counted.
    for (;;) {
        XCounts c;
        if (hinted) {
            auto bound = [&](uint32_t n) { return slack > 0 ? n + uint32_t(slack) : (n ? n - 1 : 0u); };
            c = XCounts{bound(hint[R_NEAR]), bound(hint[R_INSIDE]), bound(hint[R_S]), bound(hint[R_C]),
                        bound(hint[R_V])};
        } else {
            x_sync<WIDE>();
            if (tid < 8) cnt[tid] = 0;
            x_sync<WIDE>();
            // Sizes.
            x_for_near(A.gs, cx, cy, cz, reach + A.max_expanded, tid, T, [&](uint32_t k) {
                const uint32_t st = A.status[k];
                if (st == STATUS_CONTAINED) return;
                const double4 c = A.sph[k];
                const double d = dist3(cx, cy, cz, c.x, c.y, c.z);
                if (d < c.w + reach) atomicAdd(&cnt[0], 1u);
                if (d < c.w + rho) atomicAdd(&cnt[1], 1u);
                if (st == STATUS_EXPOSED && fabs(d - c.w) <= reach) atomicAdd(&cnt[2], 1u);
            });
            x_for_near(A.gc, cx, cy, cz, reach + A.rho_max, tid, T, [&](uint32_t ci) {
                if (circle_reach_dist(A, cx, cy, cz, ci) <= reach) atomicAdd(&cnt[3], 1u);
            });
            x_for_near(A.gv, cx, cy, cz, reach, tid, T, [&](uint32_t vi) {
                const double4 p = A.vert[vi];
                if (dist3(cx, cy, cz, p.x, p.y, p.z) <= reach) atomicAdd(&cnt[4], 1u);
            });
            x_sync<WIDE>();
            c = XCounts{cnt[0], cnt[1], cnt[2], cnt[3], cnt[4]};
        }
        size_t tail = 0;
        const size_t need = x_layout(c, base, v, &tail);
        x_sync<WIDE>();
        if (need > cap) {
            if (hinted) {
                hinted = false;
                continue;
            }
            return false;
        }
        if (tid < 8) cnt[tid] = 0;
        x_sync<WIDE>();
        // Spheres: near (scratch ids), inside (direct), S (scratch pairs).
        // Writes stay within the laid-out sizes; cnt[5] flags a list that
        // went past them (only a hinted attempt can), which sends the ball
        // to the counted attempt.
        x_for_near(A.gs, cx, cy, cz, reach + A.max_expanded, tid, T, [&](uint32_t k) {
            const uint32_t st = A.status[k];
            if (st == STATUS_CONTAINED) return;
            const double4 s = A.sph[k];
            const double d = dist3(cx, cy, cz, s.x, s.y, s.z);
            if (d < s.w + reach) {
                const uint32_t p = atomicAdd(&cnt[0], 1u);
                if (p < c.nn) v.t_id[p] = k;
                else cnt[5] = 1;
            }
            if (d < s.w + rho) {
                const uint32_t p = atomicAdd(&cnt[1], 1u);
                if (p < c.ni) v.in_c[p] = s;
                else cnt[5] = 1;
            }
            const double lb = fabs(d - s.w);
            if (st == STATUS_EXPOSED && lb <= reach) {
                const uint32_t p = atomicAdd(&cnt[2], 1u);
                if (p < c.ns) v.t_key[p] = lb, v.t_id[c.nn + p] = k;
                else cnt[5] = 1;
            }
        });
        x_sync<WIDE>();
        if (cnt[5]) {
            hinted = false;
            continue;
        }
        const uint32_t nn = cnt[0], ni = cnt[1], ns = cnt[2];
        for (uint32_t i = tid; i < nn; i += T) {
            const uint32_t id = v.t_id[i];
            uint32_t r = 0;
            for (uint32_t q = 0; q < nn; q++) r += v.t_id[q] < id ? 1u : 0u;
            v.near_id[r] = id;
            v.near_c[r] = A.sph[id];
        }
        for (uint32_t i = tid; i < ns; i += T) {
            const double lb = v.t_key[i];
            const uint32_t k = v.t_id[c.nn + i];
            const uint32_t r = x_rank(v.t_key, v.t_id + c.nn, ns, lb, k);
            v.s_id[r] = k;
            v.s_key[r] = lb - rho - X_PRUNE;
            v.s_c[r] = A.sph[k];
        }
        // Circles.
        x_sync<WIDE>();
        x_for_near(A.gc, cx, cy, cz, reach + A.rho_max, tid, T, [&](uint32_t ci) {
            const double d = circle_reach_dist(A, cx, cy, cz, ci);
            if (d <= reach) {
                const uint32_t p = atomicAdd(&cnt[3], 1u);
                if (p < c.nc) v.t_key[p] = d, v.t_id[p] = ci;
                else cnt[5] = 1;
            }
        });
        x_sync<WIDE>();
        if (cnt[5]) {
            hinted = false;
            continue;
        }
        const uint32_t nc = cnt[3];
        for (uint32_t i = tid; i < nc; i += T) {
            const double d = v.t_key[i];
            const uint32_t ci = v.t_id[i];
            const uint32_t r = x_rank(v.t_key, v.t_id, nc, d, ci);
            const double* C = A.circ + 12 * size_t(ci);
            v.c_id[r] = ci;
            v.c_key[r] = d - rho - X_PRUNE;
            v.c_m[r] = make_double4(C[0], C[1], C[2], C[9]);
            v.c_u[r] = make_double4(C[3], C[4], C[5], C[6]);
        }
        x_sync<WIDE>();
        // SAS vertices.
        x_for_near(A.gv, cx, cy, cz, reach, tid, T, [&](uint32_t vi) {
            const double4 p = A.vert[vi];
            const double d = dist3(cx, cy, cz, p.x, p.y, p.z);
            if (d <= reach) {
                const uint32_t q = atomicAdd(&cnt[4], 1u);
                if (q < c.nv) v.t_key[q] = d, v.t_id[q] = vi;
                else cnt[5] = 1;
            }
        });
        x_sync<WIDE>();
        if (cnt[5]) {
            hinted = false;
            continue;
        }
        const uint32_t nv = cnt[4];
        for (uint32_t i = tid; i < nv; i += T) {
            const double d = v.t_key[i];
            const uint32_t vi = v.t_id[i];
            const uint32_t r = x_rank(v.t_key, v.t_id, nv, d, vi);
            v.v_id[r] = vi;
            v.v_key[r] = d - rho - X_PRUNE;
            v.v_p[r] = A.vert[vi];
        }
        v.nn = nn, v.ni = ni, v.ns = ns, v.nc = nc, v.nv = nv;
        // Blockers, kept to near spheres, in the scratch's place.
        if (x_blockers<WIDE>(A, base, cap, tail, tid, T, v)) return true;
        if (!hinted) return false;
        hinted = false;  // the laid-out bounds took the room: lay out the counted sizes
    }
}

struct XEval {
    double value, qx, qy, qz;
    uint32_t kind, id;
};

// eval_local (point.rs:686-738) against the ball's lists: value, feature and
// closest point.  COUNT: adds the f64 arithmetic operations executed to ops
// (sqrt and division one each; compares, selects, fabs not counted): 9 per
// inside sphere tested; if inside, 1, then 10 per S candidate visited (+7
// for the projection, +10 per blocker tested), 26 per C candidate (+9 or +6,
// +10 per blocker), 9 per SAS vertex, 1 final.
template <bool COUNT = false>
__device__ __forceinline__ XEval x_eval(const XView& v, const double* circ, double probe, double band, double x,
                                        double y, double z, unsigned long long* ops = nullptr) {
    XEval e;
    e.qx = x, e.qy = y, e.qz = z, e.id = 0;
    bool inside = false;
    unsigned long long n_ops = 0;
    for (uint32_t k = 0; k < v.ni; k++) {
        const double4 c = v.in_c[k];
        if (COUNT) n_ops += 9;
        if (sqrt_lt(sq3(x, y, z, c.x, c.y, c.z), c.w)) {
            inside = true;
            break;
        }
    }
    if (!inside) {
        e.value = probe, e.kind = XF_SOLVENT;
        if (COUNT) *ops += n_ops;
        return e;
    }
    double best = probe + band;
    if (COUNT) n_ops += 1;
    e.kind = XF_BEYOND;
    // Pruning at this point: a candidate's value here is at least its value
    // at the ball's centre minus |x - centre| (each is 1-Lipschitz), so with
    // slack = rho - |x - centre| (less a 1e-12 rounding margin, at least 0)
    // the keys (centre value - rho - 1e-9, ascending) can stop a loop at
    // best - slack instead of best: every candidate skipped could not go
    // below best, so the result is the unpruned one.
    const double ddx = x - v.cx, ddy = y - v.cy, ddz = z - v.cz;
    const double slack = fmax(v.rho - sqrt(ddx * ddx + ddy * ddy + ddz * ddz) - 1e-12, 0.0);
    for (uint32_t i = 0; i < v.ns && v.s_key[i] < best - slack; i++) {
        const double4 c = v.s_c[i];
        const double vx = x - c.x, vy = y - c.y, vz = z - c.z;
        const double len = sqrt(vx * vx + vy * vy + vz * vz);
        const double lb = fabs(len - c.w);
        if (COUNT) n_ops += 10;
        if (lb >= best || len < 1e-12) continue;
        const double s = c.w / len;
        const double qx = c.x + vx * s, qy = c.y + vy * s, qz = c.z + vz * s;
        if (COUNT) n_ops += 7;
        bool free = true;
        for (uint32_t p = v.s_off[i], pe = v.s_off[i + 1]; p < pe; p++) {
            const double4 k = v.near_c[v.s_blk[p]];
            if (COUNT) n_ops += 10;
            if (!sqrt_ge(sq3(qx, qy, qz, k.x, k.y, k.z), k.w - X_EPS)) {
                free = false;
                break;
            }
        }
        if (free) best = lb, e.kind = XF_SPHERE, e.id = v.s_id[i], e.qx = qx, e.qy = qy, e.qz = qz;
    }
    for (uint32_t i = 0; i < v.nc && v.c_key[i] < best - slack; i++) {
        const double4 m = v.c_m[i], u = v.c_u[i];
        const double yx = x - m.x, yy = y - m.y, yz = z - m.z;
        const double along = yx * u.x + yy * u.y + yz * u.z;
        const double wx = yx - u.x * along, wy = yy - u.y * along, wz = yz - u.z * along;
        const double wl = sqrt(wx * wx + wy * wy + wz * wz);
        const double dist2 = along * along + (wl - m.w) * (wl - m.w);
        if (COUNT) n_ops += 26;
        if (sqrt_ge(dist2, best)) continue;
        const double dist = sqrt(dist2);
        double dx, dy, dz;
        if (wl > 1e-12) {
            dx = wx / wl, dy = wy / wl, dz = wz / wl;
            if (COUNT) n_ops += 3;
        } else {  // on the axis: e1 (A.circ words 6..8)
            const double* C = circ + 12 * size_t(v.c_id[i]);
            dx = u.w, dy = C[7], dz = C[8];
        }
        const double qx = m.x + dx * m.w, qy = m.y + dy * m.w, qz = m.z + dz * m.w;
        if (COUNT) n_ops += 6;
        bool free = true;
        for (uint32_t p = v.c_off[i], pe = v.c_off[i + 1]; p < pe; p++) {
            const double4 k = v.near_c[v.c_blk[p]];
            if (COUNT) n_ops += 10;
            if (!sqrt_ge(sq3(qx, qy, qz, k.x, k.y, k.z), k.w - X_EPS)) {
                free = false;
                break;
            }
        }
        if (free) best = dist, e.kind = XF_CIRCLE, e.id = v.c_id[i], e.qx = qx, e.qy = qy, e.qz = qz;
    }
    for (uint32_t i = 0; i < v.nv && v.v_key[i] < best - slack; i++) {
        const double4 p = v.v_p[i];
        const double d2 = sq3(x, y, z, p.x, p.y, p.z);
        if (COUNT) n_ops += 9;
        if (!sqrt_lt(d2, best)) continue;
        best = sqrt(d2), e.kind = XF_VERTEX, e.id = v.v_id[i], e.qx = p.x, e.qy = p.y, e.qz = p.z;
    }
    if (COUNT) *ops += n_ops + 1;
    e.value = probe - best;
    return e;
}

// x_eval by a group of RG lanes that all hold the same point: the lanes
// take RG candidates of a list at a time (each skipping one whose key
// reaches best - slack) and the group keeps the least value, the earliest
// candidate on ties; a candidate replaces the best only when strictly
// smaller, as in x_eval's walk, so the result is x_eval's.  gl: the lane's
// place in the group, gm: the group's lanes.
template <int RG>
__device__ __forceinline__ void x_argmin(uint32_t gm, double& v, int& i) {
#pragma unroll
    for (int o = RG / 2; o; o >>= 1) {
        const double v2 = __shfl_xor_sync(gm, v, o);
        const int i2 = __shfl_xor_sync(gm, i, o);
        if (v2 < v || (v2 == v && i2 < i)) v = v2, i = i2;
    }
}

template <int RG>
__device__ __forceinline__ XEval x_eval_group(const XView& v, const double* circ, double probe, double band, double x,
                                              double y, double z, int gl, uint32_t gm) {
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    XEval e;
    e.qx = x, e.qy = y, e.qz = z, e.id = 0;
    bool inside = false;
    for (uint32_t k0 = 0; k0 < v.ni; k0 += RG) {
        const uint32_t k = k0 + gl;
        bool in = false;
        if (k < v.ni) {
            const double4 c = v.in_c[k];
            in = sqrt_lt(sq3(x, y, z, c.x, c.y, c.z), c.w);
        }
        if (__any_sync(gm, in)) {
            inside = true;
            break;
        }
    }
    if (!inside) {
        e.value = probe, e.kind = XF_SOLVENT;
        return e;
    }
    double best = probe + band;
    e.kind = XF_BEYOND;
    const double ddx = x - v.cx, ddy = y - v.cy, ddz = z - v.cz;
    const double slack = fmax(v.rho - sqrt(ddx * ddx + ddy * ddy + ddz * ddz) - 1e-12, 0.0);
    const int g0 = int(threadIdx.x & 31) & ~(RG - 1);
    for (uint32_t i0 = 0; i0 < v.ns && v.s_key[i0] < best - slack; i0 += RG) {
        const uint32_t i = i0 + gl;
        double val = inf, qx = 0.0, qy = 0.0, qz = 0.0;
        if (i < v.ns && v.s_key[i] < best - slack) {
            const double4 c = v.s_c[i];
            const double vx = x - c.x, vy = y - c.y, vz = z - c.z;
            const double len = sqrt(vx * vx + vy * vy + vz * vz);
            const double lb = fabs(len - c.w);
            if (!(lb >= best || len < 1e-12)) {
                const double s = c.w / len;
                qx = c.x + vx * s, qy = c.y + vy * s, qz = c.z + vz * s;
                bool free = true;
                for (uint32_t p = v.s_off[i], pe = v.s_off[i + 1]; p < pe; p++) {
                    const double4 k = v.near_c[v.s_blk[p]];
                    if (!sqrt_ge(sq3(qx, qy, qz, k.x, k.y, k.z), k.w - X_EPS)) {
                        free = false;
                        break;
                    }
                }
                if (free) val = lb;
            }
        }
        int w = int(i);
        x_argmin<RG>(gm, val, w);
        if (val < best) {
            const int src = g0 + (w - int(i0));
            best = val, e.kind = XF_SPHERE, e.id = v.s_id[w];
            e.qx = __shfl_sync(gm, qx, src), e.qy = __shfl_sync(gm, qy, src), e.qz = __shfl_sync(gm, qz, src);
        }
    }
    for (uint32_t i0 = 0; i0 < v.nc && v.c_key[i0] < best - slack; i0 += RG) {
        const uint32_t i = i0 + gl;
        double val = inf, qx = 0.0, qy = 0.0, qz = 0.0;
        if (i < v.nc && v.c_key[i] < best - slack) {
            const double4 m = v.c_m[i], u = v.c_u[i];
            const double yx = x - m.x, yy = y - m.y, yz = z - m.z;
            const double along = yx * u.x + yy * u.y + yz * u.z;
            const double wx = yx - u.x * along, wy = yy - u.y * along, wz = yz - u.z * along;
            const double wl = sqrt(wx * wx + wy * wy + wz * wz);
            const double dist2 = along * along + (wl - m.w) * (wl - m.w);
            if (!sqrt_ge(dist2, best)) {
                const double dist = sqrt(dist2);
                double dx, dy, dz;
                if (wl > 1e-12) {
                    dx = wx / wl, dy = wy / wl, dz = wz / wl;
                } else {  // on the axis: e1 (A.circ words 6..8)
                    const double* C = circ + 12 * size_t(v.c_id[i]);
                    dx = u.w, dy = C[7], dz = C[8];
                }
                qx = m.x + dx * m.w, qy = m.y + dy * m.w, qz = m.z + dz * m.w;
                bool free = true;
                for (uint32_t p = v.c_off[i], pe = v.c_off[i + 1]; p < pe; p++) {
                    const double4 k = v.near_c[v.c_blk[p]];
                    if (!sqrt_ge(sq3(qx, qy, qz, k.x, k.y, k.z), k.w - X_EPS)) {
                        free = false;
                        break;
                    }
                }
                if (free) val = dist;
            }
        }
        int w = int(i);
        x_argmin<RG>(gm, val, w);
        if (val < best) {
            const int src = g0 + (w - int(i0));
            best = val, e.kind = XF_CIRCLE, e.id = v.c_id[w];
            e.qx = __shfl_sync(gm, qx, src), e.qy = __shfl_sync(gm, qy, src), e.qz = __shfl_sync(gm, qz, src);
        }
    }
    for (uint32_t i0 = 0; i0 < v.nv && v.v_key[i0] < best - slack; i0 += RG) {
        const uint32_t i = i0 + gl;
        double val = inf;
        if (i < v.nv && v.v_key[i] < best - slack) {
            const double4 p = v.v_p[i];
            const double d2 = sq3(x, y, z, p.x, p.y, p.z);
            if (sqrt_lt(d2, best)) val = sqrt(d2);
        }
        int w = int(i);
        x_argmin<RG>(gm, val, w);
        if (val < best) {
            const double4 p = v.v_p[w];
            best = val, e.kind = XF_VERTEX, e.id = v.v_id[w], e.qx = p.x, e.qy = p.y, e.qz = p.z;
        }
    }
    e.value = probe - best;
    return e;
}

// eval_local of a sphere field (point.rs:723-736): the least |x - c| - R
// over the ball's spheres, band when none is below it; the closest point
// carries the minimising sphere's centre (the gradient's x - c).  COUNT: 9
// per sphere.
template <bool COUNT = false>
__device__ __forceinline__ XEval x_eval_spheres(const XView& v, double band, double x, double y, double z,
                                                unsigned long long* ops = nullptr) {
    XEval e;
    e.qx = x, e.qy = y, e.qz = z, e.kind = XF_BEYOND, e.id = 0;
    double best = band;
    for (uint32_t i = 0; i < v.ni; i++) {
        const double4 c = v.in_c[i];
        const double val = dist3(x, y, z, c.x, c.y, c.z) - c.w;
        if (val < best) best = val, e.kind = XF_SPHERE, e.id = v.s_id[i], e.qx = c.x, e.qy = c.y, e.qz = c.z;
    }
    if (COUNT) *ops += 9ull * v.ni;
    e.value = best;
    return e;
}

// The same by a group of RG lanes (x_eval_group's rules: the least value,
// the earliest sphere on ties, so the result is the one-lane walk's).
template <int RG>
__device__ __forceinline__ XEval x_eval_spheres_group(const XView& v, double band, double x, double y, double z,
                                                      int gl, uint32_t gm) {
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    XEval e;
    e.qx = x, e.qy = y, e.qz = z, e.kind = XF_BEYOND, e.id = 0;
    double best = band;
    for (uint32_t i0 = 0; i0 < v.ni; i0 += RG) {
        const uint32_t i = i0 + gl;
        double val = inf;
        if (i < v.ni) {
            const double4 c = v.in_c[i];
            val = dist3(x, y, z, c.x, c.y, c.z) - c.w;
        }
        int w = int(i);
        x_argmin<RG>(gm, val, w);
        if (val < best) {
            const double4 c = v.in_c[w];
            best = val, e.kind = XF_SPHERE, e.id = v.s_id[w], e.qx = c.x, e.qy = c.y, e.qz = c.z;
        }
    }
    e.value = best;
    return e;
}

__device__ __forceinline__ double x_clamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

// The atom nearest to p among ids (extract.rs:566-576): its input index.
__device__ __forceinline__ uint32_t x_nearest(const DArr& A, const ExactAttr& X, const uint32_t* ids, int n, double px,
                                              double py, double pz) {
    double best = __longlong_as_double(0x7ff0000000000000LL);
    uint32_t bi = ids[0];
    for (int q = 0; q < n; q++) {
        const double4 c = A.sph[ids[q]];
        const double d = dist3(px, py, pz, c.x, c.y, c.z) - A.rvdw[ids[q]];
        if (d < best) best = d, bi = ids[q];
    }
    return X.orig[bi];
}

// sphere_eval (point.rs:742-757): the non-contained sphere with the lowest
// |p - c| - R below cutoff, in cell-scan order (first on ties); -1: none.
__device__ long long x_sphere_eval(const DArr& A, double px, double py, double pz, double cutoff) {
    double best = cutoff;
    long long bi = -1;
    const CellBox bx = cell_box(A.gs, px, py, pz, cutoff + A.max_expanded);
    for (uint32_t zc = bx.z0; zc <= bx.z1; zc++)
        for (uint32_t yc = bx.y0; yc <= bx.y1; yc++) {
            const size_t row = (size_t(zc) * A.gs.dy + yc) * A.gs.dx;
            for (uint32_t i = A.gs.starts[row + bx.x0], e = A.gs.starts[row + bx.x1 + 1]; i < e; i++) {
                const uint32_t k = A.gs.items[i];
                if (A.status[k] == STATUS_CONTAINED) continue;
                const double4 c = A.sph[k];
                const double v = dist3(px, py, pz, c.x, c.y, c.z) - c.w;
                if (v < best) best = v, bi = k;
            }
        }
    return bi;
}

// extract::attributes (extract.rs:553-597) of a vertex at p on the edge
// (pa, pa + d) whose last evaluation had feature (kind, id) and closest
// point q: normal, patch, input atom.
__device__ void x_attributes(const DArr& A, const DLat& L, const ExactAttr& X, uint32_t kind, uint32_t id, double qx,
                             double qy, double qz, double px, double py, double pz, double dx, double dy, double dz,
                             double fa, double& nx, double& ny, double& nz, uint32_t& atom, uint32_t& patch) {
    double ox = dx, oy = dy, oz = dz;
    if (!(fa < 0.0)) ox = dx * -1.0, oy = dy * -1.0, oz = dz * -1.0;
    const double on = sqrt(ox * ox + oy * oy + oz * oz);
    ox = ox / on, oy = oy / on, oz = oz / on;
    if ((A.flags & DARR_SPHERES) && kind == XF_SPHERE) {  // extract.rs:583-587: unit(v - c)
        const double4 c = A.sph[id];
        nx = px - c.x, ny = py - c.y, nz = pz - c.z;
        const double nl = sqrt(nx * nx + ny * ny + nz * nz);
        if (nl > 1e-9) nx = nx / nl, ny = ny / nl, nz = nz / nl;
        else nx = ox, ny = oy, nz = oz;
        atom = X.orig[id], patch = 0;
        return;
    }
    if ((A.flags & DARR_SPHERES) == 0 && (kind == XF_SPHERE || kind == XF_CIRCLE || kind == XF_VERTEX)) {
        nx = qx - px, ny = qy - py, nz = qz - pz;
        const double nl = sqrt(nx * nx + ny * ny + nz * nz);
        if (nl > 1e-9) nx = nx / nl, ny = ny / nl, nz = nz / nl;
        else nx = ox, ny = oy, nz = oz;
        if (kind == XF_SPHERE) atom = X.orig[id], patch = 0;
        else if (kind == XF_CIRCLE) atom = x_nearest(A, X, X.circle_ij + 2 * size_t(id), 2, px, py, pz), patch = 1;
        else atom = x_nearest(A, X, X.vertex_atoms + 3 * size_t(id), 3, px, py, pz), patch = 2;
        return;
    }
    nx = ox, ny = oy, nz = oz;
    patch = 0;
    const long long bi = x_sphere_eval(A, px, py, pz, A.probe + L.band + 8.0);
    atom = bi < 0 ? 0u : X.orig[bi];
}

// extract::vertex of edge k (exact mode) and its attributes; RG > 1: by a
// group of RG lanes (x_eval_group), the group's first lane placing it.
template <bool COUNT = false, int RG = 1>
__device__ __forceinline__ void x_edge(const XView& v, const DArr& A, const DLat& L, const ExactAttr& X, int4 key, uint32_t k,
                       uint32_t code, float2 fv, const ExactOut& out, unsigned long long* ops = nullptr, int gl = 0,
                       uint32_t gm = 0xffffffffu) {
    static_assert(RG == 1 || !COUNT, "operations are counted one lane per edge");
    const int b = L.b;
    const double h = L.h;
    const uint32_t cell = code / 3, axis = code % 3;
    const long long ix = (long long)key.x * b + (long long)(cell % uint32_t(b)),
                    iy = (long long)key.y * b + (long long)((cell / uint32_t(b)) % uint32_t(b)),
                    iz = (long long)key.z * b + (long long)(cell / uint32_t(b * b));
    const double pax = double(ix) * h, pay = double(iy) * h, paz = double(iz) * h;
    const double pbx = double(ix + (axis == 0)) * h, pby = double(iy + (axis == 1)) * h,
                 pbz = double(iz + (axis == 2)) * h;
    const double fa = double(fv.x), fb = double(fv.y);
    const double dx = pbx - pax, dy = pby - pay, dz = pbz - paz;
    const double probe = A.probe, band = L.band;
    double t = x_clamp(fa / (fa - fb), 0.0, 1.0);
    XEval last;
    double t0 = 0.0, g0 = fa, t1 = 1.0, g1 = fb;
    int side = 0;
    bool converged = false;
    uint32_t evals = 0;
    const bool spheres = A.flags & DARR_SPHERES;
    auto eval = [&](double x, double y, double z) {
        if (spheres)
            return RG == 1 ? x_eval_spheres<COUNT>(v, band, x, y, z, ops) : x_eval_spheres_group<RG>(v, band, x, y, z, gl, gm);
        return RG == 1 ? x_eval<COUNT>(v, A.circ, probe, band, x, y, z, ops)
                       : x_eval_group<RG>(v, A.circ, probe, band, x, y, z, gl, gm);
    };
    for (int it = 0; it < X_MAX_ITER; it++) {
        const double x = pax + dx * t, y = pay + dy * t, z = paz + dz * t;
        const XEval e = eval(x, y, z);
        evals++;
        last = e;
        const double g = e.value;
        if (fabs(g) <= X_TOL) {
            converged = true;
            break;
        }
        if ((g < 0.0) == (g0 < 0.0)) {
            t0 = t, g0 = g;
            if (side == -1) g1 *= 0.5;
            side = -1;
        } else {
            t1 = t, g1 = g;
            if (side == 1) g0 *= 0.5;
            side = 1;
        }
        double slope = 0.0;
        if (e.kind != XF_SOLVENT && e.kind != XF_BEYOND) {
            // gradient (extract.rs:539-549): towards the closest point (SES)
            // or away from the sphere's centre (a sphere field).
            const double wx = spheres ? x - e.qx : e.qx - x, wy = spheres ? y - e.qy : e.qy - y,
                         wz = spheres ? z - e.qz : e.qz - z;
            const double len = sqrt(wx * wx + wy * wy + wz * wz);
            if (len > 1e-12) slope = (wx / len) * dx + (wy / len) * dy + (wz / len) * dz;
        }
        const double newton = t - g / slope;
        if (fabs(slope) > 1e-3 * sqrt(dx * dx + dy * dy + dz * dz) && newton > t0 && newton < t1) {
            t = newton;
        } else {
            const double s = (t0 * g1 - t1 * g0) / (g1 - g0);
            t = (isfinite(s) && s > t0 && s < t1) ? s : 0.5 * (t0 + t1);
        }
    }
    if (!converged) {
        const double len = sqrt(dx * dx + dy * dy + dz * dz);
        const bool neg0 = g0 < 0.0;
        for (int it = 0; it < X_MAX_BISECT; it++) {
            t = 0.5 * (t0 + t1);
            const double x = pax + dx * t, y = pay + dy * t, z = paz + dz * t;
            const XEval e = eval(x, y, z);
            evals++;
            last = e;
            if (fabs(e.value) <= X_TOL || (t1 - t0) * len <= 2.0 * X_TOL) break;
            if ((e.value < 0.0) == neg0) t0 = t;
            else t1 = t;
        }
    }
    if (gl) return;
    const double ct = x_clamp(t, X.t_min, 1.0 - X.t_min);
    const double px = pax + dx * ct, py = pay + dy * ct, pz = paz + dz * ct;
    double nx, ny, nz;
    uint32_t atom, patch;
    x_attributes(A, L, X, last.kind, last.id, last.qx, last.qy, last.qz, px, py, pz, dx, dy, dz, fa, nx, ny, nz, atom,
                 patch);
    out.pos[3 * size_t(k)] = float(px), out.pos[3 * size_t(k) + 1] = float(py), out.pos[3 * size_t(k) + 2] = float(pz);
    out.nrm[3 * size_t(k)] = float(nx), out.nrm[3 * size_t(k) + 1] = float(ny), out.nrm[3 * size_t(k) + 2] = float(nz);
    out.atom[k] = atom;
    out.patch[k] = uint8_t(patch);
    out.t[k] = float(t);
    out.evals[k] = evals;
}

// Persistent CTAs of X_WARPS warps; each warp claims a work item, builds
// the item's ball in its own region and refines the item's edges lane per
// edge.  SLAB = false: the region is `region` bytes of shared memory, items
// come from counters[CNT_QUEUE] over all items, and an item whose lists do
// not fit goes to ovf (ovf[0] = count, then the items).  SLAB = true: the
// region is `region` bytes of a global slab per warp (read back through
// L1), items come from ovf through counters[CNT_XQUEUE], and an item that
// does not fit either stays with the host (*left counts them).  RG > 1: a
// group of RG lanes per edge instead of a lane.
template <bool SLAB, bool COUNT = false, int RG = 1>
__global__ void __launch_bounds__(32 * X_WARPS, 4) k_refine_exact(DArr A, DLat L, ExactAttr X, const int4* keys,
                                                               const uint32_t* work, const uint32_t* edges,
                                                               const float2* edge_vals, const uint32_t* item_off,
                                                               const uint32_t* item_edges, uint32_t n_items,
                                                               ExactOut out, size_t region, uint32_t* ovf,
                                                               unsigned char* slab, unsigned int* left,
                                                               unsigned long long* counters, const uint32_t* rec,
                                                               int slack, const uint32_t* gids,
                                                               const uint8_t* window) {
    extern __shared__ __align__(16) unsigned char xs[];
    __shared__ uint32_t sh_cnt[X_WARPS][8];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* mine = SLAB ? slab + (size_t(blockIdx.x) * X_WARPS + warp) * region : xs + size_t(warp) * region;
    uint32_t* cnt = sh_cnt[warp];
    unsigned int* queue = reinterpret_cast<unsigned int*>(&counters[SLAB ? CNT_XQUEUE : CNT_QUEUE]);
    const uint32_t n_claim = SLAB ? ovf[0] : n_items;
    unsigned long long ops = 0;
    for (;;) {
        uint32_t q = 0;
        if (lane == 0) q = atomicAdd(queue, 1u);
        q = __shfl_sync(0xffffffffu, q, 0);
        if (q >= n_claim) break;
        const uint32_t i = SLAB ? ovf[1 + q] : q;
        const uint32_t a0 = item_off[i], a1 = item_off[i + 1];
        if (a0 == a1) continue;
        const uint32_t j = work[i];
        const int4 key = keys[j >> 3];
        XView v;
        if (!x_ball<false>(A, L, key, j, mine, region, cnt, lane, 32u, v,
                           rec ? rec + size_t(j) * REC_WORDS : nullptr, slack, gids, window)) {
            if (lane == 0) {
                if (SLAB) atomicAdd(left, 1u);
                else ovf[1 + atomicAdd(&ovf[0], 1u)] = i;
            }
            continue;
        }
        const uint32_t gm = (0xffffffffu >> (32 - RG)) << (lane & ~uint32_t(RG - 1));
        for (uint32_t e = a0 + lane / RG; e < a1; e += 32 / RG) {
            const uint32_t k = item_edges[e];
            x_edge<COUNT, RG>(v, A, L, X, key, k, edges[k], edge_vals[k], out, &ops, int(lane % RG), gm);
        }
    }
    if (COUNT) {
        for (int o = 16; o; o >>= 1) ops += __shfl_down_sync(0xffffffffu, ops, o);
        if (lane == 0 && ops) atomicAdd(&counters[CNT_OPS], ops);
    }
}

// Sum of the edges' evaluation counts and the number of edges left to the
// host (evals = 0): out[0], out[1].
__global__ void k_exact_summary(const uint32_t* evals, size_t n, unsigned long long* out) {
    unsigned long long sum = 0, zero = 0;
    for (size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x; k < n; k += size_t(gridDim.x) * blockDim.x) {
        const uint32_t e = evals[k];
        sum += e;
        zero += e == 0;
    }
    for (int o = 16; o; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        zero += __shfl_down_sync(0xffffffffu, zero, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (sum) atomicAdd(&out[0], sum);
        if (zero) atomicAdd(&out[1], zero);
    }
}

// mesh_brick_device (extract.rs:274-365) on the device: each edge the f32
// refinement converged on (t in [0, 1], a valid feature) is placed at
// pa + d clamp(t) with the exact attributes of its feature and closest
// point (brick origin + the f32 offset); every other edge is marked in
// need[] for the exact refinement.  counters[0] += the marked edges.
__global__ void k_place_fast(DArr A, DLat L, ExactAttr X, const int4* keys, uint32_t n_bricks,
                             const uint32_t* edge_off, const uint32_t* edges, const float2* edge_vals, size_t n_edges,
                             const float* t_in, const uint32_t* feat, const float* q, const uint32_t* ev_in,
                             ExactOut out, uint8_t* need, unsigned long long* marked) {
    const size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    unsigned long long mine = 0;
    if (k < n_edges) {
        const uint32_t ev = ev_in[k];
        const double t = double(t_in[k]);
        const uint32_t kind = feat[k] >> 29, id = feat[k] & ((1u << 29) - 1);
        bool ok = (ev & 0x80000000u) && t >= 0.0 && t <= 1.0;
        if (ok) {
            if (kind == XF_SPHERE) ok = id < A.n;
            else if (kind == XF_CIRCLE) ok = id < A.nc;
            else if (kind == XF_VERTEX) ok = id < A.nv;
            else ok = kind == XF_SOLVENT || kind == XF_BEYOND;
        }
        if (!ok) {
            need[k] = 1;
            out.evals[k] = 0;
            mine = 1;
        } else {
            need[k] = 0;
            uint32_t lo = 0, hi = n_bricks;  // the brick of edge k: edge_off[lo] <= k < edge_off[lo + 1]
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (edge_off[mid] <= k) lo = mid;
                else hi = mid;
            }
            const int4 key = keys[lo];
            const int b = L.b;
            const double h = L.h;
            const uint32_t code = edges[k], cell = code / 3, axis = code % 3;
            const long long ix = (long long)key.x * b + (long long)(cell % uint32_t(b)),
                            iy = (long long)key.y * b + (long long)((cell / uint32_t(b)) % uint32_t(b)),
                            iz = (long long)key.z * b + (long long)(cell / uint32_t(b * b));
            const double pax = double(ix) * h, pay = double(iy) * h, paz = double(iz) * h;
            const double dx = double(ix + (axis == 0)) * h - pax, dy = double(iy + (axis == 1)) * h - pay,
                         dz = double(iz + (axis == 2)) * h - paz;
            const double ct = x_clamp(t, X.t_min, 1.0 - X.t_min);
            const double px = pax + dx * ct, py = pay + dy * ct, pz = paz + dz * ct;
            const double bx = double((long long)key.x * b) * h, by = double((long long)key.y * b) * h,
                         bz = double((long long)key.z * b) * h;
            const double qx = bx + double(q[3 * k]), qy = by + double(q[3 * k + 1]), qz = bz + double(q[3 * k + 2]);
            double nx, ny, nz;
            uint32_t atom, patch;
            x_attributes(A, L, X, kind, id, qx, qy, qz, px, py, pz, dx, dy, dz, double(edge_vals[k].x), nx, ny, nz,
                         atom, patch);
            out.pos[3 * k] = float(px), out.pos[3 * k + 1] = float(py), out.pos[3 * k + 2] = float(pz);
            out.nrm[3 * k] = float(nx), out.nrm[3 * k + 1] = float(ny), out.nrm[3 * k + 2] = float(nz);
            out.atom[k] = atom;
            out.patch[k] = uint8_t(patch);
            out.t[k] = t_in[k];
            out.evals[k] = ev & 0x7fffffffu;
        }
    }
    for (int o = 16; o; o >>= 1) mine += __shfl_down_sync(0xffffffffu, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(marked, mine);
}

}  // namespace

cudaError_t launch_place_fast(const DArr& A, const DLat& L, const ExactAttr& X, const int4* keys, uint32_t n_bricks,
                              const uint32_t* edge_off, const uint32_t* edges, const float2* edge_vals, size_t n_edges,
                              const float* t, const uint32_t* feat, const float* q, const uint32_t* evals,
                              const ExactOut& out, uint8_t* need, unsigned long long* marked, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(marked, 0, 8, s);
    if (e != cudaSuccess || !n_edges) return e;
    count_launches(1);
    k_place_fast<<<unsigned((n_edges + 255) / 256), 256, 0, s>>>(A, L, X, keys, n_bricks, edge_off, edges, edge_vals,
                                                                  n_edges, t, feat, q, evals, out, need, marked);
    return cudaGetLastError();
}

cudaError_t launch_exact_summary(const uint32_t* evals, size_t n, unsigned long long* out, int sms, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(out, 0, 16, s);
    if (e != cudaSuccess || !n) return e;
    const size_t want = (n + 255) / 256;
    count_launches(1);
    k_exact_summary<<<unsigned(std::min<size_t>(want, size_t(sms) * 8)), 256, 0, s>>>(evals, n, out);
    return cudaGetLastError();
}

template <bool COUNT, int RG, int RGS>
static cudaError_t launch_exact_levels(const DArr& A, const DLat& L, const ExactAttr& X, const int4* keys,
                                       const uint32_t* work, const uint32_t* edges, const float2* edge_vals,
                                       const uint32_t* item_off, const uint32_t* item_edges, uint32_t n_items,
                                       const ExactOut& out, uint32_t* ovf, unsigned char* slab, size_t slab_bytes,
                                       unsigned long long* counters, int sms, size_t region, cudaStream_t s,
                                       const uint32_t* rec, int slack, const uint32_t* gids,
                                       const uint8_t* window);

size_t exact_slab_bytes(int sms) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_refine_exact<true>, 32 * X_WARPS, 0);
    return size_t(std::max(sms, 1)) * size_t(std::max(per_sm, 1)) * X_WARPS * EXACT_SLAB;
}

cudaError_t launch_refine_exact(const DArr& A, const DLat& L, const ExactAttr& X, const int4* keys,
                                const uint32_t* work, const uint32_t* edges, const float2* edge_vals,
                                const uint32_t* item_off, const uint32_t* item_edges, uint32_t n_items,
                                const ExactOut& out, uint32_t* ovf, unsigned char* slab, size_t slab_bytes,
                                unsigned long long* counters, int sms, size_t region, cudaStream_t s, bool count,
                                int group, const uint32_t* rec, int hint, const uint32_t* gids,
                                const uint8_t* window) {
    const int slack = hint == 2 ? 0 : X_HINT_SLACK;
    if (hint == 0) rec = nullptr;
    if (count) {
        cudaError_t e = cudaMemsetAsync(&counters[CNT_OPS], 0, 8, s);
        if (e != cudaSuccess) return e;
        return launch_exact_levels<true, 1, 1>(A, L, X, keys, work, edges, edge_vals, item_off, item_edges,
                                               n_items, out, ovf, slab, slab_bytes, counters, sms, region, s, rec, slack, gids, window);
    }
    // The slab pass takes the largest lists: at least 8 lanes per edge.
    if (group == 32)
        return launch_exact_levels<false, 32, 32>(A, L, X, keys, work, edges, edge_vals, item_off, item_edges,
                                                  n_items, out, ovf, slab, slab_bytes, counters, sms, region, s, rec, slack, gids, window);
    if (group == 8)
        return launch_exact_levels<false, 8, 8>(A, L, X, keys, work, edges, edge_vals, item_off, item_edges, n_items,
                                                out, ovf, slab, slab_bytes, counters, sms, region, s, rec, slack, gids, window);
    return launch_exact_levels<false, 1, 8>(A, L, X, keys, work, edges, edge_vals, item_off, item_edges, n_items,
                                            out, ovf, slab, slab_bytes, counters, sms, region, s, rec, slack, gids, window);
}

template <bool COUNT, int RG, int RGS>
static cudaError_t launch_exact_levels(const DArr& A, const DLat& L, const ExactAttr& X, const int4* keys,
                                       const uint32_t* work, const uint32_t* edges, const float2* edge_vals,
                                       const uint32_t* item_off, const uint32_t* item_edges, uint32_t n_items,
                                       const ExactOut& out, uint32_t* ovf, unsigned char* slab, size_t slab_bytes,
                                       unsigned long long* counters, int sms, size_t region, cudaStream_t s,
                                       const uint32_t* rec, int slack, const uint32_t* gids,
                                       const uint8_t* window) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(&counters[CNT_QUEUE], 0, 8, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(&counters[CNT_XQUEUE], 0, 8, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(ovf, 0, 8, s)) != cudaSuccess) return e;
    if (!n_items) return cudaSuccess;
    region = (region + 15) & ~size_t(15);
    const size_t narrow = size_t(X_WARPS) * region;
    auto kn = k_refine_exact<false, COUNT, RG>;
    auto kg = k_refine_exact<true, COUNT, RGS>;
    if ((e = cudaFuncSetAttribute(kn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(narrow))) != cudaSuccess)
        return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kn, 32 * X_WARPS, narrow)) != cudaSuccess)
        return e;
    const uint32_t warps = (n_items + X_WARPS - 1) / X_WARPS;
    const uint32_t grid = std::min<uint32_t>(warps, uint32_t(sms * std::max(per_sm, 1)));
    count_launches(2);
    // ovf[0]: items over the shared region, ovf[1..]: those items; the word
    // after the list counts the items over a slab (left to the host).
    unsigned int* left = reinterpret_cast<unsigned int*>(ovf) + 1 + n_items;
    if ((e = cudaMemsetAsync(left, 0, 4, s)) != cudaSuccess) return e;
    kn<<<grid, 32 * X_WARPS, narrow, s>>>(A, L, X, keys, work, edges, edge_vals, item_off, item_edges, n_items, out,
                                          region, ovf, nullptr, left, counters, rec, slack, gids, window);
    // The overflowed items: a warp each, lists in a global slab.
    const uint32_t slabs = uint32_t(slab_bytes / EXACT_SLAB);
    const uint32_t grid_g = std::max<uint32_t>(1, slabs / X_WARPS);
    if (!slab || !grid_g) return cudaErrorInvalidValue;
    kg<<<grid_g, 32 * X_WARPS, 0, s>>>(A, L, X, keys, work, edges, edge_vals, item_off, item_edges, n_items, out,
                                       EXACT_SLAB, ovf, slab, left, counters, rec, slack, gids, window);
    return cudaGetLastError();
}

}  // namespace smb
