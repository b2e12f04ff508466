// The SES arrangement of a sphere set built on the device, in f64:
// active spheres in Morton order (geom/arrangement.rs:476-489), the cell
// grids (geom/cells.rs:27-84), containment (:497-514), neighbour rows
// (:522-545), the exposed intersection circles of each pair with their
// blockers and the exposed triple points (:674-752; as host/arrangement.cpp
// restates them), statuses, the rows of exposed spheres and the grids of
// circle centres and vertices (field/point.rs:235-270).
//
// Every value is the host build's bit for bit: the same f64 operations in
// the same order (no FMA contraction, IEEE division and square root), sets
// ordered by the same unique keys (stable radix sorts keep input order on
// equal keys, as the host's stable counting sort and pair sort do).  One
// decision uses a transcendental function: whether an angular gap between
// buried runs of a circle exceeds 1e-12 rad (atan2 of two crossing
// vectors).  The device's atan2 and the host's differ by a few ulps; a gap
// whose device value lies within 1e-13 rad of that threshold, or of the
// wrap at 0 / 2 pi, cannot be decided the same way with certainty, and the
// device then declines the whole build (the host builds it).  So does a
// circle with more candidate blockers than a thread keeps.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "common.cuh"
#include "kernels.hpp"
#include "sas.hpp"
#include "scan.cuh"

namespace smb {
namespace {

constexpr double S_EPS = 1e-9;           // arrangement.rs:26
constexpr double S_ANG_EPS = 1e-12;      // arrangement.rs:29
constexpr double S_PERIOD = 4.0;         // arrangement.rs:277
constexpr double S_PSEUDO_EPS = 1e-12;   // arrangement.rs:279
constexpr double S_TWO_PI = 6.283185307179586;
constexpr double S_ANG_MARGIN = 1e-13;   // device/host atan2 disagreement bound on a gap
constexpr int MAX_SPANS = 48;            // candidate blockers a thread keeps per circle
constexpr int RED_BLOCKS = 1024;         // partial reductions

enum : uint32_t { DECLINE_ANGLE = 1, DECLINE_SPANS = 2 };

struct D3 {
    double x, y, z;
};
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ D3 operator/(D3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
__device__ __forceinline__ double dotp(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 crossp(D3 a, D3 o) {
    return {a.y * o.z - a.z * o.y, a.z * o.x - a.x * o.z, a.x * o.y - a.y * o.x};
}
__device__ __forceinline__ double normp(D3 a) { return sqrt(dotp(a, a)); }
__device__ __forceinline__ double distp(D3 a, D3 b) { return normp(a - b); }
__device__ __forceinline__ D3 xyz(double4 v) { return {v.x, v.y, v.z}; }

__host__ __device__ __forceinline__ unsigned long long to_u64d(double v) {  // Rust's saturating cast
    if (!(v > 0.0)) return 0;
    return v >= 18446744073709551616.0 ? ~0ull : (unsigned long long)v;
}

__device__ __forceinline__ unsigned long long interleave(uint32_t v) {  // cells.rs:135-143
    unsigned long long x = (unsigned long long)v & 0x1fffff;
    x = (x | (x << 32)) & 0x001f00000000ffffULL;
    x = (x | (x << 16)) & 0x001f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

// Bounding box (and, for spheres, the largest expanded radius and the
// count of spheres with r > 0) per block.
struct Box {
    double lo[3], hi[3], mx;
    unsigned long long cnt;
};

__device__ void box_reduce(Box b, Box* out) {
    __shared__ Box sh[256];
    sh[threadIdx.x] = b;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (int(threadIdx.x) < o) {
            Box& a = sh[threadIdx.x];
            const Box& c = sh[threadIdx.x + o];
            for (int k = 0; k < 3; k++) a.lo[k] = fmin(a.lo[k], c.lo[k]), a.hi[k] = fmax(a.hi[k], c.hi[k]);
            a.mx = fmax(a.mx, c.mx);
            a.cnt += c.cnt;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

__device__ __forceinline__ Box box_empty() {
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    return Box{{inf, inf, inf}, {-inf, -inf, -inf}, 0.0, 0};
}

// Active spheres (r > 0): centres' box, max(r + probe), count.
__global__ void k_box_active(const double* xyzr, size_t n, double probe, Box* out) {
    Box b = box_empty();
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double* s = xyzr + 4 * i;
        if (!(s[3] > 0.0)) continue;
        for (int k = 0; k < 3; k++) b.lo[k] = fmin(b.lo[k], s[k]), b.hi[k] = fmax(b.hi[k], s[k]);
        b.mx = fmax(b.mx, s[3] + probe);
        b.cnt++;
    }
    box_reduce(b, out);
}

// Points at p + stride * i: box; mx = the largest word `wmax` of each point.
__global__ void k_box_points(const double* p, size_t stride, size_t n, int wmax, Box* out) {
    Box b = box_empty();
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double* q = p + stride * i;
        for (int k = 0; k < 3; k++) b.lo[k] = fmin(b.lo[k], q[k]), b.hi[k] = fmax(b.hi[k], q[k]);
        if (wmax >= 0) b.mx = fmax(b.mx, q[wmax]);
        b.cnt++;
    }
    box_reduce(b, out);
}

// Morton keys of the active spheres' cells, ties by input index (the sort
// is stable); inactive spheres sort last.
__global__ void k_morton(const double* xyzr, size_t n, double lx, double ly, double lz, double cell,
                         unsigned long long* keys, uint32_t* vals) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double* s = xyzr + 4 * i;
    vals[i] = uint32_t(i);
    if (!(s[3] > 0.0)) {
        keys[i] = ~0ull;
        return;
    }
    const double px = (s[0] - lx) / cell, py = (s[1] - ly) / cell, pz = (s[2] - lz) / cell;
    const uint32_t qx = uint32_t(min(to_u64d(px), 0x1fffffull)), qy = uint32_t(min(to_u64d(py), 0x1fffffull)),
                   qz = uint32_t(min(to_u64d(pz), 0x1fffffull));
    keys[i] = interleave(qx) | (interleave(qy) << 1) | (interleave(qz) << 2);
}

__global__ void k_take_spheres(const double* xyzr, const uint32_t* order, size_t n, double probe, double4* sph,
                               double* rvdw, uint32_t* orig) {
    const size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (k >= n) return;
    const uint32_t i = order[k];
    const double* s = xyzr + 4 * size_t(i);
    sph[k] = make_double4(s[0], s[1], s[2], s[3] + probe);
    rvdw[k] = s[3];
    orig[k] = i;
}

// Grid::coord (geom/cells.rs:91-104).
__device__ __forceinline__ uint32_t grid_coord(double p, double o, double cell, uint32_t dim) {
    const double c = floor((p - o) / cell);
    if (!(c > 0.0)) return 0;
    const unsigned long long v = to_u64d(c);
    return v >= dim - 1 ? dim - 1 : uint32_t(v);
}

__global__ void k_cell_keys(const double* p, size_t stride, size_t n, double ox, double oy, double oz, double cell,
                            uint32_t dx, uint32_t dy, uint32_t dz, uint32_t* keys, uint32_t* vals) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double* q = p + stride * i;
    keys[i] = (grid_coord(q[2], oz, cell, dz) * dy + grid_coord(q[1], oy, cell, dy)) * dx + grid_coord(q[0], ox, cell, dx);
    vals[i] = uint32_t(i);
}

// starts[c] = first position of cell c among the sorted keys (cells + 1).
__global__ void k_cell_starts(const uint32_t* sorted, size_t n, size_t cells, uint32_t* starts) {
    const size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (c > cells) return;
    size_t lo = 0, hi = n;
    while (lo < hi) {
        const size_t mid = (lo + hi) >> 1;
        if (sorted[mid] < c) lo = mid + 1;
        else hi = mid;
    }
    starts[c] = uint32_t(lo);
}

template <class F>
__device__ __forceinline__ void grid_near(const DGrid& g, D3 c, double r, F&& f) {
    const uint32_t x0 = grid_coord(c.x - r, g.ox, g.cell, g.dx), y0 = grid_coord(c.y - r, g.oy, g.cell, g.dy),
                   z0 = grid_coord(c.z - r, g.oz, g.cell, g.dz);
    const uint32_t x1 = grid_coord(c.x + r, g.ox, g.cell, g.dx), y1 = grid_coord(c.y + r, g.oy, g.cell, g.dy),
                   z1 = grid_coord(c.z + r, g.oz, g.cell, g.dz);
    for (uint32_t z = z0; z <= z1; z++)
        for (uint32_t y = y0; y <= y1; y++) {
            const size_t row = (size_t(z) * g.dy + y) * g.dx;
            for (uint32_t i = g.starts[row + x0], e = g.starts[row + x1 + 1]; i < e; i++) f(g.items[i]);
        }
}

// Containment (arrangement.rs:497-514).
__global__ void k_contained(const double4* sph, const uint32_t* orig, size_t n, DGrid g, double max_expanded,
                            uint32_t* contained) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const double4 si = sph[i];
    const D3 ci = xyz(si);
    const double Ri = si.w;
    bool found = false;
    grid_near(g, ci, Ri + max_expanded, [&](uint32_t j) {
        if (found || j == i) return;
        const double4 sj = sph[j];
        const double d = distp(ci, xyz(sj));
        if (d + Ri <= sj.w + S_EPS && (sj.w - Ri > S_EPS || d > S_EPS || orig[j] < orig[i])) found = true;
    });
    contained[i] = found ? 1u : 0u;
}

// Neighbour rows (arrangement.rs:522-545): count, then fill and sort.
template <bool FILL>
__global__ void k_rows(const double4* sph, const uint32_t* contained, size_t n, DGrid g, double max_expanded,
                       uint32_t* count, const uint32_t* off, uint32_t* items) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    if (contained[i]) {
        if (!FILL) count[i] = 0;
        return;
    }
    const double4 si = sph[i];
    const D3 ci = xyz(si);
    uint32_t c = 0;
    uint32_t* row = FILL ? items + off[i] : nullptr;
    grid_near(g, ci, si.w + max_expanded, [&](uint32_t j) {
        if (j == i || contained[j]) return;
        const double4 sj = sph[j];
        const D3 dc = ci - xyz(sj);
        if (sqrt_lt(dotp(dc, dc), si.w + sj.w - S_EPS)) {  // |ci - cj| < Ri + Rj - eps
            if (FILL) row[c] = j;
            c++;
        }
    });
    if constexpr (!FILL) {
        count[i] = c;
    } else {
        for (uint32_t a = 1; a < c; a++) {  // insertion sort: rows are short
            const uint32_t v = row[a];
            uint32_t b = a;
            for (; b > 0 && row[b - 1] > v; b--) row[b] = row[b - 1];
            row[b] = v;
        }
    }
}

// The circle of an (i, j) pair (arrangement.rs:674-700) and its cut by a
// third sphere (:251-274).
struct Circle {
    D3 m, u, e1, e2;
    double rho;
};

__device__ __forceinline__ int cut(const Circle& c, D3 s, double R, double en[2], double lv[2]) {
    const D3 g = c.m - s;
    const double a = 2.0 * c.rho * dotp(c.e1, g);
    const double b = 2.0 * c.rho * dotp(c.e2, g);
    const double rhs = R * R - dotp(g, g) - c.rho * c.rho;
    const double amp = sqrt(a * a + b * b);
    if (amp <= rhs) return 1;
    if (amp <= -rhs || amp == 0.0) return 0;
    const double cp = a / amp, sp = b / amp, ca = rhs / amp;
    const double sa = sqrt(fmax(1.0 - ca * ca, 0.0));
    en[0] = cp * ca - sp * sa, en[1] = sp * ca + cp * sa;
    lv[0] = cp * ca + sp * sa, lv[1] = sp * ca - cp * sa;
    return 2;
}

__device__ __forceinline__ double diamond(double x, double y) {  // arrangement.rs:282-297
    if (y >= 0.0) return x >= 0.0 ? y / (x + y) : 1.0 - x / (y - x);
    return x < 0.0 ? 2.0 - y / (-x - y) : 3.0 + x / (x - y);
}

__device__ __forceinline__ long long order_bits(double v) {  // f64::total_cmp as an integer key
    const long long b = __double_as_longlong(v);
    return b ^ (long long)((unsigned long long)(b >> 63) >> 1);
}

__device__ __forceinline__ double wrap_tau(double a) {  // f64::rem_euclid(TAU)
    const double r = fmod(a, S_TWO_PI);
    return r < 0.0 ? r + S_TWO_PI : r;
}

// A circle's blocked spans: start and end parameters and the blocking
// sphere (its cut points are recomputed where needed, which keeps each
// thread's local memory small).
struct Spans {
    double start[MAX_SPANS], end[MAX_SPANS];
    uint32_t sphere[MAX_SPANS];
    uint8_t ord[MAX_SPANS];
    int n;
};

// any_exposed (arrangement.rs:340-405): 1 exposed, 0 buried, -1 declined.
// Runs keep the span that opened them (its start and entry point) and the
// span that gave their end (its exit point).
__device__ int any_exposed(Spans& S, const Circle& C, const double4* sph) {
    if (S.n == 0) return 1;
    for (int a = 0; a < S.n; a++) S.ord[a] = uint8_t(a);
    auto less = [&](int a, int b) {
        long long x = order_bits(S.start[a]), y = order_bits(S.start[b]);
        if (x != y) return x < y;
        x = order_bits(S.end[b]), y = order_bits(S.end[a]);
        if (x != y) return x < y;
        return S.sphere[a] < S.sphere[b];
    };
    for (int a = 1; a < S.n; a++) {
        const uint8_t v = S.ord[a];
        int b = a;
        for (; b > 0 && less(v, S.ord[b - 1]); b--) S.ord[b] = S.ord[b - 1];
        S.ord[b] = v;
    }
    // Runs, in place of nothing: at most n of them.
    double re[MAX_SPANS];
    uint8_t first[MAX_SPANS], last[MAX_SPANS];
    int m = 0;
    for (int a = 0; a < S.n; a++) {
        const int s = S.ord[a];
        if (m > 0 && S.start[s] <= re[m - 1]) {
            if (S.end[s] > re[m - 1]) re[m - 1] = S.end[s], last[m - 1] = uint8_t(s);
        } else {
            re[m] = S.end[s], first[m] = uint8_t(s), last[m] = uint8_t(s);
            m++;
        }
    }
    int b0 = 0;  // runs[b0 .. m)
    while (m - b0 > 1) {
        const double fs = S.start[first[b0]], fe = re[b0];
        const int l = m - 1;
        if (re[l] - S_PERIOD < fs) break;
        if (fe + S_PERIOD > re[l]) re[l] = fe + S_PERIOD, last[l] = last[b0];
        b0++;
    }
    const int cnt = m - b0;
    for (int k = 0; k < cnt; k++) {
        const int cur = b0 + k, nxt = b0 + (k + 1) % cnt;
        const double ns = S.start[first[nxt]];
        const double next_start = k + 1 < cnt ? ns : ns + S_PERIOD;
        if (next_start - re[cur] > S_PSEUDO_EPS) {
            double en[2], lv[2], en2[2], lv2[2];
            const double4 sc = sph[S.sphere[last[cur]]], sn = sph[S.sphere[first[nxt]]];
            cut(C, xyz(sc), sc.w, en, lv);
            cut(C, xyz(sn), sn.w, en2, lv2);
            const double a0 = wrap_tau(atan2(lv[1], lv[0]));
            const double a1 = atan2(en2[1], en2[0]);
            const double w = wrap_tau(a1 - a0);
            if (w < S_ANG_EPS + S_ANG_MARGIN || w > S_TWO_PI - S_ANG_MARGIN) return -1;
            if (w > S_ANG_EPS) return 1;
        }
    }
    return 0;
}

// The row entries (i, j) with j > i, whose circles k_circles builds: rows
// ascend, so they are each row's tail; per row their count, then (at the
// scanned offsets) each one's entry index and row.
__global__ void k_upper_count(const uint32_t* nb_off, const uint32_t* nb_items, size_t n, uint32_t* cnt) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    uint32_t lo = nb_off[i], hi = nb_off[i + 1];
    const uint32_t end = hi;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (nb_items[mid] <= uint32_t(i)) lo = mid + 1;
        else hi = mid;
    }
    cnt[i] = end - lo;
}

__global__ void k_upper_fill(const uint32_t* nb_off, const uint32_t* cnt, const uint32_t* uoff, size_t n,
                             uint32_t* uent, uint32_t* urow) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = cnt[i], end = nb_off[i + 1], o = uoff[i];
    for (uint32_t t = 0; t < c; t++) uent[o + t] = end - c + t, urow[o + t] = uint32_t(i);
}

// The upper entries whose circle is exposed, at their circle's index.
__global__ void k_exposed_list(const uint32_t* uent, size_t n_upper, const uint32_t* c_ex, const uint32_t* o_circ,
                               uint32_t* xlist) {
    const size_t u = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (u >= n_upper) return;
    const uint32_t e = uent[u];
    if (c_ex[e]) xlist[o_circ[e]] = uint32_t(u);
}

// Circles, blockers and triple points of each row entry (i, j > i)
// (arrangement.rs:674-752), a thread per upper entry (uent, urow).  Count
// pass: per entry the circle's exposure (0/1), blocker and vertex counts
// (zero beforehand for every entry), exposed[] of both spheres; fill pass,
// a thread per exposed circle (xlist): the records at the scanned offsets.
template <bool FILL>
__global__ void __launch_bounds__(128) k_circles(const double4* sph, size_t n, const uint32_t* nb_off,
                                                 const uint32_t* nb_items, size_t n_threads, const uint32_t* uent,
                                                 const uint32_t* urow, const uint32_t* xlist, uint32_t* c_ex,
                                                 uint32_t* c_blk, uint32_t* c_vtx, uint32_t* exposed,
                                                 const uint32_t* o_circ, const uint32_t* o_blk, const uint32_t* o_vtx,
                                                 double* circ, uint32_t* ij, uint32_t* cb_off, uint32_t* cb_items,
                                                 double4* vert, uint32_t* vatoms, uint32_t* decline) {
    const size_t id = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (id >= n_threads) return;
    const uint32_t u = FILL ? xlist[id] : uint32_t(id);
    const size_t e = uent[u];
    auto zero = [&] {
        if (!FILL) c_ex[e] = 0, c_blk[e] = 0, c_vtx[e] = 0;
    };
    const uint32_t i = urow[u], j = nb_items[e];
    if (j <= i) return zero();
    if (FILL && !c_ex[e]) return;
    const double4 si = sph[i], sj = sph[j];
    const D3 ci = xyz(si), cj = xyz(sj);
    const double Ri = si.w, Rj = sj.w;
    const double d = distp(ci, cj);
    const D3 axis = (cj - ci) / d;
    const double t = (d * d + Ri * Ri - Rj * Rj) / (2.0 * d);
    const double rho2 = Ri * Ri - t * t;
    if (rho2 <= 0.0) return zero();
    const double ax = fabs(axis.x), ay = fabs(axis.y), az = fabs(axis.z);  // orthonormal_basis (geom/vec.rs:112-125)
    const D3 helper = (ax <= ay && ax <= az) ? D3{1, 0, 0} : (ay <= az ? D3{0, 1, 0} : D3{0, 0, 1});
    const D3 hx = crossp(helper, axis);
    const D3 e1 = hx / normp(hx);
    const D3 e2 = crossp(axis, e1);
    Circle C{ci + axis * t, axis, e1, e2, sqrt(rho2)};
    const uint32_t ri0 = nb_off[i], ri1 = nb_off[i + 1], rj1 = nb_off[j + 1];
    uint32_t q = nb_off[j];
    Spans S;
    S.n = 0;
    for (uint32_t pk = ri0; pk < ri1; pk++) {
        const uint32_t k = nb_items[pk];
        while (q < rj1 && nb_items[q] < k) q++;
        if (q == rj1 || nb_items[q] != k) continue;
        double en[2], lv[2];
        const double4 sk = sph[k];
        const int kind = cut(C, xyz(sk), sk.w, en, lv);
        if (kind == 0) continue;
        if (kind == 1) return zero();  // buried
        if (S.n == MAX_SPANS) {
            atomicOr(decline, DECLINE_SPANS);
            return zero();
        }
        const int a = S.n++;
        S.start[a] = diamond(en[0], en[1]);
        S.end[a] = diamond(lv[0], lv[1]);
        if (S.end[a] <= S.start[a]) S.end[a] += S_PERIOD;
        S.sphere[a] = k;
    }
    const int ex = any_exposed(S, C, sph);
    if (ex < 0) {
        atomicOr(decline, DECLINE_ANGLE);
        return zero();
    }
    if (ex == 0) return zero();
    // Triple points with the blockers k > j.
    uint32_t nv = 0;
    const uint32_t v0 = FILL ? o_vtx[e] : 0;
    for (int a = 0; a < S.n; a++) {
        const uint32_t k = S.sphere[a];
        if (k <= j) continue;
        double en[2], lv[2];
        const double4 sk = sph[k];
        if (cut(C, xyz(sk), sk.w, en, lv) != 2) continue;
        const double* ends[2] = {lv, en};
        for (int w = 0; w < 2; w++) {
            const double* cs = ends[w];
            const D3 p = C.m + (C.e1 * cs[0] + e2 * cs[1]) * C.rho;
            bool free = true;
            for (uint32_t pl = ri0; pl < ri1 && free; pl++) {
                const uint32_t l = nb_items[pl];
                if (l != j && l != k) {
                    // |p - c| >= R - eps, decided from the square where it
                    // is clear (sqrt_ge: the same result as the rounded root).
                    const double4 sl = sph[l];
                    const D3 dp = p - xyz(sl);
                    free = sqrt_ge(dotp(dp, dp), sl.w - S_EPS);
                }
            }
            if (free) {
                if (FILL) {
                    vert[v0 + nv] = make_double4(p.x, p.y, p.z, 0.0);
                    uint32_t* va = vatoms + 3 * size_t(v0 + nv);
                    va[0] = i, va[1] = j, va[2] = k;
                }
                nv++;
            }
        }
    }
    if (!FILL) {
        c_ex[e] = 1, c_blk[e] = uint32_t(S.n), c_vtx[e] = nv;
        exposed[i] = 1, exposed[j] = 1;
        return;
    }
    const uint32_t c = o_circ[e], b = o_blk[e];
    double* rec = circ + 12 * size_t(c);
    rec[0] = C.m.x, rec[1] = C.m.y, rec[2] = C.m.z, rec[3] = axis.x, rec[4] = axis.y, rec[5] = axis.z;
    rec[6] = e1.x, rec[7] = e1.y, rec[8] = e1.z, rec[9] = C.rho, rec[10] = 0.0, rec[11] = 0.0;
    ij[2 * size_t(c)] = i, ij[2 * size_t(c) + 1] = j;
    cb_off[c] = b;
    for (int a = 0; a < S.n; a++) cb_items[b + a] = S.sphere[a];
}

// Status (contained 2, exposed 0, buried 1) and the row lengths kept
// (exposed spheres only; point.rs:244-245).
__global__ void k_status(const uint32_t* contained, const uint32_t* exposed, const uint32_t* nb_off, size_t n,
                         uint32_t* status, uint32_t* keep_len) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n) return;
    const uint32_t len = nb_off[i + 1] - nb_off[i];
    const bool ex = !contained[i] && (len == 0 || exposed[i]);
    status[i] = contained[i] ? STATUS_CONTAINED : (ex ? STATUS_EXPOSED : STATUS_BURIED);
    keep_len[i] = ex ? len : 0;
}

__global__ void k_keep_rows(const uint32_t* nb_off, const uint32_t* nb_items, const uint32_t* keep_len,
                            const uint32_t* new_off, size_t n, uint32_t* out) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i >= n || !keep_len[i]) return;
    for (uint32_t a = 0; a < keep_len[i]; a++) out[new_off[i] + a] = nb_items[nb_off[i] + a];
}

__global__ void k_put(uint32_t* dst, uint32_t v) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *dst = v;
}

// Host side.
struct Ctx {
    cudaStream_t s;
    DevArrangement& out;
    std::vector<void*> temp;
    std::string* msg;
    bool ok = true;
    void* alloc(size_t bytes, bool keep) {
        void* p = nullptr;
        if (mem_alloc(&p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            ok = false;
            if (msg) *msg = "device memory for the arrangement";
            return nullptr;
        }
        if (keep) out.owned.push_back(p), out.bytes += bytes;
        else temp.push_back(p);
        return p;
    }
    ~Ctx() {
        for (void* p : temp) mem_free(p);
    }
};

unsigned blocks_for(size_t n, unsigned t = 256) { return unsigned(std::max<size_t>(1, (n + t - 1) / t)); }

bool reduce_box(Ctx& X, Box* part, Box& b) {
    std::vector<Box> h(RED_BLOCKS);
    if (cudaMemcpyAsync(h.data(), part, sizeof(Box) * RED_BLOCKS, cudaMemcpyDeviceToHost, X.s) != cudaSuccess ||
        cudaStreamSynchronize(X.s) != cudaSuccess)
        return false;
    const double inf = std::numeric_limits<double>::infinity();
    b = Box{{inf, inf, inf}, {-inf, -inf, -inf}, 0.0, 0};
    for (const Box& p : h) {
        for (int k = 0; k < 3; k++) b.lo[k] = std::fmin(b.lo[k], p.lo[k]), b.hi[k] = std::fmax(b.hi[k], p.hi[k]);
        b.mx = std::fmax(b.mx, p.mx);
        b.cnt += p.cnt;
    }
    return true;
}

// Grid::build (geom/cells.rs:27-84) over n points at p + stride * i.
bool build_grid(Ctx& X, const double* p, size_t stride, size_t n, double cell_in, Box* part, DGrid& G) {
    G = DGrid{};
    G.cell = cell_in;
    if (n == 0) {
        G.dx = G.dy = G.dz = 1;
        uint32_t* st = static_cast<uint32_t*>(X.alloc(8, true));
        if (!st || cudaMemsetAsync(st, 0, 8, X.s) != cudaSuccess) return false;
        G.starts = st;
        G.items = static_cast<uint32_t*>(X.alloc(4, true));
        return G.items != nullptr;
    }
    k_box_points<<<RED_BLOCKS, 256, 0, X.s>>>(p, stride, n, -1, part);
    Box b;
    if (!reduce_box(X, part, b)) return false;
    const double e[3] = {b.hi[0] - b.lo[0], b.hi[1] - b.lo[1], b.hi[2] - b.lo[2]};
    const size_t max_cells = std::max<size_t>(8 * n, size_t(1) << 16);
    double cell = cell_in;
    uint32_t dims[3];
    for (;;) {
        unsigned __int128 total = 1;
        bool ok = true;
        for (int a = 0; a < 3; a++) {
            const uint64_t v = to_u64d(std::floor(e[a] / cell));
            if (v >= UINT32_MAX) ok = false;
            dims[a] = ok ? uint32_t(v + 1) : 1;
            total *= (unsigned __int128)(v + 1);
        }
        if (ok && total <= max_cells) break;
        cell *= 2.0;
    }
    G.ox = b.lo[0], G.oy = b.lo[1], G.oz = b.lo[2], G.cell = cell;
    G.dx = dims[0], G.dy = dims[1], G.dz = dims[2];
    const size_t cells = size_t(dims[0]) * dims[1] * dims[2];
    if (cells >= (size_t(1) << 32) - 1 || n >= (size_t(1) << 31)) return false;
    uint32_t* keys = static_cast<uint32_t*>(X.alloc(n * 4, false));
    uint32_t* keys2 = static_cast<uint32_t*>(X.alloc(n * 4, false));
    uint32_t* vals = static_cast<uint32_t*>(X.alloc(n * 4, false));
    uint32_t* items = static_cast<uint32_t*>(X.alloc(n * 4, true));
    uint32_t* starts = static_cast<uint32_t*>(X.alloc((cells + 1) * 4, true));
    if (!X.ok) return false;
    k_cell_keys<<<blocks_for(n), 256, 0, X.s>>>(p, stride, n, G.ox, G.oy, G.oz, cell, dims[0], dims[1], dims[2], keys,
                                                vals);
    unsigned bits = 1;
    while (bits < 32 && (uint64_t(1) << bits) < cells) bits++;
    size_t tmp = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys2, vals, items, int(n), 0, int(bits), X.s);
    void* t = X.alloc(tmp, false);
    if (!t) return false;
    if (cub::DeviceRadixSort::SortPairs(t, tmp, keys, keys2, vals, items, int(n), 0, int(bits), X.s) != cudaSuccess)
        return false;
    k_cell_starts<<<blocks_for(cells + 1), 256, 0, X.s>>>(keys2, n, cells, starts);
    G.starts = starts;
    G.items = items;
    count_launches(4);
    return cudaGetLastError() == cudaSuccess;
}

}  // namespace

void DevArrangement::release() {
    for (void* p : owned) mem_free(p);
    owned.clear();
    bytes = 0;
}

int build_arrangement_device(smb_device* d, const double* xyzr, size_t ns, double probe, DevArrangement& out,
                             std::string* msg) {
    out = DevArrangement();
    Ctx X{d->stream, out, {}, msg};
    cudaStream_t s = d->stream;
    auto fail = [&](const char* what) {
        if (msg && msg->empty()) *msg = what;
        out.release();
        return 2;
    };
    if (ns >= (size_t(1) << 31)) return fail("too many spheres for the device arrangement");
    double* dx = static_cast<double*>(X.alloc(ns * 32, false));
    Box* part = static_cast<Box*>(X.alloc(sizeof(Box) * RED_BLOCKS, false));
    if (!X.ok) return fail("device memory");
    if (ns && cudaMemcpyAsync(dx, xyzr, ns * 32, cudaMemcpyHostToDevice, s) != cudaSuccess) return fail("upload");
    // Active spheres, max_expanded, Morton order.
    k_box_active<<<RED_BLOCKS, 256, 0, s>>>(dx, ns, probe, part);
    count_launches(1);
    Box ba;
    if (!reduce_box(X, part, ba)) return fail("reduction");
    const size_t n = size_t(ba.cnt);
    const double max_expanded = ba.mx;
    const double cell = std::fmax(2.0 * max_expanded, 1e-6);
    DArr& A = out.A;
    A.n = uint32_t(n);
    A.max_expanded = max_expanded;
    A.probe = probe;
    out.n = n;
    double4* sph = static_cast<double4*>(X.alloc(n * 32, true));
    double* rvdw = static_cast<double*>(X.alloc(n * 8, true));
    uint32_t* orig = static_cast<uint32_t*>(X.alloc(n * 4, true));
    uint32_t* status = static_cast<uint32_t*>(X.alloc(n * 4, true));
    if (!X.ok) return fail("device memory");
    if (ns) {
        unsigned long long* keys = static_cast<unsigned long long*>(X.alloc(ns * 8, false));
        unsigned long long* keys2 = static_cast<unsigned long long*>(X.alloc(ns * 8, false));
        uint32_t* vals = static_cast<uint32_t*>(X.alloc(ns * 4, false));
        uint32_t* order = static_cast<uint32_t*>(X.alloc(ns * 4, false));
        if (!X.ok) return fail("device memory");
        k_morton<<<blocks_for(ns), 256, 0, s>>>(dx, ns, ba.lo[0], ba.lo[1], ba.lo[2], cell, keys, vals);
        size_t tmp = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, tmp, keys, keys2, vals, order, int(ns), 0, 64, s);
        void* t = X.alloc(tmp, false);
        if (!t || cub::DeviceRadixSort::SortPairs(t, tmp, keys, keys2, vals, order, int(ns), 0, 64, s) != cudaSuccess)
            return fail("sort");
        if (n) k_take_spheres<<<blocks_for(n), 256, 0, s>>>(dx, order, n, probe, sph, rvdw, orig);
        count_launches(2);
    }
    A.sph = sph, A.rvdw = rvdw, A.status = status;
    out.orig = orig;
    for (int k = 0; k < 3; k++) out.lo[k] = n ? ba.lo[k] : 0.0, out.hi[k] = n ? ba.hi[k] : 0.0;
    if (!build_grid(X, reinterpret_cast<const double*>(sph), 4, n, cell, part, A.gs)) return fail("sphere grid");
    // Containment, rows.
    uint32_t* contained = static_cast<uint32_t*>(X.alloc(n * 4, false));
    uint32_t* rlen = static_cast<uint32_t*>(X.alloc(n * 4, false));
    uint32_t* roff = static_cast<uint32_t*>(X.alloc((n + 1) * 4, false));
    unsigned long long* tiles = static_cast<unsigned long long*>(X.alloc(size_t(scan_tiles_needed(uint32_t(n + 1))) * 8 + 64, false));
    unsigned long long* total = static_cast<unsigned long long*>(X.alloc(64, false));
    if (!X.ok) return fail("device memory");
    unsigned long long h_tot[3] = {0, 0, 0};
    if (n) {
        k_contained<<<blocks_for(n), 256, 0, s>>>(sph, orig, n, A.gs, max_expanded, contained);
        k_rows<false><<<blocks_for(n), 256, 0, s>>>(sph, contained, n, A.gs, max_expanded, rlen, nullptr, nullptr);
        launch_scan(rlen, uint32_t(n), roff, nullptr, tiles, total, s);
        if (cudaMemcpyAsync(h_tot, total, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return fail("rows");
        count_launches(2);
    }
    const size_t n_entries = size_t(h_tot[0]);
    if (n_entries >= (size_t(1) << 32)) return fail("too many neighbour pairs for the device arrangement");
    k_put<<<1, 32, 0, s>>>(roff + n, uint32_t(n_entries));
    uint32_t* items = static_cast<uint32_t*>(X.alloc(n_entries * 4, false));
    if (!X.ok) return fail("device memory");
    if (n) k_rows<true><<<blocks_for(n), 256, 0, s>>>(sph, contained, n, A.gs, max_expanded, nullptr, roff, items);
    // Circles: count, scans, fill.
    uint32_t* c_ex = static_cast<uint32_t*>(X.alloc(n_entries * 4, false));
    uint32_t* c_blk = static_cast<uint32_t*>(X.alloc(n_entries * 4, false));
    uint32_t* c_vtx = static_cast<uint32_t*>(X.alloc(n_entries * 4, false));
    uint32_t* o_circ = static_cast<uint32_t*>(X.alloc(n_entries * 4, false));
    uint32_t* o_blk = static_cast<uint32_t*>(X.alloc(n_entries * 4, false));
    uint32_t* o_vtx = static_cast<uint32_t*>(X.alloc(n_entries * 4, false));
    uint32_t* exposed = static_cast<uint32_t*>(X.alloc((n + 1) * 4, false));
    uint32_t* decline = static_cast<uint32_t*>(X.alloc(16, false));
    unsigned long long* tiles_e =
        static_cast<unsigned long long*>(X.alloc(size_t(scan_tiles_needed(uint32_t(n_entries))) * 8 + 64, false));
    if (!X.ok) return fail("device memory");
    uint32_t* ucnt = static_cast<uint32_t*>(X.alloc(n * 4 + 4, false));
    uint32_t* uoff = static_cast<uint32_t*>(X.alloc(n * 4 + 4, false));
    if (!X.ok) return fail("device memory");
    cudaMemsetAsync(exposed, 0, n * 4 + 4, s);
    cudaMemsetAsync(decline, 0, 16, s);
    // The upper entries (j > i) as a list, so that every thread of the
    // circle passes has a pair to build.
    size_t n_upper = 0;
    uint32_t *uent = nullptr, *urow = nullptr;
    if (n_entries) {
        k_upper_count<<<blocks_for(n), 256, 0, s>>>(roff, items, n, ucnt);
        launch_scan(ucnt, uint32_t(n), uoff, nullptr, tiles, total, s);
        unsigned long long h_up = 0;
        if (cudaMemcpyAsync(&h_up, total, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return fail("upper entries");
        n_upper = size_t(h_up);
        uent = static_cast<uint32_t*>(X.alloc(n_upper * 4 + 4, false));
        urow = static_cast<uint32_t*>(X.alloc(n_upper * 4 + 4, false));
        if (!X.ok) return fail("device memory");
        k_upper_fill<<<blocks_for(n), 256, 0, s>>>(roff, ucnt, uoff, n, uent, urow);
        count_launches(3);
    }
    if (n_entries) {
        cudaMemsetAsync(c_ex, 0, n_entries * 4, s);
        cudaMemsetAsync(c_blk, 0, n_entries * 4, s);
        cudaMemsetAsync(c_vtx, 0, n_entries * 4, s);
        if (n_upper)
            k_circles<false><<<blocks_for(n_upper, 128), 128, 0, s>>>(
                sph, n, roff, items, n_upper, uent, urow, nullptr, c_ex, c_blk, c_vtx, exposed, nullptr, nullptr,
                nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, decline);
        launch_scan(c_ex, uint32_t(n_entries), o_circ, nullptr, tiles_e, total, s);
        launch_scan(c_blk, uint32_t(n_entries), o_blk, nullptr, tiles_e, total + 1, s);
        launch_scan(c_vtx, uint32_t(n_entries), o_vtx, nullptr, tiles_e, total + 2, s);
        count_launches(3);
    } else {
        cudaMemsetAsync(total, 0, 24, s);
    }
    uint32_t h_decline = 0;
    if (cudaMemcpyAsync(h_tot, total, 24, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&h_decline, decline, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail("circles");
    if (h_decline) {
        if (msg)
            *msg = (h_decline & DECLINE_ANGLE) ? "a circle's exposure is within the device's atan2 error of its threshold"
                                               : "a circle has more candidate blockers than the device keeps";
        out.release();
        return 1;
    }
    const size_t nc = size_t(h_tot[0]), ncb = size_t(h_tot[1]), nv = size_t(h_tot[2]);
    if (ncb >= (size_t(1) << 32) || nv >= (size_t(1) << 32)) return fail("arrangement too large for the device");
    double* circ = static_cast<double*>(X.alloc(nc * 96, true));
    uint32_t* ij = static_cast<uint32_t*>(X.alloc(nc * 8, true));
    uint32_t* cb_off = static_cast<uint32_t*>(X.alloc((nc + 1) * 4, true));
    uint32_t* cb_items = static_cast<uint32_t*>(X.alloc(ncb * 4, true));
    double4* vert = static_cast<double4*>(X.alloc(nv * 32, true));
    uint32_t* vatoms = static_cast<uint32_t*>(X.alloc(nv * 12, true));
    uint32_t* keep_len = static_cast<uint32_t*>(X.alloc(n * 4, false));
    uint32_t* nb_off = static_cast<uint32_t*>(X.alloc((n + 1) * 4, true));
    if (!X.ok) return fail("device memory");
    if (nc) {
        uint32_t* xlist = static_cast<uint32_t*>(X.alloc(nc * 4, false));
        if (!X.ok) return fail("device memory");
        k_exposed_list<<<blocks_for(n_upper), 256, 0, s>>>(uent, n_upper, c_ex, o_circ, xlist);
        k_circles<true><<<blocks_for(nc, 128), 128, 0, s>>>(sph, n, roff, items, nc, uent, urow, xlist, c_ex, c_blk,
                                                          c_vtx, exposed, o_circ, o_blk, o_vtx, circ, ij, cb_off,
                                                          cb_items, vert, vatoms, decline);
        count_launches(1);
    }
    k_put<<<1, 32, 0, s>>>(cb_off + nc, uint32_t(ncb));
    // Statuses and the rows of exposed spheres.
    if (n) {
        k_status<<<blocks_for(n), 256, 0, s>>>(contained, exposed, roff, n, status, keep_len);
        launch_scan(keep_len, uint32_t(n), nb_off, nullptr, tiles, total, s);
    } else {
        cudaMemsetAsync(total, 0, 8, s);
    }
    unsigned long long h_nb = 0;
    if (cudaMemcpyAsync(&h_nb, total, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return fail("status");
    k_put<<<1, 32, 0, s>>>(nb_off + n, uint32_t(h_nb));
    uint32_t* nb_items = static_cast<uint32_t*>(X.alloc(size_t(h_nb) * 4, true));
    if (!X.ok) return fail("device memory");
    if (n) k_keep_rows<<<blocks_for(n), 256, 0, s>>>(roff, items, keep_len, nb_off, n, nb_items);
    count_launches(7);
    A.nb_off = nb_off, A.nb_items = nb_items;
    A.nc = uint32_t(nc), A.nv = uint32_t(nv);
    A.flags = DARR_ROWS_SORTED;  // rows sorted in k_rows, blockers listed in row order
    A.circ = circ, A.cb_off = cb_off, A.cb_items = cb_items, A.vert = vert;
    out.circle_ij = ij, out.vertex_atoms = vatoms;
    out.n_circles = nc, out.n_vertices = nv, out.nb_items = size_t(h_nb), out.cb_items = ncb;
    // Grids of circle centres and vertices, rho_max, extent.
    if (!build_grid(X, circ, 12, nc, cell, part, A.gc)) return fail("circle grid");
    if (!build_grid(X, reinterpret_cast<const double*>(vert), 4, nv, cell, part, A.gv)) return fail("vertex grid");
    A.rho_max = 0.0;
    if (nc) {
        k_box_points<<<RED_BLOCKS, 256, 0, s>>>(circ, 12, nc, 9, part);
        count_launches(1);
        Box bc;
        if (!reduce_box(X, part, bc)) return fail("reduction");
        A.rho_max = bc.mx;
    }
    if (n) {
        const double ex = out.hi[0] - out.lo[0], ey = out.hi[1] - out.lo[1], ez = out.hi[2] - out.lo[2];
        out.extent = std::sqrt(ex * ex + ey * ey + ez * ez) + 4.0 * max_expanded + 4.0 * probe + 1.0;
    }
    // Containment count.
    std::vector<uint32_t> hc(n);
    if (n && (cudaMemcpyAsync(hc.data(), contained, n * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
              cudaStreamSynchronize(s) != cudaSuccess))
        return fail("containment");
    out.n_contained = 0;
    for (uint32_t c : hc) out.n_contained += c;
    if (cudaGetLastError() != cudaSuccess) return fail("kernel launch");
    return 0;
}

bool arrangement_to_host(const DevArrangement& D, smbh::Arrangement& H) {
    const DArr& A = D.A;
    const size_t n = D.n, nc = D.n_circles, nv = D.n_vertices;
    H = smbh::Arrangement();
    H.probe = A.probe;
    H.n = n;
    H.n_contained = D.n_contained;
    H.max_expanded = A.max_expanded;
    H.rho_max = A.rho_max;
    H.extent = D.extent;
    std::vector<double> sph(4 * n), circ(12 * nc), vert(4 * nv);
    H.radius.resize(n), H.orig.resize(n), H.status.resize(n), H.nb_off.resize(n + 1), H.nb_items.resize(D.nb_items);
    H.circle_ij.resize(2 * nc), H.cb_off.resize(nc + 1), H.cb_items.resize(D.cb_items), H.vertex_atoms.resize(3 * nv);
    auto get = [](void* dst, const void* src, size_t bytes) {
        return !bytes || cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
    };
    bool ok = get(sph.data(), A.sph, n * 32) && get(H.radius.data(), A.rvdw, n * 8) &&
              get(H.orig.data(), D.orig, n * 4) && get(H.status.data(), A.status, n * 4) &&
              get(H.nb_off.data(), A.nb_off, (n + 1) * 4) && get(H.nb_items.data(), A.nb_items, D.nb_items * 4) &&
              get(circ.data(), A.circ, nc * 96) && get(H.circle_ij.data(), D.circle_ij, nc * 8) &&
              get(H.cb_off.data(), A.cb_off, (nc + 1) * 4) && get(H.cb_items.data(), A.cb_items, D.cb_items * 4) &&
              get(vert.data(), A.vert, nv * 32) && get(H.vertex_atoms.data(), D.vertex_atoms, nv * 12);
    if (!ok) return false;
    H.center.resize(3 * n), H.expanded.resize(n);
    for (size_t i = 0; i < n; i++)
        H.center[3 * i] = sph[4 * i], H.center[3 * i + 1] = sph[4 * i + 1], H.center[3 * i + 2] = sph[4 * i + 2],
        H.expanded[i] = sph[4 * i + 3];
    H.circle.resize(10 * nc);
    for (size_t c = 0; c < nc; c++)
        for (int k = 0; k < 10; k++) H.circle[10 * c + k] = circ[12 * c + k];
    H.vertex.resize(3 * nv);
    for (size_t v = 0; v < nv; v++)
        for (int k = 0; k < 3; k++) H.vertex[3 * v + k] = vert[4 * v + k];
    const DGrid* g[3] = {&A.gs, &A.gc, &A.gv};
    smbh::Grid* h[3] = {&H.cells, &H.circle_cells, &H.vertex_cells};
    const size_t cnt[3] = {n, nc, nv};
    for (int k = 0; k < 3; k++) {
        smbh::Grid& G = *h[k];
        G.origin[0] = g[k]->ox, G.origin[1] = g[k]->oy, G.origin[2] = g[k]->oz, G.cell = g[k]->cell;
        G.dims[0] = g[k]->dx, G.dims[1] = g[k]->dy, G.dims[2] = g[k]->dz;
        const size_t cells = size_t(G.dims[0]) * G.dims[1] * G.dims[2];
        G.starts.resize(cells + 1);
        G.items.resize(cnt[k]);
        if (!get(G.starts.data(), g[k]->starts, (cells + 1) * 4) || !get(G.items.data(), g[k]->items, cnt[k] * 4))
            return false;
    }
    return true;
}

}  // namespace smb
