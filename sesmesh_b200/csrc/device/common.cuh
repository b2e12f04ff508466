// Device-side data layout and the f64 geometry shared by the kernels.
//
// Every f64 and f32 expression here keeps the operation order of the
// sesmesh CPU code it restates (left to right, no FMA: the library is built
// with -fmad=false -prec-div=true -prec-sqrt=true -ftz=false), so brick
// classes, candidate lists and sample values equal the CPU back end's bit
// for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace smb {

constexpr double CLASSIFY_EPS = 2e-3;      // field/lattice.rs:20
constexpr double GEOM_EPS = 1e-9;          // geom/arrangement.rs:26
constexpr float INSIDE_TOL = 2e-5f;        // field/kernel.rs:40
constexpr int64_t KEY_BIAS = int64_t(1) << 20;  // field/lattice.rs:15
constexpr double PRUNE_MARGIN = 1e-3;      // f32 safety margin of the sampler's candidate pruning

constexpr uint32_t ST_SAMPLE = 0, ST_OUT = 1, ST_IN = 2;
constexpr uint32_t STATUS_EXPOSED = 0, STATUS_BURIED = 1, STATUS_CONTAINED = 2;

// Record words per sub-block (see include/sesmesh_b200.h).
constexpr int REC_WORDS = 12;
enum RecWord {
    R_STATE = 0, R_IDS = 1, R_INSIDE = 2, R_NEAR = 3, R_S = 4, R_C = 5, R_V = 6, R_SBLK = 7, R_CBLK = 8,
    R_PACK = 9, R_PACKLEN = 10, R_FLAGS = 11
};
constexpr uint32_t REC_OVERFLOW = 1;

// A cell grid over points (geom/cells.rs:12): items of cell c are
// items[starts[c]..starts[c+1]], cells x-fastest.
struct DGrid {
    double ox, oy, oz, cell;
    uint32_t dx, dy, dz, pad;
    const uint32_t* starts;
    const uint32_t* items;
};

// DArr::pad flags.
constexpr uint32_t DARR_ROWS_SORTED = 1;  // every neighbour row and circle-blocker list ascends
// A sphere field (SAS or vdW, field/mod.rs:33-41): min(|x - c| - R) over the
// spheres, no circles or vertices, every sphere not contained exposed.
constexpr uint32_t DARR_SPHERES = 2;

// The resident arrangement, internal (Morton) sphere order.
struct DArr {
    uint32_t n, nc, nv, flags;  // DARR_* bits
    const double4* sph;      // centre x, y, z, expanded radius R
    const double* rvdw;      // vdW radius r
    const uint32_t* status;  // STATUS_*
    const uint32_t* nb_off;  // class-S blockers: neighbour CSR of exposed spheres
    const uint32_t* nb_items;
    const double* circ;      // 12 per circle: centre xyz, axis xyz, e1 xyz, radius, 0, 0
    const uint32_t* cb_off;  // circle blocker CSR
    const uint32_t* cb_items;
    const double4* vert;     // SAS vertex x, y, z, 0
    DGrid gs, gc, gv;
    double max_expanded, rho_max, probe;
};

// Lattice and sampling constants (field/lattice.rs:26-45, kernel.rs:204-271).
struct DLat {
    double h;
    double fx, fy, fz;       // frame origin (a lattice point), f64
    long long frame[3];      // lattice index of the frame origin
    double band;             // sqrt(3) h 1.01
    double rho_sub;          // 0.5 sqrt(3) sub h
    double rho_brick;        // 0.5 sqrt(3) b h
    float h32, band32, probe32, cutoff2;
    int b, sub, spb, kind;   // brick edge, sub-block edge, samples per brick; 1: a sphere field
};

// geom/cells.rs:91-104 on one axis.
__device__ __forceinline__ uint32_t cell_coord(double p, double o, double cell, uint32_t dim) {
    double c = floor((p - o) / cell);
    if (!(c > 0.0)) return 0;
    if (c >= double(dim - 1)) return dim - 1;
    return uint32_t(c);
}

struct CellBox {
    uint32_t x0, x1, y0, y1, z0, z1;
};

// The cells overlapping the cube of half-size r around (x, y, z)
// (geom/cells.rs:113-130: coord(center - r) .. coord(center + r)).
__device__ __forceinline__ CellBox cell_box(const DGrid& g, double x, double y, double z, double r) {
    CellBox b;
    b.x0 = cell_coord(x - r, g.ox, g.cell, g.dx);
    b.y0 = cell_coord(y - r, g.oy, g.cell, g.dy);
    b.z0 = cell_coord(z - r, g.oz, g.cell, g.dz);
    b.x1 = cell_coord(x + r, g.ox, g.cell, g.dx);
    b.y1 = cell_coord(y + r, g.oy, g.cell, g.dy);
    b.z1 = cell_coord(z + r, g.oz, g.cell, g.dz);
    return b;
}

// |a - b| as Vec3::dist computes it (geom/vec.rs:27-55).
__device__ __forceinline__ double dist3(double ax, double ay, double az, double bx, double by, double bz) {
    double dx = ax - bx, dy = ay - by, dz = az - bz;
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Comparisons of a correctly rounded square root with a threshold T >= 0,
// decided from the square when it is clear of T^2: t2 = fl(T T) is within
// 2^-53 of T^2, so d2 >= fl(t2 (1 + 2^-49)) gives sqrt(d2) >= T (1 + 6 2^-53)
// and fl(sqrt(d2)) > T; d2 <= fl(t2 (1 - 2^-49)) with t2 > 0 gives
// fl(sqrt(d2)) < T.  Only in between is the square root taken.  The results
// are those of fl(sqrt(d2)) >= T and fl(sqrt(d2)) < T exactly (NaN: false
// for both).
__device__ __forceinline__ bool sqrt_ge(double d2, double T) {
    const double t2 = T * T;
    if (d2 >= t2 * (1.0 + 0x1p-49)) return true;
    if (d2 <= t2 * (1.0 - 0x1p-49)) return false;
    return sqrt(d2) >= T;
}
__device__ __forceinline__ bool sqrt_lt(double d2, double T) {
    const double t2 = T * T;
    if (d2 <= t2 * (1.0 - 0x1p-49) && t2 > 0.0) return true;
    if (d2 >= t2 * (1.0 + 0x1p-49)) return false;
    return sqrt(d2) < T;
}
__device__ __forceinline__ double sq3(double ax, double ay, double az, double bx, double by, double bz) {
    const double dx = ax - bx, dy = ay - by, dz = az - bz;
    return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The items of a box's rows as one sequence in the rows' order (z, then y,
// then the row's cells from x0 to x1), visited by a warp in chunks of 32
// consecutive items: f(valid, item) on every lane, lane l holding the
// chunk's l-th item (valid false past the end).  The row bounds of 32 rows
// are loaded at once and the rows' items flattened by a prefix sum, so a
// box costs a dependent load round per 32 rows and one per 32 items rather
// than one per row.
template <class F>
__device__ __forceinline__ void warp_box_items(const DGrid& g, const CellBox& bx, int lane, F&& f) {
    const uint32_t ny = bx.y1 - bx.y0 + 1, nrows = ny * (bx.z1 - bx.z0 + 1);
    for (uint32_t r0 = 0; r0 < nrows; r0 += 32) {
        const uint32_t rr = r0 + uint32_t(lane);
        uint32_t a = 0, cnt = 0;
        if (rr < nrows) {
            const size_t row = (size_t(bx.z0 + rr / ny) * g.dy + (bx.y0 + rr % ny)) * g.dx;
            a = g.starts[row + bx.x0];
            cnt = g.starts[row + bx.x1 + 1] - a;
        }
        uint32_t inc = cnt;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, inc, 31), excl = inc - cnt;
        for (uint32_t b = 0; b < total; b += 32) {
            const uint32_t t = b + uint32_t(lane);
            // The row holding item t: the last lane q with excl_q <= t
            // (excl ascends; such a row is not empty while t < total).
            int q = 0;
#pragma unroll
            for (int step = 16; step; step >>= 1) {
                const uint32_t e = __shfl_sync(0xffffffffu, excl, q + step);
                if (e <= t) q += step;
            }
            const uint32_t aq = __shfl_sync(0xffffffffu, a, q), eq = __shfl_sync(0xffffffffu, excl, q);
            const bool valid = t < total;
            f(valid, valid ? g.items[aq + (t - eq)] : 0u);
        }
    }
}

// Every item of the box visited once, by some lane of the warp.
template <class F>
__device__ __forceinline__ void warp_for_near(const DGrid& g, double x, double y, double z, double r, int lane, F&& f) {
    warp_box_items(g, cell_box(g, x, y, z, r), lane, [&](bool valid, uint32_t k) {
        if (valid) f(k);
    });
}

// No sphere of items[p .. e) blocks q (each centre at least R - GEOM_EPS
// from q), in list order, stopping at the first that does; two spheres'
// loads in flight at a time (the tests have no side effects, so reading one
// past the first blocker changes nothing).
__device__ __forceinline__ bool unblocked(const DArr& A, const uint32_t* items, uint32_t p, uint32_t e, double qx,
                                          double qy, double qz) {
    for (; p + 2 <= e; p += 2) {
        const uint32_t i0 = items[p], i1 = items[p + 1];
        const double4 k0 = A.sph[i0], k1 = A.sph[i1];
        if (!sqrt_ge(sq3(qx, qy, qz, k0.x, k0.y, k0.z), k0.w - GEOM_EPS)) return false;
        if (!sqrt_ge(sq3(qx, qy, qz, k1.x, k1.y, k1.z), k1.w - GEOM_EPS)) return false;
    }
    if (p < e) {
        const double4 k = A.sph[items[p]];
        if (!sqrt_ge(sq3(qx, qy, qz, k.x, k.y, k.z), k.w - GEOM_EPS)) return false;
    }
    return true;
}

// SesField::try_sphere_with (field/point.rs:422-444): the candidate's
// distance if its radial projection is unblocked and below best, else best.
// Threshold tests on distances go through sqrt_ge / sqrt_lt (the root only
// where the square leaves them open), with the results of the plain
// comparisons.
__device__ __forceinline__ double try_sphere(const DArr& A, double x, double y, double z, uint32_t i, double best) {
    double4 c = A.sph[i];
    double vx = x - c.x, vy = y - c.y, vz = z - c.z;
    double len = sqrt(vx * vx + vy * vy + vz * vz);
    double lb = fabs(len - c.w);
    if (lb >= best || len < 1e-12) return best;
    double s = c.w / len;
    double qx = c.x + vx * s, qy = c.y + vy * s, qz = c.z + vz * s;
    return unblocked(A, A.nb_items, A.nb_off[i], A.nb_off[i + 1], qx, qy, qz) ? lb : best;
}

// SesField::try_circle_with (field/point.rs:452-476).
__device__ __forceinline__ double try_circle(const DArr& A, double x, double y, double z, uint32_t ci, double best) {
    const double* c = A.circ + 12 * size_t(ci);
    double yx = x - c[0], yy = y - c[1], yz = z - c[2];
    double along = yx * c[3] + yy * c[4] + yz * c[5];
    const double a2 = along * along;
    double wx = yx - c[3] * along, wy = yy - c[4] * along, wz = yz - c[5] * along;
    double wl = sqrt(wx * wx + wy * wy + wz * wz);
    double t = wl - c[9];
    const double dist2 = a2 + t * t;
    if (sqrt_ge(dist2, best)) return best;
    double dist = sqrt(dist2);
    double dx, dy, dz;
    if (wl > 1e-12) {
        dx = wx / wl, dy = wy / wl, dz = wz / wl;
    } else {
        dx = c[6], dy = c[7], dz = c[8];
    }
    double qx = c[0] + dx * c[9], qy = c[1] + dy * c[9], qz = c[2] + dz * c[9];
    return unblocked(A, A.cb_items, A.cb_off[ci], A.cb_off[ci + 1], qx, qy, qz) ? dist : best;
}

// Distance from (x, y, z) to the circle ci as gather_ses / gather_local
// compute it for the reach test (field/kernel.rs:714-722).
__device__ __forceinline__ double circle_reach_dist(const DArr& A, double x, double y, double z, uint32_t ci) {
    const double* c = A.circ + 12 * size_t(ci);
    double yx = x - c[0], yy = y - c[1], yz = z - c[2];
    double along = yx * c[3] + yy * c[4] + yz * c[5];
    double wx = yx - c[3] * along, wy = yy - c[4] * along, wz = yz - c[5] * along;
    double wl = sqrt(wx * wx + wy * wy + wz * wz);
    return sqrt(along * along + (wl - c[9]) * (wl - c[9]));
}

// circle_reach_dist, or +infinity where the distance to the circle's plane
// alone puts it above T: the distance squared fl(a2 + t t) is at least a2,
// and a2 >= fl(T T (1 + 2^-49)) gives fl(sqrt(a2)) > T (sqrt_ge's margin),
// so the distance exceeds T too and every test against a threshold up to
// T comes out as with it.
__device__ __forceinline__ double circle_reach_dist_above(const DArr& A, double x, double y, double z, uint32_t ci,
                                                          double T) {
    const double* c = A.circ + 12 * size_t(ci);
    double yx = x - c[0], yy = y - c[1], yz = z - c[2];
    double along = yx * c[3] + yy * c[4] + yz * c[5];
    const double a2 = along * along;
    if (a2 >= T * T * (1.0 + 0x1p-49)) return __longlong_as_double(0x7ff0000000000000LL);
    double wx = yx - c[3] * along, wy = yy - c[4] * along, wz = yz - c[5] * along;
    double wl = sqrt(wx * wx + wy * wy + wz * wz);
    return sqrt(a2 + (wl - c[9]) * (wl - c[9]));
}

// SesField::ses_eval distance (field/point.rs:385-411), one warp.  The result
// is min(cutoff, min over unblocked candidates), which does not depend on the
// visiting order, so lanes keep partial minima that are merged at the end.
// inside_known: 1 or 0 when the caller's scan already settled whether some
// sphere contains the point (it covered every sphere that can), -1 to scan.
__device__ inline double ses_eval_warp(const DArr& A, double x, double y, double z, double cutoff, int lane,
                                       int inside_known = -1) {
    bool inside = inside_known > 0;
    if (inside_known < 0)
        warp_for_near(A.gs, x, y, z, A.max_expanded, lane, [&](uint32_t k) {
            if (!inside && A.status[k] != STATUS_CONTAINED) {
                double4 c = A.sph[k];
                if (sqrt_lt(sq3(x, y, z, c.x, c.y, c.z), c.w)) inside = true;
            }
        });
    if (!__any_sync(0xffffffffu, inside)) return 0.0;
    double best = cutoff;
    warp_for_near(A.gs, x, y, z, cutoff + A.max_expanded, lane, [&](uint32_t i) {
        if (A.status[i] == STATUS_EXPOSED) best = try_sphere(A, x, y, z, i, best);
    });
    best = warp_min(best);
    warp_for_near(A.gc, x, y, z, cutoff + A.rho_max, lane, [&](uint32_t ci) { best = try_circle(A, x, y, z, ci, best); });
    warp_for_near(A.gv, x, y, z, cutoff, lane, [&](uint32_t vi) {
        double4 p = A.vert[vi];
        const double d2 = sq3(x, y, z, p.x, p.y, p.z);
        if (sqrt_lt(d2, best)) best = sqrt(d2);
    });
    return warp_min(best);
}

// lattice::uniform_sign (field/lattice.rs:190-227), one warp: 1 uniformly
// outside, 0 uniformly inside, -1 the surface may pass.
// A sphere with fl(|x - c|) - R clear of margin by a factor 2^-40 (decided
// from the square, as sqrt_ge does) enters neither minimum's tests: its
// terms are above +margin (R >= r), so s_sas >= margin, s_vdw <= -margin and
// the sphere field's s_sas > margin and s_sas < -margin come out as with it;
// the square root is taken for the others alone.
__device__ inline int uniform_sign_warp(const DArr& A, double x, double y, double z, double rho, int lane) {
    double margin = rho + CLASSIFY_EPS;
    double s_sas = __longlong_as_double(0x7ff0000000000000LL), s_vdw = s_sas;
    // The same scan answers ses_eval's inside test (some sphere with
    // |x - c| < R: every such sphere lies in this box and is not skipped).
    bool inside = false;
    warp_for_near(A.gs, x, y, z, margin + A.max_expanded, lane, [&](uint32_t k) {
        if (A.status[k] != STATUS_CONTAINED) {
            double4 c = A.sph[k];
            const double d2 = sq3(x, y, z, c.x, c.y, c.z);
            const double T = c.w + margin;
            if (d2 >= T * T * (1.0 + 0x1p-38)) return;
            double d = sqrt(d2);
            inside = inside || d < c.w;
            s_sas = fmin(s_sas, d - c.w);
            s_vdw = fmin(s_vdw, d - A.rvdw[k]);
        }
    });
    s_sas = warp_min(s_sas);
    s_vdw = warp_min(s_vdw);
    if (A.flags & DARR_SPHERES) return s_sas > margin ? 1 : (s_sas < -margin ? 0 : -1);  // lattice.rs:213-215
    if (s_sas >= margin) return 1;
    if (s_vdw <= -margin) return 0;
    double cutoff = A.probe + margin + CLASSIFY_EPS;
    double v = A.probe - ses_eval_warp(A, x, y, z, cutoff, lane, __any_sync(0xffffffffu, inside) ? 1 : 0);
    if (v > margin) return 1;
    if (v < -margin) return 0;
    return -1;
}

}  // namespace smb
