// Host stages of sesmesh's mesh stage (exact f64 refinement, assembly,
// measurement, OBJ).  Restates crates/sesmesh/src/field/point.rs:496-738,
// crates/sesmesh/src/mesh/{extract.rs,mod.rs,post.rs} and
// crates/sesmesh/src/export/{obj.rs,fmt.rs}.
#include "mesher.hpp"

#include <algorithm>
#include <atomic>
#include <cstring>

namespace smbh {

namespace {
constexpr double EPS = 1e-9;
constexpr int MAX_ITER = 8;
constexpr int MAX_BISECT = 64;
constexpr double TOL = 1e-5;
constexpr uint32_t CODE_SHIFT = 28, ID_MASK = (1u << 28) - 1;
constexpr uint32_t FEAT_SHIFT = 29, EDGE_CONVERGED = 1u << 31;

inline double clamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

void nearest_first(std::vector<std::pair<double, uint32_t>>& v) {
    std::sort(v.begin(), v.end(), [](const auto& a, const auto& b) {
        return a.first < b.first || (a.first == b.first && a.second < b.second);
    });
}

struct Best {
    double d;
    V3 q;
    Feature f;
};

// try_sphere_with (point.rs:422-444)
inline void try_sphere(const Arrangement& A, const V3& x, uint32_t i, const uint32_t* b0, const uint32_t* b1, Best& best) {
    V3 c = A.c(i), v = x - c;
    double len = v.norm();
    double lb = std::fabs(len - A.expanded[i]);
    if (lb >= best.d || len < 1e-12) return;
    V3 q = c + v * (A.expanded[i] / len);
    for (const uint32_t* k = b0; k != b1; k++)
        if (!(q.dist(A.c(*k)) >= A.expanded[*k] - EPS)) return;
    best = Best{lb, q, Feature{F_SPHERE, i}};
}

// try_circle_with (point.rs:452-476)
inline void try_circle(const Arrangement& A, const V3& x, uint32_t ci, const uint32_t* b0, const uint32_t* b1, Best& best) {
    const double* c = &A.circle[10 * size_t(ci)];
    V3 m = V3::at(c), u = V3::at(c + 3);
    V3 y = x - m;
    double along = y.dot(u);
    V3 w = y - u * along;
    double wl = w.norm();
    double dist = std::sqrt(along * along + (wl - c[9]) * (wl - c[9]));
    if (dist >= best.d) return;
    V3 dir = wl > 1e-12 ? w / wl : V3::at(c + 6);
    V3 q = m + dir * c[9];
    for (const uint32_t* k = b0; k != b1; k++)
        if (!(q.dist(A.c(*k)) >= A.expanded[*k] - EPS)) return;
    best = Best{dist, q, Feature{F_CIRCLE, ci}};
}

// sphere_eval (point.rs:742-757)
std::pair<double, int64_t> sphere_eval(const Arrangement& A, const V3& x, double cutoff) {
    std::pair<double, int64_t> best{cutoff, -1};
    A.cells.near(x, cutoff + A.max_expanded, [&](uint32_t k) {
        if (A.status[k] == CONTAINED) return;
        double v = x.dist(A.c(k)) - A.expanded[k];
        if (v < best.first) best = {v, int64_t(k)};
    });
    return best;
}

// extract::attributes (extract.rs:553-597), SES.
void attributes(const Arrangement& A, const MeshParams& P, const V3& v, const NearEval& e, const V3& outward,
                V3& normal, uint8_t& patch, uint32_t& atom) {
    auto unit = [&](const V3& w) {
        double len = w.norm();
        return len > 1e-9 ? w / len : outward;
    };
    auto nearest = [&](const uint32_t* ids, int k) {
        double best = INFINITY;
        uint32_t bi = ids[0];
        for (int q = 0; q < k; q++) {
            double d = v.dist(A.c(ids[q])) - A.radius[ids[q]];
            if (d < best) best = d, bi = ids[q];
        }
        return A.orig[bi];
    };
    if (A.kind != 0 && e.feature.kind == F_SPHERE) {  // extract.rs:583-587
        normal = unit(v - A.c(e.feature.id)), patch = 0, atom = A.orig[e.feature.id];
        return;
    }
    const uint32_t kind = A.kind != 0 ? uint32_t(F_BEYOND) : uint32_t(e.feature.kind);
    switch (kind) {
        case F_SPHERE:
            normal = unit(e.closest - v), patch = 0, atom = A.orig[e.feature.id];
            return;
        case F_CIRCLE:
            normal = unit(e.closest - v), patch = 1, atom = nearest(&A.circle_ij[2 * size_t(e.feature.id)], 2);
            return;
        case F_VERTEX:
            normal = unit(e.closest - v), patch = 2, atom = nearest(&A.vertex_atoms[3 * size_t(e.feature.id)], 3);
            return;
        default: {
            auto r = sphere_eval(A, v, A.probe + P.band + 8.0);
            normal = outward, patch = 0, atom = r.second < 0 ? 0 : A.orig[size_t(r.second)];
        }
    }
}

struct Vertex {
    V3 pos, normal;
    uint8_t patch;
    uint32_t atom;
    double t;  // root parameter before the edge clamp
};

// extract::vertex (extract.rs:425-535), exact mode.
Vertex refine_edge(const Arrangement& A, const MeshParams& P, const V3& pa, const V3& pb, double fa, double fb,
                   const Local& local, uint32_t& evals) {
    const V3 d = pb - pa;
    double t = clamp(fa / (fa - fb), 0.0, 1.0);
    NearEval last{};
    bool have = false;
    double t0 = 0.0, g0 = fa, t1 = 1.0, g1 = fb;
    int side = 0;
    bool converged = false;
    for (int it = 0; it < MAX_ITER; it++) {
        const V3 x = pa + d * t;
        NearEval e = eval_local(A, x, P.band, local);
        evals++;
        last = e, have = true;
        double g = e.value;
        if (std::fabs(g) <= TOL) {
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
        double slope = 0.0;  // gradient (extract.rs:539-549) along the edge
        if (e.feature.kind != F_SOLVENT && e.feature.kind != F_BEYOND) {
            V3 w = A.kind != 0 ? x - A.c(e.feature.id) : e.closest - x;
            double len = w.norm();
            if (len > 1e-12) slope = (w / len).dot(d);
        }
        double newton = t - g / slope;
        if (std::fabs(slope) > 1e-3 * d.norm() && newton > t0 && newton < t1) {
            t = newton;
        } else {
            double s = (t0 * g1 - t1 * g0) / (g1 - g0);
            t = (std::isfinite(s) && s > t0 && s < t1) ? s : 0.5 * (t0 + t1);
        }
    }
    if (!converged) {
        double len = d.norm();
        bool neg0 = g0 < 0.0;
        for (int it = 0; it < MAX_BISECT; it++) {
            t = 0.5 * (t0 + t1);
            NearEval e = eval_local(A, pa + d * t, P.band, local);
            evals++;
            last = e, have = true;
            if (std::fabs(e.value) <= TOL || (t1 - t0) * len <= 2.0 * TOL) break;
            if ((e.value < 0.0) == neg0) t0 = t;
            else t1 = t;
        }
    }
    Vertex out;
    out.t = t;
    out.pos = pa + d * clamp(t, P.t_min, 1.0 - P.t_min);
    if (!have) {
        evals++;
        last = eval_local(A, out.pos, P.band, local);
    }
    V3 outward = (fa < 0.0 ? d : d * -1.0).unit();
    attributes(A, P, out.pos, last, outward, out.normal, out.patch, out.atom);
    return out;
}

// The lattice geometry of one brick edge.
struct EdgeGeom {
    V3 pa, pb;
    int sb;
};

inline EdgeGeom edge_geom(const MeshParams& P, const int32_t* key, uint32_t e) {
    const int b = P.b;
    uint32_t cell = e / 3, axis = e % 3;
    int64_t x = cell % b, y = (cell / b) % b, z = cell / (b * b);
    int64_t ia[3] = {int64_t(key[0]) * b + x, int64_t(key[1]) * b + y, int64_t(key[2]) * b + z};
    EdgeGeom g;
    g.pa = V3(double(ia[0]) * P.h, double(ia[1]) * P.h, double(ia[2]) * P.h);
    ia[axis] += 1;
    g.pb = V3(double(ia[0]) * P.h, double(ia[1]) * P.h, double(ia[2]) * P.h);
    g.sb = int(std::min<int64_t>(x / P.sub, 1) + 2 * std::min<int64_t>(y / P.sub, 1) + 4 * std::min<int64_t>(z / P.sub, 1));
    return g;
}

// gather_local ball of a sub-block (extract.rs:165-177, 195-206).
inline void local_of(const Arrangement& A, const MeshParams& P, const int32_t* key, int sb, Local& l) {
    const double h = P.h, sub = double(P.sub);
    V3 base(double(int64_t(key[0]) * P.b) * h, double(int64_t(key[1]) * P.b) * h, double(int64_t(key[2]) * P.b) * h);
    V3 c = base + V3(double((sb & 1) * P.sub) + 0.5 * sub, double(((sb >> 1) & 1) * P.sub) + 0.5 * sub,
                     double((sb >> 2) * P.sub) + 0.5 * sub) * h;
    double rho = 0.5 * std::sqrt(3.0) * sub * h * (1.0 + 1e-9) + 1e-9;
    gather_local(A, c, rho, P.band, l);
}

void put(MeshOut& out, size_t at, const Vertex& v) {
    out.positions[at] = {float(v.pos.x), float(v.pos.y), float(v.pos.z)};
    out.normals[at] = {float(v.normal.x), float(v.normal.y), float(v.normal.z)};
    out.atoms[at] = v.atom;
    out.patches[at] = v.patch;
    out.t[at] = float(v.t);
}

void resize(MeshOut& out, size_t nv, size_t nb) {
    out.positions.resize(nv);
    out.normals.resize(nv);
    out.atoms.resize(nv);
    out.patches.resize(nv);
    out.t.resize(nv);
    out.evals.assign(nb, 0);
    out.cpu_refined.assign(nb, 0);
}

}  // namespace

// point.rs:496-582 (SES)
// Pruning: every point evaluated with a ball's candidates lies in the ball,
// and |d - R|, the circle distance and the vertex distance are 1-Lipschitz,
// so a candidate whose centre value minus the radius exceeds the current best
// by more than f64 rounding cannot pass its test; the lists are sorted by
// that centre value, so evaluation stops at the first such candidate.  The
// result (value, feature, closest point) is unchanged.
constexpr double PRUNE_MARGIN = 1e-9;

void gather_local(const Arrangement& A, const V3& b, double rho, double band, Local& out) {
    out.inside.clear(), out.near.clear(), out.spheres.clear(), out.s_blk.clear(), out.circles.clear();
    out.c_blk.clear(), out.vertices.clear(), out.order.clear();
    out.s_key.clear(), out.c_key.clear(), out.v_key.clear();
    out.s_off.assign(1, 0), out.c_off.assign(1, 0);
    if (A.kind != 0) {  // point.rs:566-579: sphere fields, by (centre value, index)
        const double reach = band + rho;
        A.cells.near(b, reach + A.max_expanded, [&](uint32_t k) {
            if (A.status[k] != CONTAINED && b.dist(A.c(k)) - A.expanded[k] < reach)
                out.order.push_back({b.dist(A.c(k)) - A.expanded[k], k});
        });
        nearest_first(out.order);
        for (auto& o : out.order) out.inside.push_back(o.second);
        out.order.clear();
        return;
    }
    const double reach = A.probe + band + rho;
    A.cells.near(b, reach + A.max_expanded, [&](uint32_t k) {
        if (A.status[k] == CONTAINED) return;
        double d = b.dist(A.c(k));
        if (d < A.expanded[k] + reach) out.near.push_back(k);
        if (d < A.expanded[k] + rho) out.inside.push_back(k);
        double lb = std::fabs(d - A.expanded[k]);
        if (A.status[k] == EXPOSED && lb <= reach) out.order.push_back({lb, k});
    });
    std::sort(out.near.begin(), out.near.end());
    nearest_first(out.order);
    auto keep_near = [&](const uint32_t* r0, const uint32_t* r1, std::vector<uint32_t>& dst) {
        for (const uint32_t* p = r0; p != r1; p++)
            if (std::binary_search(out.near.begin(), out.near.end(), *p)) dst.push_back(*p);
    };
    for (auto& o : out.order) {
        out.spheres.push_back(o.second);
        out.s_key.push_back(o.first - rho - PRUNE_MARGIN);
        keep_near(A.nb_items.data() + A.nb_off[o.second], A.nb_items.data() + A.nb_off[o.second + 1], out.s_blk);
        out.s_off.push_back(uint32_t(out.s_blk.size()));
    }
    out.order.clear();
    A.circle_cells.near(b, reach + A.rho_max, [&](uint32_t ci) {
        const double* c = &A.circle[10 * size_t(ci)];
        V3 y = b - V3::at(c), u = V3::at(c + 3);
        double along = y.dot(u);
        double wl = (y - u * along).norm();
        double dist = std::sqrt(along * along + (wl - c[9]) * (wl - c[9]));
        if (dist <= reach) out.order.push_back({dist, ci});
    });
    nearest_first(out.order);
    for (auto& o : out.order) {
        out.circles.push_back(o.second);
        out.c_key.push_back(o.first - rho - PRUNE_MARGIN);
        keep_near(A.cb_items.data() + A.cb_off[o.second], A.cb_items.data() + A.cb_off[o.second + 1], out.c_blk);
        out.c_off.push_back(uint32_t(out.c_blk.size()));
    }
    out.order.clear();
    A.vertex_cells.near(b, reach, [&](uint32_t vi) {
        double d = b.dist(V3::at(&A.vertex[3 * size_t(vi)]));
        if (d <= reach) out.order.push_back({d, vi});
    });
    nearest_first(out.order);
    for (auto& o : out.order) out.vertices.push_back(o.second), out.v_key.push_back(o.first - rho - PRUNE_MARGIN);
}

// point.rs:686-738 (SES)
NearEval eval_local(const Arrangement& A, const V3& x, double band, const Local& l) {
    if (A.kind != 0) {  // point.rs:723-736
        double best = band;
        int64_t bi = -1;
        for (uint32_t k : l.inside) {
            double v = x.dist(A.c(k)) - A.expanded[k];
            if (v < best) best = v, bi = k;
        }
        NearEval r;
        r.value = best;
        r.feature.kind = bi < 0 ? F_BEYOND : F_SPHERE;
        r.feature.id = bi < 0 ? 0u : uint32_t(bi);
        r.closest = x;
        return r;
    }
    bool inside = false;
    for (uint32_t k : l.inside)
        if (x.dist(A.c(k)) < A.expanded[k]) {
            inside = true;
            break;
        }
    if (!inside) return NearEval{A.probe, Feature{F_SOLVENT, 0}, x};
    Best best{A.probe + band, x, Feature{F_BEYOND, 0}};
    for (size_t k = 0; k < l.spheres.size() && l.s_key[k] < best.d; k++)
        try_sphere(A, x, l.spheres[k], l.s_blk.data() + l.s_off[k], l.s_blk.data() + l.s_off[k + 1], best);
    for (size_t k = 0; k < l.circles.size() && l.c_key[k] < best.d; k++)
        try_circle(A, x, l.circles[k], l.c_blk.data() + l.c_off[k], l.c_blk.data() + l.c_off[k + 1], best);
    for (size_t k = 0; k < l.vertices.size() && l.v_key[k] < best.d; k++) {
        uint32_t vi = l.vertices[k];
        V3 p = V3::at(&A.vertex[3 * size_t(vi)]);
        double d = x.dist(p);
        if (d < best.d) best = Best{d, p, Feature{F_VERTEX, vi}};
    }
    return NearEval{A.probe - best.d, best.f, best.q};
}

void refine_exact(const Arrangement& A, const MeshParams& P, const int32_t* keys, size_t n, const uint32_t* edge_off,
                  const uint32_t* edges, const float* vals, MeshOut& out) {
    resize(out, edge_off[n], n);
    const size_t chunk = 16;
    parallel_for((n + chunk - 1) / chunk, [&](size_t c, int) {
        Local locals[8];
        for (size_t i = c * chunk; i < std::min(n, (c + 1) * chunk); i++) {
            bool have[8] = {false};
            uint32_t evals = 0;
            for (uint32_t k = edge_off[i]; k < edge_off[i + 1]; k++) {
                EdgeGeom g = edge_geom(P, keys + 3 * i, edges[k]);
                if (!have[g.sb]) local_of(A, P, keys + 3 * i, g.sb, locals[g.sb]), have[g.sb] = true;
                put(out, k, refine_edge(A, P, g.pa, g.pb, double(vals[2 * k]), double(vals[2 * k + 1]), locals[g.sb], evals));
            }
            out.evals[i] = evals;
        }
    });
}

void place_fast(const Arrangement& A, const MeshParams& P, const int32_t* keys, size_t n, const uint32_t* edge_off,
                const uint32_t* edges, const float* vals, const DeviceRefine& dev, MeshOut& out) {
    resize(out, edge_off[n], n);
    const size_t chunk = 16;
    parallel_for((n + chunk - 1) / chunk, [&](size_t c, int) {
        Local locals[8];
        for (size_t i = c * chunk; i < std::min(n, (c + 1) * chunk); i++) {
            bool have[8] = {false};
            uint32_t evals = 0, cpu = 0;
            const int32_t* key = keys + 3 * i;
            V3 base(double(int64_t(key[0]) * P.b) * P.h, double(int64_t(key[1]) * P.b) * P.h,
                    double(int64_t(key[2]) * P.b) * P.h);
            for (uint32_t k = edge_off[i]; k < edge_off[i + 1]; k++) {
                EdgeGeom g = edge_geom(P, key, edges[k]);
                double fa = double(vals[2 * k]), fb = double(vals[2 * k + 1]);
                // DeviceEdges::get (field/gpu.rs:155-179)
                uint32_t ev = dev.evals[k];
                double t = double(dev.t[k]);
                uint32_t kind = dev.feat[k] >> FEAT_SHIFT, id = dev.feat[k] & ((1u << FEAT_SHIFT) - 1);
                bool ok = (ev & EDGE_CONVERGED) && t >= 0.0 && t <= 1.0;
                if (ok) {
                    if (kind == F_SPHERE) ok = id < A.n;
                    else if (kind == F_CIRCLE) ok = id < A.n_circles();
                    else if (kind == F_VERTEX) ok = id < A.n_vertices();
                    else ok = kind == F_SOLVENT || kind == F_BEYOND;
                }
                if (ok) {
                    V3 d = g.pb - g.pa;
                    Vertex v;
                    v.t = t;
                    v.pos = g.pa + d * clamp(t, P.t_min, 1.0 - P.t_min);
                    NearEval e{0.0, Feature{kind, id},
                               base + V3(double(dev.closest[3 * k]), double(dev.closest[3 * k + 1]), double(dev.closest[3 * k + 2]))};
                    V3 outward = (fa < 0.0 ? d : d * -1.0).unit();
                    attributes(A, P, v.pos, e, outward, v.normal, v.patch, v.atom);
                    put(out, k, v);
                    evals += ev & ~EDGE_CONVERGED;
                } else {
                    if (!have[g.sb]) local_of(A, P, key, g.sb, locals[g.sb]), have[g.sb] = true;
                    put(out, k, refine_edge(A, P, g.pa, g.pb, fa, fb, locals[g.sb], evals));
                    cpu++;
                }
            }
            out.evals[i] = evals;
            out.cpu_refined[i] = cpu;
        }
    });
}

void place_exact(const Arrangement& A, const MeshParams& P, const int32_t* keys, size_t n, const uint32_t* edge_off,
                 const uint32_t* edges, const float* vals, const uint32_t* dev_evals, MeshOut& out) {
    resize(out, edge_off[n], n);
    const size_t chunk = 64;
    parallel_for((n + chunk - 1) / chunk, [&](size_t c, int) {
        Local locals[8];
        for (size_t i = c * chunk; i < std::min(n, (c + 1) * chunk); i++) {
            bool have[8] = {false};
            uint32_t evals = 0, cpu = 0;
            for (uint32_t k = edge_off[i]; k < edge_off[i + 1]; k++) {
                if (dev_evals[k]) {
                    evals += dev_evals[k];
                    continue;
                }
                EdgeGeom g = edge_geom(P, keys + 3 * i, edges[k]);
                if (!have[g.sb]) local_of(A, P, keys + 3 * i, g.sb, locals[g.sb]), have[g.sb] = true;
                put(out, k, refine_edge(A, P, g.pa, g.pb, double(vals[2 * k]), double(vals[2 * k + 1]), locals[g.sb], evals));
                cpu++;
            }
            out.evals[i] = evals;
            out.cpu_refined[i] = cpu;
        }
    });
}

static uint64_t pack_key(int32_t x, int32_t y, int32_t z) {  // lattice.rs:93-96
    const int64_t bias = int64_t(1) << 20;
    return uint64_t(int64_t(x) + bias) | (uint64_t(int64_t(y) + bias) << 21) | (uint64_t(int64_t(z) + bias) << 42);
}

std::string assemble(const int32_t* keys, size_t n, const uint32_t* edge_off, const uint32_t* edges,
                     const uint32_t* tri_off, const uint32_t* refs, Mesh& mesh) {
    std::vector<uint64_t> packed(n);
    for (size_t i = 0; i < n; i++) packed[i] = pack_key(keys[3 * i], keys[3 * i + 1], keys[3 * i + 2]);
    for (size_t i = 1; i < n; i++)
        if (packed[i] <= packed[i - 1]) return "bricks are not in packed-key order";
    mesh.triangles.resize(tri_off[n]);
    std::atomic<int> bad{0};
    parallel_for((n + 63) / 64, [&](size_t c, int) {
        for (size_t i = c * 64; i < std::min(n, (c + 1) * 64); i++) {
            int64_t target[8];
            for (auto& t : target) t = -1;
            target[0] = int64_t(i);
            for (uint32_t t = tri_off[i]; t < tri_off[i + 1]; t++)
                for (int k = 0; k < 3; k++) {
                    uint32_t r = refs[3 * size_t(t) + k], code = r >> CODE_SHIFT, id = r & ID_MASK;
                    if (target[code] < 0) {
                        uint64_t want = pack_key(keys[3 * i] + int32_t(code & 1), keys[3 * i + 1] + int32_t((code >> 1) & 1),
                                                 keys[3 * i + 2] + int32_t((code >> 2) & 1));
                        auto it = std::lower_bound(packed.begin(), packed.end(), want);
                        if (it == packed.end() || *it != want) {
                            bad = 1;
                            return;
                        }
                        target[code] = it - packed.begin();
                    }
                    size_t tb = size_t(target[code]);
                    const uint32_t *e0 = edges + edge_off[tb], *e1 = edges + edge_off[tb + 1];
                    const uint32_t* pos = std::lower_bound(e0, e1, id);
                    if (pos == e1 || *pos != id) {
                        bad = 2;
                        return;
                    }
                    mesh.triangles[t][k] = uint32_t(edge_off[tb] + uint32_t(pos - e0));
                }
        }
    });
    if (bad == 1) return "triangle references an edge of a missing brick";
    if (bad == 2) return "triangle references an edge without vertex";
    return "";
}

// Sums in fixed chunks of 2^14 triangles (mesh/mod.rs:86) merged in order.
static constexpr size_t SUM_CHUNK = size_t(1) << 14;

static void area_volume(const Mesh& m, const std::array<uint32_t, 3>& t, const double o[3], double& a, double& v) {
    double p[3][3];
    for (int q = 0; q < 3; q++)
        for (int k = 0; k < 3; k++) p[q][k] = double(m.positions[t[q]][k]) - o[k];
    double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    double c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    a = 0.5 * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
    double x[3] = {p[1][1] * p[2][2] - p[1][2] * p[2][1], p[1][2] * p[2][0] - p[1][0] * p[2][2],
                   p[1][0] * p[2][1] - p[1][1] * p[2][0]};
    v = (p[0][0] * x[0] + p[0][1] * x[1] + p[0][2] * x[2]) / 6.0;
}


void EdgeUses::build(const Mesh& m) {
    size_t nv = m.positions.size(), nt = m.triangles.size();
    std::vector<std::atomic<uint32_t>> cnt(nv + 1);
    for (auto& c : cnt) c.store(0, std::memory_order_relaxed);
    parallel_for((nt + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
        for (size_t t = c * SUM_CHUNK; t < std::min(nt, (c + 1) * SUM_CHUNK); t++)
            for (int k = 0; k < 3; k++) {
                uint32_t a = m.triangles[t][k], b = m.triangles[t][(k + 1) % 3];
                cnt[std::min(a, b)].fetch_add(1, std::memory_order_relaxed);
            }
    });
    start.assign(nv + 1, 0);
    for (size_t v = 0; v < nv; v++) start[v + 1] = start[v] + cnt[v].load(std::memory_order_relaxed);
    std::vector<std::atomic<uint64_t>> fill(nv);
    for (size_t v = 0; v < nv; v++) fill[v].store(start[v], std::memory_order_relaxed);
    uses.resize(start[nv]);
    parallel_for((nt + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
        for (size_t t = c * SUM_CHUNK; t < std::min(nt, (c + 1) * SUM_CHUNK); t++)
            for (int k = 0; k < 3; k++) {
                uint32_t a = m.triangles[t][k], b = m.triangles[t][(k + 1) % 3];
                uint32_t lo = std::min(a, b), hi = std::max(a, b);
                uses[fill[lo].fetch_add(1, std::memory_order_relaxed)] = (uint64_t(hi) << 1) | (a < b ? 1u : 0u);
            }
    });
    parallel_for((nv + 4095) / 4096, [&](size_t c, int) {
        for (size_t v = c * 4096; v < std::min(nv, (c + 1) * 4096); v++) std::sort(uses.begin() + start[v], uses.begin() + start[v + 1]);
    });
}

size_t defects(const Mesh& m, EdgeUses* keep) {
    const size_t nv = m.positions.size(), nt = m.triangles.size();
    std::atomic<size_t> bad{0};
    parallel_for((nv + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
        size_t b = 0;
        for (size_t v = c * SUM_CHUNK; v < std::min(nv, (c + 1) * SUM_CHUNK); v++) {
            const auto& p = m.positions[v];
            if (!(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]))) b++;
            if (!m.normals.empty()) {
                const auto& q = m.normals[v];
                float len2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
                if (!(std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]) && std::fabs(len2 - 1.0f) < 1e-3f)) b++;
            }
        }
        bad += b;
    });
    for (auto& t : m.triangles)
        if (t[0] >= nv || t[1] >= nv || t[2] >= nv) return bad + 1;
    double o[3] = {0, 0, 0};
    if (nv) o[0] = m.positions[0][0], o[1] = m.positions[0][1], o[2] = m.positions[0][2];
    parallel_for((nt + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
        size_t b = 0;
        for (size_t t = c * SUM_CHUNK; t < std::min(nt, (c + 1) * SUM_CHUNK); t++) {
            const auto& T = m.triangles[t];
            double a, v;
            area_volume(m, T, o, a, v);
            if (T[0] == T[1] || T[1] == T[2] || T[0] == T[2] || a == 0.0) b++;
        }
        bad += b;
    });
    EdgeUses local;
    EdgeUses& E = keep ? *keep : local;
    E.build(m);
    parallel_for((nv + 4095) / 4096, [&](size_t c, int) {
        size_t b = 0;
        for (size_t v = c * 4096; v < std::min(nv, (c + 1) * 4096); v++)
            for (uint64_t i = E.start[v]; i < E.start[v + 1];) {
                uint64_t j = i;
                size_t fwd = 0, bwd = 0;
                while (j < E.start[v + 1] && (E.uses[j] >> 1) == (E.uses[i] >> 1)) (E.uses[j] & 1 ? fwd : bwd)++, j++;
                if (!(fwd == 1 && bwd == 1)) b++;
                i = j;
            }
        bad += b;
    });
    // Duplicate triangles: equal sorted vertex triples, bucketed by the
    // smallest vertex (counting sort), pairs (s1, s2) sorted per bucket.
    {
        std::vector<std::atomic<uint32_t>> cnt(nv + 1);
        for (auto& c : cnt) c.store(0, std::memory_order_relaxed);
        auto sorted3 = [&](size_t t) {
            std::array<uint32_t, 3> a = m.triangles[t];
            if (a[0] > a[1]) std::swap(a[0], a[1]);
            if (a[1] > a[2]) std::swap(a[1], a[2]);
            if (a[0] > a[1]) std::swap(a[0], a[1]);
            return a;
        };
        parallel_for((nt + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
            for (size_t t = c * SUM_CHUNK; t < std::min(nt, (c + 1) * SUM_CHUNK); t++)
                cnt[sorted3(t)[0]].fetch_add(1, std::memory_order_relaxed);
        });
        std::vector<uint64_t> start(nv + 1, 0);
        for (size_t v = 0; v < nv; v++) start[v + 1] = start[v] + cnt[v].load(std::memory_order_relaxed);
        std::vector<std::atomic<uint64_t>> fill(nv);
        for (size_t v = 0; v < nv; v++) fill[v].store(start[v], std::memory_order_relaxed);
        std::vector<uint64_t> pairs(nt);
        parallel_for((nt + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
            for (size_t t = c * SUM_CHUNK; t < std::min(nt, (c + 1) * SUM_CHUNK); t++) {
                auto a = sorted3(t);
                pairs[fill[a[0]].fetch_add(1, std::memory_order_relaxed)] = (uint64_t(a[1]) << 32) | a[2];
            }
        });
        parallel_for((nv + 4095) / 4096, [&](size_t c, int) {
            size_t b = 0;
            for (size_t v = c * 4096; v < std::min(nv, (c + 1) * 4096); v++) {
                std::sort(pairs.begin() + start[v], pairs.begin() + start[v + 1]);
                for (uint64_t i = start[v] + 1; i < start[v + 1]; i++) b += pairs[i] == pairs[i - 1];
            }
            bad += b;
        });
    }
    return bad.load();
}

void components_and_group(Mesh& m, std::vector<Component>& comps, const EdgeUses* uses) {
    const size_t nv = m.positions.size(), nt = m.triangles.size();
    // Lock-free union-find linking the larger root to the smaller (mesh/
    // mod.rs:190-230): parents only decrease, every root is its component's
    // smallest vertex, and the partition does not depend on scheduling.
    std::vector<std::atomic<uint32_t>> parent(nv);
    for (size_t v = 0; v < nv; v++) parent[v].store(uint32_t(v), std::memory_order_relaxed);
    auto find = [&](uint32_t x) {
        for (;;) {
            uint32_t p = parent[x].load(std::memory_order_relaxed);
            if (p == x) return x;
            uint32_t g = parent[p].load(std::memory_order_relaxed);
            if (g != p) parent[x].compare_exchange_weak(p, g, std::memory_order_relaxed);
            x = g;
        }
    };
    auto unite = [&](uint32_t a, uint32_t b) {
        for (;;) {
            uint32_t ra = find(a), rb = find(b);
            if (ra == rb) return;
            uint32_t lo = std::min(ra, rb), hi = std::max(ra, rb);
            if (parent[hi].compare_exchange_strong(hi, lo, std::memory_order_relaxed)) return;
        }
    };
    parallel_for((nt + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
        for (size_t t = c * SUM_CHUNK; t < std::min(nt, (c + 1) * SUM_CHUNK); t++) {
            unite(m.triangles[t][0], m.triangles[t][1]);
            unite(m.triangles[t][0], m.triangles[t][2]);
        }
    });
    std::vector<uint32_t> root(nv);
    parallel_for((nv + SUM_CHUNK - 1) / SUM_CHUNK, [&](size_t c, int) {
        for (size_t v = c * SUM_CHUNK; v < std::min(nv, (c + 1) * SUM_CHUNK); v++) root[v] = find(uint32_t(v));
    });
    std::vector<uint32_t>& id = m.vertex_component;
    id.assign(nv, 0);
    comps.clear();
    for (size_t v = 0; v < nv; v++) {
        uint32_t r = root[v];
        if (r == v) id[v] = uint32_t(comps.size()), comps.emplace_back();
        else id[v] = id[r];
        comps[id[v]].vertices++;
    }
    double o[3] = {0, 0, 0};
    if (nv) o[0] = m.positions[0][0], o[1] = m.positions[0][1], o[2] = m.positions[0][2];
    struct Acc {
        uint32_t comp;
        size_t t;
        double a, v;
    };
    size_t chunks = (nt + SUM_CHUNK - 1) / SUM_CHUNK;
    std::vector<std::vector<Acc>> parts(chunks);
    parallel_for(chunks, [&](size_t c, int) {
        auto& acc = parts[c];
        for (size_t t = c * SUM_CHUNK; t < std::min(nt, (c + 1) * SUM_CHUNK); t++) {
            uint32_t comp = id[m.triangles[t][0]];
            double a, v;
            area_volume(m, m.triangles[t], o, a, v);
            Acc* e = nullptr;
            for (auto& x : acc)
                if (x.comp == comp) {
                    e = &x;
                    break;
                }
            if (e) e->t++, e->a += a, e->v += v;
            else acc.push_back(Acc{comp, 1, a, v});
        }
    });
    for (auto& p : parts)
        for (auto& x : p) comps[x.comp].triangles += x.t, comps[x.comp].area += x.a, comps[x.comp].volume += x.v;
    EdgeUses local;
    if (!uses) local.build(m);
    const EdgeUses& E = uses ? *uses : local;
    std::vector<int64_t> ecount(comps.size(), 0);
    for (size_t v = 0; v < nv; v++)
        for (uint64_t i = E.start[v]; i < E.start[v + 1]; i++)
            if (i == E.start[v] || (E.uses[i] >> 1) != (E.uses[i - 1] >> 1)) ecount[id[v]]++;
    for (size_t c = 0; c < comps.size(); c++) comps[c].euler = int64_t(comps[c].vertices) - ecount[c] + int64_t(comps[c].triangles);
    // Triangles grouped by component, relative order kept (post.rs:14-32).
    size_t start = 0;
    std::vector<size_t> next(comps.size());
    for (size_t c = 0; c < comps.size(); c++) comps[c].first_triangle = next[c] = start, start += comps[c].triangles;
    std::vector<std::array<uint32_t, 3>> out(nt);
    for (auto& t : m.triangles) out[next[id[t[0]]]++] = t;
    m.triangles.swap(out);
}

// Decimal digits of v (what "%llu" prints) at the end of d[20]; their count.
static inline int u64_digits(uint64_t v, char d[20]) {
    int n = 0;
    do {
        d[19 - n++] = char('0' + v % 10);
        v /= 10;
    } while (v);
    return n;
}

static inline void push_u64(std::string& buf, uint64_t v) {
    char d[20];
    const int n = u64_digits(v, d);
    buf.append(d + 20 - n, size_t(n));
}

// export/fmt.rs:30-53: exact for f32 because x * 10^prec is exact in f64.
void push_fixed(std::string& buf, float x, int prec) {
    static const uint64_t P10[10] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000, 100000000, 1000000000};
    double scaled = std::nearbyint(double(x) * double(P10[prec]));
    if (!std::isfinite(scaled) || std::fabs(scaled) >= 1e18) {
        if (std::isnan(x)) buf += "NaN";
        else if (std::isinf(x)) buf += x < 0 ? "-inf" : "inf";
        else {
            char tmp[512];
            std::snprintf(tmp, sizeof tmp, "%.*f", prec, double(x));
            buf += tmp;
        }
        return;
    }
    if (std::signbit(x)) buf.push_back('-');
    uint64_t mnt = uint64_t(std::fabs(scaled));
    push_u64(buf, mnt / P10[prec]);
    if (prec > 0) {
        buf.push_back('.');
        uint64_t f = mnt % P10[prec];
        char d[10];
        for (int k = prec - 1; k >= 0; k--) d[k] = char('0' + f % 10), f /= 10;
        buf.append(d, size_t(prec));
    }
}

// push_fixed into a raw buffer (room for 64 bytes at p); the end.  The
// common case (finite, |x 10^prec| < 1e18) is written directly, the rest
// through push_fixed.  P is the precision when it is known at compile time
// (the default 4), else 0 and prec is used.
template <int P>
static inline char* put_fixed(char* p, float x, int prec) {
    static const uint64_t P10[10] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000, 100000000, 1000000000};
    const int pr = P ? P : prec;
    const double scaled = std::nearbyint(double(x) * double(P ? P10[P] : P10[pr]));
    if (!std::isfinite(scaled) || std::fabs(scaled) >= 1e18) {
        std::string tmp;
        push_fixed(tmp, x, pr);
        std::memcpy(p, tmp.data(), tmp.size());
        return p + tmp.size();
    }
    if (std::signbit(x)) *p++ = '-';
    const uint64_t mnt = uint64_t(std::fabs(scaled));
    const uint64_t ip = P ? mnt / P10[P] : mnt / P10[pr];
    uint64_t f = mnt - ip * (P ? P10[P] : P10[pr]);
    char d[20];
    const int n = u64_digits(ip, d);
    std::memcpy(p, d + 20 - n, size_t(n));
    p += n;
    if (pr > 0) {
        *p++ = '.';
        for (int k = pr - 1; k >= 0; k--) p[k] = char('0' + f % 10), f /= 10;
        p += pr;
    }
    return p;
}

// Bytes put_fixed writes for x.
template <int P>
static inline size_t fixed_len(float x, int prec) {
    static const uint64_t P10[10] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000, 100000000, 1000000000};
    const int pr = P ? P : prec;
    const double scaled = std::nearbyint(double(x) * double(P ? P10[P] : P10[pr]));
    if (!std::isfinite(scaled) || std::fabs(scaled) >= 1e18) {
        std::string tmp;
        push_fixed(tmp, x, pr);
        return tmp.size();
    }
    const uint64_t ip = uint64_t(std::fabs(scaled)) / (P ? P10[P] : P10[pr]);
    size_t n = 1;
    for (uint64_t v = ip; v >= 10; v /= 10) n++;
    return (std::signbit(x) ? 1 : 0) + n + (pr > 0 ? 1 + size_t(pr) : 0);
}

static inline size_t u64_len(uint64_t v) {
    size_t n = 1;
    for (; v >= 10; v /= 10) n++;
    return n;
}

// export/obj.rs:144-236, default options: header, object "ses", v, vn, f a//a.
// Two passes over chunks of lines on the host threads: the exact byte count
// of each chunk, then each chunk formatted straight into its place, so the
// text is written once into one buffer (no intermediate copies).
static const char OBJ_HEAD[] = "# sesmesh 1.3.2\no ses\n";
constexpr size_t OBJ_CH = 1 << 15;

struct ObjPlan {
    std::vector<size_t> at;  // chunk start offsets: v chunks, vn chunks, f chunks, then the end
    size_t nvc = 0, nfc = 0;
    bool normals = false;
};

static ObjPlan obj_plan(const MeshRef& m, int precision, bool normals) {
    ObjPlan P;
    P.normals = normals && m.nrm;
    const size_t nv = m.nv, nt = m.nt;
    P.nvc = (nv + OBJ_CH - 1) / OBJ_CH, P.nfc = (nt + OBJ_CH - 1) / OBJ_CH;
    const size_t nvec = P.normals ? 2 : 1, nch = nvec * P.nvc + P.nfc;
    std::vector<size_t> len(nch, 0);
    parallel_for(nch, [&](size_t c, int) {
        size_t n = 0;
        if (c < nvec * P.nvc) {
            const bool nrm = c >= P.nvc;
            const float* data = nrm ? m.nrm : m.pos;
            const size_t ch = nrm ? c - P.nvc : c;
            for (size_t i = ch * OBJ_CH, e = std::min(nv, (ch + 1) * OBJ_CH); i < e; i++) {
                n += (nrm ? 3 : 2) + 2 + 1;  // tag, two spaces, newline
                for (int k = 0; k < 3; k++)
                    n += precision == 4 ? fixed_len<4>(data[3 * i + k], 4) : fixed_len<0>(data[3 * i + k], precision);
            }
        } else {
            const size_t ch = c - nvec * P.nvc;
            for (size_t t = ch * OBJ_CH, e = std::min(nt, (ch + 1) * OBJ_CH); t < e; t++) {
                n += 2;  // 'f', newline
                for (int k = 0; k < 3; k++) {
                    const size_t d = u64_len(uint64_t(m.tris[3 * t + k]) + 1);
                    n += 1 + (P.normals ? 2 * d + 2 : d);
                }
            }
        }
        len[c] = n;
    });
    P.at.assign(nch + 1, sizeof OBJ_HEAD - 1);
    for (size_t c = 0; c < nch; c++) P.at[c + 1] = P.at[c] + len[c];
    return P;
}

static void obj_fill(const MeshRef& m, int precision, const ObjPlan& P, char* out) {
    std::memcpy(out, OBJ_HEAD, sizeof OBJ_HEAD - 1);
    const size_t nv = m.nv, nt = m.nt;
    const size_t nvec = P.normals ? 2 : 1, nch = nvec * P.nvc + P.nfc;
    parallel_for(nch, [&](size_t c, int) {
        char* p = out + P.at[c];
        if (c < nvec * P.nvc) {
            const bool nrm = c >= P.nvc;
            const float* data = nrm ? m.nrm : m.pos;
            const size_t ch = nrm ? c - P.nvc : c;
            for (size_t i = ch * OBJ_CH, e = std::min(nv, (ch + 1) * OBJ_CH); i < e; i++) {
                *p++ = 'v';
                if (nrm) *p++ = 'n';
                *p++ = ' ';
                for (int k = 0; k < 3; k++) {
                    if (k) *p++ = ' ';
                    p = precision == 4 ? put_fixed<4>(p, data[3 * i + k], 4) : put_fixed<0>(p, data[3 * i + k], precision);
                }
                *p++ = '\n';
            }
        } else {
            const size_t ch = c - nvec * P.nvc;
            for (size_t t = ch * OBJ_CH, e = std::min(nt, (ch + 1) * OBJ_CH); t < e; t++) {
                *p++ = 'f';
                for (int k = 0; k < 3; k++) {
                    char d[20];
                    const int n = u64_digits(uint64_t(m.tris[3 * t + k]) + 1, d);
                    *p++ = ' ';
                    std::memcpy(p, d + 20 - n, size_t(n));
                    p += n;
                    if (P.normals) {
                        *p++ = '/', *p++ = '/';
                        std::memcpy(p, d + 20 - n, size_t(n));
                        p += n;
                    }
                }
                *p++ = '\n';
            }
        }
    });
}

ObjText obj_text_buffer(const MeshRef& m, int precision, bool normals) {
    const ObjPlan P = obj_plan(m, precision, normals);
    ObjText t;
    t.size = P.at.back();
    t.data.reset(new char[t.size]);
    obj_fill(m, precision, P, t.data.get());
    return t;
}

std::string obj_text(const MeshRef& m, int precision, bool normals) {
    const ObjPlan P = obj_plan(m, precision, normals);
    std::string out(P.at.back(), '\0');
    obj_fill(m, precision, P, &out[0]);
    return out;
}

}  // namespace smbh
