// Oracle (test infrastructure): cell grids and the SAS arrangement.
// Restates crates/sesmesh/src/geom/{vec.rs,cells.rs,arrangement.rs}.
#include "oracle.hpp"

#include <algorithm>
#include <atomic>
#include <thread>

namespace orc {

static int g_threads = 0;
void set_threads(int n) { g_threads = n; }
int threads() {
    if (g_threads > 0) return g_threads;
    unsigned h = std::thread::hardware_concurrency();
    return h ? int(h) : 1;
}

// Dynamic schedule over [0, n); callers write results by index, so the output
// never depends on the schedule (par.rs:13-44).
void parallel_for(size_t n, const std::function<void(size_t, int)>& f) {
    int t = std::min<size_t>(size_t(threads()), n ? n : 1);
    if (t <= 1) {
        for (size_t i = 0; i < n; i++) f(i, 0);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    for (int w = 0; w < t; w++)
        pool.emplace_back([&, w] {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                f(i, w);
            }
        });
    for (auto& th : pool) th.join();
}

// geom/vec.rs:112-125
static void orthonormal_basis(const V3& u, V3& e1, V3& e2) {
    double ax = std::fabs(u.x), ay = std::fabs(u.y), az = std::fabs(u.z);
    V3 helper = (ax <= ay && ax <= az) ? V3(1, 0, 0) : (ay <= az ? V3(0, 1, 0) : V3(0, 0, 1));
    e1 = helper.cross(u).normalized();
    e2 = u.cross(e1);
}

// geom/cells.rs:27-84
void CellGrid::build(const std::vector<V3>& pts, double cell_) {
    cell = cell_;
    if (pts.empty()) {
        origin = V3();
        dims[0] = dims[1] = dims[2] = 1;
        starts.assign(2, 0);
        items.clear();
        return;
    }
    V3 lo = pts[0], hi = pts[0];
    for (auto& p : pts) {
        lo = lo.vmin(p);
        hi = hi.vmax(p);
    }
    V3 ext = hi - lo;
    size_t max_cells = std::max<size_t>(8 * pts.size(), size_t(1) << 16);
    for (;;) {
        double e[3] = {ext.x, ext.y, ext.z};
        size_t d[3];
        bool ok = true;
        unsigned __int128 total = 1;
        for (int a = 0; a < 3; a++) {
            uint64_t v = sat_u64(std::floor(e[a] / cell));
            if (v == UINT64_MAX) { ok = false; break; }
            d[a] = size_t(v) + 1;
            total *= d[a];
        }
        if (ok && total <= max_cells) {
            dims[0] = d[0], dims[1] = d[1], dims[2] = d[2];
            break;
        }
        cell *= 2.0;
    }
    origin = lo;
    size_t total = dims[0] * dims[1] * dims[2];
    std::vector<size_t> keys(pts.size());
    for (size_t i = 0; i < pts.size(); i++) {
        size_t c[3];
        coord(pts[i], c);
        keys[i] = flat(c[0], c[1], c[2]);
    }
    starts.assign(total + 1, 0);
    for (size_t k : keys) starts[k + 1]++;
    for (size_t i = 0; i < total; i++) starts[i + 1] += starts[i];
    std::vector<uint32_t> cursor(starts.begin(), starts.end());
    items.assign(pts.size(), 0);
    for (size_t i = 0; i < keys.size(); i++) items[cursor[keys[i]]++] = uint32_t(i);
}

// geom/cells.rs:91-104
void CellGrid::coord(const V3& p, size_t out[3]) const {
    double rel[3] = {p.x - origin.x, p.y - origin.y, p.z - origin.z};
    for (int a = 0; a < 3; a++) {
        double c = std::floor(rel[a] / cell);
        if (c <= 0.0 || std::isnan(c)) {
            out[a] = 0;
        } else {
            uint64_t v = sat_u64(c);
            out[a] = std::min<uint64_t>(v, dims[a] - 1);
        }
    }
}

// geom/cells.rs:135-150
static uint64_t spread(uint32_t v) {
    uint64_t x = uint64_t(v) & 0x1fffff;
    x = (x | (x << 32)) & 0x001f00000000ffffULL;
    x = (x | (x << 16)) & 0x001f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}
static uint64_t morton(uint32_t a, uint32_t b, uint32_t c) { return spread(a) | (spread(b) << 1) | (spread(c) << 2); }

// ---- arrangement.rs:246-405: circle cuts and exposed arcs ------------------
constexpr double EPS = 1e-9;
constexpr double ANG_EPS = 1e-12;
constexpr double PSEUDO_PERIOD = 4.0;
constexpr double PSEUDO_EPS = 1e-12;
constexpr double TAU = 6.283185307179586;

enum CutKind { CUT_EMPTY, CUT_FULL, CUT_INTERVAL };
struct Cut {
    CutKind kind;
    double enter[2], leave[2];
};

// arrangement.rs:251-274
static Cut cut(const Circle& c, const V3& center, double expanded) {
    V3 g = c.center - center;
    double a = 2.0 * c.radius * c.e1.dot(g);
    double b = 2.0 * c.radius * c.e2().dot(g);
    double rhs = expanded * expanded - g.norm2() - c.radius * c.radius;
    double amp = std::sqrt(a * a + b * b);
    Cut out;
    if (amp <= rhs) {
        out.kind = CUT_FULL;
    } else if (amp <= -rhs || amp == 0.0) {
        out.kind = CUT_EMPTY;
    } else {
        double cp = a / amp, sp = b / amp;
        double ca = rhs / amp;
        double sa = std::sqrt(std::fmax(1.0 - ca * ca, 0.0));
        out.kind = CUT_INTERVAL;
        out.enter[0] = cp * ca - sp * sa;
        out.enter[1] = sp * ca + cp * sa;
        out.leave[0] = cp * ca + sp * sa;
        out.leave[1] = sp * ca - cp * sa;
    }
    return out;
}

// arrangement.rs:282-297
static double pseudo_angle(const double v[2]) {
    double x = v[0], y = v[1];
    if (y >= 0.0) {
        if (x >= 0.0) return y / (x + y);
        return 1.0 - x / (y - x);
    }
    if (x < 0.0) return 2.0 - y / (-x - y);
    return 3.0 + x / (x - y);
}

struct Buried {
    double start, end;
    uint32_t sphere;
    double enter[2], leave[2];
};
struct Merged {
    double start, end;
    uint32_t first, last;
    double enter[2], leave[2];
};

// f64::total_cmp for the sort keys (finite here; kept general).
static inline int64_t total_key(double v) {
    int64_t b;
    std::memcpy(&b, &v, 8);
    return b ^ int64_t(uint64_t(b >> 63) >> 1);
}

static double rem_euclid(double a, double b) {
    double r = std::fmod(a, b);
    return r < 0.0 ? r + std::fabs(b) : r;
}

// arrangement.rs:340-405; returns whether some arc is exposed.
static bool exposed_arcs(std::vector<Buried>& iv, std::vector<Merged>& merged) {
    if (iv.empty()) return true;
    std::sort(iv.begin(), iv.end(), [](const Buried& x, const Buried& y) {
        int64_t a = total_key(x.start), b = total_key(y.start);
        if (a != b) return a < b;
        int64_t c = total_key(y.end), d = total_key(x.end);
        if (c != d) return c < d;
        return x.sphere < y.sphere;
    });
    merged.clear();
    for (auto& b : iv) {
        if (!merged.empty() && b.start <= merged.back().end) {
            Merged& last = merged.back();
            if (b.end > last.end) {
                last.end = b.end;
                last.last = b.sphere;
                last.leave[0] = b.leave[0], last.leave[1] = b.leave[1];
            }
        } else {
            Merged m{b.start, b.end, b.sphere, b.sphere, {b.enter[0], b.enter[1]}, {b.leave[0], b.leave[1]}};
            merged.push_back(m);
        }
    }
    while (merged.size() > 1) {
        Merged first = merged[0];
        Merged& last = merged.back();
        if (last.end - PSEUDO_PERIOD < first.start) break;
        if (first.end + PSEUDO_PERIOD > last.end) {
            last.end = first.end + PSEUDO_PERIOD;
            last.last = first.last;
            last.leave[0] = first.leave[0], last.leave[1] = first.leave[1];
        }
        merged.erase(merged.begin());
    }
    size_t m = merged.size();
    bool any = false;
    for (size_t idx = 0; idx < m; idx++) {
        const Merged& cur = merged[idx];
        const Merged& next = merged[(idx + 1) % m];
        double next_start = idx + 1 < m ? next.start : next.start + PSEUDO_PERIOD;
        if (next_start - cur.end > PSEUDO_EPS) {
            double a0 = rem_euclid(std::atan2(cur.leave[1], cur.leave[0]), TAU);
            double a1 = std::atan2(next.enter[1], next.enter[0]);
            double len = rem_euclid(a1 - a0, TAU);
            if (len > ANG_EPS) any = true;
        }
    }
    return any;
}

// arrangement.rs:437-646 (without arcs; with circles for the SES, without
// for SAS and vdW, as SesField::new_with builds them, point.rs:229-237).
static std::string build_arrangement(const Sphere* sp, size_t ns, double probe, Arrangement& A, bool with_circles) {
    if (!(std::isfinite(probe) && probe >= 0.0)) return "probe radius must be finite and >= 0";
    for (size_t i = 0; i < ns; i++) {
        V3 c(sp[i].c[0], sp[i].c[1], sp[i].c[2]);
        if (!c.finite()) return "sphere " + std::to_string(i) + " has a non-finite centre";
        if (!(std::isfinite(sp[i].r) && sp[i].r >= 0.0)) return "sphere " + std::to_string(i) + " has an invalid radius";
    }
    A = Arrangement();
    A.probe = probe;
    std::vector<uint32_t> active;
    for (size_t i = 0; i < ns; i++)
        if (sp[i].r > 0.0) active.push_back(uint32_t(i));
    double max_expanded = 0.0;
    for (uint32_t i : active) max_expanded = std::fmax(max_expanded, sp[i].r + probe);
    double cell = std::fmax(2.0 * max_expanded, 1e-6);
    if (!active.empty()) {
        V3 lo(sp[active[0]].c[0], sp[active[0]].c[1], sp[active[0]].c[2]);
        for (uint32_t i : active) lo = lo.vmin(V3(sp[i].c[0], sp[i].c[1], sp[i].c[2]));
        std::vector<std::pair<uint64_t, uint32_t>> keyed;
        keyed.reserve(active.size());
        for (uint32_t i : active) {
            V3 p = (V3(sp[i].c[0], sp[i].c[1], sp[i].c[2]) - lo) / cell;
            uint32_t q[3];
            double v[3] = {p.x, p.y, p.z};
            for (int a = 0; a < 3; a++) q[a] = uint32_t(std::min<uint64_t>(sat_u64(v[a]), 0x1fffff));
            keyed.push_back({morton(q[0], q[1], q[2]), i});
        }
        std::sort(keyed.begin(), keyed.end());
        for (size_t k = 0; k < active.size(); k++) active[k] = keyed[k].second;
    }
    size_t n = active.size();
    A.orig = active;
    A.centers.resize(n);
    A.radii.resize(n);
    A.expanded.resize(n);
    for (size_t k = 0; k < n; k++) {
        const Sphere& s = sp[active[k]];
        A.centers[k] = V3(s.c[0], s.c[1], s.c[2]);
        A.radii[k] = s.r;
        A.expanded[k] = s.r + probe;
    }
    A.max_expanded = max_expanded;
    A.cells.build(A.centers, cell);
    const auto& C = A.centers;
    const auto& E = A.expanded;

    // Containment (arrangement.rs:497-514).
    std::vector<uint8_t> contained(n, 0);
    parallel_for(n, [&](size_t i, int) {
        bool found = false;
        A.cells.for_each_near(C[i], E[i] + max_expanded, [&](uint32_t j) {
            if (j == i || found) return;
            double d = C[i].dist(C[j]);
            if (d + E[i] <= E[j] + EPS && (E[j] - E[i] > EPS || d > EPS || active[j] < active[i])) found = true;
        });
        contained[i] = found;
    });
    for (auto c : contained) A.n_contained += c;

    // Neighbours (arrangement.rs:522-545).
    std::vector<std::vector<uint32_t>> rows(n);
    parallel_for(n, [&](size_t i, int) {
        if (contained[i]) return;
        auto& r = rows[i];
        A.cells.for_each_near(C[i], E[i] + max_expanded, [&](uint32_t j) {
            if (j != i && !contained[j] && C[i].dist(C[j]) < E[i] + E[j] - EPS) r.push_back(j);
        });
        std::sort(r.begin(), r.end());
    });
    A.neighbors.off.assign(1, 0);
    for (size_t i = 0; i < n; i++) {
        A.neighbors.items.insert(A.neighbors.items.end(), rows[i].begin(), rows[i].end());
        A.neighbors.off.push_back(uint32_t(A.neighbors.items.size()));
    }
    rows.clear();
    rows.shrink_to_fit();

    // Circles, blockers and triple points per sphere (arrangement.rs:674-752).
    struct Part {
        std::vector<Circle> circles;
        std::vector<std::vector<uint32_t>> blockers;
        std::vector<SasVertex> vertices;
    };
    std::vector<Part> parts(n);
    const Csr& NB = A.neighbors;
    parallel_for(n, [&](size_t i, int) {
        if (contained[i] || !with_circles) return;
        Part& out = parts[i];
        std::vector<Buried> intervals;
        std::vector<Merged> merged;
        std::vector<uint32_t> blockers;
        for (const uint32_t* pj = NB.row_begin(i); pj != NB.row_end(i); pj++) {
            uint32_t j = *pj;
            if (j <= i) continue;
            double d = C[i].dist(C[j]);
            V3 axis = (C[j] - C[i]) / d;
            double t = (d * d + E[i] * E[i] - E[j] * E[j]) / (2.0 * d);
            double rho2 = E[i] * E[i] - t * t;
            if (rho2 <= 0.0) continue;
            V3 e1, e2;
            orthonormal_basis(axis, e1, e2);
            Circle circle{uint32_t(i), j, C[i] + axis * t, axis, e1, std::sqrt(rho2)};
            intervals.clear();
            blockers.clear();
            bool buried = false;
            // sorted_intersection(N(i), N(j)) (arrangement.rs:756-765)
            const uint32_t *b = NB.row_begin(j), *be = NB.row_end(j);
            for (const uint32_t* pk = NB.row_begin(i); pk != NB.row_end(i); pk++) {
                uint32_t k = *pk;
                while (b < be && *b < k) b++;
                if (!(b < be && *b == k)) continue;
                Cut ct = cut(circle, C[k], E[k]);
                if (ct.kind == CUT_EMPTY) continue;
                if (ct.kind == CUT_FULL) {
                    buried = true;
                    break;
                }
                Buried bi;
                bi.start = pseudo_angle(ct.enter);
                bi.end = pseudo_angle(ct.leave);
                if (bi.end <= bi.start) bi.end += PSEUDO_PERIOD;
                bi.sphere = k;
                bi.enter[0] = ct.enter[0], bi.enter[1] = ct.enter[1];
                bi.leave[0] = ct.leave[0], bi.leave[1] = ct.leave[1];
                intervals.push_back(bi);
                blockers.push_back(k);
            }
            if (buried) continue;
            if (!exposed_arcs(intervals, merged)) continue;
            for (uint32_t k : blockers) {
                if (k <= j) continue;
                Cut ct = cut(circle, C[k], E[k]);
                if (ct.kind != CUT_INTERVAL) continue;
                const double* pts[2] = {ct.leave, ct.enter};
                for (int w = 0; w < 2; w++) {
                    double c = pts[w][0], s = pts[w][1];
                    V3 q = circle.center + (circle.e1 * c + e2 * s) * circle.radius;
                    bool free = true;
                    for (const uint32_t* pl = NB.row_begin(i); pl != NB.row_end(i); pl++) {
                        uint32_t l = *pl;
                        if (l == j || l == k) continue;
                        if (!(q.dist(C[l]) >= E[l] - EPS)) {
                            free = false;
                            break;
                        }
                    }
                    if (free) out.vertices.push_back(SasVertex{q, {uint32_t(i), j, k}});
                }
            }
            out.circles.push_back(circle);
            out.blockers.push_back(blockers);
        }
    });
    // arrangement.rs:568-571: without circles every sphere not contained is
    // exposed.
    std::vector<uint8_t> exposed(n);
    for (size_t i = 0; i < n; i++) exposed[i] = !contained[i] && (!with_circles || NB.row_len(i) == 0);
    A.circle_blockers.off.assign(1, 0);
    for (size_t i = 0; i < n; i++) {
        Part& p = parts[i];
        for (size_t c = 0; c < p.circles.size(); c++) {
            exposed[p.circles[c].i] = 1;
            exposed[p.circles[c].j] = 1;
            A.circles.push_back(p.circles[c]);
            auto& bl = p.blockers[c];
            A.circle_blockers.items.insert(A.circle_blockers.items.end(), bl.begin(), bl.end());
            A.circle_blockers.off.push_back(uint32_t(A.circle_blockers.items.size()));
        }
        A.vertices.insert(A.vertices.end(), p.vertices.begin(), p.vertices.end());
        Part().circles.swap(p.circles);
    }
    A.status.resize(n);
    for (size_t i = 0; i < n; i++) A.status[i] = contained[i] ? CONTAINED : (exposed[i] ? EXPOSED : BURIED);
    return "";
}

// point.rs:213-285
std::string build_field(const Sphere* s, size_t n, double probe, SesField& F, int kind) {
    if (!(std::isfinite(probe) && probe >= 0.0)) return "probe radius must be finite and >= 0";
    if (kind == KIND_SES && probe == 0.0) kind = KIND_VDW;  // point.rs:224-228
    F.kind = kind;
    std::string err = build_arrangement(s, n, kind == KIND_VDW ? 0.0 : probe, F.arr, kind == KIND_SES);
    if (!err.empty()) return err;
    F.probe = probe;
    Arrangement& A = F.arr;
    // Empty the neighbour rows of spheres that are not exposed (point.rs:244-245).
    {
        Csr nb;
        nb.off.assign(1, 0);
        for (size_t i = 0; i < A.centers.size(); i++) {
            if (A.status[i] == EXPOSED) nb.items.insert(nb.items.end(), A.neighbors.row_begin(i), A.neighbors.row_end(i));
            nb.off.push_back(uint32_t(nb.items.size()));
        }
        A.neighbors = std::move(nb);
    }
    double cell = std::fmax(2.0 * A.max_expanded, 1e-6);
    std::vector<V3> pts;
    for (auto& c : A.circles) pts.push_back(c.center);
    F.circle_cells.build(pts, cell);
    pts.clear();
    for (auto& v : A.vertices) pts.push_back(v.position);
    F.vertex_cells.build(pts, cell);
    F.rho_max = 0.0;
    for (auto& c : A.circles) F.rho_max = std::fmax(F.rho_max, c.radius);
    if (A.centers.empty()) {
        F.extent = 0.0;
    } else {
        V3 lo = A.centers[0], hi = A.centers[0];
        for (auto& c : A.centers) lo = lo.vmin(c), hi = hi.vmax(c);
        F.extent = (hi - lo).norm() + 4.0 * A.max_expanded + 4.0 * probe + 1.0;
    }
    return "";
}

}  // namespace orc
