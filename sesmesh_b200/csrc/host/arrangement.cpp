// SAS arrangement on the host (f64): containment, neighbour rows, exposed
// intersection circles with their blockers, exposed triple points.
// Restates crates/sesmesh/src/geom/arrangement.rs:246-770 (without arcs, as
// the SES field builds it, field/point.rs:235-237) and geom/cells.rs.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>

#include "geom.hpp"

namespace smbh {

static int g_threads = 0;
void set_threads(int n) { g_threads = n; }
int threads() {
    if (g_threads > 0) return g_threads;
    unsigned h = std::thread::hardware_concurrency();
    return h ? int(h) : 1;
}

static thread_local bool t_serial = false;
SerialScope::SerialScope() : prev(t_serial) { t_serial = true; }
SerialScope::~SerialScope() { t_serial = prev; }

void parallel_for(size_t n, const std::function<void(size_t, int)>& f) {
    size_t t = t_serial ? 1 : std::min<size_t>(size_t(threads()), n);
    if (t <= 1) {
        for (size_t i = 0; i < n; i++) f(i, 0);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> pool;
    pool.reserve(t);
    for (size_t w = 0; w < t; w++)
        pool.emplace_back([&, w] {
            for (size_t i; (i = next.fetch_add(1, std::memory_order_relaxed)) < n;) f(i, int(w));
        });
    for (auto& th : pool) th.join();
}

// geom/cells.rs:27-84: cell doubled until the grid has at most
// max(65 536, 8 n) cells.
void Grid::build(const double* pts, size_t n, size_t stride, double cell_) {
    cell = cell_;
    if (n == 0) {
        origin[0] = origin[1] = origin[2] = 0;
        dims[0] = dims[1] = dims[2] = 1;
        starts.assign(2, 0);
        items.clear();
        return;
    }
    V3 lo = V3::at(pts), hi = lo;
    for (size_t i = 0; i < n; i++) {
        V3 p = V3::at(pts + i * stride);
        lo = lo.lo(p), hi = hi.hi(p);
    }
    V3 ext = hi - lo;
    double e[3] = {ext.x, ext.y, ext.z};
    size_t max_cells = std::max<size_t>(8 * n, size_t(1) << 16);
    for (;;) {
        unsigned __int128 total = 1;
        bool ok = true;
        for (int a = 0; a < 3; a++) {
            uint64_t v = to_u64(std::floor(e[a] / cell));
            if (v >= UINT32_MAX) ok = false;
            dims[a] = ok ? uint32_t(v + 1) : 1;
            total *= (unsigned __int128)(v + 1);
        }
        if (ok && total <= max_cells) break;
        cell *= 2.0;
    }
    origin[0] = lo.x, origin[1] = lo.y, origin[2] = lo.z;
    size_t cells = size_t(dims[0]) * dims[1] * dims[2];
    std::vector<uint32_t> key(n);
    starts.assign(cells + 1, 0);
    for (size_t i = 0; i < n; i++) {
        const double* p = pts + i * stride;
        key[i] = uint32_t((size_t(coord(p[2], 2)) * dims[1] + coord(p[1], 1)) * dims[0] + coord(p[0], 0));
        starts[key[i] + 1]++;
    }
    for (size_t i = 0; i < cells; i++) starts[i + 1] += starts[i];
    std::vector<uint32_t> fill(starts.begin(), starts.end() - 1);
    items.resize(n);
    for (size_t i = 0; i < n; i++) items[fill[key[i]]++] = uint32_t(i);
}

namespace {

constexpr double EPS = 1e-9;             // arrangement.rs:26
constexpr double ANG_EPS = 1e-12;        // arrangement.rs:29
constexpr double PERIOD = 4.0;           // arrangement.rs:277
constexpr double PSEUDO_EPS = 1e-12;     // arrangement.rs:279
constexpr double TWO_PI = 6.283185307179586;

uint64_t interleave(uint32_t v) {  // cells.rs:135-143
    uint64_t x = uint64_t(v) & 0x1fffff;
    x = (x | (x << 32)) & 0x001f00000000ffffULL;
    x = (x | (x << 16)) & 0x001f0000ff0000ffULL;
    x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
    x = (x | (x << 2)) & 0x1249249249249249ULL;
    return x;
}

struct CircleF {
    V3 m, u, e1;
    double rho;
    V3 e2() const { return u.cross(e1); }
};

// Circle points strictly inside a sphere (arrangement.rs:251-274):
// 0 none, 1 all, 2 the arc between the crossing vectors.
int cut(const CircleF& c, const V3& s, double R, double enter[2], double leave[2]) {
    V3 g = c.m - s;
    double a = 2.0 * c.rho * c.e1.dot(g);
    double b = 2.0 * c.rho * c.e2().dot(g);
    double rhs = R * R - g.dot(g) - c.rho * c.rho;
    double amp = std::sqrt(a * a + b * b);
    if (amp <= rhs) return 1;
    if (amp <= -rhs || amp == 0.0) return 0;
    double cp = a / amp, sp = b / amp, ca = rhs / amp;
    double sa = std::sqrt(std::fmax(1.0 - ca * ca, 0.0));
    enter[0] = cp * ca - sp * sa, enter[1] = sp * ca + cp * sa;
    leave[0] = cp * ca + sp * sa, leave[1] = sp * ca - cp * sa;
    return 2;
}

double diamond(const double v[2]) {  // arrangement.rs:282-297
    double x = v[0], y = v[1];
    if (y >= 0.0) return x >= 0.0 ? y / (x + y) : 1.0 - x / (y - x);
    return x < 0.0 ? 2.0 - y / (-x - y) : 3.0 + x / (x - y);
}

struct Span {  // a buried interval in diamond-angle space
    double start, end;
    uint32_t sphere;
    double enter[2], leave[2];
};
struct Run {
    double start, end;
    double enter[2], leave[2];
};

inline int64_t order_bits(double v) {  // f64::total_cmp as an integer key
    int64_t b;
    std::memcpy(&b, &v, 8);
    return b ^ int64_t(uint64_t(b >> 63) >> 1);
}

double wrap_tau(double a) {  // f64::rem_euclid(TAU)
    double r = std::fmod(a, TWO_PI);
    return r < 0.0 ? r + TWO_PI : r;
}

// Whether any arc of the circle stays exposed (arrangement.rs:340-405).
bool any_exposed(std::vector<Span>& spans, std::vector<Run>& runs) {
    if (spans.empty()) return true;
    std::sort(spans.begin(), spans.end(), [](const Span& a, const Span& b) {
        int64_t x = order_bits(a.start), y = order_bits(b.start);
        if (x != y) return x < y;
        x = order_bits(b.end), y = order_bits(a.end);
        if (x != y) return x < y;
        return a.sphere < b.sphere;
    });
    runs.clear();
    for (const Span& s : spans) {
        if (!runs.empty() && s.start <= runs.back().end) {
            Run& r = runs.back();
            if (s.end > r.end) r.end = s.end, r.leave[0] = s.leave[0], r.leave[1] = s.leave[1];
        } else {
            runs.push_back(Run{s.start, s.end, {s.enter[0], s.enter[1]}, {s.leave[0], s.leave[1]}});
        }
    }
    while (runs.size() > 1) {
        const Run first = runs.front();
        Run& last = runs.back();
        if (last.end - PERIOD < first.start) break;
        if (first.end + PERIOD > last.end)
            last.end = first.end + PERIOD, last.leave[0] = first.leave[0], last.leave[1] = first.leave[1];
        runs.erase(runs.begin());
    }
    size_t m = runs.size();
    for (size_t k = 0; k < m; k++) {
        const Run& cur = runs[k];
        const Run& nxt = runs[(k + 1) % m];
        double next_start = k + 1 < m ? nxt.start : nxt.start + PERIOD;
        if (next_start - cur.end > PSEUDO_EPS) {
            double a0 = wrap_tau(std::atan2(cur.leave[1], cur.leave[0]));
            double a1 = std::atan2(nxt.enter[1], nxt.enter[0]);
            if (wrap_tau(a1 - a0) > ANG_EPS) return true;
        }
    }
    return false;
}

struct SpherePart {
    std::vector<double> circle;
    std::vector<uint32_t> ij, blk_len, blk, vtx_atoms;
    std::vector<double> vtx;
};

}  // namespace

std::string check_spheres(const double* xyzr, size_t ns, double probe, int kind) {
    if (kind == 0 && !(std::isfinite(probe) && probe > 0.0)) return "probe radius must be finite and > 0 for the SES";
    if (!(std::isfinite(probe) && probe >= 0.0)) return "probe radius must be finite and >= 0";
    for (size_t i = 0; i < ns; i++) {
        const double* s = xyzr + 4 * i;
        if (!(std::isfinite(s[0]) && std::isfinite(s[1]) && std::isfinite(s[2])))
            return "sphere " + std::to_string(i) + " has a non-finite centre";
        if (!(std::isfinite(s[3]) && s[3] >= 0.0)) return "sphere " + std::to_string(i) + " has an invalid radius";
    }
    return "";
}

const char* const CANCELLED = "cancelled";

// kind != 0: a sphere field (SAS, or vdW with probe 0): containment alone,
// every sphere not contained exposed, no circles or vertices
// (arrangement.rs:437-646 with with_circles false, point.rs:229-237).
std::string build_arrangement(const double* xyzr, size_t ns, double probe, Arrangement& A, const Control* ctl,
                              int kind) {
    std::string bad = check_spheres(xyzr, ns, probe, kind);
    if (!bad.empty()) return bad;
    // The flag is polled per sphere in every pass (control.rs:94-131).
    auto stop = [&] { return ctl && ctl->cancelled(); };
    if (stop()) return CANCELLED;
    A = Arrangement();
    A.kind = kind;
    A.probe = probe;
    std::vector<uint32_t> active;
    for (size_t i = 0; i < ns; i++)
        if (xyzr[4 * i + 3] > 0.0) active.push_back(uint32_t(i));
    double max_expanded = 0.0;
    for (uint32_t i : active) max_expanded = std::fmax(max_expanded, xyzr[4 * i + 3] + probe);
    const double cell = std::fmax(2.0 * max_expanded, 1e-6);
    if (!active.empty()) {  // Morton order of cells, ties by input index (arrangement.rs:476-489)
        V3 lo = V3::at(xyzr + 4 * size_t(active[0]));
        for (uint32_t i : active) lo = lo.lo(V3::at(xyzr + 4 * size_t(i)));
        std::vector<std::pair<uint64_t, uint32_t>> key(active.size());
        for (size_t k = 0; k < active.size(); k++) {
            V3 p = (V3::at(xyzr + 4 * size_t(active[k])) - lo) / cell;
            uint32_t q[3] = {uint32_t(std::min<uint64_t>(to_u64(p.x), 0x1fffff)),
                             uint32_t(std::min<uint64_t>(to_u64(p.y), 0x1fffff)),
                             uint32_t(std::min<uint64_t>(to_u64(p.z), 0x1fffff))};
            key[k] = {interleave(q[0]) | (interleave(q[1]) << 1) | (interleave(q[2]) << 2), active[k]};
        }
        std::sort(key.begin(), key.end());
        for (size_t k = 0; k < active.size(); k++) active[k] = key[k].second;
    }
    const size_t n = active.size();
    A.n = n;
    A.orig = active;
    A.center.resize(3 * n);
    A.expanded.resize(n);
    A.radius.resize(n);
    for (size_t k = 0; k < n; k++) {
        const double* s = xyzr + 4 * size_t(active[k]);
        A.center[3 * k] = s[0], A.center[3 * k + 1] = s[1], A.center[3 * k + 2] = s[2];
        A.radius[k] = s[3];
        A.expanded[k] = s[3] + probe;
    }
    A.max_expanded = max_expanded;
    A.cells.build(A.center.data(), n, 3, cell);
    const std::vector<double>& R = A.expanded;

    // Containment (arrangement.rs:497-514).
    std::vector<uint8_t> contained(n, 0);
    parallel_for(n, [&](size_t i, int) {
        if (stop()) return;
        V3 ci = A.c(uint32_t(i));
        bool found = false;
        A.cells.near(ci, R[i] + max_expanded, [&](uint32_t j) {
            if (found || j == i) return;
            double d = ci.dist(A.c(j));
            if (d + R[i] <= R[j] + EPS && (R[j] - R[i] > EPS || d > EPS || active[j] < active[i])) found = true;
        });
        contained[i] = found;
    });
    for (uint8_t c : contained) A.n_contained += c;
    if (stop()) return CANCELLED;
    if (kind != 0) {
        A.status.resize(n);
        for (size_t i = 0; i < n; i++) A.status[i] = contained[i] ? CONTAINED : EXPOSED;
        A.nb_off.assign(n + 1, 0);
        A.cb_off.assign(1, 0);
        A.circle_cells.build(A.circle.data(), 0, 10, cell);
        A.vertex_cells.build(A.vertex.data(), 0, 3, cell);
        if (n) {
            V3 lo = A.c(0), hi = lo;
            for (size_t i = 0; i < n; i++) lo = lo.lo(A.c(uint32_t(i))), hi = hi.hi(A.c(uint32_t(i)));
            A.extent = (hi - lo).norm() + 4.0 * max_expanded + 4.0 * probe + 1.0;
        }
        return "";
    }

    // Neighbour rows, ascending (arrangement.rs:522-545).
    std::vector<std::vector<uint32_t>> rows(n);
    parallel_for(n, [&](size_t i, int) {
        if (contained[i] || stop()) return;
        V3 ci = A.c(uint32_t(i));
        auto& r = rows[i];
        A.cells.near(ci, R[i] + max_expanded, [&](uint32_t j) {
            if (j != i && !contained[j] && ci.dist(A.c(j)) < R[i] + R[j] - EPS) r.push_back(j);
        });
        std::sort(r.begin(), r.end());
    });
    if (stop()) return CANCELLED;
    std::vector<uint32_t> nb_off(n + 1, 0), nb_items;
    for (size_t i = 0; i < n; i++) nb_off[i + 1] = nb_off[i] + uint32_t(rows[i].size());
    nb_items.reserve(nb_off[n]);
    for (auto& r : rows) nb_items.insert(nb_items.end(), r.begin(), r.end());
    std::vector<std::vector<uint32_t>>().swap(rows);
    auto row = [&](uint32_t i) { return std::make_pair(nb_items.data() + nb_off[i], nb_items.data() + nb_off[i + 1]); };

    // Circles (i, j > i), blockers, triple points (arrangement.rs:674-752).
    std::vector<SpherePart> parts(n);
    parallel_for(n, [&](size_t iu, int) {
        if (contained[iu] || stop()) return;
        const uint32_t i = uint32_t(iu);
        SpherePart& out = parts[i];
        std::vector<Span> spans;
        std::vector<Run> runs;
        std::vector<uint32_t> blockers;
        const V3 ci = A.c(i);
        auto [ri0, ri1] = row(i);
        for (const uint32_t* pj = ri0; pj != ri1; pj++) {
            const uint32_t j = *pj;
            if (j <= i) continue;
            const V3 cj = A.c(j);
            double d = ci.dist(cj);
            V3 axis = (cj - ci) / d;
            double t = (d * d + R[i] * R[i] - R[j] * R[j]) / (2.0 * d);
            double rho2 = R[i] * R[i] - t * t;
            if (rho2 <= 0.0) continue;
            // orthonormal_basis (geom/vec.rs:112-125)
            double ax = std::fabs(axis.x), ay = std::fabs(axis.y), az = std::fabs(axis.z);
            V3 helper = (ax <= ay && ax <= az) ? V3(1, 0, 0) : (ay <= az ? V3(0, 1, 0) : V3(0, 0, 1));
            V3 e1 = helper.cross(axis).unit();
            V3 e2 = axis.cross(e1);
            CircleF C{ci + axis * t, axis, e1, std::sqrt(rho2)};
            spans.clear();
            blockers.clear();
            bool buried = false;
            auto [rj0, rj1] = row(j);
            const uint32_t* q = rj0;
            for (const uint32_t* pk = ri0; pk != ri1 && !buried; pk++) {
                const uint32_t k = *pk;
                while (q < rj1 && *q < k) q++;
                if (q == rj1 || *q != k) continue;
                Span s;
                int kind = cut(C, A.c(k), R[k], s.enter, s.leave);
                if (kind == 0) continue;
                if (kind == 1) {
                    buried = true;
                    break;
                }
                s.start = diamond(s.enter);
                s.end = diamond(s.leave);
                if (s.end <= s.start) s.end += PERIOD;
                s.sphere = k;
                spans.push_back(s);
                blockers.push_back(k);
            }
            if (buried || !any_exposed(spans, runs)) continue;
            for (uint32_t k : blockers) {
                if (k <= j) continue;
                double en[2], lv[2];
                if (cut(C, A.c(k), R[k], en, lv) != 2) continue;
                const double* ends[2] = {lv, en};
                for (const double* cs : ends) {
                    V3 p = C.m + (C.e1 * cs[0] + e2 * cs[1]) * C.rho;
                    bool free = true;
                    for (const uint32_t* pl = ri0; pl != ri1 && free; pl++) {
                        uint32_t l = *pl;
                        if (l != j && l != k) free = p.dist(A.c(l)) >= R[l] - EPS;
                    }
                    if (free) {
                        out.vtx.insert(out.vtx.end(), {p.x, p.y, p.z});
                        out.vtx_atoms.insert(out.vtx_atoms.end(), {i, j, k});
                    }
                }
            }
            out.circle.insert(out.circle.end(), {C.m.x, C.m.y, C.m.z, axis.x, axis.y, axis.z, e1.x, e1.y, e1.z, C.rho});
            out.ij.insert(out.ij.end(), {i, j});
            out.blk_len.push_back(uint32_t(blockers.size()));
            out.blk.insert(out.blk.end(), blockers.begin(), blockers.end());
        }
    });
    if (stop()) return CANCELLED;
    std::vector<uint8_t> exposed(n);
    for (size_t i = 0; i < n; i++) exposed[i] = !contained[i] && nb_off[i + 1] == nb_off[i];
    A.cb_off.assign(1, 0);
    for (auto& p : parts) {
        for (size_t c = 0; c < p.ij.size() / 2; c++) exposed[p.ij[2 * c]] = exposed[p.ij[2 * c + 1]] = 1;
        A.circle.insert(A.circle.end(), p.circle.begin(), p.circle.end());
        A.circle_ij.insert(A.circle_ij.end(), p.ij.begin(), p.ij.end());
        size_t o = 0;
        for (uint32_t len : p.blk_len) {
            A.cb_items.insert(A.cb_items.end(), p.blk.begin() + o, p.blk.begin() + o + len);
            A.cb_off.push_back(uint32_t(A.cb_items.size()));
            o += len;
        }
        A.vertex.insert(A.vertex.end(), p.vtx.begin(), p.vtx.end());
        A.vertex_atoms.insert(A.vertex_atoms.end(), p.vtx_atoms.begin(), p.vtx_atoms.end());
        SpherePart().circle.swap(p.circle);
    }
    A.status.resize(n);
    for (size_t i = 0; i < n; i++) A.status[i] = contained[i] ? CONTAINED : (exposed[i] ? EXPOSED : BURIED);
    // Rows of spheres that are not exposed are never read (point.rs:244-245).
    A.nb_off.assign(n + 1, 0);
    for (size_t i = 0; i < n; i++) {
        if (A.status[i] == EXPOSED) A.nb_items.insert(A.nb_items.end(), nb_items.begin() + nb_off[i], nb_items.begin() + nb_off[i + 1]);
        A.nb_off[i + 1] = uint32_t(A.nb_items.size());
    }
    // Cell grids of circle centres and vertices; rho_max; extent (point.rs:246-270).
    A.circle_cells.build(A.circle.data(), A.n_circles(), 10, cell);
    A.vertex_cells.build(A.vertex.data(), A.n_vertices(), 3, cell);
    for (size_t c = 0; c < A.n_circles(); c++) A.rho_max = std::fmax(A.rho_max, A.circle[10 * c + 9]);
    if (n) {
        V3 lo = A.c(0), hi = lo;
        for (size_t i = 0; i < n; i++) lo = lo.lo(A.c(uint32_t(i))), hi = hi.hi(A.c(uint32_t(i)));
        A.extent = (hi - lo).norm() + 4.0 * max_expanded + 4.0 * probe + 1.0;
    }
    return "";
}

}  // namespace smbh
