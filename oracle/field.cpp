// Oracle (test infrastructure): exact f64 field, lattice classification and
// the f32 sampling engine.  Restates crates/sesmesh/src/field/{point.rs,
// lattice.rs,kernel.rs}.
#include "oracle.hpp"

#include <algorithm>

namespace orc {

static constexpr double EPS = 1e-9;

void LocalCandidates::clear() {
    inside.clear();
    near.clear();
    spheres.clear();
    s_off.assign(1, 0);
    s_blk.clear();
    circles.clear();
    c_off.assign(1, 0);
    c_blk.clear();
    vertices.clear();
    order.clear();
}

// point.rs:159-161: nearest first, ties by index (values are never NaN here).
static void sort_nearest(std::vector<std::pair<double, uint32_t>>& v) {
    std::sort(v.begin(), v.end(), [](const auto& a, const auto& b) {
        if (a.first != b.first) return a.first < b.first;
        return a.second < b.second;
    });
}

// point.rs:372-383
bool SesField::inside_sas(const V3& x) const {
    const Arrangement& a = arr;
    bool inside = false;
    a.cells.for_each_near(x, a.max_expanded, [&](uint32_t k) {
        if (!inside && a.status[k] != CONTAINED && x.dist(a.centers[k]) < a.expanded[k]) inside = true;
    });
    return inside;
}

// point.rs:385-411
PointEval SesField::ses_eval(const V3& x, double cutoff) const {
    const Arrangement& a = arr;
    if (!inside_sas(x)) return PointEval{0.0, x, Feature{F_SOLVENT, 0}};
    PointEval best{cutoff, x, Feature{F_BEYOND, 0}};
    a.cells.for_each_near(x, cutoff + a.max_expanded, [&](uint32_t i) {
        if (a.status[i] == EXPOSED) try_sphere_with(x, i, a.neighbors.row_begin(i), a.neighbors.row_end(i), best);
    });
    circle_cells.for_each_near(x, cutoff + rho_max, [&](uint32_t ci) {
        try_circle_with(x, ci, a.circle_blockers.row_begin(ci), a.circle_blockers.row_end(ci), best);
    });
    vertex_cells.for_each_near(x, cutoff, [&](uint32_t vi) { try_vertex(x, vi, best); });
    return best;
}

// point.rs:422-444
void SesField::try_sphere_with(const V3& x, uint32_t i, const uint32_t* b0, const uint32_t* b1, PointEval& best) const {
    const Arrangement& a = arr;
    V3 v = x - a.centers[i];
    double len = v.norm();
    double lb = std::fabs(len - a.expanded[i]);
    if (lb >= best.distance || len < 1e-12) return;
    V3 q = a.centers[i] + v * (a.expanded[i] / len);
    for (const uint32_t* k = b0; k != b1; k++)
        if (!(q.dist(a.centers[*k]) >= a.expanded[*k] - EPS)) return;
    best = PointEval{lb, q, Feature{F_SPHERE, i}};
}

// point.rs:452-476
void SesField::try_circle_with(const V3& x, uint32_t ci, const uint32_t* b0, const uint32_t* b1, PointEval& best) const {
    const Arrangement& a = arr;
    const Circle& c = a.circles[ci];
    V3 y = x - c.center;
    double along = y.dot(c.axis);
    V3 w = y - c.axis * along;
    double wl = w.norm();
    double dist = std::sqrt(along * along + (wl - c.radius) * (wl - c.radius));
    if (dist >= best.distance) return;
    V3 dir = wl > 1e-12 ? w / wl : c.e1;
    V3 q = c.center + dir * c.radius;
    for (const uint32_t* k = b0; k != b1; k++)
        if (!(q.dist(a.centers[*k]) >= a.expanded[*k] - EPS)) return;
    best = PointEval{dist, q, Feature{F_CIRCLE, ci}};
}

// point.rs:479-490
void SesField::try_vertex(const V3& x, uint32_t vi, PointEval& best) const {
    const V3& p = arr.vertices[vi].position;
    double d = x.dist(p);
    if (d < best.distance) best = PointEval{d, p, Feature{F_VERTEX, vi}};
}

// point.rs:496-582 (SES branch)
void SesField::gather_local(const V3& b, double rho, double band, LocalCandidates& out) const {
    const Arrangement& a = arr;
    out.clear();
    if (kind != KIND_SES) {  // point.rs:566-579
        double reach = band + rho;
        a.cells.for_each_near(b, reach + a.max_expanded, [&](uint32_t k) {
            if (a.status[k] != CONTAINED && b.dist(a.centers[k]) - a.expanded[k] < reach)
                out.order.push_back({b.dist(a.centers[k]) - a.expanded[k], k});
        });
        sort_nearest(out.order);
        for (auto& o : out.order) out.inside.push_back(o.second);
        out.order.clear();
        return;
    }
    double reach = probe + band + rho;
    a.cells.for_each_near(b, reach + a.max_expanded, [&](uint32_t k) {
        if (a.status[k] == CONTAINED) return;
        double d = b.dist(a.centers[k]);
        if (d < a.expanded[k] + reach) out.near.push_back(k);
        if (d < a.expanded[k] + rho) out.inside.push_back(k);
        double lb = std::fabs(d - a.expanded[k]);
        if (a.status[k] == EXPOSED && lb <= reach) out.order.push_back({lb, k});
    });
    std::sort(out.near.begin(), out.near.end());
    sort_nearest(out.order);
    auto filter = [&](const uint32_t* r0, const uint32_t* r1, std::vector<uint32_t>& dst) {
        for (const uint32_t* p = r0; p != r1; p++)
            if (std::binary_search(out.near.begin(), out.near.end(), *p)) dst.push_back(*p);
    };
    for (auto& o : out.order) {
        out.spheres.push_back(o.second);
        filter(a.neighbors.row_begin(o.second), a.neighbors.row_end(o.second), out.s_blk);
        out.s_off.push_back(uint32_t(out.s_blk.size()));
    }
    out.order.clear();
    circle_cells.for_each_near(b, reach + rho_max, [&](uint32_t ci) {
        const Circle& c = a.circles[ci];
        V3 y = b - c.center;
        double along = y.dot(c.axis);
        double wl = (y - c.axis * along).norm();
        double dist = std::sqrt(along * along + (wl - c.radius) * (wl - c.radius));
        if (dist <= reach) out.order.push_back({dist, ci});
    });
    sort_nearest(out.order);
    for (auto& o : out.order) {
        out.circles.push_back(o.second);
        filter(a.circle_blockers.row_begin(o.second), a.circle_blockers.row_end(o.second), out.c_blk);
        out.c_off.push_back(uint32_t(out.c_blk.size()));
    }
    out.order.clear();
    vertex_cells.for_each_near(b, reach, [&](uint32_t vi) {
        double d = b.dist(a.vertices[vi].position);
        if (d <= reach) out.order.push_back({d, vi});
    });
    sort_nearest(out.order);
    for (auto& o : out.order) out.vertices.push_back(o.second);
    out.order.clear();
}

// point.rs:686-738 (SES branch)
NearEval SesField::eval_local(const V3& x, double band, const LocalCandidates& l) const {
    const Arrangement& a = arr;
    if (kind != KIND_SES) {  // point.rs:723-736
        double best = band;
        int64_t bi = -1;
        for (uint32_t k : l.inside) {
            double v = x.dist(a.centers[k]) - a.expanded[k];
            if (v < best) best = v, bi = k;
        }
        return NearEval{best, bi < 0 ? Feature{F_BEYOND, 0} : Feature{F_SPHERE, uint32_t(bi)}, x};
    }
    bool inside = false;
    for (uint32_t k : l.inside)
        if (x.dist(a.centers[k]) < a.expanded[k]) {
            inside = true;
            break;
        }
    if (!inside) return NearEval{probe, Feature{F_SOLVENT, 0}, x};
    PointEval best{probe + band, x, Feature{F_BEYOND, 0}};
    for (size_t k = 0; k < l.spheres.size(); k++)
        try_sphere_with(x, l.spheres[k], l.s_blk.data() + l.s_off[k], l.s_blk.data() + l.s_off[k + 1], best);
    for (size_t k = 0; k < l.circles.size(); k++)
        try_circle_with(x, l.circles[k], l.c_blk.data() + l.c_off[k], l.c_blk.data() + l.c_off[k + 1], best);
    for (uint32_t vi : l.vertices) try_vertex(x, vi, best);
    return NearEval{probe - best.distance, best.feature, best.closest};
}

// point.rs:742-757
std::pair<double, int64_t> SesField::sphere_eval(const V3& x, double cutoff) const {
    const Arrangement& a = arr;
    std::pair<double, int64_t> best{cutoff, -1};
    a.cells.for_each_near(x, cutoff + a.max_expanded, [&](uint32_t k) {
        if (a.status[k] == CONTAINED) return;
        double v = x.dist(a.centers[k]) - a.expanded[k];
        if (v < best.first) best = {v, int64_t(k)};
    });
    return best;
}

// point.rs:760-765
double SesField::clamped_value(const V3& x, double band) const {
    if (kind != KIND_SES) return sphere_eval(x, band).first;
    return probe - ses_eval(x, probe + band).distance;
}

// point.rs:304-349 (SES): value with the growing cutoff, and the normal.
double SesField::value(const V3& x, V3* normal, bool* has_normal) const {
    if (has_normal) *has_normal = false;
    if (arr.centers.empty()) return kind == KIND_SES ? probe : INFINITY;
    if (kind != KIND_SES) {  // point.rs:340-370
        double cutoff = 4.0;
        std::pair<double, int64_t> r;
        for (;;) {
            r = sphere_eval(x, cutoff);
            if (r.second >= 0 || cutoff > extent) break;
            cutoff *= 2.0;
        }
        if (r.second >= 0) {
            V3 dir = x - arr.centers[size_t(r.second)];
            double len = dir.norm();
            if (len > 1e-12) {
                if (normal) *normal = dir / len;
                if (has_normal) *has_normal = true;
            }
        }
        return r.first;
    }
    double cutoff = probe + 4.0;
    PointEval e;
    for (;;) {
        e = ses_eval(x, cutoff);
        if (e.feature.kind != F_BEYOND || cutoff > extent) break;
        cutoff *= 2.0;
    }
    bool solvent = e.feature.kind == F_SOLVENT || e.feature.kind == F_BEYOND;
    V3 to_p = e.closest - x;
    if (!solvent && to_p.norm() > 1e-12) {
        if (normal) *normal = to_p.normalized();
        if (has_normal) *has_normal = true;
    }
    return probe - e.distance;
}

// ---- lattice.rs --------------------------------------------------------------
// lattice.rs:36-45; Rust f64::round is half away from zero, like C round().
void Lattice::init(double h_, size_t b_, const V3& fc) {
    h = h_;
    b = int64_t(b_);
    double v[3] = {fc.x, fc.y, fc.z};
    for (int a = 0; a < 3; a++) frame[a] = sat_i64(std::round(v[a] / h));
    h32 = float(h);
}

// lattice.rs:72-75
V3 Lattice::brick_center(const int32_t k[3]) const {
    auto c = [&](int32_t v) { return (double(v) + 0.5) * double(b) * h; };
    return V3(c(k[0]), c(k[1]), c(k[2]));
}

// lattice.rs:93-101
uint64_t pack_key(const int32_t k[3]) {
    uint64_t r = 0;
    for (int a = 0; a < 3; a++) r |= uint64_t(int64_t(k[a]) + KEY_BIAS) << (21 * a);
    return r;
}
void unpack_key(uint64_t p, int32_t k[3]) {
    for (int a = 0; a < 3; a++) k[a] = int32_t(int64_t((p >> (21 * a)) & 0x1fffff) - KEY_BIAS);
}

// lattice.rs:105-163
std::vector<uint64_t> touched_bricks(const Engine& e, std::string& err) {
    const Arrangement& a = e.field.arr;
    const Lattice& L = e.lattice;
    size_t n = a.centers.size();
    std::vector<std::vector<uint64_t>> per(n);
    std::vector<uint8_t> bad(n, 0);
    parallel_for(n, [&](size_t i, int) {
        if (a.status[i] == CONTAINED) return;
        double r = a.expanded[i] + CLASSIFY_EPS;
        const V3& c = a.centers[i];
        int64_t lo[3] = {L.brick_of(c.x - r), L.brick_of(c.y - r), L.brick_of(c.z - r)};
        int64_t hi[3] = {L.brick_of(c.x + r), L.brick_of(c.y + r), L.brick_of(c.z + r)};
        for (int k = 0; k < 3; k++)
            if (std::llabs(lo[k]) >= KEY_BIAS - 1 || std::llabs(hi[k]) >= KEY_BIAS - 1) {
                bad[i] = 1;
                return;
            }
        auto& keys = per[i];
        for (int64_t z = lo[2]; z <= hi[2]; z++)
            for (int64_t y = lo[1]; y <= hi[1]; y++)
                for (int64_t x = lo[0]; x <= hi[0]; x++) {
                    int32_t k[3] = {int32_t(x), int32_t(y), int32_t(z)};
                    keys.push_back(pack_key(k));
                }
    });
    for (size_t i = 0; i < n; i++)
        if (bad[i]) {
            err = "coordinates too far from the origin for the grid spacing";
            return {};
        }
    std::vector<uint64_t> keys;
    for (auto& v : per) keys.insert(keys.end(), v.begin(), v.end());
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    return keys;
}

// lattice.rs:190-227; returns 1 (uniformly outside), 0 (inside) or -1.
int uniform_sign(const SesField& f, const V3& center, double rho) {
    const Arrangement& a = f.arr;
    double margin = rho + CLASSIFY_EPS;
    double s_sas = INFINITY, s_vdw = INFINITY;
    a.cells.for_each_near(center, margin + a.max_expanded, [&](uint32_t k) {
        if (a.status[k] != CONTAINED) {
            double d = center.dist(a.centers[k]);
            s_sas = std::fmin(s_sas, d - a.expanded[k]);
            s_vdw = std::fmin(s_vdw, d - a.radii[k]);
        }
    });
    if (f.kind != KIND_SES) {  // lattice.rs:213-215: the sign of s_sas alone
        if (s_sas > margin) return 1;
        if (s_sas < -margin) return 0;
        return -1;
    }
    if (s_sas >= margin) return 1;
    if (s_vdw <= -margin) return 0;
    double cutoff = f.probe + margin + CLASSIFY_EPS;
    double v = f.probe - f.ses_eval(center, cutoff).distance;
    if (v > margin) return 1;
    if (v < -margin) return 0;
    return -1;
}

// lattice.rs:168-181
std::vector<std::array<int32_t, 3>> surface_bricks(const Engine& e, const std::vector<uint64_t>& touched) {
    double rho = e.lattice.brick_radius();
    std::vector<uint8_t> keep(touched.size());
    parallel_for(touched.size(), [&](size_t t, int) {
        int32_t k[3];
        unpack_key(touched[t], k);
        keep[t] = uniform_sign(e.field, e.lattice.brick_center(k), rho) < 0;
    });
    std::vector<std::array<int32_t, 3>> out;
    for (size_t t = 0; t < touched.size(); t++)
        if (keep[t]) {
            int32_t k[3];
            unpack_key(touched[t], k);
            out.push_back({k[0], k[1], k[2]});
        }
    return out;
}

// ---- kernel.rs ----------------------------------------------------------------
static constexpr float INSIDE_TOL = 2e-5f;
static constexpr double F32_MAX_COORD = 2000.0;
static constexpr size_t MAX_LANES = 16;

void Gathered::clear() {
    for (auto* v : {&nx, &ny, &nz, &nr, &nr2, &nr2tol, &sx, &sy, &sz, &sr, &cx, &cy, &cz, &ux, &uy, &uz, &ex,
                    &ey, &ez, &rho, &vx, &vy, &vz})
        v->clear();
    n_inside = 0;
    s_off.assign(1, 0);
    s_blk.clear();
    c_off.assign(1, 0);
    c_blk.clear();
    near_ids.clear();
    s_ids.clear();
    c_ids.clear();
    v_ids.clear();
}

// kernel.rs:204-271 (spacing and brick checks, frame, band, f32_ok, coord_max)
std::string make_engine(SesField&& field, double spacing, size_t brick, Engine& E) {
    if (!(std::isfinite(spacing) && spacing >= 0.01)) return "grid spacing must be at least 0.01";
    if (brick < 2 || brick > 32) return "brick size must be 2..=32 cells";
    E.field = std::move(field);
    const Arrangement& a = E.field.arr;
    V3 center;
    double half = 0.0;
    if (!a.centers.empty()) {
        V3 lo = a.centers[0], hi = a.centers[0];
        for (auto& c : a.centers) lo = lo.vmin(c), hi = hi.vmax(c);
        V3 d = hi - lo;
        center = (lo + hi) * 0.5;
        half = 0.5 * std::fmax(std::fmax(d.x, d.y), d.z);
    }
    E.lattice.init(spacing, brick, center);
    double reach = half + 2.0 * a.max_expanded + 2.0 * E.field.probe + 4.0 * double(brick) * spacing;
    E.f32_ok = reach < F32_MAX_COORD && reach / spacing < double(1u << 23);
    E.band = std::sqrt(3.0) * spacing * 1.01;
    E.coord_max = std::fmax(std::fmax(std::fabs(center.x), std::fabs(center.y)), std::fabs(center.z)) + half +
                  a.max_expanded + E.field.probe + 2.0 * E.band;
    int64_t b = E.lattice.b;
    E.sub = (b % 2 == 0 && b >= 4) ? b / 2 : b;
    E.nsub = b / E.sub;
    return "";
}

void BrickScratch::init(const Engine& e) {
    size_t padded = (e.samples_per_brick() + MAX_LANES - 1) / MAX_LANES * MAX_LANES;
    xs.assign(padded, 0.f);
    ys.assign(padded, 0.f);
    zs.assign(padded, 0.f);
    out.assign(padded, 0.f);
    values.assign(padded, 0.f);
    local_of.assign(e.field.arr.centers.size(), UINT32_MAX);
    touched.clear();
}

// kernel.rs:467-482
void sub_states(const Engine& e, const int32_t key[3], int st[8]) {
    for (int i = 0; i < 8; i++) st[i] = -1;
    if (e.nsub != 2) return;
    const Lattice& L = e.lattice;
    V3 base = L.point(int64_t(key[0]) * L.b, int64_t(key[1]) * L.b, int64_t(key[2]) * L.b);
    double h = L.h;
    double rho = 0.5 * std::sqrt(3.0) * double(e.sub) * h;
    for (int i = 0; i < 8; i++) {
        double half = double(e.sub) * 0.5;
        auto off = [&](int bit) { return double((i >> bit) & 1) * double(e.sub) + half; };
        V3 center = base + V3(off(0), off(1), off(2)) * h;
        st[i] = uniform_sign(e.field, center, rho);
    }
}

// Sub-block centre and radius as prepare_sub computes them (kernel.rs:575-583).
V3 sub_center(const Engine& e, const int32_t key[3], int sb, double* rho) {
    const Lattice& L = e.lattice;
    V3 base = L.point(int64_t(key[0]) * L.b, int64_t(key[1]) * L.b, int64_t(key[2]) * L.b);
    double h = L.h;
    double sub_rho = 0.5 * std::sqrt(3.0) * double(e.sub) * h, half = double(e.sub) * 0.5;
    if (e.nsub == 2) {
        auto off = [&](int bit) { return double((sb >> bit) & 1) * double(e.sub) + half; };
        *rho = sub_rho;
        return base + V3(off(0), off(1), off(2)) * h;
    }
    *rho = L.brick_radius();
    return L.brick_center(key);
}

// kernel.rs:489-546
static void assign(const Engine& e, const int32_t key[3], const int state[8], BrickScratch& s) {
    const Lattice& L = e.lattice;
    int64_t b = L.b, side = b + 1;
    int64_t origin[3] = {int64_t(key[0]) * b, int64_t(key[1]) * b, int64_t(key[2]) * b};
    float band = float(e.band);
    int64_t sub = e.sub, nsub = e.nsub;
    auto range = [&](int64_t v, int64_t& lo, int64_t& hi) {
        hi = std::min(v / sub, nsub - 1);
        lo = (v > 0 && v % sub == 0) ? std::min(v / sub - 1, nsub - 1) : hi;
    };
    for (auto& g : s.groups) g.clear();
    size_t i = 0;
    for (int64_t z = 0; z < side; z++) {
        int64_t z0, z1;
        range(z, z0, z1);
        for (int64_t y = 0; y < side; y++) {
            int64_t y0, y1;
            range(y, y0, y1);
            for (int64_t x = 0; x < side; x++) {
                int64_t x0, x1;
                range(x, x0, x1);
                int owner = -1;
                bool positive = true;
                for (int64_t sz = z0; sz <= z1 && owner < 0; sz++)
                    for (int64_t sy = y0; sy <= y1 && owner < 0; sy++)
                        for (int64_t sx = x0; sx <= x1; sx++) {
                            int sb = int(sx + 2 * sy + 4 * sz);
                            if (state[sb] < 0) {
                                owner = sb;
                                break;
                            }
                            positive = state[sb] == 1;
                        }
                if (owner < 0) {
                    s.values[i] = positive ? band : -band;
                } else if (e.f32_ok) {
                    s.groups[owner].push_back(uint32_t(i));
                } else {
                    V3 p = L.point(origin[0] + x, origin[1] + y, origin[2] + z);
                    s.values[i] = float(e.field.clamped_value(p, e.band));
                }
                i++;
            }
        }
    }
}

// kernel.rs:614-651 (two passes: spheres that can contain a sample first)
static void gather_near(const Engine& e, const V3& b, double rho, double reach, BrickScratch& s) {
    const Arrangement& a = e.field.arr;
    V3 frame = e.lattice.frame_origin();
    s.g.clear();
    s.touched.clear();
    for (int pass = 0; pass < 2; pass++) {
        a.cells.for_each_near(b, reach + a.max_expanded, [&](uint32_t k) {
            double r = a.expanded[k];
            double d = b.dist(a.centers[k]);
            bool contains_sample = d < r + rho;
            if (a.status[k] == CONTAINED || d >= r + reach || contains_sample != (pass == 0)) return;
            s.local_of[k] = uint32_t(s.g.nx.size());
            s.touched.push_back(k);
            V3 c = a.centers[k] - frame;
            s.g.nx.push_back(float(c.x));
            s.g.ny.push_back(float(c.y));
            s.g.nz.push_back(float(c.z));
            float r32 = float(r);
            s.g.nr.push_back(r32);
            s.g.nr2.push_back(r32 * r32);
            float rt = std::fmax(r32 - INSIDE_TOL, 0.0f);
            s.g.nr2tol.push_back(rt * rt);
            s.g.near_ids.push_back(k);
        });
        if (pass == 0) s.g.n_inside = s.g.nx.size();
    }
}

// kernel.rs:671-752
void gather_ses(const Engine& e, const V3& b, double rho, BrickScratch& s) {
    const Arrangement& a = e.field.arr;
    const SesField& F = e.field;
    V3 frame = e.lattice.frame_origin();
    double reach = F.probe + e.band + rho;
    gather_near(e, b, rho, reach, s);
    Gathered& g = s.g;
    s.order.clear();
    for (uint32_t k : s.touched) {
        if (a.status[k] != EXPOSED) continue;
        double lb = std::fabs(b.dist(a.centers[k]) - a.expanded[k]);
        if (lb <= reach) s.order.push_back({lb, k});
    }
    sort_nearest(s.order);
    for (auto& o : s.order) {
        uint32_t k = o.second, local = s.local_of[k];
        g.sx.push_back(g.nx[local]);
        g.sy.push_back(g.ny[local]);
        g.sz.push_back(g.nz[local]);
        g.sr.push_back(g.nr[local]);
        for (const uint32_t* p = a.neighbors.row_begin(k); p != a.neighbors.row_end(k); p++) {
            uint32_t l = s.local_of[*p];
            if (l != UINT32_MAX) g.s_blk.push_back(l);
        }
        g.s_off.push_back(uint32_t(g.s_blk.size()));
        g.s_ids.push_back(k);
    }
    s.order.clear();
    F.circle_cells.for_each_near(b, reach + F.rho_max, [&](uint32_t ci) {
        const Circle& c = a.circles[ci];
        V3 y = b - c.center;
        double along = y.dot(c.axis);
        double wl = (y - c.axis * along).norm();
        double dist = std::sqrt(along * along + (wl - c.radius) * (wl - c.radius));
        if (dist <= reach) s.order.push_back({dist, ci});
    });
    sort_nearest(s.order);
    for (auto& o : s.order) {
        const Circle& c = a.circles[o.second];
        V3 m = c.center - frame;
        g.cx.push_back(float(m.x));
        g.cy.push_back(float(m.y));
        g.cz.push_back(float(m.z));
        g.ux.push_back(float(c.axis.x));
        g.uy.push_back(float(c.axis.y));
        g.uz.push_back(float(c.axis.z));
        g.ex.push_back(float(c.e1.x));
        g.ey.push_back(float(c.e1.y));
        g.ez.push_back(float(c.e1.z));
        g.rho.push_back(float(c.radius));
        for (const uint32_t* p = a.circle_blockers.row_begin(o.second); p != a.circle_blockers.row_end(o.second); p++) {
            uint32_t l = s.local_of[*p];
            if (l != UINT32_MAX) g.c_blk.push_back(l);
        }
        g.c_off.push_back(uint32_t(g.c_blk.size()));
        g.c_ids.push_back(o.second);
    }
    F.vertex_cells.for_each_near(b, reach, [&](uint32_t vi) {
        const V3& p = a.vertices[vi].position;
        if (b.dist(p) <= reach) {
            V3 q = p - frame;
            g.vx.push_back(float(q.x));
            g.vy.push_back(float(q.y));
            g.vz.push_back(float(q.z));
            g.v_ids.push_back(vi);
        }
    });
    for (uint32_t k : s.touched) s.local_of[k] = UINT32_MAX;
}

// kernel.rs:837-952, one lane: the SIMD kernel's per-lane result does not
// depend on the vector width (masks only narrow; early exits skip work whose
// lanes are all masked off), so a scalar loop gives the same bits.
static float ses_sample(const Gathered& g, float x, float y, float z, float probe, float cutoff2) {
    bool inside = false;
    for (size_t k = 0; k < g.n_inside; k++) {
        float dx = x - g.nx[k], dy = y - g.ny[k], dz = z - g.nz[k];
        inside |= (dx * dx + dy * dy + dz * dz) < g.nr2[k];
    }
    if (!inside) return probe;
    float best2 = cutoff2;
    for (size_t v = 0; v < g.vx.size(); v++) {
        float dx = x - g.vx[v], dy = y - g.vy[v], dz = z - g.vz[v];
        best2 = std::fmin(best2, dx * dx + dy * dy + dz * dz);
    }
    for (size_t si = 0; si < g.sx.size(); si++) {
        float cx = g.sx[si], cy = g.sy[si], cz = g.sz[si], r = g.sr[si];
        float dx = x - cx, dy = y - cy, dz = z - cz;
        float dist = std::sqrt(dx * dx + dy * dy + dz * dz);
        float lb = std::fabs(dist - r);
        float lb2 = lb * lb;
        bool valid = lb2 < best2 && 1e-6f < dist;
        if (!valid) continue;
        float scale = r / dist;
        float qx = cx + dx * scale, qy = cy + dy * scale, qz = cz + dz * scale;
        for (uint32_t p = g.s_off[si]; p < g.s_off[si + 1] && valid; p++) {
            uint32_t k = g.s_blk[p];
            float ex = qx - g.nx[k], ey = qy - g.ny[k], ez = qz - g.nz[k];
            valid = (ex * ex + ey * ey + ez * ez) >= g.nr2tol[k];
        }
        if (valid) best2 = lb2;
    }
    for (size_t ci = 0; ci < g.cx.size(); ci++) {
        float mx = g.cx[ci], my = g.cy[ci], mz = g.cz[ci];
        float ux = g.ux[ci], uy = g.uy[ci], uz = g.uz[ci];
        float rho = g.rho[ci];
        float yx = x - mx, yy = y - my, yz = z - mz;
        float along = yx * ux + yy * uy + yz * uz;
        float wx = yx - ux * along, wy = yy - uy * along, wz = yz - uz * along;
        float wl = std::sqrt(wx * wx + wy * wy + wz * wz);
        float t = wl - rho;
        float d2 = along * along + t * t;
        bool valid = d2 < best2;
        if (!valid) continue;
        bool degenerate = wl < 1e-6f;
        float sc = rho / wl;
        float qx = degenerate ? mx + g.ex[ci] * rho : mx + wx * sc;
        float qy = degenerate ? my + g.ey[ci] * rho : my + wy * sc;
        float qz = degenerate ? mz + g.ez[ci] * rho : mz + wz * sc;
        for (uint32_t p = g.c_off[ci]; p < g.c_off[ci + 1] && valid; p++) {
            uint32_t k = g.c_blk[p];
            float ex = qx - g.nx[k], ey = qy - g.ny[k], ez = qz - g.nz[k];
            valid = (ex * ex + ey * ey + ez * ez) >= g.nr2tol[k];
        }
        if (valid) best2 = d2;
    }
    return probe - std::sqrt(best2);
}

// sphere_kernel (kernel.rs:957-981) at one point: the clamped union of
// spheres, min(band, min_k(|x - c_k| - R_k)) over every gathered sphere.
static float sphere_sample(const Gathered& g, float x, float y, float z, float band) {
    float best = band;
    for (size_t k = 0; k < g.nx.size(); k++) {
        float dx = x - g.nx[k], dy = y - g.ny[k], dz = z - g.nz[k];
        best = std::fmin(best, std::sqrt(dx * dx + dy * dy + dz * dz) - g.nr[k]);
    }
    return best;
}

// kernel.rs:415-446 with prepare_sub (kernel.rs:553-600)
void evaluate(const Engine& e, const int32_t key[3], BrickScratch& s) {
    int state[8];
    sub_states(e, key, state);
    assign(e, key, state, s);
    if (!e.f32_ok) return;
    float probe = float(e.field.probe);
    float cutoff = float(e.field.probe + e.band);
    float cutoff2 = cutoff * cutoff;
    const Lattice& L = e.lattice;
    int64_t side = L.b + 1;
    int64_t origin[3] = {int64_t(key[0]) * L.b, int64_t(key[1]) * L.b, int64_t(key[2]) * L.b};
    int nsb = int(e.nsub * e.nsub * e.nsub);
    for (int sb = 0; sb < nsb; sb++) {
        const auto& grp = s.groups[sb];
        if (grp.empty()) continue;
        for (size_t j = 0; j < grp.size(); j++) {
            size_t i = grp[j];
            int64_t x = int64_t(i) % side, y = (int64_t(i) / side) % side, z = int64_t(i) / (side * side);
            s.xs[j] = L.local(origin[0] + x, 0);
            s.ys[j] = L.local(origin[1] + y, 1);
            s.zs[j] = L.local(origin[2] + z, 2);
        }
        double rho;
        V3 center = sub_center(e, key, sb, &rho);
        if (e.field.kind != KIND_SES) {
            // gather_spheres + sphere_kernel (kernel.rs:651-654, 957-981).
            gather_near(e, center, rho, e.band + rho, s);
            for (size_t j = 0; j < grp.size(); j++)
                s.values[grp[j]] = sphere_sample(s.g, s.xs[j], s.ys[j], s.zs[j], float(e.band));
            continue;
        }
        gather_ses(e, center, rho, s);
        for (size_t j = 0; j < grp.size(); j++)
            s.values[grp[j]] = ses_sample(s.g, s.xs[j], s.ys[j], s.zs[j], probe, cutoff2);
    }
}

}  // namespace orc
