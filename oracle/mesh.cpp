// Oracle (test infrastructure): marching cubes with exact f64 refinement,
// assembly, components, measurement and the OBJ writer.  Restates
// crates/sesmesh/src/mesh/{extract.rs,tables.rs,mod.rs,post.rs} and
// crates/sesmesh/src/export/{obj.rs,fmt.rs}.
#include "oracle.hpp"

#include <algorithm>
#include <chrono>
#include <unordered_map>

#include "../sesmesh_b200/csrc/mc_table.inc"

namespace orc {

static constexpr int MAX_ITER = 8;      // extract.rs:29
static constexpr int MAX_BISECT = 64;   // extract.rs:33
static constexpr double TOL = 1e-5;     // extract.rs:35
static constexpr double T_MIN = 1e-4;   // extract.rs:40
static constexpr uint32_t CODE_SHIFT = 28;
static constexpr uint32_t ID_MASK = (1u << CODE_SHIFT) - 1;
static const uint8_t EDGE_LOWER[3][4] = {{0, 2, 4, 6}, {0, 1, 4, 5}, {0, 1, 2, 3}};  // tables.rs:27

static inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

// extract.rs:47-51
double edge_clamp(const Engine& e) {
    float m = float(clampd(e.coord_max, 1.0, double(3.4028234663852886e38f) / 4.0));
    uint32_t bits;
    std::memcpy(&bits, &m, 4);
    bits += 1;
    float next;
    std::memcpy(&next, &bits, 4);
    double ulp = double(next - m);
    return clampd(4.0 * ulp / e.lattice.h, T_MIN, 0.25);
}

// extract.rs:539-549
static bool gradient(const SesField& f, const V3& x, const NearEval& e, V3& out) {
    if (e.feature.kind == F_SOLVENT || e.feature.kind == F_BEYOND) return false;
    if (f.kind != KIND_SES && e.feature.kind != F_SPHERE) return false;
    V3 w = f.kind == KIND_SES ? e.closest - x : x - f.arr.centers[e.feature.id];
    double len = w.norm();
    if (!(len > 1e-12)) return false;
    out = w / len;
    return true;
}

// extract.rs:553-597 (SES)
static void attributes(const Engine& E, const V3& v, const NearEval& e, const V3& outward, V3& normal,
                       uint8_t& patch, uint32_t& atom) {
    const Arrangement& a = E.field.arr;
    auto unit = [&](const V3& w) {
        double len = w.norm();
        return len > 1e-9 ? w / len : outward;
    };
    auto nearest = [&](const uint32_t* atoms, int n) {
        double best = INFINITY;
        uint32_t bi = atoms[0];
        for (int q = 0; q < n; q++) {
            uint32_t k = atoms[q];
            double d = v.dist(a.centers[k]) - a.radii[k];
            if (d < best) best = d, bi = k;
        }
        return a.orig[bi];
    };
    if (E.field.kind != KIND_SES && e.feature.kind == F_SPHERE) {  // extract.rs:583-587
        normal = unit(v - a.centers[e.feature.id]), patch = 0, atom = a.orig[e.feature.id];
        return;
    }
    switch (E.field.kind != KIND_SES ? uint32_t(F_BEYOND) : e.feature.kind) {
        case F_SPHERE:
            normal = unit(e.closest - v), patch = 0, atom = a.orig[e.feature.id];
            return;
        case F_CIRCLE: {
            const Circle& c = a.circles[e.feature.id];
            uint32_t at[2] = {c.i, c.j};
            normal = unit(e.closest - v), patch = 1, atom = nearest(at, 2);
            return;
        }
        case F_VERTEX:
            normal = unit(e.closest - v), patch = 2, atom = nearest(a.vertices[e.feature.id].atoms, 3);
            return;
        default: {
            auto r = E.field.sphere_eval(v, E.field.probe + E.band + 8.0);
            normal = outward, patch = 0, atom = r.second < 0 ? 0 : a.orig[size_t(r.second)];
        }
    }
}

// extract.rs:425-535 (exact refinement)
static void vertex(const Engine& E, const V3& pa, const V3& pb, double fa, double fb, double t_min,
                   const LocalCandidates& local, BrickMesh& out) {
    const SesField& field = E.field;
    double band = E.band;
    V3 d = pb - pa;
    double t = clampd(fa / (fa - fb), 0.0, 1.0);
    NearEval last{};
    bool have_last = false;
    double t0 = 0.0, g0 = fa, t1 = 1.0, g1 = fb;
    int side = 0;
    bool converged = false;
    for (int it = 0; it < MAX_ITER; it++) {
        NearEval e = field.eval_local(pa + d * t, band, local);
        out.evals++;
        last = e, have_last = true;
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
        V3 n;
        double slope = gradient(field, pa + d * t, e, n) ? n.dot(d) : 0.0;
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
            NearEval e = field.eval_local(pa + d * t, band, local);
            out.evals++;
            last = e, have_last = true;
            if (std::fabs(e.value) <= TOL || (t1 - t0) * len <= 2.0 * TOL) break;
            if ((e.value < 0.0) == neg0) t0 = t;
            else t1 = t;
        }
    }
    V3 v = pa + d * clampd(t, t_min, 1.0 - t_min);
    if (!have_last) {
        out.evals++;
        last = field.eval_local(v, band, local);
    }
    V3 outward = (fa < 0.0 ? d : d * -1.0).normalized();
    V3 normal;
    uint8_t patch;
    uint32_t atom;
    attributes(E, v, last, outward, normal, patch, atom);
    out.positions.push_back({float(v.x), float(v.y), float(v.z)});
    out.normals.push_back({float(normal.x), float(normal.y), float(normal.z)});
    out.atoms.push_back(atom);
    out.patches.push_back(patch);
}

// extract.rs:226-265
void cells_pass(size_t b, const float* values, BrickMesh& out) {
    size_t s = b + 1;
    size_t corner_step[8];
    for (int c = 0; c < 8; c++) corner_step[c] = size_t(c & 1) + size_t((c >> 1) & 1) * s + size_t((c >> 2) & 1) * s * s;
    for (size_t z = 0; z < b; z++)
        for (size_t y = 0; y < b; y++)
            for (size_t x = 0; x < b; x++) {
                size_t i0 = (z * s + y) * s + x;
                int cs = 0;
                for (int c = 0; c < 8; c++)
                    if (values[i0 + corner_step[c]] < 0.0f) cs |= 1 << c;
                if (cs == 0 || cs == 255) continue;
                for (int t = SMB_TRI_OFFSET[cs]; t < SMB_TRI_OFFSET[cs + 1]; t++) {
                    std::array<uint32_t, 3> tri;
                    for (int k = 0; k < 3; k++) {
                        int e = SMB_TRI_EDGES[t][k];
                        int axis = e / 4, lo = EDGE_LOWER[axis][e % 4];
                        size_t l[3] = {x + size_t(lo & 1), y + size_t((lo >> 1) & 1), z + size_t((lo >> 2) & 1)};
                        uint32_t code = 0;
                        size_t lc[3] = {0, 0, 0};
                        for (int a = 0; a < 3; a++) {
                            if (l[a] == b) code |= 1u << a;
                            else lc[a] = l[a];
                        }
                        tri[k] = (code << CODE_SHIFT) | uint32_t(((lc[2] * b + lc[1]) * b + lc[0]) * 3 + size_t(axis));
                    }
                    out.tris.push_back(tri);
                }
            }
}

// extract.rs:146-219
void mesh_brick(const Engine& E, const int32_t key[3], const float* values, BrickMesh& out) {
    const Lattice& L = E.lattice;
    size_t b = size_t(L.b), s = b + 1;
    size_t stride[3] = {1, s, s * s};
    int64_t origin[3] = {int64_t(key[0]) * L.b, int64_t(key[1]) * L.b, int64_t(key[2]) * L.b};
    size_t sub = (b % 2 == 0 && b >= 4) ? b / 2 : b;
    size_t nsub = b / sub;
    double h = L.h;
    V3 base = L.point(origin[0], origin[1], origin[2]);
    double rho = 0.5 * std::sqrt(3.0) * double(sub) * h * (1.0 + 1e-9) + 1e-9;
    LocalCandidates locals[8];
    bool have[8] = {false};
    double t_min = edge_clamp(E);
    for (size_t z = 0; z < b; z++)
        for (size_t y = 0; y < b; y++)
            for (size_t x = 0; x < b; x++) {
                size_t i = (z * s + y) * s + x;
                float va = values[i];
                for (int axis = 0; axis < 3; axis++) {
                    float vb = values[i + stride[axis]];
                    if ((va < 0.0f) == (vb < 0.0f)) continue;
                    int64_t ia[3] = {origin[0] + int64_t(x), origin[1] + int64_t(y), origin[2] + int64_t(z)};
                    int64_t ib[3] = {ia[0], ia[1], ia[2]};
                    ib[axis] += 1;
                    V3 pa = L.point(ia[0], ia[1], ia[2]), pb = L.point(ib[0], ib[1], ib[2]);
                    size_t sb[3] = {std::min(x / sub, nsub - 1), std::min(y / sub, nsub - 1), std::min(z / sub, nsub - 1)};
                    size_t si = sb[0] + 2 * sb[1] + 4 * sb[2];
                    if (!have[si]) {
                        V3 center = base + V3(double(sb[0] * sub) + 0.5 * double(sub), double(sb[1] * sub) + 0.5 * double(sub),
                                              double(sb[2] * sub) + 0.5 * double(sub)) *
                                               h;
                        E.field.gather_local(center, rho, E.band, locals[si]);
                        have[si] = true;
                    }
                    vertex(E, pa, pb, double(va), double(vb), t_min, locals[si], out);
                    out.edges.push_back(uint32_t(((z * b + y) * b + x) * 3 + size_t(axis)));
                }
            }
    cells_pass(b, values, out);
    out.vertex_end.push_back(uint32_t(out.edges.size()));
    out.tri_end.push_back(uint32_t(out.tris.size()));
}

// extract.rs:606-691, all bricks in one part.
std::string assemble(const std::vector<std::array<int32_t, 3>>& bricks, const BrickMesh& p, Mesh& mesh) {
    size_t nb = bricks.size();
    std::vector<size_t> vstart(nb + 1, 0), tstart(nb + 1, 0);
    for (size_t i = 0; i < nb; i++) vstart[i + 1] = p.vertex_end[i], tstart[i + 1] = p.tri_end[i];
    if (p.edges.size() > UINT32_MAX) return "mesh with too many vertices";
    std::unordered_map<uint64_t, uint32_t> index;
    index.reserve(nb * 2);
    for (size_t i = 0; i < nb; i++) index[pack_key(bricks[i].data())] = uint32_t(i);
    mesh.triangles.resize(p.tris.size());
    std::string err;
    std::vector<std::string> errs(nb);
    parallel_for(nb, [&](size_t bi, int) {
        const auto& key = bricks[bi];
        int64_t cache[8];
        for (auto& c : cache) c = -1;
        cache[0] = int64_t(bi);
        for (size_t t = tstart[bi]; t < tstart[bi + 1]; t++) {
            for (int k = 0; k < 3; k++) {
                uint32_t r = p.tris[t][k];
                uint32_t code = r >> CODE_SHIFT;
                if (cache[code] < 0) {
                    int32_t nk[3] = {key[0] + int32_t(code & 1), key[1] + int32_t((code >> 1) & 1), key[2] + int32_t((code >> 2) & 1)};
                    auto it = index.find(pack_key(nk));
                    if (it == index.end()) {
                        errs[bi] = "triangle references an edge of a missing brick";
                        return;
                    }
                    cache[code] = it->second;
                }
                size_t target = size_t(cache[code]);
                uint32_t id = r & ID_MASK;
                auto b0 = p.edges.begin() + vstart[target], b1 = p.edges.begin() + vstart[target + 1];
                auto pos = std::lower_bound(b0, b1, id);
                if (pos == b1 || *pos != id) {
                    errs[bi] = "triangle references an edge without vertex";
                    return;
                }
                mesh.triangles[t][k] = uint32_t(vstart[target] + size_t(pos - b0));
            }
        }
    });
    for (auto& e : errs)
        if (!e.empty()) return e;
    mesh.positions = p.positions;
    mesh.normals = p.normals;
    mesh.vertex_atom = p.atoms;
    mesh.vertex_patch = p.patches;
    return "";
}

static constexpr size_t SUM_CHUNK = size_t(1) << 14;  // mesh/mod.rs:86

// mesh/mod.rs:111-122
static void tri_area_volume(const Mesh& m, const std::array<uint32_t, 3>& t, const double o[3], double& area, double& vol) {
    double p[3][3];
    for (int v = 0; v < 3; v++)
        for (int k = 0; k < 3; k++) p[v][k] = double(m.positions[t[v]][k]) - o[k];
    auto sub = [](const double* a, const double* b, double* r) { for (int k = 0; k < 3; k++) r[k] = a[k] - b[k]; };
    auto cross = [](const double* a, const double* b, double* r) {
        r[0] = a[1] * b[2] - a[2] * b[1];
        r[1] = a[2] * b[0] - a[0] * b[2];
        r[2] = a[0] * b[1] - a[1] * b[0];
    };
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    double e1[3], e2[3], c[3], c2[3];
    sub(p[1], p[0], e1);
    sub(p[2], p[0], e2);
    cross(e1, e2, c);
    area = 0.5 * std::sqrt(dot(c, c));
    cross(p[1], p[2], c2);
    vol = dot(p[0], c2) / 6.0;
}

// mesh/mod.rs:185-297: union-find to the smallest vertex, per-component sums
// in fixed triangle chunks merged in chunk order, Euler characteristic.
void components(const Mesh& m, std::vector<uint32_t>& id, std::vector<Component>& comps) {
    size_t n = m.positions.size();
    std::vector<uint32_t> parent(n);
    for (size_t i = 0; i < n; i++) parent[i] = uint32_t(i);
    auto find = [&](uint32_t x) {
        while (parent[x] != x) {
            parent[x] = parent[parent[x]];
            x = parent[x];
        }
        return x;
    };
    auto unite = [&](uint32_t a, uint32_t b) {
        uint32_t ra = find(a), rb = find(b);
        if (ra == rb) return;
        if (ra < rb) parent[rb] = ra;
        else parent[ra] = rb;
    };
    for (auto& t : m.triangles) {
        unite(t[0], t[1]);
        unite(t[0], t[2]);
    }
    id.assign(n, 0);
    comps.clear();
    for (size_t v = 0; v < n; v++) {
        uint32_t r = find(uint32_t(v));
        if (r == v) {
            id[v] = uint32_t(comps.size());
            comps.push_back(Component());
        } else {
            id[v] = id[r];
        }
        comps[id[v]].vertices++;
    }
    double o[3] = {0, 0, 0};
    if (n) for (int k = 0; k < 3; k++) o[k] = double(m.positions[0][k]);
    size_t nt = m.triangles.size();
    for (size_t c0 = 0; c0 < nt; c0 += SUM_CHUNK) {
        size_t end = std::min(nt, c0 + SUM_CHUNK);
        struct Acc { uint32_t comp; size_t t; double a, v; };
        std::vector<Acc> acc;
        for (size_t t = c0; t < end; t++) {
            uint32_t comp = id[m.triangles[t][0]];
            double a, v;
            tri_area_volume(m, m.triangles[t], o, a, v);
            Acc* e = nullptr;
            for (auto& x : acc) if (x.comp == comp) { e = &x; break; }
            if (e) e->t++, e->a += a, e->v += v;
            else acc.push_back({comp, 1, a, v});
        }
        for (auto& x : acc) {
            comps[x.comp].triangles += x.t;
            comps[x.comp].area += x.a;
            comps[x.comp].volume += x.v;
        }
    }
    std::vector<uint64_t> edges;
    edges.reserve(3 * nt);
    for (auto& t : m.triangles)
        for (int k = 0; k < 3; k++) {
            uint32_t a = t[k], b = t[(k + 1) % 3];
            edges.push_back((uint64_t(std::min(a, b)) << 32) | std::max(a, b));
        }
    std::sort(edges.begin(), edges.end());
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
    std::vector<int64_t> ecount(comps.size(), 0);
    for (uint64_t e : edges) ecount[id[uint32_t(e >> 32)]]++;
    for (size_t c = 0; c < comps.size(); c++)
        comps[c].euler = int64_t(comps[c].vertices) - ecount[c] + int64_t(comps[c].triangles);
}

// mesh/post.rs:14-32
void group_by_component(Mesh& m, const std::vector<uint32_t>& id, std::vector<Component>& comps) {
    size_t start = 0;
    for (auto& c : comps) c.first_triangle = start, start += c.triangles;
    std::vector<size_t> next;
    for (auto& c : comps) next.push_back(c.first_triangle);
    std::vector<std::array<uint32_t, 3>> out(m.triangles.size());
    for (auto& t : m.triangles) out[next[id[t[0]]]++] = t;
    m.triangles.swap(out);
}

// mesh/mod.rs:638-700: the defect counts that compute_surface requires to
// be zero (boundary, non-manifold and misoriented edges, degenerate or
// duplicate triangles, invalid indices, bad vertices).
size_t validate_defects(const Mesh& m) {
    size_t n = m.positions.size(), bad = 0;
    for (auto& p : m.positions)
        if (!(std::isfinite(p[0]) && std::isfinite(p[1]) && std::isfinite(p[2]))) bad++;
    for (auto& q : m.normals) {
        float len2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        if (!(std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]) && std::fabs(len2 - 1.0f) < 1e-3f)) bad++;
    }
    for (auto& t : m.triangles)
        if (t[0] >= n || t[1] >= n || t[2] >= n) return bad + 1;
    double o[3] = {0, 0, 0};
    if (n) for (int k = 0; k < 3; k++) o[k] = double(m.positions[0][k]);
    for (auto& t : m.triangles) {
        double a, v;
        tri_area_volume(m, t, o, a, v);
        if (t[0] == t[1] || t[1] == t[2] || t[0] == t[2] || a == 0.0) bad++;
    }
    // Directed edge uses: (min, max, forward).
    std::vector<uint64_t> uses;
    for (auto& t : m.triangles)
        for (int k = 0; k < 3; k++) {
            uint32_t a = t[k], b = t[(k + 1) % 3];
            uses.push_back((uint64_t(std::min(a, b)) << 33) | (uint64_t(std::max(a, b)) << 1) | (a < b ? 1 : 0));
        }
    std::sort(uses.begin(), uses.end());
    for (size_t i = 0; i < uses.size();) {
        size_t j = i, fwd = 0, bwd = 0;
        while (j < uses.size() && (uses[j] >> 1) == (uses[i] >> 1)) {
            if (uses[j] & 1) fwd++;
            else bwd++;
            j++;
        }
        if (!(fwd == 1 && bwd == 1)) bad++;
        i = j;
    }
    std::vector<std::array<uint32_t, 3>> sorted(m.triangles);
    for (auto& t : sorted) std::sort(t.begin(), t.end());
    std::sort(sorted.begin(), sorted.end());
    for (size_t i = 1; i < sorted.size(); i++)
        if (sorted[i] == sorted[i - 1]) bad++;
    return bad;
}

// export/fmt.rs:30-53
void push_fixed(std::string& buf, float x, int prec) {
    static const uint64_t P10[10] = {1, 10, 100, 1000, 10000, 100000, 1000000, 10000000, 100000000, 1000000000};
    double scaled = std::nearbyint(double(x) * double(P10[prec]));
    if (!std::isfinite(scaled) || std::fabs(scaled) >= 1e18) {
        if (std::isnan(x)) { buf += "NaN"; return; }
        if (std::isinf(x)) { buf += x < 0 ? "-inf" : "inf"; return; }
        char tmp[512];
        snprintf(tmp, sizeof tmp, "%.*f", prec, double(x));
        buf += tmp;
        return;
    }
    if (std::signbit(x)) buf.push_back('-');
    uint64_t mnt = uint64_t(std::fabs(scaled));
    buf += std::to_string(mnt / P10[prec]);
    if (prec > 0) {
        buf.push_back('.');
        uint64_t f = mnt % P10[prec];
        char d[10];
        for (int k = prec - 1; k >= 0; k--) d[k] = char('0' + f % 10), f /= 10;
        buf.append(d, size_t(prec));
    }
}

// export/obj.rs:144-236 with the default options (object "ses", normals).
std::string obj_bytes(const Mesh& m, int precision, bool normals) {
    std::string out = "# sesmesh 1.3.2\no ses\n";
    normals = normals && !m.normals.empty();
    for (auto& p : m.positions) {
        out += "v ";
        for (int k = 0; k < 3; k++) {
            if (k) out.push_back(' ');
            push_fixed(out, p[k], precision);
        }
        out.push_back('\n');
    }
    if (normals)
        for (auto& p : m.normals) {
            out += "vn ";
            for (int k = 0; k < 3; k++) {
                if (k) out.push_back(' ');
                push_fixed(out, p[k], precision);
            }
            out.push_back('\n');
        }
    for (auto& t : m.triangles) {
        out.push_back('f');
        for (int k = 0; k < 3; k++) {
            std::string n = std::to_string(uint64_t(t[k]) + 1);
            out.push_back(' ');
            out += n;
            if (normals) out += "//" + n;
        }
        out.push_back('\n');
    }
    return out;
}

// surface.rs:1001-1300 with the default parameters and the CPU back end
// (mesh stage in chunks of par::chunk_len bricks, par.rs:66).
std::string compute_surface(const Sphere* s, size_t n, double probe, double spacing, size_t brick, SurfaceOut& out,
                            int kind) {
    using clk = std::chrono::steady_clock;
    auto secs = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    auto t0 = clk::now();
    SesField field;
    std::string err = build_field(s, n, probe, field, kind);
    if (!err.empty()) return err;
    Engine E;
    err = make_engine(std::move(field), spacing, brick, E);
    if (!err.empty()) return err;
    auto t1 = clk::now();
    auto touched = touched_bricks(E, err);
    if (!err.empty()) return err;
    auto bricks = surface_bricks(E, touched);
    auto t2 = clk::now();
    size_t nb = bricks.size();
    size_t chunk = std::min<size_t>(std::max<size_t>(nb / 256, 1), 4096);
    size_t nchunks = (nb + chunk - 1) / chunk;
    std::vector<BrickMesh> parts(nchunks);
    std::vector<BrickScratch> scratch(static_cast<size_t>(threads()));
    for (auto& sc : scratch) sc.init(E);
    parallel_for(nchunks, [&](size_t c, int w) {
        BrickScratch& sc = scratch[size_t(w)];
        for (size_t i = c * chunk; i < std::min(nb, (c + 1) * chunk); i++) {
            evaluate(E, bricks[i].data(), sc);
            mesh_brick(E, bricks[i].data(), sc.values.data(), parts[c]);
        }
    });
    auto t3 = clk::now();
    BrickMesh all;
    for (auto& p : parts) {
        size_t vb = all.edges.size(), tb = all.tris.size();
        all.edges.insert(all.edges.end(), p.edges.begin(), p.edges.end());
        all.positions.insert(all.positions.end(), p.positions.begin(), p.positions.end());
        all.normals.insert(all.normals.end(), p.normals.begin(), p.normals.end());
        all.atoms.insert(all.atoms.end(), p.atoms.begin(), p.atoms.end());
        all.patches.insert(all.patches.end(), p.patches.begin(), p.patches.end());
        all.tris.insert(all.tris.end(), p.tris.begin(), p.tris.end());
        for (auto v : p.vertex_end) all.vertex_end.push_back(uint32_t(vb + v));
        for (auto v : p.tri_end) all.tri_end.push_back(uint32_t(tb + v));
        all.evals += p.evals;
        BrickMesh().edges.swap(p.edges);
    }
    err = assemble(bricks, all, out.mesh);
    if (!err.empty()) return err;
    auto t4 = clk::now();
    if (validate_defects(out.mesh) != 0) return "mesh failed validation";
    std::vector<uint32_t> id;
    components(out.mesh, id, out.comps);
    group_by_component(out.mesh, id, out.comps);
    out.mesh.vertex_component = id;
    auto t5 = clk::now();
    SurfaceStats& st = out.stats;
    st.touched = touched.size();
    st.surface_bricks = nb;
    st.vertices = out.mesh.positions.size();
    st.triangles = out.mesh.triangles.size();
    st.components = out.comps.size();
    st.area = 0, st.volume = 0, st.euler = 0;
    for (auto& c : out.comps) st.area += c.area, st.volume += c.volume, st.euler += c.euler;
    st.refine_evaluations = all.evals;
    st.t_geometry = secs(t0, t1);
    st.t_classify = secs(t1, t2);
    st.t_mesh = secs(t2, t3);
    st.t_assemble = secs(t3, t4);
    st.t_measure = secs(t4, t5);
    return "";
}

}  // namespace orc
