// Oracle (test infrastructure): C entry points for the Python test suite and
// the CPU-baseline leg of the benchmark.  Never linked by the product.
#include <chrono>
#include <cstdio>

#include "oracle.hpp"

using namespace orc;

namespace {
struct Handle {
    Engine e;
};
struct SurfaceHandle {
    SurfaceOut out;
    std::string obj;
};
void set_err(char* err, size_t len, const std::string& m) {
    if (err && len) snprintf(err, len, "%s", m.c_str());
}
std::vector<Sphere> spheres(const double* xyzr, size_t n) {
    std::vector<Sphere> s(n);
    for (size_t i = 0; i < n; i++) s[i] = Sphere{{xyzr[4 * i], xyzr[4 * i + 1], xyzr[4 * i + 2]}, xyzr[4 * i + 3]};
    return s;
}
}  // namespace

extern "C" {

void orc_set_threads(int n) { set_threads(n); }
int orc_threads(void) { return threads(); }

// kind: 0 SES, 1 SAS, 2 vdW (field/mod.rs:33-41).
void* orc_engine_new(const double* xyzr, size_t n, double probe, double spacing, size_t brick, int kind, char* err,
                     size_t errlen) {
    auto s = spheres(xyzr, n);
    SesField f;
    std::string m = build_field(s.data(), n, probe, f, kind);
    if (!m.empty()) return set_err(err, errlen, m), nullptr;
    auto* h = new Handle();
    m = make_engine(std::move(f), spacing, brick, h->e);
    if (!m.empty()) {
        delete h;
        return set_err(err, errlen, m), nullptr;
    }
    return h;
}

void orc_engine_free(void* h) { delete static_cast<Handle*>(h); }

// info: frame[3], band, coord_max, f32_ok, n_spheres, n_contained, n_circles,
// n_vertices, max_expanded, rho_max, neighbour items, circle blocker items,
// sub, nsub, edge_clamp.
void orc_engine_info(void* hp, double* out) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    const Arrangement& a = e.field.arr;
    double v[] = {double(e.lattice.frame[0]), double(e.lattice.frame[1]), double(e.lattice.frame[2]), e.band,
                  e.coord_max, e.f32_ok ? 1.0 : 0.0, double(a.centers.size()), double(a.n_contained),
                  double(a.circles.size()), double(a.vertices.size()), a.max_expanded, e.field.rho_max,
                  double(a.neighbors.items.size()), double(a.circle_blockers.items.size()), double(e.sub),
                  double(e.nsub), edge_clamp(e)};
    std::memcpy(out, v, sizeof v);
}

// Arrangement arrays in internal order: centres (3 per sphere), expanded radii,
// status, orig; circles (i, j as doubles, centre 3, axis 3, e1 3, radius);
// vertices (position 3, atoms 3 as doubles).
void orc_engine_arrangement(void* hp, double* sph, uint8_t* status, uint32_t* orig, double* circ, double* vert) {
    const Arrangement& a = static_cast<Handle*>(hp)->e.field.arr;
    for (size_t k = 0; k < a.centers.size(); k++) {
        if (sph) {
            sph[5 * k] = a.centers[k].x, sph[5 * k + 1] = a.centers[k].y, sph[5 * k + 2] = a.centers[k].z;
            sph[5 * k + 3] = a.expanded[k], sph[5 * k + 4] = a.radii[k];
        }
        if (status) status[k] = a.status[k];
        if (orig) orig[k] = a.orig[k];
    }
    if (circ)
        for (size_t c = 0; c < a.circles.size(); c++) {
            const Circle& C = a.circles[c];
            double v[12] = {double(C.i), double(C.j), C.center.x, C.center.y, C.center.z, C.axis.x,
                            C.axis.y, C.axis.z, C.e1.x, C.e1.y, C.e1.z, C.radius};
            std::memcpy(circ + 12 * c, v, sizeof v);
        }
    if (vert)
        for (size_t k = 0; k < a.vertices.size(); k++) {
            const SasVertex& V = a.vertices[k];
            double v[6] = {V.position.x, V.position.y, V.position.z, double(V.atoms[0]), double(V.atoms[1]),
                           double(V.atoms[2])};
            std::memcpy(vert + 6 * k, v, sizeof v);
        }
}

// CSR tables: which 0 = neighbours (after the exposed-only retain), 1 = circle
// blockers.  off has rows+1 entries.
void orc_engine_csr(void* hp, int which, uint32_t* off, uint32_t* items) {
    const Arrangement& a = static_cast<Handle*>(hp)->e.field.arr;
    const Csr& c = which == 0 ? a.neighbors : a.circle_blockers;
    if (off) std::memcpy(off, c.off.data(), c.off.size() * 4);
    if (items && !c.items.empty()) std::memcpy(items, c.items.data(), c.items.size() * 4);
}

// Cell grid `which` (0 spheres, 1 circle centres, 2 SAS vertices): oc gets
// origin xyz and cell; dims 3; starts (cells + 1) and items when non-null.
// Returns the number of cells.
size_t orc_engine_grid(void* hp, int which, double* oc, uint32_t* dims, uint32_t* starts, uint32_t* items) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    const CellGrid& g = which == 0 ? e.field.arr.cells : (which == 1 ? e.field.circle_cells : e.field.vertex_cells);
    if (oc) oc[0] = g.origin.x, oc[1] = g.origin.y, oc[2] = g.origin.z, oc[3] = g.cell;
    if (dims) for (int k = 0; k < 3; k++) dims[k] = uint32_t(g.dims[k]);
    if (starts) std::memcpy(starts, g.starts.data(), g.starts.size() * 4);
    if (items && !g.items.empty()) std::memcpy(items, g.items.data(), g.items.size() * 4);
    return g.starts.size() - 1;
}

// Surface bricks (3 ints each, packed-key order); returns their count, or -1
// with err set.  *touched gets the touched-brick count.
long orc_engine_classify(void* hp, int32_t* out, size_t cap, size_t* touched, char* err, size_t errlen) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    std::string m;
    auto t = touched_bricks(e, m);
    if (!m.empty()) return set_err(err, errlen, m), -1;
    auto b = surface_bricks(e, t);
    if (touched) *touched = t.size();
    for (size_t i = 0; i < b.size() && i < cap; i++) std::memcpy(out + 3 * i, b[i].data(), 12);
    return long(b.size());
}

// Sub-block states: 8 per brick; 1 uniformly outside, 0 inside, -1 sampled.
void orc_engine_sub_states(void* hp, const int32_t* bricks, size_t n, int8_t* out) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    parallel_for(n, [&](size_t i, int) {
        int st[8];
        sub_states(e, bricks + 3 * i, st);
        for (int k = 0; k < 8; k++) out[8 * i + k] = int8_t(st[k]);
    });
}

// Sample values, (b+1)^3 per brick, x fastest.
void orc_engine_values(void* hp, const int32_t* bricks, size_t n, float* out) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    size_t spb = e.samples_per_brick();
    std::vector<BrickScratch> sc(static_cast<size_t>(threads()));
    for (auto& s : sc) s.init(e);
    parallel_for(n, [&](size_t i, int w) {
        evaluate(e, bricks + 3 * i, sc[size_t(w)]);
        std::memcpy(out + spb * i, sc[size_t(w)].values.data(), spb * 4);
    });
}

// Candidate lists of sub-block sb of one brick, serialized as
// [n_inside, n_near, n_s, n_c, n_v, s_blk total, c_blk total,
//  near ids, s ids, s_off (n_s+1), s_blk (local), c ids, c_off, c_blk, v ids].
// Returns the words needed (writes at most cap).
size_t orc_engine_gather(void* hp, const int32_t* brick, int sb, uint32_t* out, size_t cap) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    BrickScratch s;
    s.init(e);
    double rho;
    V3 c = sub_center(e, brick, sb, &rho);
    gather_ses(e, c, rho, s);
    const Gathered& g = s.g;
    std::vector<uint32_t> w = {uint32_t(g.n_inside), uint32_t(g.near_ids.size()), uint32_t(g.s_ids.size()),
                               uint32_t(g.c_ids.size()), uint32_t(g.v_ids.size()), uint32_t(g.s_blk.size()),
                               uint32_t(g.c_blk.size())};
    for (auto* v : {&g.near_ids, &g.s_ids, &g.s_off, &g.s_blk, &g.c_ids, &g.c_off, &g.c_blk, &g.v_ids})
        w.insert(w.end(), v->begin(), v->end());
    for (size_t i = 0; i < w.size() && i < cap; i++) out[i] = w[i];
    return w.size();
}

// MC pass of one brick from its values: owned crossing edge ids and triangle
// references (code << 28 | local edge id).  Returns the counts in n_out[2].
void orc_mc_brick(int b, const float* values, uint32_t* edges, uint32_t* tris, size_t* n_out) {
    BrickMesh m;
    size_t s = size_t(b) + 1;
    for (size_t z = 0; z < size_t(b); z++)
        for (size_t y = 0; y < size_t(b); y++)
            for (size_t x = 0; x < size_t(b); x++) {
                size_t i = (z * s + y) * s + x;
                size_t st[3] = {1, s, s * s};
                for (int a = 0; a < 3; a++)
                    if ((values[i] < 0.0f) != (values[i + st[a]] < 0.0f))
                        m.edges.push_back(uint32_t(((z * size_t(b) + y) * size_t(b) + x) * 3 + size_t(a)));
            }
    cells_pass(size_t(b), values, m);
    if (edges) std::memcpy(edges, m.edges.data(), m.edges.size() * 4);
    if (tris) std::memcpy(tris, m.tris.data(), m.tris.size() * 12);
    n_out[0] = m.edges.size();
    n_out[1] = m.tris.size();
}

// Exact f64 field value (growing cutoff) at n points (3 doubles each).
void orc_engine_field(void* hp, const double* pts, size_t n, double* out) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    parallel_for(n, [&](size_t i, int) {
        out[i] = e.field.value(V3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), nullptr, nullptr);
    });
}

// SesField::sample at n points: value and, where it has one, the normal
// (has[i] = 1), for the accuracy checks of tests/surface.rs:23-43.
void orc_engine_field_normals(void* hp, const double* pts, size_t n, double* out, double* normals, uint8_t* has) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    parallel_for(n, [&](size_t i, int) {
        V3 nrm;
        bool h = false;
        out[i] = e.field.value(V3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), &nrm, &h);
        normals[3 * i] = nrm.x, normals[3 * i + 1] = nrm.y, normals[3 * i + 2] = nrm.z;
        has[i] = h;
    });
}

// CPU mesh stage on a sample of bricks (Engine::evaluate + mesh_brick per
// brick, chunks of bricks over all threads, as fold_brick_chunks_with):
// wall seconds; *evals gets the refinement evaluations.
double orc_engine_mesh_sample(void* hp, const int32_t* bricks, size_t n, uint64_t* evals) {
    const Engine& e = static_cast<Handle*>(hp)->e;
    auto t0 = std::chrono::steady_clock::now();
    size_t chunk = std::min<size_t>(std::max<size_t>(n / 256, 1), 4096);
    size_t nchunks = (n + chunk - 1) / chunk;
    std::vector<BrickMesh> parts(nchunks);
    std::vector<BrickScratch> sc(static_cast<size_t>(threads()));
    for (auto& s : sc) s.init(e);
    parallel_for(nchunks, [&](size_t c, int w) {
        for (size_t i = c * chunk; i < std::min(n, (c + 1) * chunk); i++) {
            evaluate(e, bricks + 3 * i, sc[size_t(w)]);
            mesh_brick(e, bricks + 3 * i, sc[size_t(w)].values.data(), parts[c]);
        }
    });
    double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    uint64_t ev = 0;
    for (auto& p : parts) ev += p.evals;
    if (evals) *evals = ev;
    return s;
}

// Whole CPU pipeline; returns a handle or null with err set.
void* orc_surface_new(const double* xyzr, size_t n, double probe, double spacing, size_t brick, int kind, char* err,
                      size_t errlen) {
    auto s = spheres(xyzr, n);
    auto* h = new SurfaceHandle();
    std::string m = compute_surface(s.data(), n, probe, spacing, brick, h->out, kind);
    if (!m.empty()) {
        delete h;
        return set_err(err, errlen, m), nullptr;
    }
    return h;
}
void orc_surface_free(void* h) { delete static_cast<SurfaceHandle*>(h); }

// stats: touched, surface_bricks, vertices, triangles, components, area,
// volume, euler, refine_evaluations, t_geometry, t_classify, t_mesh,
// t_assemble, t_measure.
void orc_surface_stats(void* hp, double* out) {
    const SurfaceStats& s = static_cast<SurfaceHandle*>(hp)->out.stats;
    double v[] = {double(s.touched), double(s.surface_bricks), double(s.vertices), double(s.triangles),
                  double(s.components), s.area, s.volume, double(s.euler), double(s.refine_evaluations),
                  s.t_geometry, s.t_classify, s.t_mesh, s.t_assemble, s.t_measure};
    std::memcpy(out, v, sizeof v);
}

void orc_surface_mesh(void* hp, float* pos, float* nrm, uint32_t* tris, uint32_t* atoms, uint8_t* patches) {
    const Mesh& m = static_cast<SurfaceHandle*>(hp)->out.mesh;
    if (pos) std::memcpy(pos, m.positions.data(), m.positions.size() * 12);
    if (nrm) std::memcpy(nrm, m.normals.data(), m.normals.size() * 12);
    if (tris) std::memcpy(tris, m.triangles.data(), m.triangles.size() * 12);
    if (atoms) std::memcpy(atoms, m.vertex_atom.data(), m.vertex_atom.size() * 4);
    if (patches) std::memcpy(patches, m.vertex_patch.data(), m.vertex_patch.size());
}

// OBJ bytes (default options); returns the length, copies at most cap.
size_t orc_surface_obj(void* hp, char* out, size_t cap) {
    auto* h = static_cast<SurfaceHandle*>(hp);
    if (h->obj.empty()) h->obj = obj_bytes(h->out.mesh);
    if (out) std::memcpy(out, h->obj.data(), std::min(cap, h->obj.size()));
    return h->obj.size();
}

// OBJ of an explicit mesh (obj_snapshot pin).
size_t orc_obj_of(const float* pos, const float* nrm, size_t nv, const uint32_t* tris, size_t nt, int precision,
                  char* out, size_t cap) {
    Mesh m;
    m.positions.resize(nv);
    std::memcpy(m.positions.data(), pos, nv * 12);
    if (nrm) {
        m.normals.resize(nv);
        std::memcpy(m.normals.data(), nrm, nv * 12);
    }
    m.triangles.resize(nt);
    std::memcpy(m.triangles.data(), tris, nt * 12);
    std::string s = obj_bytes(m, precision);
    if (out) std::memcpy(out, s.data(), std::min(cap, s.size()));
    return s.size();
}

size_t orc_push_fixed(float x, int prec, char* out, size_t cap) {
    std::string s;
    push_fixed(s, x, prec);
    if (out) std::memcpy(out, s.data(), std::min(cap, s.size()));
    return s.size();
}

}  // extern "C"
