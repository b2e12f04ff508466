// compute_surface with the CUDA back end (crates/sesmesh/src/surface.rs:
// 599-633, 953-1300) above the C ABI: host arrangement, device
// classification and mesh-stage kernels, host f64 refinement (exact) or
// placement of the device's f32 roots (fast), assembly, validation,
// components and OBJ output.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>

#include "../../../include/sesmesh_b200.h"
#include "../../../include/sesmesh_b200_surface.h"
#include "../runtime.hpp"
#include "geom.hpp"
#include "engine.hpp"
#include "mesher.hpp"

using namespace smbh;

namespace {

using clk = std::chrono::steady_clock;
double ms_since(clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); }

void set_err(char* err, size_t len, const char* fmt, ...) {
    if (!err || !len) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
}

}  // namespace

// Host stages of one structure after its device run: placement of the
// device's f32 roots (fast) or f64 refinement (exact), assembly,
// validation, components and grouping; fills the statistics it can (sizes,
// area, volume, evaluations, host stage times).  Error text or "".
std::string finish_surface(const Arrangement& arr, const MeshParams& mp, bool fast, const int32_t* keys, size_t nb,
                           const uint32_t* edge_off, const uint32_t* edges, const float* edge_vals,
                           const uint32_t* tri_off, const uint32_t* tris, const DeviceRefine& dev, smb_surface& s,
                           smb_device* device, smb::MeasureScratch* scratch, MeshOut* exact,
                           const uint32_t* exact_evals) {
    auto t1 = clk::now();
    MeshOut mo;
    if (fast) {
        place_fast(arr, mp, keys, nb, edge_off, edges, edge_vals, dev, mo);
    } else if (exact && exact_evals) {
        mo.positions.swap(exact->positions), mo.normals.swap(exact->normals), mo.atoms.swap(exact->atoms);
        mo.patches.swap(exact->patches), mo.t.swap(exact->t);
        place_exact(arr, mp, keys, nb, edge_off, edges, edge_vals, exact_evals, mo);
    } else {
        refine_exact(arr, mp, keys, nb, edge_off, edges, edge_vals, mo);
    }
    double t_host = ms_since(t1);
    auto t2 = clk::now();
    Mesh& mesh = s.mesh;
    std::string m = assemble(keys, nb, edge_off, edges, tri_off, tris, mesh);
    if (!m.empty()) return m;
    mesh.positions.swap(mo.positions);
    mesh.normals.swap(mo.normals);
    mesh.vertex_atom.swap(mo.atoms);
    mesh.vertex_patch.swap(mo.patches);
    double t_assemble = ms_since(t2);
    auto t3 = clk::now();
    bool measured = false;
    if (device && scratch) {
        size_t bad = 0;
        std::string why;
        if (smb::measure_on_device(device, mesh, s.comps, &bad, *scratch, &why)) {
            if (bad) return "mesh failed validation (" + std::to_string(bad) + " defects)";
            measured = true;
        }
    }
    if (!measured) {
        EdgeUses uses;
        size_t bad = defects(mesh, &uses);
        if (bad) return "mesh failed validation (" + std::to_string(bad) + " defects)";
        components_and_group(mesh, s.comps, &uses);
    }
    double t_measure = ms_since(t3);
    smb_surface_stats& st = s.stats;
    st.spheres = arr.n;
    st.surface_bricks = nb;
    st.samples = nb * size_t(mp.b + 1) * size_t(mp.b + 1) * size_t(mp.b + 1);
    st.vertices = mesh.positions.size();
    st.triangles = mesh.triangles.size();
    st.components = s.comps.size();
    for (auto& c : s.comps) st.area += c.area, st.volume += c.volume, st.euler += c.euler;
    for (uint32_t v : mo.evals) st.refine_evaluations += v;
    for (uint32_t v : mo.cpu_refined) st.refine_cpu_edges += v;
    st.t_host_refine = t_host;
    st.t_assemble = t_assemble;
    st.t_measure = t_measure;
    st.host_threads = threads();
    return "";
}

static size_t g_device_arrangement_min = 16384;

const Arrangement& host_arrangement(smb_engine* e) {
    if (!e->arr_ready) {
        smb::arrangement_to_host(e->darr, e->arr);
        e->arr_ready = true;
    }
    return e->arr;
}

extern "C" {

void smb_set_device_arrangement_min(size_t n) { g_device_arrangement_min = n; }

uint64_t smb_device_bytes_estimate(size_t surface_bricks, uint32_t brick, double spacing, double probe,
                                   size_t spheres, int refine, int multiprocessors) {
    // Measured on B200 (globules of 330 and 2,800 spheres at 0.1 to 1 A,
    // exact and fast mode) and rounded up:
    // * fixed: the exact refinement's global list slabs (256 KiB for each of
    //   4 warps of 4 CTAs per SM) and about 200 MB of classification,
    //   queue, scan and measure tables;
    // * per sampled sub-block (at most 6 per surface brick counted): its
    //   candidate lists, at least the 12 KiB the gather's pools start from,
    //   else 250 bytes for each sphere of its largest ball at 0.05 spheres
    //   per A^3 (at most every sphere), with the pools' 25 % growth margins;
    // * per surface brick: its sample values (and the warm start's feature
    //   words), records and work lists;
    // * per crossing edge (2 b^2 per brick counted): the marching-cubes,
    //   refinement, vertex, triangle and measure arrays.
    const double b = double(brick), sub = 0.5 * b;
    const double spb = (b + 1) * (b + 1) * (b + 1);
    const double band = std::sqrt(3.0) * spacing * 1.01, rho = 0.5 * std::sqrt(3.0) * sub * spacing;
    const double r_ball = 1.8 + probe + probe + band + rho;
    const double in_ball = std::min(double(spheres), 0.05 * 4.18879020478639 * r_ball * r_ball * r_ball);
    const double per_sub = std::max(12288.0, 250.0 * in_ball) * 1.5625;
    const double per_brick = 6.0 * per_sub + spb * (refine == SMB_REFINE_FAST ? 8.0 : 4.0) * 1.25 +
                             8.0 * (SMB_REC_WORDS * 4 + 16) * 1.25 + 2.0 * b * b * 320.0;
    const uint64_t slabs = uint64_t(std::max(multiprocessors, 1)) * 4 * 4 * (uint64_t(256) << 10);
    return uint64_t(double(surface_bricks) * per_brick) + slabs + (uint64_t(224) << 20);
}

int smb_engine_new(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p, smb_engine** out,
                   char* err, size_t errlen) {
    return smb_engine_new_with(dev, xyzr, n, p, nullptr, out, err, errlen);
}

static void set_control(smb_engine* e, const smb_control* c) {
    e->ctl = smbh::Control();
    e->max_device_bytes = 0;
    if (!c) return;
    e->ctl.cancel = c->cancel;
    e->ctl.progress = c->progress;
    e->ctl.user = c->user;
    e->max_device_bytes = c->max_device_bytes;
}

uint64_t smb_engine_device_bytes(const smb_engine* e) {
    if (!e) return 0;
    uint64_t n = e->res ? smb_resident_bytes(e->res) : 0;
    if (e->batch)
        for (smb::DBuf* b : const_cast<smb_batch*>(e->batch)->bufs()) n += b->cap;
    smb::MeasureScratch& M = const_cast<smb_engine*>(e)->measure;
    for (smb::DBuf* b : {&M.pos, &M.nrm, &M.tris, &M.tris_out, &M.keys, &M.cnt, &M.dup, &M.parent, &M.flag, &M.cid,
                         &M.id, &M.counters, &M.comp_v, &M.comp_t, &M.area, &M.volume, &M.parts, &M.pkey, &M.pidx,
                         &M.pkey2, &M.pidx2, &M.first, &M.tkey, &M.tidx, &M.tkey2, &M.tidx2, &M.tiles, &M.cub,
                         &M.packed, &M.err, &M.tri_a, &M.tri_v})
        n += b->cap;
    return n;
}

int smb_engine_set_control(smb_engine* e, const smb_control* control) {
    if (!e) return SMB_ERR_ARG;
    set_control(e, control);
    return SMB_OK;
}

int smb_engine_new_with(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p,
                        const smb_control* control, smb_engine** out, char* err, size_t errlen) {
    if (!dev || !p || !out || (n && !xyzr)) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *out = nullptr;
    if (p->kind != SMB_SES && p->kind != SMB_SAS && p->kind != SMB_VDW)
        return set_err(err, errlen, "unknown surface kind %d", p->kind), SMB_ERR_ARG;
    if (p->refine != SMB_REFINE_EXACT && p->refine != SMB_REFINE_FAST)
        return set_err(err, errlen, "refine mode must be exact or fast on the device"), SMB_ERR_ARG;
    if (!(p->spacing >= 0.01) || !std::isfinite(p->spacing))
        return set_err(err, errlen, "grid spacing must be at least 0.01 A, got %g", p->spacing), SMB_ERR_ARG;
    if (p->brick_size < 4 || p->brick_size > 32 || p->brick_size % 2)
        return set_err(err, errlen, "brick size must be even and 4..32 on the device, got %u", p->brick_size), SMB_ERR_ARG;
    set_threads(p->threads);
    auto e = std::make_unique<smb_engine>();
    e->dev = dev;
    e->params = *p;
    // SurfaceParams::effective_probe (surface.rs:411-417) and SesField::new's
    // SES with probe 0, the vdW surface (point.rs:224-228).
    if (e->params.kind == SMB_SES && p->probe_radius == 0.0) e->params.kind = SMB_VDW;
    if (e->params.kind == SMB_VDW) e->params.probe_radius = 0.0;
    const int kind = e->params.kind;
    const double probe = e->params.probe_radius;
    set_control(e.get(), control);
    auto t0 = clk::now();
    std::string m = check_spheres(xyzr, n, probe, kind);
    if (!m.empty()) return set_err(err, errlen, "%s", m.c_str()), SMB_ERR_ARG;
    const Control& ctl = e->ctl;
    if (ctl.cancelled()) return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED;
    ctl.report(SMB_STAGE_GEOMETRY, 0, 1);
    // The arrangement: on the device for large inputs (the host builds it
    // when the device declines), else on the host threads.
    bool on_device = false;
    if (n >= g_device_arrangement_min && kind == SMB_SES) {
        std::string why;
        on_device = smb::build_arrangement_device(dev, xyzr, n, probe, e->darr, &why) == 0;
    }
    if (!on_device) {
        m = build_arrangement(xyzr, n, probe, e->arr, &ctl, kind);
        if (m == CANCELLED) return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED;
        if (!m.empty()) return set_err(err, errlen, "%s", m.c_str()), SMB_ERR_ARG;
    }
    if (ctl.cancelled()) {
        if (on_device) e->darr.release();
        return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED;
    }
    ctl.report(SMB_STAGE_GEOMETRY, 1, 1);
    e->arr_ready = !on_device;
    e->arr_where = on_device ? 1 : (n >= g_device_arrangement_min ? 2 : 0);
    const Arrangement& A = e->arr;
    const double max_expanded = on_device ? e->darr.A.max_expanded : A.max_expanded;
    e->n_spheres = on_device ? e->darr.n : A.n;
    // Engine::new (field/kernel.rs:204-271).
    V3 center;
    double half = 0.0;
    if (e->n_spheres) {
        V3 lo, hi;
        if (on_device) {
            lo = V3::at(e->darr.lo), hi = V3::at(e->darr.hi);
        } else {
            lo = A.c(0), hi = lo;
            for (size_t i = 0; i < A.n; i++) lo = lo.lo(A.c(uint32_t(i))), hi = hi.hi(A.c(uint32_t(i)));
        }
        V3 d = hi - lo;
        center = (lo + hi) * 0.5;
        half = 0.5 * std::fmax(std::fmax(d.x, d.y), d.z);
    }
    MeshParams& P = e->mp;
    P.h = p->spacing;
    P.b = int(p->brick_size);
    P.sub = P.b / 2;
    P.frame[0] = to_i64(std::round(center.x / P.h));
    P.frame[1] = to_i64(std::round(center.y / P.h));
    P.frame[2] = to_i64(std::round(center.z / P.h));
    double reach = half + 2.0 * max_expanded + 2.0 * probe + 4.0 * double(P.b) * P.h;
    P.f32_ok = reach < 2000.0 && reach / P.h < double(1u << 23);
    if (!P.f32_ok)
        return set_err(err, errlen, "extent beyond the f32 frame (%g A): the device path does not take it", reach),
               SMB_ERR_RANGE;
    P.band = std::sqrt(3.0) * P.h * 1.01;
    P.coord_max = std::fmax(std::fmax(std::fabs(center.x), std::fabs(center.y)), std::fabs(center.z)) + half +
                  max_expanded + probe + 2.0 * P.band;
    {  // edge_clamp (extract.rs:47-51)
        double cm = P.coord_max < 1.0 ? 1.0 : (P.coord_max > double(3.4028234663852886e38f) / 4.0 ? double(3.4028234663852886e38f) / 4.0 : P.coord_max);
        float mf = float(cm), nx;
        uint32_t bits;
        std::memcpy(&bits, &mf, 4);
        bits++;
        std::memcpy(&nx, &bits, 4);
        double ulp = double(nx - mf), tm = 4.0 * ulp / P.h;
        P.t_min = tm < 1e-4 ? 1e-4 : (tm > 0.25 ? 0.25 : tm);
    }
    e->t_geometry = ms_since(t0);
    auto t1 = clk::now();
    smb_lattice_ref lat{};
    lat.spacing = P.h;
    lat.brick = uint32_t(P.b);
    for (int k = 0; k < 3; k++) lat.frame[k] = P.frame[k];
    lat.band = P.band;
    int rc;
    if (on_device) {  // the resident takes over the device-built arrangement
        rc = smb::resident_from_device(dev, e->darr, &lat, &e->res, err, errlen);
        if (rc != SMB_OK) return e->darr.release(), rc;
        rc = smb_batch_new(e->res, &e->batch, err, errlen);
        if (rc != SMB_OK) return rc;
        if (p->refine == SMB_REFINE_FAST && (rc = smb_resident_set_refinement(e->res, err, errlen)) != SMB_OK)
            return rc;
        smb::resident_set_exact_tmin(e->res, P.t_min);
        e->t_upload = ms_since(t1);
        e->upload_bytes = uint64_t(n) * 32;
        *out = e.release();
        return SMB_OK;
    }
    // Upload (Resident::new).
    smb_arrangement_ref r{};
    r.n_spheres = A.n;
    r.center = A.center.data();
    r.expanded = A.expanded.data();
    r.radius = A.radius.data();
    r.status = A.status.data();
    r.nb_off = A.nb_off.data();
    r.nb_items = A.nb_items.data();
    r.n_circles = A.n_circles();
    r.circle = A.circle.data();
    r.cb_off = A.cb_off.data();
    r.cb_items = A.cb_items.data();
    r.n_vertices = A.n_vertices();
    r.vertex = A.vertex.data();
    const Grid* gs[3] = {&A.cells, &A.circle_cells, &A.vertex_cells};
    smb_grid_ref* gr[3] = {&r.sphere_grid, &r.circle_grid, &r.vertex_grid};
    for (int g = 0; g < 3; g++) {
        for (int k = 0; k < 3; k++) gr[g]->origin[k] = gs[g]->origin[k], gr[g]->dims[k] = gs[g]->dims[k];
        gr[g]->cell = gs[g]->cell;
        gr[g]->starts = gs[g]->starts.data();
        gr[g]->items = gs[g]->items.data();
        gr[g]->n_items = gs[g]->items.size();
    }
    r.max_expanded = A.max_expanded;
    r.rho_max = A.rho_max;
    r.probe = A.probe;
    r.kind = kind;
    rc = smb_resident_new(dev, &r, &lat, &e->res, err, errlen);
    if (rc != SMB_OK) return rc;
    rc = smb_batch_new(e->res, &e->batch, err, errlen);
    if (rc != SMB_OK) return rc;
    if (p->refine == SMB_REFINE_FAST && (rc = smb_resident_set_refinement(e->res, err, errlen)) != SMB_OK) return rc;
    rc = smb_resident_set_exact(e->res, A.orig.data(), A.circle_ij.data(), A.n_circles(), A.vertex_atoms.data(),
                                A.n_vertices(), P.t_min, err, errlen);
    if (rc != SMB_OK) return rc;
    e->t_upload = ms_since(t1);
    e->upload_bytes = smb_resident_bytes(e->res);
    *out = e.release();
    return SMB_OK;
}

void smb_engine_free(smb_engine* e) {
    if (!e) return;
    smb_batch_free(e->batch);
    smb_resident_free(e->res);
    delete e;
}

// Device part of the mesh stage on the resident arrangement: classification,
// sub-block states, gather, sampling, marching cubes (and fast-mode
// refinement); results stay on the device.
int smb_engine_run_device(smb_engine* e, smb_batch_times* times, char* err, size_t errlen) {
    if (!e) return SMB_ERR_ARG;
    const Control& ctl = e->ctl;
    auto cancelled = [&] { return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED; };
    if (ctl.cancelled()) return cancelled();
    size_t touched = 0, surface = 0;
    ctl.report(SMB_STAGE_CLASSIFY, 0, 1);
    auto t0 = clk::now();
    int rc = smb_classify(e->res, &touched, &surface, err, errlen);
    if (rc != SMB_OK) return rc;
    e->t_classify = ms_since(t0);
    e->touched = touched;
    ctl.report(SMB_STAGE_CLASSIFY, 1, 1);
    // The memory guard, before any mesh-stage buffer is taken.
    e->last_estimate = smb_device_bytes_estimate(surface, uint32_t(e->mp.b), e->mp.h, e->params.probe_radius,
                                                 e->n_spheres, e->params.refine, e->dev->info.multiprocessors) +
                       smb_resident_bytes(e->res);
    if (e->max_device_bytes && e->last_estimate > e->max_device_bytes)
        return set_err(err, errlen,
                       "estimated device memory (%llu bytes for %zu surface bricks at %g A) exceeds the limit of "
                       "%llu bytes",
                       (unsigned long long)e->last_estimate, surface, e->mp.h,
                       (unsigned long long)e->max_device_bytes),
               SMB_ERR_MEMORY;
    if (ctl.cancelled()) return cancelled();
    ctl.report(SMB_STAGE_MESH, 0, surface);
    smb_batch_times t{};
    rc = smb_run(e->res, 0, surface, e->batch, &t, err, errlen);
    if (rc != SMB_OK) return rc;
    if (ctl.cancelled()) return cancelled();
    e->rows_ready = false;
    if (e->params.refine == SMB_REFINE_FAST) {
        double ms = 0;
        // The warm start's candidates are the SES's features; a sphere
        // field refines from the linear guess.
        rc = e->warm && e->params.kind == SMB_SES ? smb_refine_warm(e->res, e->batch, e->warm, &ms, err, errlen)
                                                  : smb_refine(e->res, e->batch, &ms, err, errlen);
        if (rc != SMB_OK) return rc;
        t.total += ms;
        if (e->exact_device) {
            if ((rc = smb_place_fast(e->res, e->batch, &ms, err, errlen)) != SMB_OK) return rc;
            t.total += ms;
        }
    } else if (e->exact_device) {
        double ms = 0;
        if ((rc = smb_refine_exact(e->res, e->batch, &ms, err, errlen)) != SMB_OK) return rc;
        t.total += ms;
    }
    e->times = t;
    if (times) *times = t;
    if (ctl.cancelled()) return cancelled();
    ctl.report(SMB_STAGE_MESH, surface, surface);
    return SMB_OK;
}

size_t smb_engine_bricks(const smb_engine* e) { return e && e->res ? e->res->n_bricks : 0; }

smb_batch* smb_engine_batch(smb_engine* e) { return e ? e->batch : nullptr; }

// Brick keys and marching-cubes lists of the last device run to the host.
static int fetch_mc(smb_engine* e, char* err, size_t errlen) {
    size_t nb = e->res->n_bricks, ne = 0, nt = 0;
    int rc;
    smb_batch_mc_counts(e->batch, &ne, &nt);
    e->keys.resize(3 * nb);
    e->edge_off.resize(nb + 1);
    e->tri_off.resize(nb + 1);
    e->edges.resize(ne);
    e->edge_vals.resize(2 * ne);
    e->tris.resize(3 * nt);
    if (nb) {
        if ((rc = smb_resident_bricks(e->res, e->keys.data(), nb)) != SMB_OK) return set_err(err, errlen, "bricks copy"), rc;
        if ((rc = smb_batch_mc(e->batch, e->edge_off.data(), e->edges.data(), e->edge_vals.data(), e->tri_off.data(),
                               e->tris.data())) != SMB_OK)
            return set_err(err, errlen, "mc copy"), rc;
    } else {
        e->edge_off.assign(1, 0);
        e->tri_off.assign(1, 0);
    }
    return SMB_OK;
}

}  // extern "C"

// Exact mode with every vertex refined on the device: assembly, validation,
// measure and grouping there too, and the finished mesh back once.
// SMB_OK, or an error code; *fallback when the device could not and the
// host stages should run instead.
int finish_exact_device(smb_engine* e, smb_surface& s, unsigned long long evals, unsigned long long cpu_edges,
                        bool* fallback, double* ms_d2h, char* err, size_t errlen) {
    *fallback = false;
    const smb_batch* b = e->batch;
    smb::DeviceMesh in{};
    in.keys = e->res->keys + b->first;
    in.n_bricks = b->n;
    in.edge_off = b->edge_off.as<uint32_t>();
    in.edges = b->edges.as<uint32_t>();
    in.tri_off = b->tri_off.as<uint32_t>();
    in.tri_refs = b->tris.as<uint32_t>();
    in.n_edges = b->n_edges;
    in.n_tris = b->n_tris;
    in.pos = b->x_pos.as<float>();
    in.nrm = b->x_nrm.as<float>();
    in.atoms = b->x_atom.as<uint32_t>();
    in.patches = b->x_patch.as<uint8_t>();
    auto t0 = clk::now();
    size_t bad = 0;
    std::string msg;
    double ms_asm = 0;
    int r = smb::finish_on_device(e->dev, in, &s.view, &s.block, s.comps, &bad, e->measure, &msg, &ms_asm);
    if (r == 1) {
        *fallback = true;
        e->note = "device finish declined: " + msg;
        return SMB_OK;
    }
    if (r == 2) return set_err(err, errlen, "%s", msg.c_str()), SMB_ERR_STATE;
    if (bad) return set_err(err, errlen, "mesh failed validation (%zu defects)", bad), SMB_ERR_STATE;
    const MeshParams& mp = e->mp;
    smb_surface_stats& st = s.stats;
    st.spheres = e->n_spheres;
    st.surface_bricks = b->n;
    st.samples = size_t(b->n) * size_t(mp.b + 1) * size_t(mp.b + 1) * size_t(mp.b + 1);
    st.vertices = s.view.nv;
    st.triangles = s.view.nt;
    st.components = s.comps.size();
    for (auto& c : s.comps) st.area += c.area, st.volume += c.volume, st.euler += c.euler;
    st.refine_evaluations = evals;
    st.refine_cpu_edges = cpu_edges;
    st.t_host_refine = 0;
    st.t_assemble = ms_asm;
    st.t_measure = ms_since(t0) - ms_asm;
    st.host_threads = threads();
    *ms_d2h = 0;  // the copies back overlap the measure
    return SMB_OK;
}

extern "C" {


// Whole mesh stage and the stages after it: device part, results to the
// host, f64 refinement (exact) or placement (fast), assembly, validation,
// components and grouping.
int smb_engine_mesh(smb_engine* e, smb_surface** out, char* err, size_t errlen) {
    if (!e || !out) return SMB_ERR_ARG;
    *out = nullptr;
    auto t_all = clk::now();
    int rc = smb_engine_run_device(e, nullptr, err, errlen);
    if (rc != SMB_OK) return rc;
    const Control& ctl = e->ctl;
    ctl.report(SMB_STAGE_ASSEMBLE, 0, 1);
    auto fill_times = [&](smb_surface_stats& st, double t_d2h) {
        st.touched_bricks = e->touched;
        st.t_geometry = e->t_geometry;
        st.t_upload = e->t_upload;
        st.t_classify = e->t_classify;
        st.t_substates = e->times.substates;
        st.t_gather = e->times.gather;
        st.t_sample = e->times.sample;
        st.t_mc = e->times.mc;
        st.t_device = e->t_classify + e->times.total;
        st.t_d2h = t_d2h;
        st.t_mesh_stage = ms_since(t_all) - st.t_assemble - st.t_measure;
        st.arrangement_where = e->arr_where;
        st.finished_on_host = e->exact_device && !e->note.empty();
        st.upload_bytes = e->upload_bytes;
        st.spacing_used = e->mp.h;
        st.device_bytes_estimate = e->last_estimate;
        ctl.report(SMB_STAGE_ASSEMBLE, 1, 1);
        ctl.report(SMB_STAGE_MEASURE, 0, 1);
        ctl.report(SMB_STAGE_MEASURE, 1, 1);
    };
    e->note.clear();
    if (e->exact_device && e->res->n_bricks) {
        unsigned long long evals = 0, host_edges = 0, exact_edges = 0;
        if ((rc = smb_batch_exact_summary(e->batch, &evals, &host_edges, &exact_edges)) != SMB_OK)
            return set_err(err, errlen, "vertex summary failed"), rc;
        if (host_edges) e->note = std::to_string(host_edges) + " edges left to the host";
        if (host_edges == 0) {
            auto s = std::make_unique<smb_surface>();
            bool fallback = false;
            double ms_d2h = 0;
            const unsigned long long cpu = e->params.refine == SMB_REFINE_FAST ? exact_edges : 0;
            if ((rc = finish_exact_device(e, *s, evals, cpu, &fallback, &ms_d2h, err, errlen)) != SMB_OK) return rc;
            if (!fallback) {
                fill_times(s->stats, ms_d2h);
                *out = s.release();
                return SMB_OK;
            }
        }
    }
    auto t0 = clk::now();
    if ((rc = fetch_mc(e, err, errlen)) != SMB_OK) return rc;
    size_t nb = e->res->n_bricks, ne = e->edges.size();
    bool fast = e->params.refine == SMB_REFINE_FAST;
    if (fast && ne) {
        e->t.resize(ne), e->feat.resize(ne), e->closest.resize(3 * ne), e->evals.resize(ne);
        if ((rc = smb_batch_edges(e->batch, e->t.data(), e->feat.data(), e->closest.data(), e->evals.data())) != SMB_OK)
            return set_err(err, errlen, "edge results copy"), rc;
    }
    const bool exact_dev = !fast && e->exact_device;
    if (exact_dev && ne) {
        smbh::MeshOut& x = e->exact_out;
        x.positions.resize(ne), x.normals.resize(ne), x.atoms.resize(ne), x.patches.resize(ne), x.t.resize(ne);
        e->exact_evals.resize(ne);
        if ((rc = smb_batch_vertices(e->batch, x.positions.data()->data(), x.normals.data()->data(), x.atoms.data(),
                                     x.patches.data(), x.t.data(), e->exact_evals.data())) != SMB_OK)
            return set_err(err, errlen, "vertex copy"), rc;
    }
    double t_d2h = ms_since(t0);
    auto s = std::make_unique<smb_surface>();
    std::string m = finish_surface(host_arrangement(e), e->mp, fast, e->keys.data(), nb, e->edge_off.data(), e->edges.data(),
                                   e->edge_vals.data(), e->tri_off.data(), e->tris.data(),
                                   DeviceRefine{e->t.data(), e->feat.data(), e->closest.data(), e->evals.data()}, *s,
                                   e->dev, &e->measure, exact_dev && ne ? &e->exact_out : nullptr,
                                   exact_dev && ne ? e->exact_evals.data() : nullptr);
    if (!m.empty()) return set_err(err, errlen, "%s", m.c_str()), SMB_ERR_STATE;
    fill_times(s->stats, t_d2h);
    *out = s.release();
    return SMB_OK;
}

int smb_engine_field(const smb_engine* e, const double* points, size_t n, double* values) {
    if (!e || (n && (!points || !values))) return SMB_ERR_ARG;
    const double band = e->mp.band;
    const Arrangement& A = host_arrangement(const_cast<smb_engine*>(e));
    // The refinement's evaluation (field/point.rs:496-738): the candidates of
    // the point (a ball of radius 0), then the exact f64 field, which equals
    // SesField::value within the band.
    parallel_for((n + 255) / 256, [&](size_t c, int) {
        Local l;
        for (size_t i = c * 256; i < std::min(n, (c + 1) * 256); i++) {
            V3 x = V3::at(points + 3 * i);
            gather_local(A, x, 0.0, band, l);
            values[i] = eval_local(A, x, band, l).value;
        }
    });
    return SMB_OK;
}

const char* smb_engine_note(const smb_engine* e) { return e ? e->note.c_str() : ""; }

int smb_engine_set_exact_device(smb_engine* e, int on) {
    if (!e) return SMB_ERR_ARG;
    e->exact_device = on != 0;
    return SMB_OK;
}

int smb_engine_set_warm_start(smb_engine* e, const smb_mlp* mlp) {
    if (!e) return SMB_ERR_ARG;
    e->warm = mlp;
    // The warm start reads the sampler's nearest features.
    return smb_batch_record_features(e->batch, mlp != nullptr);
}

int smb_engine_warm_start_rows(smb_engine* e, float* features, float* labels, float* plain, size_t cap, size_t* n,
                               char* err, size_t errlen) {
    if (!e || !n) return SMB_ERR_ARG;
    if (!e->rows_ready) {
        smb_batch_record_features(e->batch, 1);
        int rc = smb_engine_run_device(e, nullptr, err, errlen);
        smb_batch_record_features(e->batch, e->warm != nullptr);
        if (rc != SMB_OK) return rc;
        if ((rc = fetch_mc(e, err, errlen)) != SMB_OK) return rc;
        if ((rc = smb_resident_set_refinement(e->res, err, errlen)) != SMB_OK) return rc;
        size_t ne = e->edges.size();
        std::vector<float> x(ne * SMB_MLP_FEATURES);
        std::vector<uint8_t> covered(ne);
        if ((rc = smb_batch_edge_features(e->res, e->batch, x.data(), covered.data(), err, errlen)) != SMB_OK) return rc;
        // Where plain f32 refinement stops (the reference's fast mode).
        double ms = 0;
        std::vector<float> tp(ne);
        std::vector<uint32_t> fp(ne), ep(ne);
        std::vector<float> qp(3 * ne);
        if ((rc = smb_refine(e->res, e->batch, &ms, err, errlen)) != SMB_OK) return rc;
        if (ne && (rc = smb_batch_edges(e->batch, tp.data(), fp.data(), qp.data(), ep.data())) != SMB_OK)
            return set_err(err, errlen, "edge results copy"), rc;
        // The labels: exact mode's f64 root parameter (before the edge clamp)
        // from the device refinement, which equals the host's bit for bit;
        // edges it leaves to the host (evals = 0) are left out.
        if ((rc = smb_refine_exact(e->res, e->batch, &ms, err, errlen)) != SMB_OK) return rc;
        std::vector<float> pos(3 * ne), nrm(3 * ne), t(ne);
        std::vector<uint32_t> atoms(ne), evals(ne);
        std::vector<uint8_t> patches(ne);
        if (ne && (rc = smb_batch_vertices(e->batch, pos.data(), nrm.data(), atoms.data(), patches.data(), t.data(),
                                           evals.data())) != SMB_OK)
            return set_err(err, errlen, "vertex copy"), rc;
        e->row_x.clear(), e->row_t.clear(), e->row_p.clear();
        for (size_t k = 0; k < ne; k++) {
            if (!covered[k] || evals[k] == 0) continue;
            e->row_x.insert(e->row_x.end(), x.begin() + k * SMB_MLP_FEATURES, x.begin() + (k + 1) * SMB_MLP_FEATURES);
            e->row_t.push_back(t[k]);
            e->row_p.push_back((ep[k] & 0x80000000u) ? tp[k] : std::numeric_limits<float>::quiet_NaN());
        }
        e->rows_ready = true;
    }
    *n = e->row_t.size();
    if (!features || !labels || !plain) return SMB_OK;
    if (cap < *n) return set_err(err, errlen, "%zu rows do not fit in %zu", *n, cap), SMB_ERR_MEMORY;
    std::copy(e->row_x.begin(), e->row_x.end(), features);
    std::copy(e->row_t.begin(), e->row_t.end(), labels);
    std::copy(e->row_p.begin(), e->row_p.end(), plain);
    return SMB_OK;
}

int smb_compute_surface(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p, smb_surface** out,
                        char* err, size_t errlen) {
    return smb_compute_surface_with(dev, xyzr, n, p, nullptr, out, err, errlen);
}

int smb_compute_surface_with(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p,
                             const smb_control* control, smb_surface** out, char* err, size_t errlen) {
    if (!p || !out) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *out = nullptr;
    auto t0 = clk::now();
    smb_surface_params q = *p;
    const bool coarsen = control && control->auto_coarsen && control->max_device_bytes;
    // With auto_coarsen, a refused spacing is raised by the square root of
    // the estimate's excess (surface bricks go as 1 / h^2 at a fixed brick
    // edge) until it fits, at most 10 A (surface.rs:825-860 does the same
    // search on its own estimate).
    for (int attempt = 0;; attempt++) {
        smb_engine* e = nullptr;
        int rc = smb_engine_new_with(dev, xyzr, n, &q, control, &e, err, errlen);
        if (rc != SMB_OK) return rc;
        rc = smb_engine_mesh(e, out, err, errlen);
        const uint64_t est = e->last_estimate;
        smb_engine_free(e);
        if (rc == SMB_OK) {
            (*out)->stats.t_total = ms_since(t0);
            return SMB_OK;
        }
        if (rc != SMB_ERR_MEMORY || !coarsen || !est || attempt >= 12 || q.spacing >= 10.0) return rc;
        const double excess = double(est) / double(control->max_device_bytes);
        double h = q.spacing * std::sqrt(excess) * 1.05;
        if (!(h > q.spacing)) h = q.spacing * 1.05;
        q.spacing = std::min(h, 10.0);
    }
}

void smb_surface_free(smb_surface* s) { delete s; }

int smb_surface_stats_get(const smb_surface* s, smb_surface_stats* out) {
    if (!s || !out) return SMB_ERR_ARG;
    *out = s->stats;
    return SMB_OK;
}

int smb_surface_mesh(const smb_surface* s, float* pos, float* nrm, uint32_t* tris, uint32_t* atoms, uint8_t* patches,
                     uint32_t* components) {
    if (!s) return SMB_ERR_ARG;
    const smbh::MeshRef m = s->ref();
    auto copy = [](void* dst, const void* src, size_t bytes) {
        if (dst && src && bytes) std::memcpy(dst, src, bytes);
    };
    copy(pos, m.pos, m.nv * 12);
    copy(nrm, m.nrm, m.nv * 12);
    copy(tris, m.tris, m.nt * 12);
    copy(atoms, m.atom, m.nv * 4);
    copy(patches, m.patch, m.nv);
    copy(components, m.comp, m.nv * 4);
    return SMB_OK;
}

int smb_surface_arrays(const smb_surface* s, const float** pos, const float** nrm, const uint32_t** tris,
                       const uint32_t** atoms, const uint8_t** patches, const uint32_t** components) {
    if (!s) return SMB_ERR_ARG;
    const smbh::MeshRef m = s->ref();
    if (pos) *pos = m.nv ? m.pos : nullptr;
    if (nrm) *nrm = m.nv ? m.nrm : nullptr;
    if (tris) *tris = m.nt ? m.tris : nullptr;
    if (atoms) *atoms = m.nv ? m.atom : nullptr;
    if (patches) *patches = m.nv ? m.patch : nullptr;
    if (components) *components = m.nv ? m.comp : nullptr;
    return SMB_OK;
}

size_t smb_surface_obj(smb_surface* s, char* out, size_t cap) {
    if (!s) return 0;
    if (s->obj.empty()) s->obj = obj_text_buffer(s->ref());
    if (out) std::memcpy(out, s->obj.data.get(), s->obj.size < cap ? s->obj.size : cap);
    return s->obj.size;
}

int smb_surface_write_obj(smb_surface* s, const char* path, char* err, size_t errlen) {
    if (!s || !path) return SMB_ERR_ARG;
    if (s->obj.empty()) s->obj = obj_text_buffer(s->ref());
    FILE* f = std::fopen(path, "wb");
    if (!f) return set_err(err, errlen, "cannot open %s", path), SMB_ERR_ARG;
    size_t w = std::fwrite(s->obj.data.get(), 1, s->obj.size, f);
    std::fclose(f);
    if (w != s->obj.size) return set_err(err, errlen, "short write to %s", path), SMB_ERR_ARG;
    return SMB_OK;
}

// The host arrangement of an engine (tests compare it with the oracle's).
int smb_engine_arrangement(const smb_engine* e, smb_arrangement_info* out) {
    if (!e || !out) return SMB_ERR_ARG;
    const Arrangement& A = host_arrangement(const_cast<smb_engine*>(e));
    out->built_on_device = e->darr.A.sph != nullptr;
    out->n_spheres = A.n;
    out->n_contained = A.n_contained;
    out->n_circles = A.n_circles();
    out->n_vertices = A.n_vertices();
    out->center = A.center.data();
    out->expanded = A.expanded.data();
    out->status = A.status.data();
    out->orig = A.orig.data();
    out->circle = A.circle.data();
    out->circle_ij = A.circle_ij.data();
    out->vertex = A.vertex.data();
    out->vertex_atoms = A.vertex_atoms.data();
    out->nb_off = A.nb_off.data();
    out->nb_items = A.nb_items.data();
    out->cb_off = A.cb_off.data();
    out->cb_items = A.cb_items.data();
    out->max_expanded = A.max_expanded;
    out->rho_max = A.rho_max;
    for (int k = 0; k < 3; k++) out->frame[k] = e->mp.frame[k];
    out->band = e->mp.band;
    out->t_min = e->mp.t_min;
    return SMB_OK;
}

// Host-only construction (no device): the arrangement and lattice constants.
int smb_arrangement_build(const double* xyzr, size_t n, const smb_surface_params* p, smb_engine** out, char* err,
                          size_t errlen) {
    return smb_arrangement_build_with(xyzr, n, p, nullptr, out, err, errlen);
}

int smb_arrangement_build_with(const double* xyzr, size_t n, const smb_surface_params* p,
                               const smb_control* control, smb_engine** out, char* err, size_t errlen) {
    if (!p || !out) return SMB_ERR_ARG;
    *out = nullptr;
    auto e = std::make_unique<smb_engine>();
    e->params = *p;
    set_control(e.get(), control);
    set_threads(p->threads);
    e->ctl.report(SMB_STAGE_GEOMETRY, 0, 1);
    int kind = p->kind;
    double probe = p->probe_radius;
    if (kind == SMB_SES && probe == 0.0) kind = SMB_VDW;
    if (kind == SMB_VDW) probe = 0.0;
    e->params.kind = kind, e->params.probe_radius = probe;
    std::string m = build_arrangement(xyzr, n, probe, e->arr, &e->ctl, kind);
    if (m == CANCELLED) return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED;
    if (!m.empty()) return set_err(err, errlen, "%s", m.c_str()), SMB_ERR_ARG;
    e->ctl.report(SMB_STAGE_GEOMETRY, 1, 1);
    *out = e.release();
    return SMB_OK;
}

}  // extern "C"
