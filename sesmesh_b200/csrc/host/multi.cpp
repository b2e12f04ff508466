// Many structures meshed in one device pass: the structures' arrangements
// stay resident side by side, one classification pass covers every
// structure's brick box, and the mesh stage (sub-block states, candidate
// gather, sampling, marching cubes, fast-mode refinement) runs as one
// captured CUDA graph whose kernels take their work from a device queue of
// (structure, brick) items: every brick key carries its structure number,
// and the kernels find that structure's arrangement, lattice and refinement
// constants in per-structure descriptor arrays.  Buffers are sized from
// per-brick caps chosen by an autotuner (brick edge, candidate caps, gather
// block shape); a structure that meets a cap is flagged on the device and
// meshed again on its own through the single-structure engine.
//
// sesmesh meshes one structure per compute_surface call (crates/sesmesh/
// src/surface.rs:599-711); the per-structure results here are those of the
// single-structure device path at the same brick edge (same kernels, same
// arithmetic), with the host stages of crates/sesmesh/src/mesh/extract.rs:
// 274-365 and 606-691 run per structure on the host threads.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <thread>

#include "../device/kernels.hpp"
#include "../device/mlp.cuh"
#include "../runtime.hpp"
#include "engine.hpp"

using namespace smb;
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

#define MCK(call)                                                                            \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            set_err(err, errlen, "%s: %s", #call, cudaGetErrorString(e_));                   \
            return SMB_ERR_CUDA;                                                             \
        }                                                                                    \
    } while (0)

// Candidate caps of one level: the gather's per-warp shared-memory lists,
// the largest packed block of one sub-block (16-byte units; the sampler's
// shared memory), and the list pools per sub-block of the batch.
struct CapLevel {
    GatherCaps caps;
    uint32_t unit_cap;
    uint32_t ids_per_sub, units_per_sub;
};
const CapLevel CAP_LEVELS[2] = {
    {{192, 128, 384, 128}, 2048, 640, 320},
    {{384, 256, 768, 256}, 8192, 1280, 640},
};

DLat lattice_for(const DLat& L0, int b) {
    DLat L = L0;
    L.b = b;
    L.sub = b / 2;
    L.spb = (b + 1) * (b + 1) * (b + 1);
    L.rho_sub = 0.5 * std::sqrt(3.0) * double(L.sub) * L.h;  // kernel.rs:474
    L.rho_brick = 0.5 * std::sqrt(3.0) * double(L.b) * L.h;  // lattice.rs:78-80
    return L;
}

// Page-locked host memory that grows on demand (copies from the device run
// at full link speed into it).
struct Pinned {
    void* p = nullptr;
    size_t cap = 0;
    bool reserve(size_t bytes) {
        if (bytes <= cap) return true;
        smb::pinned_free(p), p = nullptr, cap = 0;
        size_t want = bytes + bytes / 4 + 4096;
        if (!(p = smb::pinned_alloc(want))) return false;
        cap = want;
        return true;
    }
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
    ~Pinned() { smb::pinned_free(p); }
};

// One group's results on the host.
struct HostGroup {
    size_t ne = 0, nt = 0;
    Pinned eo, to, edges, tris, feat, evals, ev, t, q;
};

}  // namespace

// Structures [s0, s1), surface bricks [k0, k1) of the keys, and the graph
// recorded for that pass (with the configuration it was recorded for).
struct Group {
    size_t s0 = 0, s1 = 0, k0 = 0, k1 = 0;
    cudaGraphExec_t graph = nullptr;
    smb_multi_config cfg{};
    const smb_mlp* warm = nullptr;
    const void* keys = nullptr;
    uint64_t gen = 0;
};

struct smb_multi {
    smb_device* dev = nullptr;
    std::vector<smb_engine*> eng;  // per structure: host arrangement, parameters, resident
    const smb_mlp* warm = nullptr;
    smb_multi_config cfg{};
    bool tuned = false;
    smbh::Control ctl;  // cancel flag and progress of the runs
    double t_setup = 0, t_tune = 0;
    // Descriptors of the current brick edge.
    int desc_brick = 0;
    std::vector<DLat> lat;
    std::vector<MeshParams> mp;
    std::vector<BrickBox> box;
    std::vector<unsigned long long> flag_off;
    std::vector<uint32_t> sph_off;
    DBuf d_arr, d_lat, d_rc, d_box, d_flag_off, d_sph_off, d_err, d_fail;
    // Batch buffers.
    DBuf flags, list, surf, cells, tiles, tot, keys, rec, sampled, work, retry, values, counters, totals, ids, pack;
    DBuf mc_counts, edge_off, tri_off, edges, edge_vals, tris, item_counts, item_off, item_edges;
    DBuf e_t, e_feat, e_q, e_evals;
    DBuf w_feats, w_start;  // warm start: the sampler's nearest features, each row's start
    size_t edge_cap = 0, tri_cap = 0;
    // Groups of structures, one pass (and one recorded graph) each.
    std::vector<Group> groups;
    size_t group_bricks = 0;
    bool graph_ok = true;
    uint32_t unit_cap = 0;     // the sampler's block cap (units), raised to what a pass needed
    smb_multi_config unit_cfg{};
    uint64_t gen = 0;          // buffer generation (recorded graphs hold their buffers' addresses)
    std::vector<int4> keys4;   // host copy of the keys
    HostGroup* hosts = nullptr;  // two alternating sets of results on the host
    std::vector<size_t> b0;    // first brick of each structure (n + 1)
    bool device_finish = true; // place, refine and finish each structure on the device
    cudaEvent_t ev[2] = {};
    // Results of the last run.
    std::vector<std::unique_ptr<smb_surface>> out;
    std::vector<double> latency;
    std::vector<uint8_t> redone;
    uint32_t n_bricks = 0;

    std::vector<DBuf*> bufs() {
        return {&d_arr, &d_lat, &d_rc, &d_box, &d_flag_off, &d_sph_off, &d_err, &d_fail, &flags, &list, &surf,
                &cells, &tiles, &tot, &keys, &rec, &sampled, &work, &retry, &values, &counters, &totals, &ids, &pack,
                &mc_counts, &edge_off, &tri_off, &edges, &edge_vals, &tris, &item_counts, &item_off, &item_edges, &w_feats, &w_start,
                &e_t, &e_feat, &e_q, &e_evals};
    }
    size_t n() const { return eng.size(); }
};

namespace {

// Per-structure lattice, host mesh parameters, brick boxes and the device
// descriptor arrays for brick edge b.
int set_brick(smb_multi* m, int b, char* err, size_t errlen) {
    if (m->desc_brick == b) return SMB_OK;
    const size_t n = m->n();
    m->lat.resize(n), m->mp.resize(n), m->box.resize(n);
    m->flag_off.assign(n + 1, 0);
    m->sph_off.assign(n + 1, 0);
    std::vector<DArr> arr(n);
    std::vector<RefineConsts> rc(n);
    for (size_t i = 0; i < n; i++) {
        smb_resident* r = m->eng[i]->res;
        arr[i] = r->A;
        rc[i] = r->rc;
        m->lat[i] = lattice_for(r->L, b);
        m->mp[i] = m->eng[i]->mp;
        m->mp[i].b = b, m->mp[i].sub = b / 2;
        // Box of the bricks any sphere can touch (as smb_classify).
        const DLat& L = m->lat[i];
        double rr = r->A.max_expanded + CLASSIFY_EPS, bh = double(L.b) * L.h, cells = 1;
        for (int k = 0; k < 3; k++) {
            double lo = std::floor((r->lo[k] - rr) / bh), hi = std::floor((r->hi[k] + rr) / bh);
            if (!(std::fabs(lo) < double(KEY_BIAS) && std::fabs(hi) < double(KEY_BIAS)))
                return set_err(err, errlen, "structure %zu: coordinates too far from the origin", i), SMB_ERR_RANGE;
            m->box[i].lo[k] = (long long)lo;
            m->box[i].n[k] = r->A.n ? uint32_t(hi - lo + 1) : 0;
            cells *= double(m->box[i].n[k]);
        }
        m->flag_off[i + 1] = m->flag_off[i] + (unsigned long long)cells;
        m->sph_off[i + 1] = m->sph_off[i] + r->A.n;
    }
    if (m->flag_off[n] >= (1ull << 31))
        return set_err(err, errlen, "the structures' brick boxes hold %llu bricks, more than 2^31", m->flag_off[n]),
               SMB_ERR_RANGE;
    int rc_;
    if ((rc_ = m->d_arr.reserve(n * sizeof(DArr), err, errlen)) ||
        (rc_ = m->d_lat.reserve(n * sizeof(DLat), err, errlen)) ||
        (rc_ = m->d_rc.reserve(n * sizeof(RefineConsts), err, errlen)) ||
        (rc_ = m->d_box.reserve(n * sizeof(BrickBox), err, errlen)) ||
        (rc_ = m->d_flag_off.reserve((n + 1) * 8, err, errlen)) ||
        (rc_ = m->d_sph_off.reserve((n + 1) * 4, err, errlen)) || (rc_ = m->d_err.reserve(n * 4, err, errlen)) ||
        (rc_ = m->d_fail.reserve(n * 4, err, errlen)))
        return rc_;
    cudaStream_t s = m->dev->stream;
    MCK(cudaMemcpyAsync(m->d_arr.p, arr.data(), n * sizeof(DArr), cudaMemcpyHostToDevice, s));
    MCK(cudaMemcpyAsync(m->d_lat.p, m->lat.data(), n * sizeof(DLat), cudaMemcpyHostToDevice, s));
    MCK(cudaMemcpyAsync(m->d_rc.p, rc.data(), n * sizeof(RefineConsts), cudaMemcpyHostToDevice, s));
    MCK(cudaMemcpyAsync(m->d_box.p, m->box.data(), n * sizeof(BrickBox), cudaMemcpyHostToDevice, s));
    MCK(cudaMemcpyAsync(m->d_flag_off.p, m->flag_off.data(), (n + 1) * 8, cudaMemcpyHostToDevice, s));
    MCK(cudaMemcpyAsync(m->d_sph_off.p, m->sph_off.data(), (n + 1) * 4, cudaMemcpyHostToDevice, s));
    MCK(cudaStreamSynchronize(s));
    m->desc_brick = b;
    return SMB_OK;
}

Scene scene_of(smb_multi* m) {
    Scene S{};
    S.arr = m->d_arr.as<DArr>();
    S.lat = m->d_lat.as<DLat>();
    S.rc = m->d_rc.as<RefineConsts>();
    S.box = m->d_box.as<BrickBox>();
    S.flag_off = m->d_flag_off.as<unsigned long long>();
    S.sph_off = m->d_sph_off.as<uint32_t>();
    S.n_struct = uint32_t(m->n());
    S.n_work = m->totals.as<unsigned long long>();
    S.err = m->d_err.as<int>();
    S.fail = m->d_fail.as<uint32_t>();
    return S;
}

// Every structure's surface bricks in one pass (lattice::touched_bricks +
// surface_bricks per structure); keys (x, y, z, structure) in structure
// order, each structure's in packed-key order.
int classify_all(smb_multi* m, char* err, size_t errlen) {
    const size_t n = m->n();
    cudaStream_t s = m->dev->stream;
    const uint32_t nf = uint32_t(m->flag_off[n]);
    int rc;
    if ((rc = m->flags.reserve(size_t(nf) * 4 + 4, err, errlen)) || (rc = m->list.reserve(size_t(nf) * 4 + 4, err, errlen)) ||
        (rc = m->surf.reserve(size_t(nf) * 4 + 4, err, errlen)) || (rc = m->cells.reserve(size_t(nf) * 4 + 4, err, errlen)) ||
        (rc = m->tiles.reserve(size_t(scan_tiles_needed(std::max(nf, 8u))) * 8 + 64, err, errlen)) ||
        (rc = m->tot.reserve(16, err, errlen)) || (rc = m->totals.reserve(64, err, errlen)))
        return rc;
    Scene S = scene_of(m);
    MCK(cudaMemsetAsync(m->flags.p, 0, size_t(nf) * 4 + 4, s));
    MCK(cudaMemsetAsync(m->surf.p, 0, size_t(nf) * 4 + 4, s));
    MCK(cudaMemsetAsync(m->d_err.p, 0, n * 4, s));
    launch_mark_touched(DArr{}, DLat{}, BrickBox{}, m->flags.as<uint32_t>(), nullptr, s, &S, m->sph_off[n]);
    launch_scan(m->flags.as<uint32_t>(), nf, nullptr, m->list.as<uint32_t>(), m->tiles.as<unsigned long long>(),
                m->tot.as<unsigned long long>(), s);
    unsigned long long n_touched = 0;
    std::vector<int> kerr(n);
    MCK(cudaMemcpyAsync(&n_touched, m->tot.p, 8, cudaMemcpyDeviceToHost, s));
    MCK(cudaMemcpyAsync(kerr.data(), m->d_err.p, n * 4, cudaMemcpyDeviceToHost, s));
    MCK(cudaStreamSynchronize(s));
    for (size_t i = 0; i < n; i++)
        if (kerr[i]) return set_err(err, errlen, "structure %zu: coordinates too far from the origin", i), SMB_ERR_RANGE;
    launch_classify_bricks(DArr{}, DLat{}, BrickBox{}, m->list.as<uint32_t>(), uint32_t(n_touched),
                           m->surf.as<uint32_t>(), s, &S);
    launch_scan(m->surf.as<uint32_t>(), nf, nullptr, m->cells.as<uint32_t>(), m->tiles.as<unsigned long long>(),
                m->tot.as<unsigned long long>(), s);
    unsigned long long n_surface = 0;
    MCK(cudaMemcpyAsync(&n_surface, m->tot.p, 8, cudaMemcpyDeviceToHost, s));
    MCK(cudaStreamSynchronize(s));
    if ((rc = m->keys.reserve(std::max<size_t>(n_surface, 1) * sizeof(int4), err, errlen))) return rc;
    launch_cells_to_keys(BrickBox{}, m->cells.as<uint32_t>(), uint32_t(n_surface), m->keys.as<int4>(), s, &S);
    m->n_bricks = uint32_t(n_surface);
    return SMB_OK;
}

// Device bytes one surface brick of a pass needs at the configured caps
// (records, values, list pools, marching-cubes and refinement outputs).
size_t bytes_per_brick(const smb_multi_config& c) {
    const int b = int(c.brick);
    const CapLevel& C = CAP_LEVELS[c.caps_level];
    const size_t spb = size_t(b + 1) * (b + 1) * (b + 1), edges = size_t(3) * b * b;
    return spb * 4 + 8 * (REC_WORDS * 4 + 12) + 4 * (size_t(C.ids_per_sub) * 4 + size_t(C.units_per_sub) * 16) +
           edges * (4 + 8 + 4 + 4 + 4 + 12 + 4) + 2 * edges * 12 + 8;
}

// Structures in order, grouped so that each group's surface bricks fit the
// pass buffers (a structure larger than that is a group of its own).
void form_groups(smb_multi* m) {
    const size_t n = m->n();
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t budget = std::max<size_t>(size_t(1) << 28, free_b / 3);
    m->group_bricks = std::max<size_t>(4096, budget / bytes_per_brick(m->cfg));
    std::vector<Group> g;
    size_t s0 = 0;
    while (s0 < n) {
        size_t s1 = s0 + 1;
        while (s1 < n && m->b0[s1 + 1] - m->b0[s0] <= m->group_bricks) s1++;
        Group G;
        G.s0 = s0, G.s1 = s1, G.k0 = m->b0[s0], G.k1 = m->b0[s1];
        g.push_back(G);
        s0 = s1;
    }
    // Keep recorded graphs whose group is unchanged.
    for (Group& G : g)
        for (Group& O : m->groups)
            if (O.graph && O.s0 == G.s0 && O.s1 == G.s1 && O.k0 == G.k0 && O.k1 == G.k1) std::swap(G.graph, O.graph),
                G.cfg = O.cfg, G.warm = O.warm, G.keys = O.keys, G.gen = O.gen;
    for (Group& O : m->groups)
        if (O.graph) cudaGraphExecDestroy(O.graph);
    m->groups.swap(g);
}

// Buffers of one pass of up to max_nb surface bricks at the configured caps.
int reserve_pass(smb_multi* m, size_t max_nb, char* err, size_t errlen) {
    const size_t nb = std::max<size_t>(max_nb, 1), nsub = nb * 8;
    const int b = m->cfg.brick;
    const CapLevel& C = CAP_LEVELS[m->cfg.caps_level];
    const size_t spb = size_t(b + 1) * (b + 1) * (b + 1);
    m->edge_cap = std::min<size_t>(size_t(0xFFFFFFF0u), nb * size_t(3) * b * b);
    m->tri_cap = std::min<size_t>(size_t(0xFFFFFFF0u), 2 * m->edge_cap);
    int rc;
    if ((rc = m->rec.reserve(nsub * REC_WORDS * 4, err, errlen)) || (rc = m->sampled.reserve(nsub * 4, err, errlen)) ||
        (rc = m->work.reserve(nsub * 4, err, errlen)) || (rc = m->retry.reserve(nsub * 4, err, errlen)) ||
        (rc = m->values.reserve(nb * spb * 4, err, errlen)) ||
        (rc = m->tiles.reserve(size_t(scan_tiles_needed(uint32_t(nsub))) * 8 + 64, err, errlen)) ||
        (rc = m->counters.reserve(CNT_N * 8, err, errlen)) ||
        (rc = m->ids.reserve(nsub / 2 * C.ids_per_sub * 4, err, errlen)) ||
        (rc = m->pack.reserve(nsub / 2 * C.units_per_sub * 16, err, errlen)) ||
        (rc = m->mc_counts.reserve(nb * 8, err, errlen)) || (rc = m->edge_off.reserve(nb * 4 + 4, err, errlen)) ||
        (rc = m->tri_off.reserve(nb * 4 + 4, err, errlen)) || (rc = m->edges.reserve(m->edge_cap * 4, err, errlen)) ||
        (rc = m->edge_vals.reserve(m->edge_cap * 8, err, errlen)) ||
        (rc = m->tris.reserve(m->tri_cap * 12, err, errlen)) || (rc = m->item_counts.reserve(nsub * 4, err, errlen)) ||
        (rc = m->item_off.reserve(nsub * 4 + 4, err, errlen)) ||
        (rc = m->item_edges.reserve(m->edge_cap * 4, err, errlen)) || (rc = m->e_t.reserve(m->edge_cap * 4, err, errlen)) ||
        (rc = m->e_feat.reserve(m->edge_cap * 4, err, errlen)) || (rc = m->e_q.reserve(m->edge_cap * 12, err, errlen)) ||
        (rc = m->e_evals.reserve(m->edge_cap * 4, err, errlen)) ||
        (m->warm && ((rc = m->w_feats.reserve(nb * spb * 4, err, errlen)) ||
                     (rc = m->w_start.reserve(m->edge_cap * 8, err, errlen)))))
        return rc;
    return SMB_OK;
}

// The mesh-stage pass over one group's surface bricks (keys [k0, k1)), all
// sizes fixed (no host synchronisation inside), as one stream of launches:
// recorded once into a CUDA graph, then replayed.
int enqueue_pass(smb_multi* m, const Group& G, char* err, size_t errlen) {
    cudaStream_t s = m->dev->stream;
    smb_device* d = m->dev;
    const uint32_t nb = uint32_t(G.k1 - G.k0), nsub = nb * 8;
    const int b = m->cfg.brick;
    const CapLevel& C = CAP_LEVELS[m->cfg.caps_level];
    const size_t spb = size_t(b + 1) * (b + 1) * (b + 1);
    Scene S = scene_of(m);
    const int4* keys = m->keys.as<int4>() + G.k0;
    unsigned long long* cnt = m->counters.as<unsigned long long>();
    unsigned long long* tot = m->totals.as<unsigned long long>();
    DLat L{};  // per-structure lattices come from the scene; b and spb are shared
    L.b = b, L.sub = b / 2, L.spb = int(spb);
    MCK(cudaMemsetAsync(cnt, 0, CNT_N * 8, s));
    MCK(cudaMemsetAsync(m->values.p, 0, size_t(nb) * spb * 4, s));
    launch_substates(DArr{}, DLat{}, keys, nb, m->rec.as<uint32_t>(), m->sampled.as<uint32_t>(), s, &S);
    launch_scan(m->sampled.as<uint32_t>(), nsub, nullptr, m->work.as<uint32_t>(), m->tiles.as<unsigned long long>(),
                tot, s);
    GatherOut O{m->rec.as<uint32_t>(), m->ids.as<uint32_t>(), m->pack.as<uint4>(), m->retry.as<uint32_t>(), cnt,
                m->ids.cap / 4, m->pack.cap / 16, m->unit_cap, m->d_fail.as<uint32_t>()};
    cudaError_t e = launch_gather(DArr{}, DLat{}, keys, m->work.as<uint32_t>(), nsub, O, C.caps,
                                  int(m->cfg.gather_warps), s, &S);
    if (e != cudaSuccess) return set_err(err, errlen, "gather launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    // Sub-blocks over the shared-memory list caps: once more, a warp per
    // block with four times the caps (the count is kept first: the retry
    // pass counts its own overflows in the same counter).
    {
        GatherCaps big = C.caps;
        big.near *= 4, big.s *= 4, big.c *= 4, big.v *= 4;
        launch_copy_count(cnt + CNT_RETRY, cnt + CNT_OVERFLOW, s);
        Scene R = S;
        R.n_work = cnt + CNT_RETRY;
        GatherOut O2 = O;
        O2.retry = nullptr;
        e = launch_gather(DArr{}, DLat{}, keys, m->retry.as<uint32_t>(), nsub, O2, big, 1, s, &R);
        if (e != cudaSuccess) return set_err(err, errlen, "gather launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    }
    e = launch_sample(DLat{}, keys, m->work.as<uint32_t>(), nsub, m->rec.as<uint32_t>(), m->pack.as<uint4>(),
                      m->unit_cap, m->values.as<float>(), cnt, true, false, s, &S, nullptr, 0, m->ids.as<uint32_t>(),
                      m->warm ? m->w_feats.as<uint32_t>() : nullptr);
    if (e != cudaSuccess) return set_err(err, errlen, "sample launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    e = launch_mc(L, nb, m->values.as<float>(), m->rec.as<uint32_t>(), m->mc_counts.as<uint32_t>(), nullptr, nullptr,
                  nullptr, nullptr, nullptr, false, s, keys, ~0ull, ~0ull, &S);
    if (e != cudaSuccess) return set_err(err, errlen, "mc launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    launch_scan(m->mc_counts.as<uint32_t>(), nb, m->edge_off.as<uint32_t>(), nullptr, m->tiles.as<unsigned long long>(),
                tot + 1, s);
    launch_scan(m->mc_counts.as<uint32_t>() + nb, nb, m->tri_off.as<uint32_t>(), nullptr,
                m->tiles.as<unsigned long long>(), tot + 2, s);
    launch_put_total(m->edge_off.as<uint32_t>() + nb, tot + 1, s);
    launch_put_total(m->tri_off.as<uint32_t>() + nb, tot + 2, s);
    e = launch_mc(L, nb, m->values.as<float>(), m->rec.as<uint32_t>(), nullptr, m->edge_off.as<uint32_t>(),
                  m->tri_off.as<uint32_t>(), m->edges.as<uint32_t>(), m->edge_vals.as<float2>(), m->tris.as<uint32_t>(),
                  true, s, keys, m->edge_cap, m->tri_cap, &S);
    if (e != cudaSuccess) return set_err(err, errlen, "mc launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    launch_item_edges(L, m->work.as<uint32_t>(), nsub, m->rec.as<uint32_t>(), m->edge_off.as<uint32_t>(),
                      m->edges.as<uint32_t>(), m->item_counts.as<uint32_t>(), m->item_off.as<uint32_t>(),
                      m->item_edges.as<uint32_t>(), m->tiles.as<unsigned long long>(), tot + 3, cnt, s, &S, keys);
    const int mode = m->warm ? REFINE_WARM : REFINE_PLAIN;
    if (m->warm) {
        e = launch_warm_starts(DArr{}, DLat{}, RefineConsts{}, keys, m->work.as<uint32_t>(), nsub,
                               m->rec.as<uint32_t>(), m->edges.as<uint32_t>(), m->edge_vals.as<float2>(),
                               m->item_off.as<uint32_t>(), m->item_edges.as<uint32_t>(), m->values.as<float>(),
                               m->w_feats.as<uint32_t>(), mlp_dev(m->warm), mlp_use(m->warm), m->w_start.as<float2>(),
                               cnt, m->edge_cap, d->info.multiprocessors, s, &S);
        if (e != cudaSuccess) return set_err(err, errlen, "warm start launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    }
    const size_t cand = size_t(m->unit_cap) * 16 + 64;
    e = launch_refine(DArr{}, DLat{}, RefineConsts{}, keys, m->work.as<uint32_t>(), m->rec.as<uint32_t>(),
                      m->ids.as<uint32_t>(), m->edges.as<uint32_t>(), m->edge_vals.as<float2>(),
                      m->item_off.as<uint32_t>(), m->item_edges.as<uint32_t>(), nsub, m->e_t.as<float>(),
                      m->e_feat.as<uint32_t>(), m->e_q.as<float>(), m->e_evals.as<uint32_t>(), cand, mode,
                      m->warm ? m->w_start.as<float2>() : nullptr, cnt, d->info.multiprocessors, d->smem_optin, s,
                      nullptr, &S);
    if (e != cudaSuccess) return set_err(err, errlen, "refine launch: %s", cudaGetErrorString(e)), SMB_ERR_CUDA;
    return SMB_OK;
}

// Runs one group's pass: from its recorded graph when that matches the
// configuration, else directly once (setting the kernels' attributes) and
// then records it; direct launches if recording is refused.
int run_group(smb_multi* m, Group& G, float* device_ms, char* err, size_t errlen) {
    cudaStream_t s = m->dev->stream;
    int rc;
    if (!m->ev[0]) cudaEventCreate(&m->ev[0]), cudaEventCreate(&m->ev[1]);
    *device_ms = 0;
    if (G.k1 == G.k0) return SMB_OK;
    const bool same = G.graph && G.cfg.brick == m->cfg.brick && G.cfg.caps_level == m->cfg.caps_level &&
                      G.cfg.gather_warps == m->cfg.gather_warps && G.warm == m->warm && G.keys == m->keys.p &&
                      G.gen == m->gen;
    if (!same) {
        if (G.graph) cudaGraphExecDestroy(G.graph), G.graph = nullptr;
        // Direct passes: the first sets the kernels' attributes; when lists
        // ran past the pools or the sampler's block cap, those grow to what
        // the pass counted and the pass runs again (twice at most).
        for (int attempt = 0;; attempt++) {
            MCK(cudaEventRecord(m->ev[0], s));
            if ((rc = enqueue_pass(m, G, err, errlen))) return rc;
            MCK(cudaEventRecord(m->ev[1], s));
            MCK(cudaStreamSynchronize(s));
            unsigned long long c[CNT_N];
            MCK(cudaMemcpy(c, m->counters.p, sizeof c, cudaMemcpyDeviceToHost));
            if (!c[CNT_NOMEM] || attempt >= 2) break;
            bool grow = false;
            if (c[CNT_IDS] > m->ids.cap / 4) {
                if ((rc = m->ids.reserve(size_t(c[CNT_IDS]) * 4, err, errlen))) return rc;
                grow = true;
            }
            if (c[CNT_PACK] > m->pack.cap / 16) {
                if ((rc = m->pack.reserve(size_t(c[CNT_PACK]) * 16, err, errlen))) return rc;
                grow = true;
            }
            const unsigned long long unit_limit = (m->dev->smem_optin - 64) / 16;
            if (c[CNT_MAXPACK] > m->unit_cap && c[CNT_MAXPACK] <= unit_limit) {
                m->unit_cap = uint32_t(c[CNT_MAXPACK]);
                grow = true;
            }
            if (!grow) break;
            m->gen++;
            MCK(cudaMemsetAsync(m->d_fail.as<uint32_t>() + G.s0, 0, (G.s1 - G.s0) * 4, s));
        }
        cudaGraph_t g = nullptr;
        if (m->graph_ok && cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            char e2[256] = {0};
            int prc = enqueue_pass(m, G, e2, sizeof e2);
            cudaError_t ce = cudaStreamEndCapture(s, &g);
            if (prc == SMB_OK && ce == cudaSuccess && g && cudaGraphInstantiate(&G.graph, g, 0) == cudaSuccess) {
                G.cfg = m->cfg, G.warm = m->warm, G.keys = m->keys.p, G.gen = m->gen;
            } else {
                G.graph = nullptr;
                m->graph_ok = false;
                cudaGetLastError();
            }
            if (g) cudaGraphDestroy(g);
        }
        cudaEventElapsedTime(device_ms, m->ev[0], m->ev[1]);
        return SMB_OK;
    }
    MCK(cudaEventRecord(m->ev[0], s));
    MCK(cudaGraphLaunch(G.graph, s));
    MCK(cudaEventRecord(m->ev[1], s));
    MCK(cudaStreamSynchronize(s));
    cudaEventElapsedTime(device_ms, m->ev[0], m->ev[1]);
    return SMB_OK;
}

// Classification of every structure, brick ranges and groups, buffers.
int prepare_run(smb_multi* m, double* classify_ms, char* err, size_t errlen) {
    int rc;
    if ((rc = set_brick(m, m->cfg.brick, err, errlen))) return rc;
    auto t0 = clk::now();
    if ((rc = classify_all(m, err, errlen))) return rc;
    const size_t n = m->n(), nb = m->n_bricks;
    m->keys4.resize(nb);
    if (nb) MCK(cudaMemcpy(m->keys4.data(), m->keys.p, nb * sizeof(int4), cudaMemcpyDeviceToHost));
    *classify_ms = ms_since(t0);
    m->b0.assign(n + 1, nb);
    for (size_t i = nb; i-- > 0;) m->b0[size_t(m->keys4[i].w)] = i;
    for (size_t i = n; i-- > 0;) m->b0[i] = std::min(m->b0[i], m->b0[i + 1]);
    form_groups(m);
    const smb_multi_config& c = m->cfg;
    if (!m->unit_cap || c.brick != m->unit_cfg.brick || c.caps_level != m->unit_cfg.caps_level) {
        m->unit_cap = CAP_LEVELS[c.caps_level].unit_cap;
        m->unit_cfg = c;
        m->gen++;
    }
    size_t max_nb = 0;
    for (const Group& G : m->groups) max_nb = std::max(max_nb, G.k1 - G.k0);
    if ((rc = reserve_pass(m, max_nb, err, errlen))) return rc;
    MCK(cudaMemsetAsync(m->d_fail.p, 0, n * 4, m->dev->stream));
    return SMB_OK;
}

int fetch_group(smb_multi* m, const Group& G, HostGroup& H, char* err, size_t errlen, bool full = true) {
    const size_t nb = G.k1 - G.k0;
    cudaStream_t s = m->dev->stream;
    H.ne = H.nt = 0;
    if (!H.eo.reserve((nb + 1) * 4) || !H.to.reserve((nb + 1) * 4))
        return set_err(err, errlen, "page-locked host memory"), SMB_ERR_MEMORY;
    if (!nb) {
        H.eo.as<uint32_t>()[0] = H.to.as<uint32_t>()[0] = 0;
        return SMB_OK;
    }
    unsigned long long t3[4] = {0, 0, 0, 0};
    MCK(cudaMemcpy(t3, m->totals.p, 32, cudaMemcpyDeviceToHost));
    H.ne = std::min<size_t>(t3[1], m->edge_cap), H.nt = std::min<size_t>(t3[2], m->tri_cap);
    const size_t ne = H.ne, nt = H.nt;
    if (!H.edges.reserve(ne * 4 + 4) || !H.tris.reserve(nt * 12 + 4) || !H.feat.reserve(ne * 4 + 4) ||
        !H.evals.reserve(ne * 4 + 4) || !H.ev.reserve(ne * 8 + 8) || !H.t.reserve(ne * 4 + 4) ||
        !H.q.reserve(ne * 12 + 12))
        return set_err(err, errlen, "page-locked host memory"), SMB_ERR_MEMORY;
    MCK(cudaMemcpyAsync(H.eo.p, m->edge_off.p, (nb + 1) * 4, cudaMemcpyDeviceToHost, s));
    MCK(cudaMemcpyAsync(H.to.p, m->tri_off.p, (nb + 1) * 4, cudaMemcpyDeviceToHost, s));
    if (!full) {
        MCK(cudaStreamSynchronize(s));
        return SMB_OK;
    }
    if (ne) {
        MCK(cudaMemcpyAsync(H.edges.p, m->edges.p, ne * 4, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(H.ev.p, m->edge_vals.p, ne * 8, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(H.t.p, m->e_t.p, ne * 4, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(H.feat.p, m->e_feat.p, ne * 4, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(H.q.p, m->e_q.p, ne * 12, cudaMemcpyDeviceToHost, s));
        MCK(cudaMemcpyAsync(H.evals.p, m->e_evals.p, ne * 4, cudaMemcpyDeviceToHost, s));
    }
    if (nt) MCK(cudaMemcpyAsync(H.tris.p, m->tris.p, nt * 12, cudaMemcpyDeviceToHost, s));
    MCK(cudaStreamSynchronize(s));
    return SMB_OK;
}

}  // namespace

extern "C" {

int smb_multi_new(smb_device* dev, size_t n, const double* const* xyzr, const size_t* counts,
                  const smb_surface_params* params, const smb_multi_config* cfg, smb_multi** out, char* err,
                  size_t errlen) {
    if (!dev || !out || (n && (!xyzr || !counts || !params))) return set_err(err, errlen, "null argument"), SMB_ERR_ARG;
    *out = nullptr;
    if (n == 0 || n >= (size_t(1) << 31)) return set_err(err, errlen, "structure count must be 1..2^31"), SMB_ERR_ARG;
    smb_multi_config c = cfg ? *cfg : smb_multi_config{};
    if (c.brick && (c.brick < 4 || c.brick > 32 || c.brick % 2))
        return set_err(err, errlen, "brick must be 0 (tuned) or even and 4..32, got %u", c.brick), SMB_ERR_ARG;
    if (c.caps_level > 1) return set_err(err, errlen, "caps level must be 0 or 1"), SMB_ERR_ARG;
    if (c.gather_warps && c.gather_warps != 1 && c.gather_warps != 2 && c.gather_warps != 4 && c.gather_warps != 8)
        return set_err(err, errlen, "gather warps must be 0 (tuned), 1, 2, 4 or 8"), SMB_ERR_ARG;
    for (size_t i = 0; i < n; i++) {
        if (params[i].refine != SMB_REFINE_FAST)
            return set_err(err, errlen, "structure %zu: the batch meshes in fast mode", i), SMB_ERR_ARG;
        if (params[i].kind != SMB_SES || !(params[i].probe_radius > 0.0))
            return set_err(err, errlen, "structure %zu: the batch meshes the SES (probe > 0)", i), SMB_ERR_ARG;
    }
    auto t0 = clk::now();
    auto m = std::make_unique<smb_multi>();
    m->dev = dev;
    dev_retain(dev);
    m->cfg = c;
    m->tuned = c.brick != 0 && c.gather_warps != 0;
    m->eng.assign(n, nullptr);
    for (size_t i = 0; i < n; i++) {
        smb_surface_params p = params[i];
        p.brick_size = c.brick ? c.brick : 8;
        int rc = smb_engine_new(dev, xyzr[i], counts[i], &p, &m->eng[i], err, errlen);
        if (rc != SMB_OK) {
            char tmp[512];
            snprintf(tmp, sizeof tmp, "structure %zu: %s", i, err ? err : "");
            set_err(err, errlen, "%s", tmp);
            smb_multi_free(m.release());
            return rc;
        }
    }
    if (!m->cfg.gather_warps) m->cfg.gather_warps = 4;
    if (!m->cfg.brick) m->cfg.brick = 8;
    m->t_setup = ms_since(t0);
    *out = m.release();
    return SMB_OK;
}

void smb_multi_free(smb_multi* m) {
    if (!m) return;
    cudaSetDevice(m->dev->index);
    cudaStreamSynchronize(m->dev->stream);
    for (Group& G : m->groups)
        if (G.graph) cudaGraphExecDestroy(G.graph);
    for (auto& ev : m->ev)
        if (ev) cudaEventDestroy(ev);
    for (DBuf* b : m->bufs()) b->release();
    delete[] m->hosts;
    for (smb_engine* e : m->eng) smb_engine_free(e);
    smb_device* d = m->dev;
    delete m;
    dev_release(d);
}

int smb_multi_set_control(smb_multi* m, const smb_control* c) {
    if (!m) return SMB_ERR_ARG;
    m->ctl = smbh::Control();
    if (c) m->ctl.cancel = c->cancel, m->ctl.progress = c->progress, m->ctl.user = c->user;
    return SMB_OK;
}

int smb_multi_set_warm_start(smb_multi* m, const smb_mlp* mlp) {
    if (!m) return SMB_ERR_ARG;
    m->warm = mlp;
    for (smb_engine* e : m->eng) smb_engine_set_warm_start(e, mlp);
    return SMB_OK;
}

int smb_multi_tune(smb_multi* m, char* err, size_t errlen) {
    if (!m) return SMB_ERR_ARG;
    if (cudaSetDevice(m->dev->index) != cudaSuccess) return set_err(err, errlen, "cudaSetDevice failed"), SMB_ERR_CUDA;
    auto t0 = clk::now();
    // Candidates: brick edge 8 or 16, candidate caps level 0 or 1, 2 or 4
    // warps per gather block.  Each runs the device part over every group
    // (first pass of a configuration, so recording included); score: its
    // time plus classification plus the single-structure cost of the
    // structures over a cap (their share of the pass, times four).
    smb_multi_config best = m->cfg;
    double best_score = 1e300;
    std::string last;
    const int bricks[2] = {8, 16};
    const uint32_t warps[2] = {2, 4};
    for (int b : bricks)
        for (uint32_t lvl = 0; lvl < 2; lvl++)
            for (uint32_t w : warps) {
                m->cfg.brick = uint32_t(b), m->cfg.caps_level = lvl, m->cfg.gather_warps = w;
                double cms = 0, dev = 0;
                float dms = 0;
                int rc = prepare_run(m, &cms, err, errlen);
                for (size_t gi = 0; rc == SMB_OK && gi < m->groups.size(); gi++)
                    rc = run_group(m, m->groups[gi], &dms, err, errlen), dev += dms;
                if (rc != SMB_OK) {
                    last = err ? err : "";
                    continue;
                }
                std::vector<uint32_t> f(m->n());
                if (cudaMemcpy(f.data(), m->d_fail.p, m->n() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) continue;
                const double all = double(std::max<uint32_t>(m->n_bricks, 1));
                double fails = 0;
                for (size_t i = 0; i < m->n(); i++) fails += f[i] ? double(m->b0[i + 1] - m->b0[i]) : 0.0;
                double score = cms + dev + 4.0 * dev * fails / all;
                if (score < best_score) best_score = score, best = m->cfg;
            }
    if (best_score >= 1e300) return set_err(err, errlen, "no configuration ran: %s", last.c_str()), SMB_ERR_CUDA;
    m->cfg = best;
    m->tuned = true;
    m->t_tune = ms_since(t0);
    return SMB_OK;
}

int smb_multi_set_device_finish(smb_multi* m, int on) {
    if (!m) return SMB_ERR_ARG;
    m->device_finish = on != 0;
    return SMB_OK;
}

int smb_multi_config_get(const smb_multi* m, smb_multi_config* out) {
    if (!m || !out) return SMB_ERR_ARG;
    *out = m->cfg;
    return SMB_OK;
}

namespace {

__global__ void k_rebase(uint32_t* dst, const uint32_t* src, size_t n, uint32_t delta) {
    const size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    if (i < n) dst[i] = src[i] + delta;
}

// Structure i of group G finished on the device: its slice of the group's
// results (bricks, sub-block records, work items, marching-cubes lists, f32
// roots) is copied into its engine's own batch in the single-structure
// layout (offsets rebased to the slice), then placed (smb_place_fast: the
// converged roots with their exact attributes, the rest refined exactly),
// assembled, validated and measured there.  work: the group's work list on
// the host.  *fallback when the device left the structure to the host.
int finish_structure_device(smb_multi* m, const Group& G, size_t i, const uint32_t* eo, const uint32_t* to,
                            const uint32_t* work, size_t n_work, smb_surface& s, bool* fallback, char* err,
                            size_t errlen) {
    *fallback = false;
    smb_engine* e = m->eng[i];
    smb_resident* r = e->res;
    smb_batch* b = e->batch;
    cudaStream_t st = m->dev->stream;
    const size_t lo = m->b0[i] - G.k0, hi = m->b0[i + 1] - G.k0, nb = hi - lo;
    const uint32_t e0 = eo[lo], e1 = eo[hi], t0 = to[lo], t1 = to[hi];
    const size_t ne = e1 - e0, nt = t1 - t0;
    const uint32_t* w0 = std::lower_bound(work, work + n_work, uint32_t(8 * lo));
    const uint32_t* w1 = std::lower_bound(work, work + n_work, uint32_t(8 * hi));
    const size_t nw = size_t(w1 - w0), wo = size_t(w0 - work);
    r->L = m->lat[i];
    e->mp = m->mp[i];
    if (r->keys) mem_free(r->keys);
    r->keys = nullptr;
    if (nb && mem_alloc(reinterpret_cast<void**>(&r->keys), nb * sizeof(int4)) != cudaSuccess)
        return set_err(err, errlen, "device memory for structure %zu", i), SMB_ERR_MEMORY;
    r->n_bricks = uint32_t(nb);
    r->classified = true;
    int rc;
    if ((rc = b->rec.reserve(std::max<size_t>(nb, 1) * 8 * REC_WORDS * 4, err, errlen)) ||
        (rc = b->work.reserve(std::max<size_t>(nw, 1) * 4, err, errlen)) ||
        (rc = b->edge_off.reserve((nb + 1) * 4, err, errlen)) || (rc = b->tri_off.reserve((nb + 1) * 4, err, errlen)) ||
        (rc = b->edges.reserve(std::max<size_t>(ne, 1) * 4, err, errlen)) ||
        (rc = b->edge_vals.reserve(std::max<size_t>(ne, 1) * 8, err, errlen)) ||
        (rc = b->tris.reserve(std::max<size_t>(nt, 1) * 12, err, errlen)) ||
        (rc = b->e_t.reserve(std::max<size_t>(ne, 1) * 4, err, errlen)) ||
        (rc = b->e_feat.reserve(std::max<size_t>(ne, 1) * 4, err, errlen)) ||
        (rc = b->e_q.reserve(std::max<size_t>(ne, 1) * 12, err, errlen)) ||
        (rc = b->e_evals.reserve(std::max<size_t>(ne, 1) * 4, err, errlen)) ||
        (rc = b->totals.reserve(64, err, errlen)) || (rc = b->counters.reserve(CNT_N * 8, err, errlen)))
        return rc;
    auto d2d = [&](void* dst, const void* src, size_t bytes) {
        return !bytes || cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    };
    auto rebase = [&](uint32_t* dst, const uint32_t* src, size_t n, uint32_t delta) {
        if (n) k_rebase<<<unsigned((n + 255) / 256), 256, 0, st>>>(dst, src, n, delta);
        return cudaGetLastError() == cudaSuccess;
    };
    const size_t sub0 = 8 * lo;
    if (!d2d(r->keys, m->keys.as<int4>() + G.k0 + lo, nb * sizeof(int4)) ||
        !d2d(b->rec.p, m->rec.as<uint32_t>() + sub0 * REC_WORDS, nb * 8 * REC_WORDS * 4) ||
        !rebase(b->work.as<uint32_t>(), m->work.as<uint32_t>() + wo, nw, uint32_t(0) - uint32_t(sub0)) ||
        !rebase(b->edge_off.as<uint32_t>(), m->edge_off.as<uint32_t>() + lo, nb + 1, uint32_t(0) - e0) ||
        !rebase(b->tri_off.as<uint32_t>(), m->tri_off.as<uint32_t>() + lo, nb + 1, uint32_t(0) - t0) ||
        !d2d(b->edges.p, m->edges.as<uint32_t>() + e0, ne * 4) ||
        !d2d(b->edge_vals.p, m->edge_vals.as<float2>() + e0, ne * 8) ||
        !d2d(b->tris.p, m->tris.as<uint32_t>() + 3 * size_t(t0), nt * 12) ||
        !d2d(b->e_t.p, m->e_t.as<float>() + e0, ne * 4) || !d2d(b->e_feat.p, m->e_feat.as<uint32_t>() + e0, ne * 4) ||
        !d2d(b->e_q.p, m->e_q.as<float>() + 3 * size_t(e0), ne * 12) ||
        !d2d(b->e_evals.p, m->e_evals.as<uint32_t>() + e0, ne * 4))
        return set_err(err, errlen, "copy of structure %zu's results failed", i), SMB_ERR_CUDA;
    count_launches(3);
    b->first = 0;
    b->window_ok = false;  // the slice brings records, not the gather's ids or marks
    b->n = uint32_t(nb);
    b->n_work = uint32_t(nw);
    b->n_edges = ne;
    b->n_tris = nt;
    b->refined = true;
    b->refined_exact = false;
    // The engine's buffers go back to the memory cache afterwards: the next
    // structure takes them from there (one structure's worth held at a time).
    auto release = [&](int code) {
        cudaDeviceSynchronize();
        for (DBuf* x : b->bufs()) x->release_synced();
        e->measure.release(true);
        mem_free_synced(r->keys);
        r->keys = nullptr;
        r->n_bricks = 0;
        b->refined = b->refined_exact = false;
        return code;
    };
    double ms = 0;
    if ((rc = smb_place_fast(r, b, &ms, err, errlen)) != SMB_OK) return release(rc);
    unsigned long long evals = 0, host_edges = 0, exact_edges = 0;
    if ((rc = smb_batch_exact_summary(b, &evals, &host_edges, &exact_edges)) != SMB_OK)
        return release((set_err(err, errlen, "vertex summary failed"), rc));
    if (host_edges || !nb) {
        *fallback = true;
        return release(SMB_OK);
    }
    double ms_d2h = 0;
    return release(finish_exact_device(e, s, evals, exact_edges, fallback, &ms_d2h, err, errlen));
}

}  // namespace

int smb_multi_run(smb_multi* m, smb_multi_times* times, char* err, size_t errlen) {
    if (!m) return SMB_ERR_ARG;
    if (cudaSetDevice(m->dev->index) != cudaSuccess) return set_err(err, errlen, "cudaSetDevice failed"), SMB_ERR_CUDA;
    int rc;
    if (!m->tuned && (rc = smb_multi_tune(m, err, errlen))) return rc;
    auto t_start = clk::now();
    double cms = 0;
    if ((rc = prepare_run(m, &cms, err, errlen))) return rc;
    const size_t n = m->n();
    m->out.clear();
    m->out.resize(n);
    m->latency.assign(n, 0.0);
    m->redone.assign(n, 0);
    std::vector<std::string> errs(n);
    double t_device = 0, t_d2h = 0, t_finish = 0;
    unsigned long long over_lists = 0, over_memory = 0;
    bool graphs = true;
    // Group by group: the device pass of group g + 1 runs while the host
    // threads finish group g (results in two alternating page-locked sets).
    if (!m->hosts) m->hosts = new HostGroup[2];
    HostGroup* hosts = m->hosts;
    std::thread worker;
    auto t_host0 = clk::now();
    double t_host = 0;
    size_t finished = 0;
    m->ctl.report(SMB_STAGE_MESH, 0, n);
    for (size_t gi = 0; gi < m->groups.size(); gi++) {
        Group& G = m->groups[gi];
        float dms = 0;
        // Cancellation between groups (the host stages of the group before
        // finish first).
        if (m->ctl.cancelled()) {
            if (worker.joinable()) worker.join();
            return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED;
        }
        if ((rc = run_group(m, G, &dms, err, errlen))) {
            if (worker.joinable()) worker.join();
            return rc;
        }
        if (gi) m->ctl.report(SMB_STAGE_MESH, finished, n);
        finished = G.s1;
        graphs = graphs && (G.graph != nullptr || G.k1 == G.k0);
        t_device += dms;
        auto t1 = clk::now();
        std::vector<uint32_t> fail(n);
        HostGroup& Hc = hosts[gi % 2];
        if ((rc = fetch_group(m, G, Hc, err, errlen, !m->device_finish)) ||
            cudaMemcpy(fail.data(), m->d_fail.p, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            if (worker.joinable()) worker.join();
            return rc ? rc : (set_err(err, errlen, "copy of the failure flags failed"), SMB_ERR_CUDA);
        }
        t_d2h += ms_since(t1);
        unsigned long long c[CNT_N];
        if (cudaMemcpy(c, m->counters.p, sizeof c, cudaMemcpyDeviceToHost) == cudaSuccess) {
            over_lists += c[CNT_OVERFLOW] - c[CNT_RETRY];  // after the retry pass
            over_memory += c[CNT_NOMEM];
        }
        for (size_t i = G.s0; i < G.s1; i++) {
            const size_t hi = m->b0[i + 1] - G.k0;
            if (fail[i] || Hc.eo.as<uint32_t>()[hi] > Hc.ne || Hc.to.as<uint32_t>()[hi] > Hc.nt) m->redone[i] = 1;
        }
        // On the device: each structure placed, refined where the f32 search
        // left edges, assembled and measured; those it declines (host[i])
        // are finished on the host threads below.
        std::vector<uint8_t> host(n, m->device_finish ? 0 : 1);
        if (m->device_finish) {
            auto t2 = clk::now();
            std::vector<uint32_t> work;
            unsigned long long nw = 0;
            if (G.k1 > G.k0) {
                if (cudaMemcpy(&nw, m->totals.p, 8, cudaMemcpyDeviceToHost) != cudaSuccess) {
                    if (worker.joinable()) worker.join();
                    return set_err(err, errlen, "copy of the work count failed"), SMB_ERR_CUDA;
                }
                work.resize(size_t(nw));
                if (nw && cudaMemcpy(work.data(), m->work.p, size_t(nw) * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
                    if (worker.joinable()) worker.join();
                    return set_err(err, errlen, "copy of the work list failed"), SMB_ERR_CUDA;
                }
            }
            for (size_t i = G.s0; i < G.s1; i++) {
                if (m->redone[i]) continue;
                auto s = std::make_unique<smb_surface>();
                bool fallback = false;
                if ((rc = finish_structure_device(m, G, i, Hc.eo.as<uint32_t>(), Hc.to.as<uint32_t>(), work.data(),
                                                  work.size(), *s, &fallback, err, errlen))) {
                    if (worker.joinable()) worker.join();
                    return rc;
                }
                if (fallback) {
                    host[i] = 1;
                    continue;
                }
                s->stats.t_geometry = m->eng[i]->t_geometry;
                s->stats.t_upload = m->eng[i]->t_upload;
                m->out[i] = std::move(s);
                m->latency[i] = ms_since(t_start);
            }
            t_finish += ms_since(t2);
            bool any = false;
            for (size_t i = G.s0; i < G.s1; i++) any = any || (host[i] && !m->redone[i]);
            if (any) {  // the host threads need the group's lists
                if (worker.joinable()) worker.join();
                auto t3 = clk::now();
                if ((rc = fetch_group(m, G, Hc, err, errlen, true))) return rc;
                t_d2h += ms_since(t3);
            }
        }
        if (worker.joinable()) worker.join();
        worker = std::thread([m, gi, hosts, &errs, t_start, host] {
            const Group& G = m->groups[gi];
            const HostGroup& H = hosts[gi % 2];
            const uint32_t* eo = H.eo.as<uint32_t>();
            const uint32_t* to = H.to.as<uint32_t>();
            auto one = [&](size_t i) {
                const size_t lo = m->b0[i] - G.k0, hi = m->b0[i + 1] - G.k0, nbi = hi - lo;
                std::vector<int32_t> k3(3 * nbi);
                std::vector<uint32_t> leo(nbi + 1), lto(nbi + 1);
                for (size_t j = 0; j < nbi; j++) {
                    const int4& k = m->keys4[G.k0 + lo + j];
                    k3[3 * j] = k.x, k3[3 * j + 1] = k.y, k3[3 * j + 2] = k.z;
                }
                for (size_t j = 0; j <= nbi; j++) leo[j] = eo[lo + j] - eo[lo], lto[j] = to[lo + j] - to[lo];
                const size_t e0 = eo[lo], tr0 = to[lo];
                auto s = std::make_unique<smb_surface>();
                smb_engine* e = m->eng[i];
                std::string msg = finish_surface(
                    host_arrangement(e), m->mp[i], true, k3.data(), nbi, leo.data(), H.edges.as<uint32_t>() + e0,
                    H.ev.as<float>() + 2 * e0, lto.data(), H.tris.as<uint32_t>() + 3 * tr0,
                    DeviceRefine{H.t.as<float>() + e0, H.feat.as<uint32_t>() + e0, H.q.as<float>() + 3 * e0,
                                 H.evals.as<uint32_t>() + e0},
                    *s);
                if (!msg.empty()) {
                    errs[i] = msg;
                    return;
                }
                s->stats.t_geometry = e->t_geometry;
                s->stats.t_upload = e->t_upload;
                m->out[i] = std::move(s);
                m->latency[i] = ms_since(t_start);
            };
            // One host thread per structure, the largest first (longest
            // processing time first keeps the threads evenly loaded).
            std::vector<size_t> order;
            for (size_t i = G.s0; i < G.s1; i++)
                if (!m->redone[i] && host[i]) order.push_back(i);
            auto edges_of = [&](size_t i) { return eo[m->b0[i + 1] - G.k0] - eo[m->b0[i] - G.k0]; };
            std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return edges_of(a) > edges_of(b); });
            parallel_for(order.size(), [&](size_t k, int) {
                SerialScope serial;
                one(order[k]);
            });
        });
    }
    if (worker.joinable()) worker.join();
    t_host = ms_since(t_host0) - t_device - t_d2h - t_finish;
    for (size_t i = 0; i < n; i++)
        if (!errs[i].empty()) return set_err(err, errlen, "structure %zu: %s", i, errs[i].c_str()), SMB_ERR_STATE;
    auto t3b = clk::now();
    size_t n_redone = 0;
    for (size_t i = 0; i < n; i++) {
        if (!m->redone[i]) continue;
        if (m->ctl.cancelled()) return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED;
        n_redone++;
        smb_surface* s = nullptr;
        smb_engine* e = m->eng[i];
        // The engine meshes on its own, at the batch's brick edge, with
        // retries on every cap.
        e->res->L = m->lat[i];
        e->mp = m->mp[i];
        if ((rc = smb_engine_mesh(e, &s, err, errlen))) return rc;
        m->out[i].reset(s);
        m->latency[i] = ms_since(t_start);
    }
    double t_redo = ms_since(t3b);
    if (m->ctl.cancelled()) return set_err(err, errlen, "cancelled"), SMB_ERR_CANCELLED;
    m->ctl.report(SMB_STAGE_MESH, n, n);
    if (times) {
        smb_multi_times& T = *times;
        T = smb_multi_times{};
        T.structures = n;
        T.redone = n_redone;
        T.bricks = m->n_bricks;
        T.samples = size_t(m->n_bricks) * size_t(m->cfg.brick + 1) * size_t(m->cfg.brick + 1) * size_t(m->cfg.brick + 1);
        T.t_setup = m->t_setup;
        T.t_tune = m->t_tune;
        T.t_classify = cms;
        T.t_device = t_device + t_finish;
        T.t_d2h = t_d2h;
        T.t_host = t_host;
        T.t_redo = t_redo;
        T.t_total = ms_since(t_start);
        T.graph = graphs ? 1 : 0;
        T.groups = m->groups.size();
        T.over_lists = over_lists;
        T.over_memory = over_memory;
    }
    return SMB_OK;
}

smb_surface* smb_multi_surface(smb_multi* m, size_t i) {
    if (!m || i >= m->out.size()) return nullptr;
    return m->out[i].get();
}

int smb_multi_latency(const smb_multi* m, double* ms) {
    if (!m || !ms) return SMB_ERR_ARG;
    if (m->latency.size() != m->n()) return SMB_ERR_STATE;
    std::copy(m->latency.begin(), m->latency.end(), ms);
    return SMB_OK;
}

}  // extern "C"
