// Test and benchmark infrastructure, not part of the product: runs the
// reference's own CUDA kernels (crates/sesmesh-gpu/kernels/sesmesh.cuh,
// compiled from their source by oracle/Makefile's ref-gpu target into
// oracle/_ref/) on one batch of surface bricks, in the order of
// cuda::Resident::run (crates/sesmesh-gpu/src/cuda/resident.rs:494-572):
// count pass, host scan of the list sizes (resident.rs:541-558), fill pass,
// sample pass, 64 threads per sub-block (resident.rs:29); and, for fast
// mode, cuda::Resident::refine's edge count, host scan and refine passes
// (resident.rs:632-687).  It gives the reference's device sample values and
// f32 roots (compared with this library's in tests) and its kernel times on
// this GPU (the bar the benchmark reports).
//
// The two structs below restate the parameter layout the reference kernels
// take by value (sesmesh.cuh:58-81); the kernels are declared, not defined,
// here and link from the reference's translation unit.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

struct RefGrid {
    const unsigned* starts;
    const unsigned* items;
    float ox, oy, oz, cell;
    unsigned dx, dy, dz, n_items;
};

struct RefParams {
    const float *px, *py, *pz, *pr, *pr2, *pr2tol, *pvdw;
    const unsigned* status;
    const unsigned *nb_off, *nb_items;
    const float *cx, *cy, *cz, *ux, *uy, *uz, *ex, *ey, *ez, *crho;
    const unsigned *cb_off, *cb_items;
    const float *vx, *vy, *vz;
    RefGrid gs, gc, gv;
    const int* bricks;
    unsigned* rec;
    unsigned* ids;
    float* values;
    unsigned long long ids_len, values_len;
    unsigned n_sub, kind, n_spheres, n_circles, n_vertices, b, sub, near;
    float probe, band, cutoff2, rho, reach, margin, slack, cutoffc2, h, max_expanded, rho_max, pad2;
};

// RefineParams (sesmesh.cuh:430-442), by value to the fast-mode kernels.
struct RefRefine {
    const float *plx, *ply, *plz;
    const float *clx, *cly, *clz;
    const float *vlx, *vly, *vlz;
    unsigned* edge_count;
    const unsigned* edge_off;
    float* t_out;
    unsigned* feat_out;
    float* q_out;
    unsigned* evals_out;
    unsigned n_edges, max_iter, max_bisect, pad0;
    float h_hi, h_lo, tol, pad;
};

extern "C" __global__ void sesmesh_resident_count(RefParams p);
extern "C" __global__ void sesmesh_resident_fill(RefParams p);
extern "C" __global__ void sesmesh_resident_sample(RefParams p);
extern "C" __global__ void sesmesh_resident_edge_count(RefParams p, RefRefine r);
extern "C" __global__ void sesmesh_resident_refine(RefParams p, RefRefine r);

extern "C" {

// Host inputs, the reference's ArrangementRef (batch.rs:59-83) and
// BatchParams (batch.rs:86-115) as gpu.rs builds them (host_arrangement,
// grid, batch_params, frame_origins; field/gpu.rs:233-414).
typedef struct {
    unsigned n_spheres, n_circles, n_vertices;
    const float* sphere;  // 7 x n_spheres SoA: x, y, z, R, R^2, (R - tol)^2, r_vdw
    const unsigned* status;
    const unsigned *nb_off, *nb_items;
    unsigned nb_items_len;
    const float* circle;  // 10 x n_circles SoA: centre, axis, e1, radius
    const unsigned *cb_off, *cb_items;
    unsigned cb_items_len;
    const float* vertex;  // 3 x n_vertices SoA
    const float* grid_f;  // 3 x (ox, oy, oz, cell)
    const unsigned* grid_dims;  // 3 x (dx, dy, dz)
    const unsigned* grid_starts[3];
    const unsigned* grid_items[3];
    unsigned grid_n_items[3];
    float max_expanded, rho_max;
    float probe, band, cutoff2, rho, reach, margin, slack, cutoffc2, h;
    unsigned b, sub;
    const int* bricks;  // 3 per brick: brick origin minus frame, lattice units
    unsigned n_bricks;
} RefInput;

typedef struct {
    double count_ms, scan_ms, fill_ms, sample_ms, total_ms;  // per pass, best of the repetitions
    unsigned long long ids;
} RefTimes;

// Fast mode (cuda::Resident::set_refinement + refine, resident.rs:446-474,
// 632-687): the f32 residuals of the frame-local centres (Residuals,
// field/gpu.rs:182-222), the iteration constants, and the outputs per
// refined edge (sub-block order) with the per-sub-block offsets.
typedef struct {
    const float* sphere_lo;  // 3 x n_spheres SoA
    const float* circle_lo;  // 3 x n_circles
    const float* vertex_lo;  // 3 x n_vertices
    float h_hi, h_lo, tol;
    unsigned max_iter, max_bisect;
    unsigned* edge_off;      // out: 8 n_bricks + 1
    float* t;                // out: cap each
    unsigned* feat;
    float* q;                // out: 3 cap
    unsigned* evals;
    unsigned long long cap, n_edges;  // in: capacity; out: edges refined
    double edge_count_ms, scan_ms, refine_ms;  // best of the repetitions
} RefFast;

static int run_fast(RefParams& P, RefFast* f, int reps, std::vector<void*>& owned);

// Runs the batch `reps` times (the first a warm-up); values gets (b+1)^3
// floats per brick of the last run.  With fast, then the fast-mode passes
// (edge count, host scan, refine) on the last run's values, `reps` times.
// 0 on success.
int refgpu_run_fast(const RefInput* in, int reps, float* values, RefTimes* t, RefFast* fast);
int refgpu_run(const RefInput* in, int reps, float* values, RefTimes* t) {
    return refgpu_run_fast(in, reps, values, t, nullptr);
}

int refgpu_run_fast(const RefInput* in, int reps, float* values, RefTimes* t, RefFast* fast) {
    std::vector<void*> owned;
    auto up = [&](const void* src, size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes ? bytes : 4) != cudaSuccess) return nullptr;
        owned.push_back(p);
        if (bytes && src) cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
        return p;
    };
    auto cleanup = [&] {
        for (void* p : owned) cudaFree(p);
    };
    RefParams P;
    std::memset(&P, 0, sizeof P);
    const unsigned n = in->n_spheres, nc = in->n_circles, nv = in->n_vertices;
    const float* sd = static_cast<const float*>(up(in->sphere, size_t(7) * n * 4));
    const float** sph[7] = {&P.px, &P.py, &P.pz, &P.pr, &P.pr2, &P.pr2tol, &P.pvdw};
    for (int k = 0; k < 7; k++) *sph[k] = sd + size_t(k) * n;
    P.status = static_cast<const unsigned*>(up(in->status, size_t(n) * 4));
    P.nb_off = static_cast<const unsigned*>(up(in->nb_off, (size_t(n) + 1) * 4));
    P.nb_items = static_cast<const unsigned*>(up(in->nb_items, size_t(in->nb_items_len) * 4));
    const float* cd = static_cast<const float*>(up(in->circle, size_t(10) * nc * 4));
    const float** cir[10] = {&P.cx, &P.cy, &P.cz, &P.ux, &P.uy, &P.uz, &P.ex, &P.ey, &P.ez, &P.crho};
    for (int k = 0; k < 10; k++) *cir[k] = cd + size_t(k) * nc;
    P.cb_off = static_cast<const unsigned*>(up(in->cb_off, (size_t(nc) + 1) * 4));
    P.cb_items = static_cast<const unsigned*>(up(in->cb_items, size_t(in->cb_items_len) * 4));
    const float* vd = static_cast<const float*>(up(in->vertex, size_t(3) * nv * 4));
    P.vx = vd, P.vy = vd + nv, P.vz = vd + 2 * size_t(nv);
    RefGrid* grids[3] = {&P.gs, &P.gc, &P.gv};
    for (int g = 0; g < 3; g++) {
        RefGrid& G = *grids[g];
        const unsigned* d = in->grid_dims + 3 * g;
        size_t cells = size_t(d[0]) * d[1] * d[2];
        G.starts = static_cast<const unsigned*>(up(in->grid_starts[g], (cells + 1) * 4));
        G.items = static_cast<const unsigned*>(up(in->grid_items[g], size_t(in->grid_n_items[g]) * 4));
        G.ox = in->grid_f[4 * g], G.oy = in->grid_f[4 * g + 1], G.oz = in->grid_f[4 * g + 2];
        G.cell = in->grid_f[4 * g + 3];
        G.dx = d[0], G.dy = d[1], G.dz = d[2], G.n_items = in->grid_n_items[g];
    }
    const unsigned nb = in->n_bricks, n_sub = 8 * nb, side = in->b + 1;
    const size_t spb = size_t(side) * side * side;
    P.bricks = static_cast<const int*>(up(in->bricks, size_t(nb) * 12));
    P.rec = static_cast<unsigned*>(up(nullptr, size_t(n_sub) * 7 * 4));
    P.values = static_cast<float*>(up(nullptr, spb * nb * 4));
    P.values_len = spb * nb;
    P.n_sub = n_sub, P.kind = 0, P.n_spheres = n, P.n_circles = nc, P.n_vertices = nv;
    P.b = in->b, P.sub = in->sub, P.near = 0;
    P.probe = in->probe, P.band = in->band, P.cutoff2 = in->cutoff2, P.rho = in->rho, P.reach = in->reach;
    P.margin = in->margin, P.slack = in->slack, P.cutoffc2 = in->cutoffc2, P.h = in->h;
    P.max_expanded = in->max_expanded, P.rho_max = in->rho_max;
    for (void* p : owned)
        if (!p) return cleanup(), 1;
    cudaEvent_t e[5];
    for (auto& ev : e) cudaEventCreate(&ev);
    std::vector<unsigned> rec(size_t(n_sub) * 7);
    void* ids = nullptr;
    size_t ids_cap = 0;
    RefTimes best{1e30, 1e30, 1e30, 1e30, 1e30, 0};
    for (int r = 0; r < reps; r++) {
        auto w0 = std::chrono::steady_clock::now();
        cudaEventRecord(e[0]);
        sesmesh_resident_count<<<n_sub, 64>>>(P);
        cudaEventRecord(e[1]);
        cudaEventSynchronize(e[1]);
        auto s0 = std::chrono::steady_clock::now();
        cudaMemcpy(rec.data(), P.rec, rec.size() * 4, cudaMemcpyDeviceToHost);
        unsigned long long total = 0;
        for (size_t j = 0; j < n_sub; j++) {
            rec[7 * j + 1] = unsigned(total);
            for (int k = 2; k < 7; k++) total += rec[7 * j + k];
        }
        cudaMemcpy(P.rec, rec.data(), rec.size() * 4, cudaMemcpyHostToDevice);
        if (total > ids_cap) {
            if (ids) cudaFree(ids);
            ids = nullptr;
            if (cudaMalloc(&ids, total * 4) != cudaSuccess) {
                for (auto& ev : e) cudaEventDestroy(ev);
                return cleanup(), 2;
            }
            ids_cap = total;
        }
        P.ids = static_cast<unsigned*>(ids);
        P.ids_len = total;
        double scan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s0).count();
        cudaEventRecord(e[2]);
        sesmesh_resident_fill<<<n_sub, 64>>>(P);
        cudaEventRecord(e[3]);
        sesmesh_resident_sample<<<n_sub, 64>>>(P);
        cudaEventRecord(e[4]);
        if (cudaEventSynchronize(e[4]) != cudaSuccess) {
            if (ids) cudaFree(ids);
            for (auto& ev : e) cudaEventDestroy(ev);
            return cleanup(), 3;
        }
        float c = 0, f = 0, sa = 0;
        cudaEventElapsedTime(&c, e[0], e[1]);
        cudaEventElapsedTime(&f, e[2], e[3]);
        cudaEventElapsedTime(&sa, e[3], e[4]);
        double total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
        if (r > 0 || reps == 1) {
            if (total_ms < best.total_ms) best.total_ms = total_ms;
            if (c < best.count_ms) best.count_ms = c;
            if (scan_ms < best.scan_ms) best.scan_ms = scan_ms;
            if (f < best.fill_ms) best.fill_ms = f;
            if (sa < best.sample_ms) best.sample_ms = sa;
        }
        best.ids = total;
    }
    if (values) cudaMemcpy(values, P.values, spb * nb * 4, cudaMemcpyDeviceToHost);
    int frc = 0;
    if (fast) {
        P.ids = static_cast<unsigned*>(ids);
        frc = run_fast(P, fast, reps, owned);
    }
    cudaError_t err = cudaGetLastError();
    for (auto& ev : e) cudaEventDestroy(ev);
    if (ids) cudaFree(ids);
    cleanup();
    if (t) *t = best;
    if (frc) return frc;
    return err == cudaSuccess ? 0 : 4;
}

static int run_fast(RefParams& P, RefFast* f, int reps, std::vector<void*>& owned) {
    auto up = [&](const void* src, size_t bytes) -> void* {
        void* p = nullptr;
        if (cudaMalloc(&p, bytes ? bytes : 4) != cudaSuccess) return nullptr;
        owned.push_back(p);
        if (bytes && src) cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
        return p;
    };
    RefRefine R;
    std::memset(&R, 0, sizeof R);
    const unsigned n = P.n_spheres, nc = P.n_circles, nv = P.n_vertices, n_sub = P.n_sub;
    const float* sl = static_cast<const float*>(up(f->sphere_lo, size_t(3) * n * 4));
    const float* cl = static_cast<const float*>(up(f->circle_lo, size_t(3) * nc * 4));
    const float* vl = static_cast<const float*>(up(f->vertex_lo, size_t(3) * nv * 4));
    if (!sl || !cl || !vl) return 5;
    R.plx = sl, R.ply = sl + n, R.plz = sl + 2 * size_t(n);
    R.clx = cl, R.cly = cl + nc, R.clz = cl + 2 * size_t(nc);
    R.vlx = vl, R.vly = vl + nv, R.vlz = vl + 2 * size_t(nv);
    R.max_iter = f->max_iter, R.max_bisect = f->max_bisect, R.h_hi = f->h_hi, R.h_lo = f->h_lo, R.tol = f->tol;
    R.edge_count = static_cast<unsigned*>(up(nullptr, size_t(n_sub) * 4));
    unsigned* d_off = static_cast<unsigned*>(up(nullptr, (size_t(n_sub) + 1) * 4));
    if (!R.edge_count || !d_off) return 5;
    R.edge_off = d_off;
    std::vector<unsigned> off(size_t(n_sub) + 1, 0);
    float *d_t = nullptr, *d_q = nullptr;
    unsigned *d_feat = nullptr, *d_ev = nullptr;
    size_t cap = 0;
    cudaEvent_t e[4];
    for (auto& ev : e) cudaEventCreate(&ev);
    f->edge_count_ms = f->scan_ms = f->refine_ms = 1e30;
    for (int r = 0; r < reps; r++) {
        cudaEventRecord(e[0]);
        sesmesh_resident_edge_count<<<n_sub, 64>>>(P, R);
        cudaEventRecord(e[1]);
        cudaEventSynchronize(e[1]);
        auto s0 = std::chrono::steady_clock::now();
        cudaMemcpy(off.data() + 1, R.edge_count, size_t(n_sub) * 4, cudaMemcpyDeviceToHost);
        for (size_t j = 1; j <= n_sub; j++) off[j] += off[j - 1];
        cudaMemcpy(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice);
        const size_t ne = off[n_sub];
        if (ne > cap) {
            for (void* p : {(void*)d_t, (void*)d_q, (void*)d_feat, (void*)d_ev})
                if (p) cudaFree(p);
            cap = ne;
            if (cudaMalloc(&d_t, cap * 4) != cudaSuccess || cudaMalloc(&d_feat, cap * 4) != cudaSuccess ||
                cudaMalloc(&d_q, cap * 12) != cudaSuccess || cudaMalloc(&d_ev, cap * 4) != cudaSuccess) {
                for (auto& ev : e) cudaEventDestroy(ev);
                return 6;
            }
        }
        R.t_out = d_t, R.feat_out = d_feat, R.q_out = d_q, R.evals_out = d_ev, R.n_edges = unsigned(ne);
        const double scan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s0).count();
        cudaEventRecord(e[2]);
        sesmesh_resident_refine<<<n_sub, 64>>>(P, R);
        cudaEventRecord(e[3]);
        if (cudaEventSynchronize(e[3]) != cudaSuccess) {
            for (auto& ev : e) cudaEventDestroy(ev);
            return 7;
        }
        float c = 0, rf = 0;
        cudaEventElapsedTime(&c, e[0], e[1]);
        cudaEventElapsedTime(&rf, e[2], e[3]);
        if (r > 0 || reps == 1) {
            if (c < f->edge_count_ms) f->edge_count_ms = c;
            if (scan_ms < f->scan_ms) f->scan_ms = scan_ms;
            if (rf < f->refine_ms) f->refine_ms = rf;
        }
    }
    const size_t ne = off[n_sub];
    f->n_edges = ne;
    if (f->edge_off) std::memcpy(f->edge_off, off.data(), off.size() * 4);
    if (ne <= f->cap) {
        if (f->t) cudaMemcpy(f->t, d_t, ne * 4, cudaMemcpyDeviceToHost);
        if (f->feat) cudaMemcpy(f->feat, d_feat, ne * 4, cudaMemcpyDeviceToHost);
        if (f->q) cudaMemcpy(f->q, d_q, ne * 12, cudaMemcpyDeviceToHost);
        if (f->evals) cudaMemcpy(f->evals, d_ev, ne * 4, cudaMemcpyDeviceToHost);
    }
    for (void* p : {(void*)d_t, (void*)d_q, (void*)d_feat, (void*)d_ev})
        if (p) cudaFree(p);
    for (auto& ev : e) cudaEventDestroy(ev);
    return ne <= f->cap ? 0 : 8;
}

}  // extern "C"
