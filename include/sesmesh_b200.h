/*
 * sesmesh_b200 — C ABI of the B200 (sm_100a) SES mesh-stage back end.
 *
 * The entry points replace sesmesh's CUDA back-end crate
 * (crates/sesmesh-gpu/src/cuda/*.rs behind the DeviceResident / DeviceBatch
 * traits of crates/sesmesh-gpu/src/batch.rs:165-236), which
 * crates/sesmesh/src/field/gpu.rs drives from the mesh stage
 * (crates/sesmesh/src/surface.rs:953-999).  Each declaration names the
 * reference interface it stands in for.  Plain pointers and sizes only; all
 * functions return SMB_OK or an SMB_ERR_* code and write a message to
 * err[0..errlen) on failure (the reference panics on malformed shapes; this
 * ABI reports them instead).
 *
 * Differences from the reference boundary, each additive:
 *   - the arrangement is passed in f64 (the reference passes frame-local f32
 *     copies); brick classes, candidate lists and sample values are then
 *     computed with the CPU back end's f64 decisions and are bit-identical;
 *   - brick classification (lattice::touched_bricks / surface_bricks,
 *     crates/sesmesh/src/field/lattice.rs:105-181) runs on the device;
 *   - a run also extracts marching-cubes edges and triangle references per
 *     brick in the host mesher's encoding (crates/sesmesh/src/mesh/
 *     extract.rs:59-72, 146-265).
 */
#ifndef SESMESH_B200_H
#define SESMESH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    SMB_OK = 0,
    SMB_ERR_ARG = 1,       /* invalid argument or malformed table */
    SMB_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    SMB_ERR_NODEVICE = 3,  /* no such device */
    SMB_ERR_SELFTEST = 4,  /* device arithmetic differs from IEEE */
    SMB_ERR_RANGE = 5,     /* coordinates beyond the brick key range */
    SMB_ERR_MEMORY = 6,    /* allocation failed or a list exceeds a limit */
    SMB_ERR_STATE = 7,     /* call out of order (e.g. run before classify) */
    SMB_ERR_TIMEOUT = 8,   /* a bounded device wait gave up */
    SMB_ERR_CANCELLED = 9  /* stopped by its cancel flag (Error::Cancelled, control.rs:114-121) */
};

typedef struct smb_device smb_device;
typedef struct smb_resident smb_resident;
typedef struct smb_batch smb_batch;

typedef struct {
    char name[256];
    int major, minor;
    int multiprocessors;
    size_t memory;
} smb_device_info;

/* Opens CUDA device `index` and runs the arithmetic self-test.
 * Replaces cuda::Runtime::load/open + Device (crates/sesmesh-gpu/src/cuda/
 * mod.rs:93-240, 418-485) and the K0 self-test (cuda/selftest.rs:16-40). */
int smb_open(int index, smb_device** out, char* err, size_t errlen);
/* Handles may be freed in any order: a closed device stays open until the
 * residents and MLPs made on it are freed, a freed resident until its
 * batches are (the handle must not be used after its own free). */
void smb_close(smb_device* dev);
/* Device::info (cuda/mod.rs:418-470). */
int smb_device_info_get(const smb_device* dev, smb_device_info* out);
/* Device self-test on n pairs (tests/cuda.rs:65-71 runs 2^20). */
int smb_self_test(smb_device* dev, uint32_t n, char* err, size_t errlen);

/* A cell grid (GridRef, batch.rs:44-56; CellGrid::parts, geom/cells.rs:86-89):
 * items of cell c are items[starts[c]..starts[c+1]], cells x-fastest. */
typedef struct {
    double origin[3];
    double cell;
    uint32_t dims[3];
    const uint32_t* starts; /* dims[0]*dims[1]*dims[2] + 1 */
    const uint32_t* items;
    size_t n_items;
} smb_grid_ref;

/* The SAS arrangement in sesmesh's internal sphere order (ArrangementRef,
 * batch.rs:59-83, extended to f64; geom/arrangement.rs:205-228). */
typedef struct {
    size_t n_spheres;
    const double* center;     /* 3 per sphere */
    const double* expanded;   /* R = r + probe */
    const double* radius;     /* vdW radius r */
    const uint32_t* status;   /* 0 exposed, 1 buried, 2 contained */
    const uint32_t* nb_off;   /* n_spheres + 1: neighbour rows of exposed spheres */
    const uint32_t* nb_items;
    size_t n_circles;
    const double* circle;     /* 10 per circle: centre xyz, axis xyz, e1 xyz, radius */
    const uint32_t* cb_off;   /* n_circles + 1: circle blockers */
    const uint32_t* cb_items;
    size_t n_vertices;
    const double* vertex;     /* 3 per SAS vertex */
    smb_grid_ref sphere_grid, circle_grid, vertex_grid;
    double max_expanded, rho_max, probe;
    /* The surface (SurfaceKind, field/mod.rs:33-41): SMB_KIND_SES, or a
     * sphere field, SMB_KIND_SAS / SMB_KIND_VDW (min |x - c| - R over the
     * spheres; expanded = r + probe for the SAS, r for the vdW surface; no
     * circles or vertices; field/kernel.rs:957-981, point.rs:566-579,
     * 723-736). */
    int kind;
} smb_arrangement_ref;
enum { SMB_KIND_SES = 0, SMB_KIND_SAS = 1, SMB_KIND_VDW = 2 };

/* The sampling lattice (Lattice, field/lattice.rs:26-45; Engine::new,
 * field/kernel.rs:204-271).  brick must be even, 4..32 (the device path
 * splits bricks into 2x2x2 sub-blocks, field/gpu.rs:243-250). */
typedef struct {
    double spacing;
    uint32_t brick;
    int64_t frame[3]; /* lattice index of the f32 frame origin */
    double band;      /* sqrt(3) * spacing * 1.01 */
} smb_lattice_ref;

/* Uploads the arrangement (cuda::Resident::new, cuda/resident.rs:407-480;
 * tables are validated as batch.rs:323-338 does). */
int smb_resident_new(smb_device* dev, const smb_arrangement_ref* arr, const smb_lattice_ref* lat,
                     smb_resident** out, char* err, size_t errlen);
void smb_resident_free(smb_resident* res);
/* DeviceResident::resident_bytes (batch.rs:203). */
size_t smb_resident_bytes(const smb_resident* res);

/* Surface bricks on the device: lattice::touched_bricks + surface_bricks
 * (field/lattice.rs:105-181, f64).  Keeps the list (packed-key order) on the
 * device; *touched and *surface get the counts. */
int smb_classify(smb_resident* res, size_t* touched, size_t* surface, char* err, size_t errlen);
/* Copies up to cap surface-brick keys (3 int32 each) to out. */
int smb_resident_bricks(const smb_resident* res, int32_t* out, size_t cap);

/* Empty batch buffers (DeviceResident::new_batch, batch.rs:175-181). */
int smb_batch_new(smb_resident* res, smb_batch** out, char* err, size_t errlen);
void smb_batch_free(smb_batch* batch);

/* Device times of one run, milliseconds (BatchTimes, batch.rs:118-129). */
typedef struct {
    double substates, gather, sample, mc, total;
} smb_batch_times;

/* Sub-block classification, candidate gather, field sampling and marching
 * cubes for surface bricks [first, first + count) of the classified list
 * (cuda::Resident::run, cuda/resident.rs:494-572, plus the MC pass). */
int smb_run(smb_resident* res, size_t first, size_t count, smb_batch* batch, smb_batch_times* times, char* err,
            size_t errlen);

/* Accessors of the last run (DeviceBatch, batch.rs:211-236), copied to
 * caller memory. */
size_t smb_batch_bricks(const smb_batch* batch);
/* SMB_REC_WORDS words per sub-block (8 per brick, sub-block sb = x | y<<1 |
 * z<<2): state (0 sampled, 1 uniformly outside, 2 inside), ids base,
 * n_inside, n_near, n_s, n_c, n_v, n_s_blockers, n_c_blockers, pack base,
 * pack units, flags. */
#define SMB_REC_WORDS 12
int smb_batch_records(const smb_batch* batch, uint32_t* out);
/* (b+1)^3 values per brick, x fastest (DeviceBatch::brick_values). */
int smb_batch_values(const smb_batch* batch, float* out);
/* Candidate lists of all sampled sub-blocks: at each record's ids base,
 * near ids (n_near, those that can contain a sample first), S ids, S
 * offsets (n_s + 1), S blockers (near positions), C ids, C offsets,
 * C blockers, V ids -- the lists of Engine::gather_ses (kernel.rs:671-752). */
size_t smb_batch_ids_words(const smb_batch* batch);
int smb_batch_ids(const smb_batch* batch, uint32_t* out);
/* Marching cubes: totals, then per brick (count + 1 offsets) the owned
 * crossing edges (local ids ((z*b+y)*b+x)*3+axis, ascending), their sample
 * values (fa, fb) and the triangle references (code << 28 | local id). */
int smb_batch_mc_counts(const smb_batch* batch, size_t* edges, size_t* triangles);
int smb_batch_mc(const smb_batch* batch, uint32_t* edge_off, uint32_t* edges, float* edge_vals, uint32_t* tri_off,
                 uint32_t* tris);

/* Fast mode: refinement settings (Resident::set_refinement and RefineRef,
 * batch.rs:133-150, field/gpu.rs:207-221): tolerance 1e-5 A, at most 8
 * Newton / Illinois evaluations then 64 bisection steps, f32 brick-local
 * coordinates from double-float pairs. */
int smb_resident_set_refinement(smb_resident* res, char* err, size_t errlen);
/* Refines the crossing edges of the last run in f32 on the device
 * (cuda::Resident::refine, cuda/resident.rs:632-688); *ms gets the device
 * time.  Results are indexed like the marching-cubes edges. */
int smb_refine(smb_resident* res, smb_batch* batch, double* ms, char* err, size_t errlen);
/* Per edge: parameter t, feature (kind << 29 | id; kinds 0 solvent,
 * 1 beyond, 2 sphere, 3 circle, 4 SAS vertex), closest point relative to the
 * brick origin (3 floats), evaluations | 1 << 31 if Newton / Illinois
 * converged (DeviceBatch::edge_*, batch.rs:222-232). */
int smb_batch_edges(const smb_batch* batch, float* t, uint32_t* feat, float* closest, uint32_t* evals);

/* Exact mode on the device (additive: the reference refines exact-mode
 * vertices on the host, extract::mesh_brick, mesh/extract.rs:146-219 with
 * vertex :425-535 and attributes :553-597).  Uploads the tables the vertex
 * attributes read: the input index of each sphere (orig, n_spheres), the
 * atom pair of each circle (2 per circle) and the atom triple of each SAS
 * vertex (3 per vertex), in the resident arrangement's order, and the edge
 * clamp t_min (extract.rs:47-51). */
int smb_resident_set_exact(smb_resident* res, const uint32_t* orig, const uint32_t* circle_ij, size_t n_circles,
                           const uint32_t* vertex_atoms, size_t n_vertices, double t_min, char* err, size_t errlen);
/* Refines the crossing edges of the last run in f64 on the device: for each
 * sampled sub-block the candidates of its ball (SesField::gather_local,
 * field/point.rs:496-582), then extract::vertex's Newton / Illinois /
 * bisection search and the vertex attributes, operation by operation as the
 * CPU does them, so every vertex equals the CPU's.  Edges left to the host
 * (evals = 0 in smb_batch_vertices): those whose last evaluation is solvent
 * or beyond the band, and those of a sub-block whose lists exceed a block's
 * shared memory.  *ms gets the device time. */
int smb_refine_exact(smb_resident* res, smb_batch* batch, double* ms, char* err, size_t errlen);
/* Results of smb_refine_exact per marching-cubes edge: position and normal
 * (3 f32 each), input atom index, patch (0 sphere, 1 circle, 2 vertex),
 * root parameter before the clamp, evaluations (0: not refined on the
 * device).  Null pointers are skipped. */
int smb_batch_vertices(const smb_batch* batch, float* positions, float* normals, uint32_t* atoms, uint8_t* patches,
                       float* t, uint32_t* evals);
/* Fast mode's vertex placement on the device (mesh_brick_device,
 * mesh/extract.rs:274-365; additive, the reference places on the host):
 * after smb_refine, every edge the f32 refinement converged on is placed at
 * pa + d clamp(t) with the exact attributes of its feature, and every other
 * edge is refined exactly as smb_refine_exact does.  Needs
 * smb_resident_set_exact.  Results through smb_batch_vertices. */
int smb_place_fast(smb_resident* res, smb_batch* batch, double* ms, char* err, size_t errlen);
/* Over the vertices of the last smb_refine_exact / smb_place_fast: the total
 * evaluation count, the number of edges left to the host (evals = 0) and
 * the number of edges the exact refinement took. */
int smb_batch_exact_summary(const smb_batch* batch, unsigned long long* evaluations, unsigned long long* host_edges,
                            unsigned long long* exact_edges);
/* Re-runs the last smb_refine_exact counting the f64 arithmetic operations
 * of its field evaluations (the algorithmic count of its roofline; sqrt and
 * division one each; vertices are rewritten identically). */
int smb_batch_count_exact_ops(smb_batch* batch, unsigned long long* ops, char* err, size_t errlen);
/* Shared memory per warp for one sub-block's f64 lists in smb_refine_exact
 * (1 KiB..48 KiB; default 13 KiB); larger sub-blocks go to warps with global list slabs. */
int smb_batch_set_exact_region(smb_batch* batch, size_t bytes);
/* Shared memory for one sub-block's f32 lists in smb_refine, staged once
 * for a block of two warps (1 KiB..56 KiB; 0, the default: the largest
 * sub-block's lists when they fit 20 KiB and the groups are of 8 lanes,
 * else an eighth of the SM's shared memory); larger sub-blocks go to a
 * second pass that gives each a whole block.  The roots do not depend on
 * it. */
int smb_batch_set_refine_region(smb_batch* batch, size_t bytes);
/* Lanes that evaluate one edge's points together in smb_refine and
 * smb_refine_warm: 8 or 32 (0, the default: 32 when the sub-blocks' lists
 * average 16 KiB or more, else 8).  The roots do not depend on it. */
int smb_batch_set_refine_group(smb_batch* batch, int lanes);
/* Lanes per edge in smb_refine_exact and the exact pass of smb_place_fast:
 * 1, 8 or 32 (0, the default: 32 when the sub-blocks' lists average 16 KiB
 * or more, else 1); the pass over sub-blocks with global list slabs takes
 * at least 8.  The vertices do not depend on it. */
int smb_batch_set_exact_group(smb_batch* batch, int lanes);
/* smb_refine_exact lays each sub-block's lists out from the gather's list
 * sizes (1, the default), counts them first (0), or takes bounds one short
 * of the gather's (2: every sub-block goes through the recount, for tests).
 * The vertices do not depend on it. */
int smb_batch_set_exact_hint(smb_batch* batch, int mode);
/* Shared memory of each sampling CTA in a first pass over the sub-blocks
 * whose packed lists fit it (>= 1 KiB; 0, the default: 55 KiB); the others
 * run in a second pass with room for the largest. */
int smb_batch_set_sample_region(smb_batch* batch, size_t bytes);

/* Sizes and times of the last run of a batch (diagnostics; BatchTimes and
 * DeviceBatch::bytes, batch.rs:118-129, 233). */
typedef struct {
    size_t bricks, sampled_subblocks, ids_words, max_pack_units, edges, triangles, touched, resident_bytes;
    unsigned long long pack_units;
    double classify_ms;
    size_t exact_block_items;  /* smb_refine_exact: sub-blocks refined by a whole block (lists over a warp's share) */
    uint32_t gather_caps[4];   /* the gather's per-warp list caps (near, S, C, V) for the next run */
    uint32_t gather_warps;     /* warps per gather block for the next run */
} smb_batch_info;
int smb_batch_info_get(const smb_batch* batch, smb_batch_info* out);
/* Re-runs the sampling pass of the last run counting its f32 arithmetic
 * operations as executed and the samples it evaluated (the algorithmic
 * count of the roofline; values are rewritten identically). */
int smb_batch_count_ops(smb_batch* batch, unsigned long long* ops, unsigned long long* samples, char* err,
                        size_t errlen);
/* Learned warm start of fast mode (no counterpart in the reference; the
 * reference's fast mode starts every edge from the linear guess,
 * mesh/extract.rs:425-535 with field/gpu.rs:207-221): an MLP
 * 32 -> 64 -> 64 -> 1 (GELU, sigmoid output in [0, 1]) with BF16 weights
 * on the tensor cores and FP32 accumulation, proposing where each crossing
 * edge's root search starts.  Parameters are SMB_MLP_NPARAM f32 values:
 * W1 [64][32], b1 [64], W2 [64][64], b2 [64], w3 [64], b3 (row-major,
 * out x in). */
#define SMB_MLP_NPARAM 6337
#define SMB_MLP_FEATURES 32
typedef struct smb_mlp smb_mlp;
int smb_mlp_new(smb_device* dev, const float* params, smb_mlp** out, char* err, size_t errlen);
void smb_mlp_free(smb_mlp* mlp);
int smb_mlp_set_params(smb_mlp* mlp, const float* params, char* err, size_t errlen);
int smb_mlp_get_params(const smb_mlp* mlp, float* params);
/* How smb_refine_warm uses the output: SMB_MLP_GATE (default) starts an edge
 * at t_c (below) where the output is >= 0.5 and both samples name t_c's
 * candidate, and at the linear guess elsewhere; SMB_MLP_ROOT starts it at
 * the output itself, a root parameter
 * in [0, 1] (parameters trained on the exact root). */
#define SMB_MLP_GATE 0
#define SMB_MLP_ROOT 1
int smb_mlp_set_use(smb_mlp* mlp, int use);
/* t[i] = MLP(x[32 i .. 32 i + 31]) for host arrays (tests, diagnostics). */
int smb_mlp_forward(smb_mlp* mlp, const float* x, size_t n, float* t, char* err, size_t errlen);
/* Loss (mean squared error of t, *loss) and its gradient over the
 * parameter vector for n rows as one batch (at most 2^20 rows); the
 * products of forward and backward run on the tensor cores. */
int smb_mlp_gradient(smb_mlp* mlp, const float* x, const float* target, size_t n, float* loss, float* grad,
                     char* err, size_t errlen);
/* One epoch of Adam over the rows in order, minibatches of `batch` rows (a
 * multiple of 128); losses[k] gets minibatch k's loss before its step
 * (ceil(n / batch) values) when non-null. */
int smb_mlp_train_epoch(smb_mlp* mlp, const float* x, const float* target, size_t n, size_t batch, float lr,
                        float* losses, char* err, size_t errlen);
/* on = 1: the sampling pass of the batch's later runs also records every
 * sampled point's nearest feature (the candidate that sets its value, in
 * the smb_batch_edges feature encoding; the values are unchanged), which
 * the warm start reads; on = 0 (default) skips it. */
int smb_batch_record_features(smb_batch* batch, int on);
/* The last run's nearest-feature words, (b+1)^3 per brick like
 * smb_batch_values; meaningful at samples a sampled sub-block owns
 * (SMB_ERR_STATE when the run did not record them). */
int smb_batch_sample_features(const smb_batch* batch, uint32_t* out);
/* smb_refine with each edge's starting point chosen by the MLP.  The
 * sampler's nearest features at the edge's two samples name one candidate
 * (a sphere, a circle or a SAS vertex); a feature pass runs smb_refine's
 * own iteration (the same f32 operations) on that candidate alone, without
 * evaluating the field: where the candidate is the surface's nearest
 * feature at its iterates, that result t_c is where smb_refine would stop.
 * The MLP, over each edge's features (smb_batch_edge_features), then gives
 * the start (smb_mlp_set_use): t_c where both samples name the candidate,
 * its iteration converged and the gate answers >= 0.5, else the linear
 * guess fa / (fa - fb) that smb_refine always takes.  The iteration that
 * follows is smb_refine's, with its bracket, tolerance, budgets and
 * outputs: a start at which the field is within the tolerance and names
 * the candidate is accepted after one evaluation, any other falls back to
 * the bracketed refinement from the linear guess.  The last smb_run must have
 * recorded the features (smb_batch_record_features; else SMB_ERR_STATE).
 * A null mlp is smb_refine. */
int smb_refine_warm(smb_resident* res, smb_batch* batch, const smb_mlp* mlp, double* ms, char* err, size_t errlen);
/* Re-runs the last run's f32 refinement (smb_refine, or smb_refine_warm
 * with mlp) counting the f32 arithmetic operations of its field
 * evaluations into *ops (the algorithmic count of its roofline: sqrt and
 * division one each, compares and selects not counted; groups of 8 lanes;
 * the edge results are written again, identically).  Discards the last
 * placement (smb_place_fast). */
int smb_batch_count_refine_ops(smb_batch* batch, const smb_mlp* mlp, unsigned long long* ops, char* err,
                               size_t errlen);
/* The MLP's input for every crossing edge of the last run (32 f32 per edge,
 * marching-cubes edge order; zeros for edges the device does not refine)
 * and covered[k] = 1 where the device refines edge k.  With t_lin = fa /
 * (fa - fb) and t_c as above: fa / h, fb / h; finite-difference gradients
 * of the samples at both ends (6); t_lin; the candidate's kind, one-hot
 * (sphere, circle, vertex: 3); both samples name the same feature; they
 * name two different candidates; t_c's iteration converged; its steps / 8;
 * (t_c - t_lin) * 8 clamped to [-4, 4]; t_c (t_lin where it did not
 * converge); log10(max(m, 1e-9)) / 9 + 1 of its last |g| and of the
 * candidate's mismatch at both samples (3); the candidate's centre (or
 * position) less the edge midpoint / 4 A (3) and its radius / 4 A; h; the
 * probe radius; both gradients along the edge times h / (fb - fa), clamped
 * to [-10, 10] (2); |gradient| - 1 at both ends, clamped to [-4, 4] (2);
 * the other sample's feature kind / 4.  The last run must have recorded
 * the features.  Discards the last refinement. */
int smb_batch_edge_features(smb_resident* res, smb_batch* batch, float* features, uint8_t* covered, char* err,
                            size_t errlen);

/* Marching cubes (the last pass of smb_run) over caller-owned device
 * buffers, with no device allocation at all.  This entry point has no
 * counterpart in the reference: it serves callers that cannot allocate
 * device memory while they mesh, such as services that reserve a fixed
 * device-memory budget up front and must not grow it while serving, and
 * hosts whose device memory belongs to another framework's caching
 * allocator (a cudaMalloc beside it can fail once that allocator holds the
 * free memory).  Its scratch (per-brick counts, scan tiles, totals;
 * 524,832 bytes = 512.5 KiB) is one static device array that every GPU
 * loading the library holds until exit; at most SMB_MC_NOALLOC_MAX_BRICKS
 * bricks per call, more are rejected with SMB_ERR_ARG before any work.
 *   values:  (b+1)^3 floats per brick, as smb_batch_values returns them (the
 *            +-band samples are rewritten in place with the same values);
 *   records: SMB_REC_WORDS words per sub-block, as smb_batch_records;
 *   outputs: edge_off and tri_off (n_bricks + 1), edges (edges_cap),
 *            edge_vals (2 * edges_cap floats), tris (3 * tris_cap), encoded as
 *            smb_batch_mc; *n_edges and *n_tris get the totals.
 * When the totals exceed edges_cap / tris_cap (or reach 2^32, past the
 * 32-bit offsets) the call returns SMB_ERR_MEMORY with the totals reported;
 * by then it has written edge_off[0..n_bricks-1], tri_off[0..n_bricks-1]
 * and the +-band samples of values, and nothing else.
 * All pointers but n_edges and n_tris are device pointers.  The call runs
 * on the resident's device stream and returns once its work there has
 * finished; the caller's current device is left as it was.  The first call
 * on a device looks the scratch address up (cudaGetSymbolAddress); make it
 * before any stream capture.  Calls share the scratch and it keeps the last
 * call's contents: calls that overlap on the GPU (other threads, other
 * streams) race. */
#define SMB_MC_NOALLOC_MAX_BRICKS 65536
int smb_mc_noalloc(const smb_resident* res, float* values, const uint32_t* records, size_t n_bricks,
                   uint32_t* edge_off, uint32_t* edges, float* edge_vals, size_t edges_cap, uint32_t* tri_off,
                   uint32_t* tris, size_t tris_cap, size_t* n_edges, size_t* n_tris, char* err, size_t errlen);

/* Kernels this library has launched in the process (diagnostics). */
unsigned long long smb_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif
