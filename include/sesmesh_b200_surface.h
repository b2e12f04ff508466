/*
 * sesmesh_b200 — host API of the mesh stage with the B200 back end: the
 * counterpart of compute_surface / SurfaceEngine with Backend::Cuda
 * (crates/sesmesh/src/surface.rs:599-711) for the SES, refine exact or fast.
 * The host keeps the arrangement, assembly and OBJ output; the device runs
 * classification, gather, sampling, marching cubes, the vertex refinement
 * (f64 in exact mode, f32 in fast mode), validation and measure through
 * include/sesmesh_b200.h.
 */
#ifndef SESMESH_B200_SURFACE_H
#define SESMESH_B200_SURFACE_H

#include "sesmesh_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Surface kinds (SurfaceKind, field/mod.rs:33-41): the SES, the SAS (the
 * spheres expanded by the probe) and the vdW surface (the spheres; also the
 * SES with probe 0).  Equal to SMB_KIND_*. */
enum { SMB_SES = 0, SMB_SAS = 1, SMB_VDW = 2 };
enum { SMB_REFINE_EXACT = 0, SMB_REFINE_LINEAR = 1, SMB_REFINE_FAST = 2 };

/* SurfaceParams (surface.rs:195-241) restricted to what the device path
 * takes: kind (SES, SAS or vdW; the vdW surface ignores the probe radius,
 * SurfaceParams::effective_probe), spacing, brick_size (even, 4..32;
 * reference default 10), refine exact | fast (a sphere field refines fast
 * mode from the linear guess: the learned warm start is the SES's).
 * threads: host threads (0 = all cores). */
typedef struct {
    int kind;
    double probe_radius;
    double spacing;
    uint32_t brick_size;
    int refine;
    int threads;
} smb_surface_params;

/* SurfaceStats (surface.rs:506-562) plus per-stage times in milliseconds. */
typedef struct {
    size_t spheres, touched_bricks, surface_bricks, samples, vertices, triangles, components;
    double area, volume;
    int64_t euler;
    uint64_t refine_evaluations, refine_cpu_edges;
    double t_geometry, t_upload, t_classify, t_substates, t_gather, t_sample, t_mc, t_device, t_d2h, t_host_refine,
        t_mesh_stage, t_assemble, t_measure, t_total;
    int host_threads;
    /* Where the work ran.  arrangement_where: 1 the device built the
     * arrangement, 0 the host did (input below the device threshold), 2 the
     * device declined and the host built it.  finished_on_host: 1 when the
     * device path was on but the mesh was finished on the host threads
     * (smb_engine_note says why).  upload_bytes: bytes copied host to device
     * for the arrangement (the sphere rows when the device builds it, else
     * the uploaded arrangement). */
    int arrangement_where, finished_on_host;
    uint64_t upload_bytes;
    /* The grid spacing meshed (the requested one unless the memory guard
     * coarsened it) and the guard's estimate of the device bytes there. */
    double spacing_used;
    uint64_t device_bytes_estimate;
} smb_surface_stats;

/* Cooperative cancellation, progress and a device-memory guard for one
 * computation: Control (crates/sesmesh/src/control.rs:54-131) and
 * SurfaceParams::with_max_memory / with_auto_coarsen (surface.rs:226-236,
 * 309-370; the guard, fit_memory, surface.rs:776-890, estimates host peak
 * bytes; this one estimates the device stage's bytes).
 *   cancel: when *cancel becomes nonzero the computation returns
 *     SMB_ERR_CANCELLED promptly: it is polled per sphere while the host
 *     builds the arrangement, and between device passes and host stages.
 *   progress: called with (stage, 0, total) when a stage starts and
 *     (stage, total, total) when it ends (total = surface bricks for
 *     SMB_STAGE_MESH, 1 otherwise; structures for a batch's mesh stage),
 *     from the calling thread.
 *   max_device_bytes: with a nonzero limit, after classification the
 *     device stage's bytes are estimated from the surface bricks
 *     (smb_device_bytes_estimate) plus the resident arrangement; above the
 *     limit the call returns SMB_ERR_MEMORY before any mesh-stage buffer is
 *     taken, or, with auto_coarsen (smb_compute_surface_with only), meshes
 *     at the smallest spacing up to 10 A whose estimate fits
 *     (stats.spacing_used). */
enum {
    SMB_STAGE_GEOMETRY = 0,
    SMB_STAGE_CLASSIFY = 1,
    SMB_STAGE_MESH = 2,
    SMB_STAGE_ASSEMBLE = 3,
    SMB_STAGE_MEASURE = 4
};
typedef void (*smb_progress_fn)(void* user, int stage, uint64_t done, uint64_t total);
typedef struct {
    const volatile int32_t* cancel;
    smb_progress_fn progress;
    void* user;
    uint64_t max_device_bytes;
    int auto_coarsen;
} smb_control;
/* Device bytes of the mesh stage for this many surface bricks of this edge
 * at this spacing and probe, for an input of `spheres` spheres on a device
 * of `multiprocessors` SMs (values, records, candidate lists,
 * marching-cubes and refinement outputs, exact-mode vertices, the exact
 * refinement's list slabs and the device finish; conservative). */
uint64_t smb_device_bytes_estimate(size_t surface_bricks, uint32_t brick, double spacing, double probe_radius,
                                   size_t spheres, int refine, int multiprocessors);

typedef struct smb_engine smb_engine;
typedef struct smb_surface smb_surface;

/* compute_surface (surface.rs:599): spheres as n rows (x, y, z, r). */
int smb_compute_surface(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p,
                        smb_surface** out, char* err, size_t errlen);
/* compute_surface_with (surface.rs:614-631) with a control (may be null). */
int smb_compute_surface_with(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p,
                             const smb_control* control, smb_surface** out, char* err, size_t errlen);
/* SurfaceEngine-style reuse: arrangement and upload once, then meshes. */
int smb_engine_new(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p, smb_engine** out,
                   char* err, size_t errlen);
void smb_engine_free(smb_engine* e);
/* smb_engine_new under a control (its cancel flag and progress cover the
 * arrangement); the engine keeps the control for its later calls. */
int smb_engine_new_with(smb_device* dev, const double* xyzr, size_t n, const smb_surface_params* p,
                        const smb_control* control, smb_engine** out, char* err, size_t errlen);
/* Replaces the engine's control (null: none). */
int smb_engine_set_control(smb_engine* e, const smb_control* control);
/* Device bytes the engine holds now: the resident arrangement, the batch's
 * buffers and the measure's tables (what the memory guard estimates). */
uint64_t smb_engine_device_bytes(const smb_engine* e);
int smb_engine_run_device(smb_engine* e, smb_batch_times* times, char* err, size_t errlen);
size_t smb_engine_bricks(const smb_engine* e);
int smb_engine_mesh(smb_engine* e, smb_surface** out, char* err, size_t errlen);
/* The exact SES field (f64) at n points (3 doubles each), on the host
 * threads: SesField::value (field/point.rs:496-738) wherever |F| is below
 * the refinement band sqrt(3) h 1.01 (the candidates of the point, as the
 * refinement evaluates them), clamped to -band beyond it inside.  For the
 * distance of mesh vertices to the surface. */
int smb_engine_field(const smb_engine* e, const double* points, size_t n, double* values);
/* Vertex refinement (exact mode, smb_refine_exact) and placement (fast
 * mode, smb_place_fast) on the device, then assembly, validation, measure
 * and grouping there too (the default, on = 1); or all of these on the
 * host threads (on = 0, as the reference).  Both give the same mesh bytes;
 * a mesh with edges the device leaves is finished on the host. */
int smb_engine_set_exact_device(smb_engine* e, int on);
/* Why the engine's last mesh was finished on the host threads rather than
 * on the device ("" when it was not; valid until the next mesh). */
const char* smb_engine_note(const smb_engine* e);
/* The engine's device batch (sizes, counters, operation counts). */
smb_batch* smb_engine_batch(smb_engine* e);
/* Learned warm start of fast mode (no counterpart in the reference): the
 * engine's device refinement starts each edge from the MLP's proposal
 * (smb_refine_warm); null restores the linear start.  The MLP must stay
 * alive while the engine uses it. */
int smb_engine_set_warm_start(smb_engine* e, const smb_mlp* mlp);
/* Training rows of the warm start (no counterpart in the reference): runs
 * the device stage, then for every edge the device refines (marching-cubes
 * order) its SMB_MLP_FEATURES features, as the label the root parameter
 * that exact mode's f64 refinement finds on that edge (before the edge
 * clamp), and the root parameter plain f32 refinement (smb_refine) stops
 * at (NaN where it does not converge).  Edges the device's exact
 * refinement leaves to the host are left out.  *n gets the row count; the
 * rows are copied when features, labels and plain are non-null
 * (SMB_ERR_MEMORY if cap < *n).  The rows are kept until the next device
 * run, so a first call with null buffers sizes them and a second one
 * copies them. */
int smb_engine_warm_start_rows(smb_engine* e, float* features, float* labels, float* plain, size_t cap, size_t* n,
                               char* err, size_t errlen);

void smb_surface_free(smb_surface* s);
int smb_surface_stats_get(const smb_surface* s, smb_surface_stats* out);
/* Mesh arrays (Mesh, mesh/mod.rs:48-67), triangles grouped by component. */
int smb_surface_mesh(const smb_surface* s, float* positions, float* normals, uint32_t* triangles, uint32_t* atoms,
                     uint8_t* patches, uint32_t* components);
/* The same arrays without a copy: pointers into the surface, valid until
 * smb_surface_free (null for empty arrays). */
int smb_surface_arrays(const smb_surface* s, const float** positions, const float** normals,
                       const uint32_t** triangles, const uint32_t** atoms, const uint8_t** patches,
                       const uint32_t** components);
/* OBJ bytes with the default options (export/obj.rs:37-73): returns the
 * length, copies at most cap bytes. */
size_t smb_surface_obj(smb_surface* s, char* out, size_t cap);
int smb_surface_write_obj(smb_surface* s, const char* path, char* err, size_t errlen);

/* Many structures in one device pass (no counterpart in the reference,
 * which meshes one structure per compute_surface call, surface.rs:599-711):
 * structures stay resident side by side, one classification pass covers
 * them all, and the mesh stage runs as one captured CUDA graph whose
 * kernels take (structure, brick) items from a device queue; fast mode,
 * optionally with the learned warm start.  Each structure's mesh is the
 * single-structure device path's at the same brick edge.  Buffers are
 * sized from per-brick caps; a structure over a cap is meshed again on its
 * own (counted in smb_multi_times.redone).  Structures are taken in groups
 * whose buffers fit a third of the free device memory, one pass (one
 * recorded graph) per group; the host stages of one group run while the
 * device meshes the next.  The autotuner picks the brick
 * edge (8 or 16), the candidate caps (level 0 or 1) and the gather block
 * shape (2 or 4 warps) by timing the device pass; a config with every
 * field set skips it. */
typedef struct smb_multi smb_multi;
typedef struct {
    uint32_t brick;        /* 0: tuned; else even, 4..32 */
    uint32_t caps_level;   /* 0 or 1 (tuned when brick or gather_warps is 0) */
    uint32_t gather_warps; /* 0: tuned; else 1, 2, 4 or 8 */
} smb_multi_config;
typedef struct {
    size_t structures, redone, bricks, samples;
    /* ms: arrangements and uploads (once), tuning (once), classification,
     * device pass, copies back, host stages, structures redone, whole run */
    double t_setup, t_tune, t_classify, t_device, t_d2h, t_host, t_redo, t_total;
    int graph;     /* every pass ran from a captured CUDA graph */
    size_t groups; /* passes: structures are grouped to fit the device buffers */
    /* sub-blocks whose lists exceeded the shared-memory caps even on the
     * retry with four times the caps, and that exceeded the list pools or
     * the sampler's block cap (their structures are redone) */
    unsigned long long over_lists, over_memory;
} smb_multi_times;
/* n structures: xyzr[i] holds counts[i] rows (x, y, z, r); params[i] its
 * SES parameters (refine must be SMB_REFINE_FAST; brick_size is set by the
 * batch). */
int smb_multi_new(smb_device* dev, size_t n, const double* const* xyzr, const size_t* counts,
                  const smb_surface_params* params, const smb_multi_config* cfg, smb_multi** out, char* err,
                  size_t errlen);
void smb_multi_free(smb_multi* m);
int smb_multi_set_warm_start(smb_multi* m, const smb_mlp* mlp);
/* Runs the autotuner now (smb_multi_run runs it first when needed). */
int smb_multi_tune(smb_multi* m, char* err, size_t errlen);
int smb_multi_config_get(const smb_multi* m, smb_multi_config* out);
/* Meshes every structure; per-structure results and latencies (ms from the
 * start of the run until that structure's mesh is complete) until the next
 * run. */
int smb_multi_run(smb_multi* m, smb_multi_times* times, char* err, size_t errlen);
/* Each structure's placement, assembly, validation and measure on the
 * device after its group's pass (on = 1, the default; results then live in
 * page-locked memory until the next run), or on the host threads while the
 * device meshes the next group (on = 0).  Same mesh bytes either way. */
int smb_multi_set_device_finish(smb_multi* m, int on);
smb_surface* smb_multi_surface(smb_multi* m, size_t i);
int smb_multi_latency(const smb_multi* m, double* ms);
/* A batch's control: the cancel flag is polled between groups and between
 * structures' host stages (SMB_ERR_CANCELLED); progress reports the mesh
 * stage in structures finished.  The memory fields are not used (the batch
 * sizes its groups to a third of the free device memory). */
int smb_multi_set_control(smb_multi* m, const smb_control* control);

/* The host arrangement of an engine (views valid while it lives; an
 * arrangement built on the device is copied to the host on first use).
 * built_on_device: 1 when the device built it. */
typedef struct {
    size_t n_spheres, n_contained, n_circles, n_vertices;
    const double *center, *expanded, *circle, *vertex;
    const uint32_t *status, *orig, *circle_ij, *vertex_atoms, *nb_off, *nb_items, *cb_off, *cb_items;
    double max_expanded, rho_max, band, t_min;
    int64_t frame[3];
    int built_on_device;
} smb_arrangement_info;
/* Inputs of at least n spheres get their arrangement built on the device
 * (geom/arrangement.rs:246-770 with the host build's values bit for bit;
 * the host builds it when the device declines).  Process-wide; default
 * 16384; 0 = always, SIZE_MAX = never. */
void smb_set_device_arrangement_min(size_t n);
int smb_engine_arrangement(const smb_engine* e, smb_arrangement_info* out);
/* Structure input (io::read_bytes + Structure::select + radii::assign,
 * crates/sesmesh/src/io/mod.rs:188-260, structure/select.rs:140-360,
 * radii/mod.rs:166-250): the atoms of PDB (ATOM / HETATM records, MODEL /
 * ENDMDL) or mmCIF (the _atom_site loop) bytes as (x, y, z, r) rows in file
 * order, under a selection: `model` 0 the first model, else the model with
 * that number; alternate locations resolved per residue by the highest
 * total occupancy (first on ties); hydrogens (H, D, T), waters (HOH, WAT,
 * TIP3, ...) and hetero atoms kept or dropped (default: drop, drop, keep).
 * Radii: the element's Bondi radius (Bondi 1964 completed with Mantina
 * 2009 and Alvarez 2013), 1.80 A for elements without one; the element comes
 * from the element column or type_symbol, else from the atom name.  *n gets
 * the atom count; xyzr (4 doubles per atom) is filled when non-null
 * (SMB_ERR_MEMORY when cap < *n).  format: SMB_FORMAT_AUTO (mmCIF when the
 * bytes open a data_ block), _PDB or _MMCIF.  No device is used. */
enum { SMB_FORMAT_AUTO = 0, SMB_FORMAT_PDB = 1, SMB_FORMAT_MMCIF = 2 };
typedef struct {
    int model;
    int hydrogens, waters, hetero;
} smb_selection;
int smb_read_structure(const char* data, size_t len, int format, const smb_selection* selection, double* xyzr,
                       size_t cap, size_t* n, char* err, size_t errlen);

/* Builds only the host arrangement (no device; smb_engine_arrangement). */
int smb_arrangement_build(const double* xyzr, size_t n, const smb_surface_params* p, smb_engine** out, char* err,
                          size_t errlen);
/* The same under a control (cancel flag polled per sphere, geometry
 * progress). */
int smb_arrangement_build_with(const double* xyzr, size_t n, const smb_surface_params* p,
                               const smb_control* control, smb_engine** out, char* err, size_t errlen);

#ifdef __cplusplus
}
#endif
#endif
