// Host-visible declarations of the device kernels' launchers.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace smb {

// Dense box of brick keys [lo, lo + n) per axis (touched-brick flags).
struct BrickBox {
    long long lo[3];
    uint32_t n[3], pad;
};

enum : int { ERR_NONE = 0, ERR_KEY_RANGE = 1, ERR_BOX = 2 };

// Per-warp shared-memory capacities of the gather kernel.
struct GatherCaps {
    int near, s, c, v;
};

__host__ __device__ inline size_t gather_smem_bytes(const GatherCaps& c) {
    size_t b = size_t(c.near) * 12 + size_t(c.s) * 24 + size_t(c.c) * 20 + size_t(c.v) * 4 + 8;
    return (b + 15) & ~size_t(15);
}

// Device counters of one gather/sample pass.
enum : int {
    CNT_IDS = 0, CNT_PACK = 1, CNT_MAXPACK = 2, CNT_OVERFLOW = 3, CNT_NOMEM = 4, CNT_TIMEOUT = 5, CNT_OPS = 6,
    CNT_OWNED = 7, CNT_MAXNN = 8, CNT_MAXNS = 9, CNT_MAXNC = 10, CNT_MAXNV = 11, CNT_MAXITEM = 12, CNT_QUEUE = 13, CNT_RETRY = 14, CNT_XQUEUE = 15, CNT_N = 16
};
constexpr uint32_t REC_NOMEM = 2;

struct GatherOut {
    uint32_t* rec;
    uint32_t* ids;
    uint4* pack;
    uint32_t* retry;  // sub-blocks whose lists exceeded the shared-memory caps
    unsigned long long* counters;
    unsigned long long ids_cap, pack_cap;
    unsigned long long unit_cap;  // largest packed block of one sub-block
    uint32_t* fail;               // per structure (many-structure runs), else null
    // Per sub-block (null: not kept): 1 when some candidate passes the
    // exact refinement's ball test (rho with its margins) but not the
    // gather's or the other way round, else 0.
    uint8_t* window = nullptr;
};

// Fast-mode refinement constants (RefineRef, sesmesh-gpu batch.rs:133-150).
struct RefineConsts {
    float h_hi, h_lo, tol;
    uint32_t max_iter, max_bisect;
};

// Many structures in one launch: per-structure descriptors, indexed by the
// structure number each brick key carries in .w (int4 keys (x, y, z, s)).
// Every structure's arrays are slices of shared device buffers and use
// structure-local indices, so the kernels' bodies are those of one structure.
struct Scene {
    const DArr* arr;
    const DLat* lat;
    const RefineConsts* rc;
    const BrickBox* box;                 // classification: each structure's brick box
    const unsigned long long* flag_off;  // its first flag (n_struct + 1)
    const uint32_t* sph_off;             // its first sphere (n_struct + 1)
    uint32_t n_struct;
    const unsigned long long* n_work;    // sampled sub-blocks, on the device (graph replays)
    int* err;                            // per structure: classification errors
    uint32_t* fail;                      // per structure: a list or buffer limit was exceeded
};

size_t refine_smem_bytes(uint32_t nn, uint32_t ns, uint32_t nc, uint32_t nv, uint32_t nsb, uint32_t ncb);
enum : int { REFINE_PLAIN = 0, REFINE_WARM = 1 };
// Per refinable work item, its edge list (counts, exclusive offsets with the
// total at item_off[n], edge indices); the largest count goes to
// counters[CNT_MAXITEM].  With a mask, only the edges k with mask[k] != 0.
// Flagged sub-blocks (sampler lists over their caps) are left out unless
// all_items or a mask is given (the exact refinement builds its own lists).
void launch_item_edges(const DLat& L, const uint32_t* work, uint32_t n, const uint32_t* rec, const uint32_t* edge_off,
                       const uint32_t* edges, uint32_t* counts, uint32_t* item_off, uint32_t* item_edges,
                       unsigned long long* tiles, unsigned long long* total, unsigned long long* counters,
                       cudaStream_t s, const Scene* many = nullptr, const int4* keys = nullptr,
                       const uint8_t* mask = nullptr, bool all_items = false);
void launch_put_total(uint32_t* dst, const unsigned long long* total, cudaStream_t s);
void launch_copy_count(unsigned long long* dst, const unsigned long long* src, cudaStream_t s);
// Persistent refinement over the items' edge lists, each edge started at the
// linear guess (REFINE_PLAIN) or as start[e], row e of the lists, says
// (REFINE_WARM: the start and the candidate its first evaluation must name
// to be accepted, as float bits, 0 for none); grid = SMs x resident CTAs.  *smem_out gets the shared memory it needs (also
// when it does not launch, for n_items = 0).  With ovf (n_items + 1 words)
// the plain single-structure pass runs per-warp regions of `region` bytes
// (0: an eighth of smem_limit, two blocks to an SM) where four regions for the largest sub-block
// would not fit or `region` is smaller, then a whole-block pass over the
// sub-blocks that outgrow them.  group: lanes per edge in the single-
// structure passes, 8 or 32 (32 pays for long candidate lists).  count
// (single structure): the f32 operations of the field evaluations are added
// to counters[CNT_OPS] (groups of 8, every sub-block in one pass).
cudaError_t launch_refine(const DArr& A, const DLat& L, const RefineConsts& RC, const int4* keys, const uint32_t* work,
                          const uint32_t* rec, const uint32_t* ids, const uint32_t* edges, const float2* edge_vals,
                          const uint32_t* item_off, const uint32_t* item_edges, uint32_t n_items, float* t,
                          uint32_t* feat, float* q, uint32_t* evals, size_t cand_bytes, int mode, const float2* start,
                          unsigned long long* counters, int sms, size_t smem_limit, cudaStream_t s, size_t* smem_out,
                          const Scene* many = nullptr, uint32_t* ovf = nullptr, size_t region = 0, int group = 8,
                          bool count = false);
// The warm start's features of every row of the items' edge lists (32 f32
// per row into x_out); feats: the sampler's nearest-feature words
// (launch_sample with feats).  Grid-strided over at most max_rows rows (the
// many-structure pass reads its item count on the device).
void launch_warm_features(const DArr& A, const DLat& L, const RefineConsts& RC, const int4* keys, const uint32_t* work,
                          uint32_t n_items, const uint32_t* rec, const uint32_t* edges, const float2* edge_vals,
                          const uint32_t* item_off, const uint32_t* item_edges, const float* values,
                          const uint32_t* feats, float* x_out, size_t max_rows, int sms, cudaStream_t s,
                          const Scene* many = nullptr);
// The warm start's start per row (features and the MLP in one kernel, the
// tensor cores for the MLP): start[e] for the REFINE_WARM refinement.
struct MlpDev;
cudaError_t launch_warm_starts(const DArr& A, const DLat& L, const RefineConsts& RC, const int4* keys,
                               const uint32_t* work, uint32_t n_items, const uint32_t* rec, const uint32_t* edges,
                               const float2* edge_vals, const uint32_t* item_off, const uint32_t* item_edges,
                               const float* values, const uint32_t* feats, const MlpDev& P, int use, float2* start,
                               unsigned long long* counters, size_t max_rows, int sms, cudaStream_t s,
                               const Scene* many = nullptr);

unsigned long long kernel_launches();
void count_launches(unsigned long long n);

// Exact mode on the device (exact.cu): the vertex attribute tables (input
// index per sphere, atom pair per circle, atom triple per SAS vertex) and
// the edge clamp t_min (extract.rs:47-51).
struct ExactAttr {
    const uint32_t* orig;
    const uint32_t* circle_ij;
    const uint32_t* vertex_atoms;
    double t_min;
};
// Per edge: position and normal (3 f32 each), input atom, patch, root
// parameter before the clamp, evaluations (0: left to the host).
struct ExactOut {
    float* pos;
    float* nrm;
    uint32_t* atom;
    uint8_t* patch;
    float* t;
    uint32_t* evals;
};
// Fast mode's placement on the device (mesh_brick_device, extract.rs:274-365):
// converged edges placed with their exact attributes into out; need[k] = 1
// (and *marked counts them) for the edges the exact refinement must take.
cudaError_t launch_place_fast(const DArr& A, const DLat& L, const ExactAttr& X, const int4* keys, uint32_t n_bricks,
                              const uint32_t* edge_off, const uint32_t* edges, const float2* edge_vals, size_t n_edges,
                              const float* t, const uint32_t* feat, const float* q, const uint32_t* evals,
                              const ExactOut& out, uint8_t* need, unsigned long long* marked, cudaStream_t s);
// out[0] = sum of evals[0..n), out[1] = how many are 0.
cudaError_t launch_exact_summary(const uint32_t* evals, size_t n, unsigned long long* out, int sms, cudaStream_t s);
// f64 refinement of the work items' edge lists (k_item_edges): a warp per
// item with `region` bytes of shared memory for the item's candidate lists,
// then the items that did not fit with a warp each and a 256 KiB list slab
// in global memory (slab: exact_slab_bytes(sms) bytes).  ovf: n_items + 2
// words (overflow count, items, then the count of items over a slab, whose
// edges keep evals = 0).  count: counters[CNT_OPS] gets the f64 operations
// of the field evaluations (x_eval's rules).  rec: the gather's records of
// the sub-blocks (their list sizes bound each ball's), or null; hint 0: do
// not use them, 2: bounds one short (every ball through the counted layout).
// gids, window: the gather's candidate ids and its per-sub-block marks
// (GatherOut::window); an unmarked sub-block takes its lists from the ids.
size_t exact_slab_bytes(int sms);
cudaError_t launch_refine_exact(const DArr& A, const DLat& L, const ExactAttr& X, const int4* keys,
                                const uint32_t* work, const uint32_t* edges, const float2* edge_vals,
                                const uint32_t* item_off, const uint32_t* item_edges, uint32_t n_items,
                                const ExactOut& out, uint32_t* ovf, unsigned char* slab, size_t slab_bytes,
                                unsigned long long* counters, int sms, size_t region, cudaStream_t s,
                                bool count = false, int group = 1, const uint32_t* rec = nullptr, int hint = 1,
                                const uint32_t* gids = nullptr, const uint8_t* window = nullptr);
void launch_selftest(const float* a, const float* b, uint32_t* out, uint32_t n, cudaStream_t s);
void launch_scan(const uint32_t* in, uint32_t n, uint32_t* out, uint32_t* keep, unsigned long long* tiles,
                 unsigned long long* total, cudaStream_t s);
uint32_t scan_tiles_needed(uint32_t n);
void launch_mark_touched(const DArr& A, const DLat& L, const BrickBox& box, uint32_t* flags, int* err, cudaStream_t s,
                         const Scene* many = nullptr, uint32_t n_total = 0);
void launch_classify_bricks(const DArr& A, const DLat& L, const BrickBox& box, const uint32_t* touched, uint32_t n,
                            uint32_t* surface, cudaStream_t s, const Scene* many = nullptr);
void launch_cells_to_keys(const BrickBox& box, const uint32_t* cells, uint32_t n, int4* keys, cudaStream_t s,
                          const Scene* many = nullptr);
void launch_substates(const DArr& A, const DLat& L, const int4* keys, uint32_t n, uint32_t* rec, uint32_t* sampled,
                      cudaStream_t s, const Scene* many = nullptr);
cudaError_t launch_gather(const DArr& A, const DLat& L, const int4* keys, const uint32_t* work, uint32_t n,
                          const GatherOut& O, const GatherCaps& caps, int warps, cudaStream_t s,
                          const Scene* many = nullptr);
// One CTA per sampled sub-block with the largest packed block's bytes of
// shared memory; with list (n + 1 words) and small, two passes: the blocks
// of up to small bytes with small bytes each, then the others.
cudaError_t launch_sample(const DLat& L, const int4* keys, const uint32_t* work, uint32_t n, const uint32_t* rec,
                          const uint4* pack, uint32_t max_units, float* values, unsigned long long* counters, bool tma,
                          bool count, cudaStream_t s, const Scene* many = nullptr, uint32_t* list = nullptr,
                          size_t small = 0, const uint32_t* ids = nullptr, uint32_t* feats = nullptr);
cudaError_t launch_mc(const DLat& L, uint32_t n, float* values, const uint32_t* rec, uint32_t* counts, const uint32_t* edge_off,
                      const uint32_t* tri_off, uint32_t* edges, float2* edge_vals, uint32_t* tris, bool fill,
                      cudaStream_t s, const int4* keys = nullptr,
                      unsigned long long edge_cap = ~0ull, unsigned long long tri_cap = ~0ull,
                      const Scene* many = nullptr);

}  // namespace smb
