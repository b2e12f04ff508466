// Internal state behind the opaque handles of include/sesmesh_b200.h.
#pragma once
#include <atomic>
#include <mutex>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/sesmesh_b200.h"
#include "device/kernels.hpp"

namespace smb {

// A device buffer that grows on demand (contents are not preserved).
struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
    int reserve(size_t bytes, char* err, size_t errlen);
    void release();
    void release_synced();  // the device has finished every use of it (no synchronize here)
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

int dev_alloc(void** p, size_t bytes, std::vector<void*>* owned, size_t* total, char* err, size_t errlen);

// Device memory through the process-wide cache (runtime.cu): mem_free
// synchronizes the device and keeps the block for the next mem_alloc of a
// similar size on that device; mem_trim returns a device's cached blocks.
cudaError_t mem_alloc(void** p, size_t bytes);
void mem_free(void* p);
// mem_free for a block the device has finished with (the caller synchronized).
void mem_free_synced(void* p);
void mem_trim(int device);
void mem_device_open(int device);
// Page-locked host memory through a process-wide cache (null on failure).
void* pinned_alloc(size_t bytes);
void pinned_free(void* p);
void mem_device_close(int device);

// Handle lifetimes: a device stays open while residents or MLPs made on it
// live, a resident while batches made on it live, whatever order the caller
// frees them in (a garbage-collected host may finalize them in any order).
void dev_retain(smb_device* d);
void dev_release(smb_device* d);

// The warm-start MLP's device parameters and device (mlp.cu).
struct MlpDev;
MlpDev mlp_dev(const smb_mlp* m);
const smb_device* mlp_device(const smb_mlp* m);
size_t mlp_smem_bytes();
// How the warm start uses the MLP's output (SMB_MLP_GATE or SMB_MLP_ROOT).
int mlp_use(const smb_mlp* m);

}  // namespace smb

struct smb_device {
    int index = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy = nullptr;  // device-to-host copies that overlap the main stream's kernels
    smb_device_info info{};
    size_t smem_optin = 0;
    std::atomic<int> refs{0};
    std::atomic<bool> closed{false}, gone{false};
    // Gather caps and block shape the last batch with these lattice and probe
    // values settled on; new batches with the same values start from them.
    std::mutex hint_mu;
    struct CapsHint {
        double h = 0, probe = 0;
        int b = 0;
        smb::GatherCaps caps{};
        int warps = 0;
    } hint;
};

struct smb_resident {
    smb_device* dev = nullptr;
    smb::DArr A{};
    smb::DLat L{};
    std::vector<void*> owned;
    size_t bytes = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // bounding box of the centres
    int4* keys = nullptr;                          // surface bricks, packed-key order
    uint32_t n_bricks = 0;
    size_t n_touched = 0;
    bool classified = false;
    float classify_ms = 0;
    smb::RefineConsts rc{};
    bool refine_ready = false;
    smb::ExactAttr xa{};  // exact mode on the device (smb_resident_set_exact)
    bool exact_ready = false;
    std::atomic<int> refs{0};  // batches made on this resident
    std::atomic<bool> freed{false}, gone{false};
};

// Shared memory of the sampling's first-pass CTAs (sub-blocks whose packed
// lists are larger wait for a second pass with room for the largest): four
// CTAs fit an SM's 228 KiB with their 1 KiB reserve and static bytes.
constexpr size_t SAMPLE_REGION = 55 * 1024;

struct smb_batch {
    smb_resident* res = nullptr;
    uint32_t n = 0, n_work = 0, max_pack = 0;
    size_t first = 0;
    bool refined = false;
    size_t n_edges = 0, n_tris = 0, ids_words = 0;
    smb::DBuf rec, sampled, work, retry_a, retry_b, values, tiles, totals, counters;
    smb::DBuf ids, pack, mc_counts, edge_off, tri_off, edges, edge_vals, tris;
    smb::DBuf e_t, e_feat, e_q, e_evals;  // fast-mode refinement results
    smb::DBuf e_x;                        // warm-start features (32 f32 per row of the items' edge lists)
    smb::DBuf w_feats;                    // per sample: the sampler's nearest feature (record_features)
    smb::DBuf w_start;                    // per row: the warm start's chosen start
    bool record_features = false;         // the sampler records w_feats
    bool have_features = false;           // the last run recorded them
    smb::DBuf item_counts, item_off, item_edges;  // per sampled sub-block edge lists
    // Vertices refined or placed on the device: position, normal, atom, patch,
    // t, evaluations; overflowed items, summary words, fast-mode exact mask.
    smb::DBuf x_pos, x_nrm, x_atom, x_patch, x_t, x_evals, x_ovf, x_sum, x_mask, x_slab;
    smb::DBuf x_window;  // per sub-block: the gather's and the exact ball's tests disagree somewhere
    bool window_ok = false;  // x_window and ids are this batch's last gather's (smb_run)
    bool refined_exact = false;
    size_t x_exact_edges = 0;  // edges the exact refinement took in the last pass
    size_t x_block_items = 0;  // items of the last exact pass refined by a whole block
    size_t x_region = 13312;  // shared-memory bytes per warp for one sub-block's f64 candidate lists
    size_t s_region = 0;  // sampling: shared memory of the first pass's CTAs (0: SAMPLE_REGION)
    smb::DBuf s_list;     // sampling: the sub-blocks left to the second pass
    int x_hint = 1;   // smb_refine_exact: list sizes from the gather's records (0 off, 2 one short)
    int x_group = 0;  // smb_refine_exact: lanes per edge (0: by the lists' mean size)
    int r_group = 0;  // smb_refine: lanes per edge (0: by the lists' mean size)
    unsigned long long pack_units = 0;  // the last run's list units (16 bytes each)
    size_t r_region = 0;  // smb_refine: bytes per warp's f32 region when four whole ones do not fit (0: an eighth of the SM's)
    smb::GatherCaps caps{192, 128, 384, 128};
    int gather_warps = 4;
    bool use_tma = true;
    cudaEvent_t ev[6] = {};
    std::vector<smb::DBuf*> bufs() {
        return {&rec, &sampled, &work, &retry_a, &retry_b, &values, &tiles, &totals, &counters,
                &ids, &pack, &mc_counts, &edge_off, &tri_off, &edges, &edge_vals, &tris, &e_t, &e_feat, &e_q, &e_evals, &e_x, &w_feats, &w_start, &item_counts, &item_off, &item_edges,
                &x_pos, &x_nrm, &x_atom, &x_patch, &x_t, &x_evals, &x_ovf, &x_sum, &x_mask, &x_slab, &s_list, &x_window};
    }
};
