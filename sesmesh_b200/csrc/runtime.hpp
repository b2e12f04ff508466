// Internal state behind the opaque handles of include/sesmesh_b200.h.
#pragma once
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
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

int dev_alloc(void** p, size_t bytes, std::vector<void*>* owned, size_t* total, char* err, size_t errlen);

}  // namespace smb

struct smb_device {
    int index = 0;
    cudaStream_t stream = nullptr;
    smb_device_info info{};
    size_t smem_optin = 0;
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
};

struct smb_batch {
    smb_resident* res = nullptr;
    uint32_t n = 0, n_work = 0, max_pack = 0;
    size_t first = 0;
    bool refined = false;
    size_t n_edges = 0, n_tris = 0, ids_words = 0;
    smb::DBuf rec, sampled, work, retry_a, retry_b, values, tiles, totals, counters;
    smb::DBuf ids, pack, mc_counts, edge_off, tri_off, edges, edge_vals, tris;
    smb::DBuf e_t, e_feat, e_q, e_evals;  // fast-mode refinement results
    smb::GatherCaps caps{192, 128, 384, 128};
    int gather_warps = 4;
    bool use_tma = true;
    cudaEvent_t ev[6] = {};
    std::vector<smb::DBuf*> bufs() {
        return {&rec, &sampled, &work, &retry_a, &retry_b, &values, &tiles, &totals, &counters,
                &ids, &pack, &mc_counts, &edge_off, &tri_off, &edges, &edge_vals, &tris, &e_t, &e_feat, &e_q, &e_evals};
    }
};
