// Host objects behind the opaque handles of include/sesmesh_b200_surface.h,
// shared by the single-structure engine and the many-structure batch.
#pragma once
#include <string>
#include <vector>

#include "../../../include/sesmesh_b200.h"
#include "../../../include/sesmesh_b200_surface.h"
#include "../device/measure.hpp"
#include "../device/sas.hpp"
#include "../runtime.hpp"
#include "geom.hpp"
#include "mesher.hpp"

using smbh::Arrangement;
using smbh::Component;
using smbh::DeviceRefine;
using smbh::Mesh;
using smbh::MeshParams;

struct smb_engine {
    smb_device* dev = nullptr;
    smb_surface_params params{};
    Arrangement arr;           // the host arrangement (of a device-built one: copied on first use)
    bool arr_ready = true;     // arr holds the arrangement
    smb::DevArrangement darr;  // the device-built arrangement's descriptors (its buffers belong to res)
    size_t n_spheres = 0;      // spheres with r > 0
    MeshParams mp;
    smb_resident* res = nullptr;
    smb_batch* batch = nullptr;
    double t_geometry = 0, t_upload = 0;
    int arr_where = 0;          // smb_surface_stats::arrangement_where
    smbh::Control ctl;          // cancel flag and progress of the engine's calls
    uint64_t max_device_bytes = 0;  // the memory guard's limit (0: none)
    uint64_t last_estimate = 0;     // the guard's estimate at the last classification
    uint64_t upload_bytes = 0;  // bytes copied host to device for the arrangement
    // Host copies of the last device run.
    std::vector<int32_t> keys;
    std::vector<uint32_t> edge_off, edges, tri_off, tris;
    std::vector<float> edge_vals, t, closest;
    std::vector<uint32_t> feat, evals;
    size_t touched = 0;
    smb_batch_times times{};
    double t_classify = 0;
    const smb_mlp* warm = nullptr;  // warm start of fast-mode refinement
    bool exact_device = true;       // exact mode: f64 refinement on the device (else on the host threads)
    smbh::MeshOut exact_out;        // its vertices, at their edge index
    std::string note;               // why the last mesh was finished on the host, if it was
    std::vector<uint32_t> exact_evals;
    smb::MeasureScratch measure;    // device buffers of the validation and measure
    // Warm-start training rows of the last device run.
    bool rows_ready = false;
    std::vector<float> row_x, row_t, row_p;
};

// The engine's host arrangement (copied from the device on first use when
// the device built it).
const Arrangement& host_arrangement(smb_engine* e);

struct smb_surface {
    Mesh mesh;
    std::vector<Component> comps;
    smb_surface_stats stats{};
    smbh::ObjText obj;
    // A mesh finished on the device stays in the page-locked block its
    // results came back in (view points into it); else view is of mesh.
    void* block = nullptr;
    smbh::MeshRef view;
    smbh::MeshRef ref() const { return block ? view : smbh::MeshRef::of(mesh); }
    smb_surface() = default;
    smb_surface(const smb_surface&) = delete;
    smb_surface& operator=(const smb_surface&) = delete;
    ~smb_surface() { smb::pinned_free(block); }
};


// Host stages of one structure after its device run: placement of the
// device's f32 roots (fast) or f64 refinement (exact), assembly,
// validation, components and grouping; fills the statistics it can (sizes,
// area, volume, evaluations, host stage times).  With a device, the
// validation and measure run there (same results), else on the host
// threads.  Exact mode with the device's f64 vertices: `exact` holds them
// (consumed) and exact_evals their evaluation counts (0: refined here).
// Error text or "".
std::string finish_surface(const Arrangement& arr, const MeshParams& mp, bool fast, const int32_t* keys, size_t nb,
                           const uint32_t* edge_off, const uint32_t* edges, const float* edge_vals,
                           const uint32_t* tri_off, const uint32_t* tris, const DeviceRefine& dev, smb_surface& s,
                           smb_device* device = nullptr, smb::MeasureScratch* scratch = nullptr,
                           smbh::MeshOut* exact = nullptr, const uint32_t* exact_evals = nullptr);

// The engine's batch, with every vertex on the device (smb_refine_exact or
// smb_place_fast ran and left no edge to the host), assembled, validated,
// measured and grouped on the device into s (surface.cpp).  evals: the
// vertices' evaluation count; cpu_edges: the statistic refine_cpu_edges.
// SMB_OK or an error code; *fallback when the device declined (the host
// stages must finish the mesh).
int finish_exact_device(smb_engine* e, smb_surface& s, unsigned long long evals, unsigned long long cpu_edges,
                        bool* fallback, double* ms_d2h, char* err, size_t errlen);
