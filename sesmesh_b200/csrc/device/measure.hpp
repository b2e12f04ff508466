// Validation, components, area and volume, and triangle grouping of an
// assembled mesh on the device (measure.cu).
#pragma once
#include <string>
#include <vector>

#include "../host/mesher.hpp"
#include "../runtime.hpp"

namespace smb {

// Device buffers of the measure, kept between meshes.
struct MeasureScratch {
    DBuf pos, nrm, tris, tris_out, keys, cnt, dup, parent, flag, cid, id, counters, comp_v, comp_t, area,
        volume, parts, pkey, pidx, pkey2, pidx2, first, tkey, tidx, tkey2, tidx2, tiles, cub, packed, err, tri_a,
        tri_v;
    void* host = nullptr;  // page-locked staging of the results
    size_t host_cap = 0;
    // Page-locked words the device writes counters into directly: reading
    // them does not queue behind large copies on the device's copy engines.
    unsigned long long* words = nullptr;
    void* staging(size_t bytes);  // null when page-locked memory cannot be had
    void release(bool synced = false);  // synced: the device has finished every use of them
    ~MeasureScratch() { release(); }
};

// A mesh stage's results on the device: brick keys (packed-key order),
// marching-cubes edge lists and triangle references, and one vertex per
// edge (position, normal, input atom, patch).
struct DeviceMesh {
    const int4* keys;
    size_t n_bricks;
    const uint32_t *edge_off, *edges, *tri_off, *tri_refs;
    size_t n_edges, n_tris;
    const float *pos, *nrm;
    const uint32_t* atoms;
    const uint8_t* patches;
};

// Assembly (extract::assemble, mesh/extract.rs:606-691), validation,
// components, area/volume and grouping of a mesh whose vertices are on the
// device, then the finished mesh back into one page-locked block: the
// host's assemble, defects and components_and_group results bit for bit.
// On success with no defects *block is that block (the caller releases it
// with pinned_free) and *out points into it.  *ms_assemble gets the
// assembly's time.
// 0: done (*bad defects; *out, *block and comps filled when there are none); 1: the
// device could not (*msg; the caller finishes on the host); 2: the
// assembly failed (*msg is the host assembly's error text).
int finish_on_device(smb_device* d, const DeviceMesh& in, smbh::MeshRef* out, void** block,
                     std::vector<smbh::Component>& comps, size_t* bad, MeasureScratch& S, std::string* msg,
                     double* ms_assemble);

// The mesh's defects (*bad); when there are none, its components (area,
// volume, Euler characteristic, first triangle), m.vertex_component and
// m.triangles regrouped by component: the host's defects() and
// components_and_group() results bit for bit.  False (with *msg) when the
// device could not do it; the caller then measures on the host.
bool measure_on_device(smb_device* d, smbh::Mesh& m, std::vector<smbh::Component>& comps, size_t* bad,
                       MeasureScratch& S, std::string* msg);

}  // namespace smb
