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
    DBuf pos, nrm, tris, tris_out, keys, cnt, dup, parent, flag, cid, id, counters, comp_v, comp_t, comp_e, area,
        volume, parts, pkey, pidx, pkey2, pidx2, first, tkey, tidx, tkey2, tidx2, tiles, cub;
    void release();
    ~MeasureScratch() { release(); }
};

// The mesh's defects (*bad); when there are none, its components (area,
// volume, Euler characteristic, first triangle), m.vertex_component and
// m.triangles regrouped by component: the host's defects() and
// components_and_group() results bit for bit.  False (with *msg) when the
// device could not do it; the caller then measures on the host.
bool measure_on_device(smb_device* d, smbh::Mesh& m, std::vector<smbh::Component>& comps, size_t* bad,
                       MeasureScratch& S, std::string* msg);

}  // namespace smb
