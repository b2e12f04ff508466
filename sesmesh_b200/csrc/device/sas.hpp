// The SAS arrangement built on the device (sas.cu).
#pragma once
#include <string>
#include <vector>

#include "../host/geom.hpp"
#include "../runtime.hpp"
#include "kernels.hpp"

namespace smb {

// A device-built arrangement in the resident layout.  The buffers are owned
// (mem_alloc'd) and released with release() unless a resident took them.
struct DevArrangement {
    std::vector<void*> owned;
    size_t bytes = 0;
    DArr A{};
    const uint32_t* orig = nullptr;          // input index per sphere
    const uint32_t* circle_ij = nullptr;     // 2 per circle
    const uint32_t* vertex_atoms = nullptr;  // 3 per SAS vertex
    size_t n = 0, n_contained = 0, n_circles = 0, n_vertices = 0, nb_items = 0, cb_items = 0;
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};  // bounding box of the centres
    double extent = 0;
    void release();
};

// build_arrangement (host/arrangement.cpp, geom/arrangement.rs:246-770) on
// the device, with the host build's values bit for bit.  0: built; 1: the
// device declines (an exposure decision within the device's error bound of
// its threshold, or a circle with more blockers than a thread keeps): the
// caller builds on the host; 2: an error (*msg).
int build_arrangement_device(smb_device* d, const double* xyzr, size_t n, double probe, DevArrangement& out,
                             std::string* msg);

// The host Arrangement of a device-built one (the host build's layout).
bool arrangement_to_host(const DevArrangement& D, smbh::Arrangement& A);

// A resident over a device-built arrangement (runtime.cu): takes over D's
// buffers (D keeps its descriptors, no longer owning); the exact-mode
// attribute tables are D's, with t_min set by resident_set_exact_tmin.
int resident_from_device(smb_device* d, DevArrangement& D, const smb_lattice_ref* lat, smb_resident** out, char* err,
                         size_t errlen);
void resident_set_exact_tmin(smb_resident* r, double t_min);

}  // namespace smb
