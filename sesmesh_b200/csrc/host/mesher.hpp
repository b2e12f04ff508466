// Host stages of the mesh stage that sesmesh keeps on the CPU: exact f64
// vertex refinement of the device's crossing edges, assembly, validation,
// components, area/volume and the OBJ writer.
#pragma once
#include <array>
#include <cstdint>
#include <string>
#include <memory>
#include <vector>

#include "geom.hpp"

namespace smbh {

enum FeatKind : uint32_t { F_SOLVENT = 0, F_BEYOND = 1, F_SPHERE = 2, F_CIRCLE = 3, F_VERTEX = 4 };

struct Feature {
    uint32_t kind = F_BEYOND, id = 0;
};

struct NearEval {
    double value;
    Feature feature;
    V3 closest;
};

// Candidates of one ball (SesField::gather_local, field/point.rs:496-582),
// with pruning keys: the candidate's value at the ball centre minus the
// ball radius and a margin, ascending like the lists.
struct Local {
    std::vector<uint32_t> inside, near, spheres, s_off, s_blk, circles, c_off, c_blk, vertices;
    std::vector<double> s_key, c_key, v_key;
    std::vector<std::pair<double, uint32_t>> order;
};

// Lattice and refinement constants of one engine (Engine::new,
// field/kernel.rs:204-271; extract::edge_clamp, mesh/extract.rs:47-51).
struct MeshParams {
    double h = 0.5, band = 0, t_min = 1e-4, coord_max = 0;
    int b = 10, sub = 5;
    int64_t frame[3] = {0, 0, 0};
    bool f32_ok = true;
};

// Output of the mesh stage for a run of bricks, vertex k of brick i at
// edge_off[i] + k (one vertex per owned crossing edge).
struct MeshOut {
    std::vector<std::array<float, 3>> positions, normals;
    std::vector<uint32_t> atoms;
    std::vector<uint8_t> patches;
    std::vector<float> t;         // per vertex: root parameter on its edge (before the clamp)
    std::vector<uint32_t> evals;  // per brick
    std::vector<uint32_t> cpu_refined;  // per brick (fast mode)
};

void gather_local(const Arrangement& A, const V3& b, double rho, double band, Local& out);
NearEval eval_local(const Arrangement& A, const V3& x, double band, const Local& l);

// Exact refinement of the owned crossing edges of bricks [0, n): keys (3 per
// brick), edge ids and (fa, fb) from the device, edge_off (n + 1).  Writes
// vertices at their edge index.  Brick order, edge order and arithmetic are
// those of mesh_brick (mesh/extract.rs:146-219, 425-535).
void refine_exact(const Arrangement& A, const MeshParams& P, const int32_t* keys, size_t n, const uint32_t* edge_off,
                  const uint32_t* edges, const float* edge_vals, MeshOut& out);

// Device f32 refinement results of fast mode (DeviceEdges::get,
// field/gpu.rs:155-179): t, feature (kind << 29 | id), closest point
// relative to the brick origin, evaluations | 1 << 31 when converged.
struct DeviceRefine {
    const float* t;
    const uint32_t* feat;
    const float* closest;
    const uint32_t* evals;
};
// mesh_brick_device (mesh/extract.rs:274-365): converged device results are
// placed with the edge clamp and the exact attributes; the rest are refined
// exactly as in refine_exact.
void place_fast(const Arrangement& A, const MeshParams& P, const int32_t* keys, size_t n, const uint32_t* edge_off,
                const uint32_t* edges, const float* edge_vals, const DeviceRefine& dev, MeshOut& out);

// Exact mode with the device's f64 vertices (smb_refine_exact): out holds
// them at their edge index (positions, normals, atoms, patches, t); edges
// with dev_evals[k] = 0 are refined here as in refine_exact.  Per-brick
// evaluations and host-refined edge counts are filled.
void place_exact(const Arrangement& A, const MeshParams& P, const int32_t* keys, size_t n, const uint32_t* edge_off,
                 const uint32_t* edges, const float* edge_vals, const uint32_t* dev_evals, MeshOut& out);

struct Mesh {
    std::vector<std::array<float, 3>> positions, normals;
    std::vector<std::array<uint32_t, 3>> triangles;
    std::vector<uint32_t> vertex_atom, vertex_component;
    std::vector<uint8_t> vertex_patch;
};

struct Component {
    size_t vertices = 0, triangles = 0, first_triangle = 0;
    double area = 0, volume = 0;
    int64_t euler = 0;
};

// extract::assemble (mesh/extract.rs:606-691): triangle references of each
// brick resolved to global vertex indices.  Keys are in packed-key order.
std::string assemble(const int32_t* keys, size_t n, const uint32_t* edge_off, const uint32_t* edges,
                     const uint32_t* tri_off, const uint32_t* tri_refs, Mesh& mesh);

// Directed edge uses of a mesh bucketed by their smaller vertex (each
// bucket sorted): use = larger vertex << 1 | (min -> max direction); the
// uses of one undirected edge are adjacent (Edges, mesh/mod.rs:300-380).
struct EdgeUses {
    std::vector<uint64_t> start;
    std::vector<uint64_t> uses;
    void build(const Mesh& m);
};

// validate_with (mesh/mod.rs:638-700): total defect count (0 = valid); the
// edge uses are kept in *keep when given.
size_t defects(const Mesh& m, EdgeUses* keep = nullptr);
// components_with + group_by_component (mesh/mod.rs:185-297, post.rs:14-32).
void components_and_group(Mesh& m, std::vector<Component>& comps, const EdgeUses* uses = nullptr);
// Read-only arrays of a finished mesh, wherever they are stored.
struct MeshRef {
    const float* pos = nullptr;      // 3 per vertex
    const float* nrm = nullptr;      // 3 per vertex, or null
    const uint32_t* tris = nullptr;  // 3 per triangle
    const uint32_t* atom = nullptr;
    const uint8_t* patch = nullptr;
    const uint32_t* comp = nullptr;
    size_t nv = 0, nt = 0;
    static MeshRef of(const Mesh& m) {
        MeshRef r;
        r.nv = m.positions.size(), r.nt = m.triangles.size();
        r.pos = r.nv ? m.positions.data()->data() : nullptr;
        r.nrm = m.normals.empty() ? nullptr : m.normals.data()->data();
        r.tris = r.nt ? m.triangles.data()->data() : nullptr;
        r.atom = m.vertex_atom.empty() ? nullptr : m.vertex_atom.data();
        r.patch = m.vertex_patch.empty() ? nullptr : m.vertex_patch.data();
        r.comp = m.vertex_component.empty() ? nullptr : m.vertex_component.data();
        return r;
    }
};

std::string obj_text(const MeshRef& m, int precision = 4, bool normals = true);
// The same text in a buffer that is written once (not zero-filled first).
struct ObjText {
    std::unique_ptr<char[]> data;
    size_t size = 0;
    bool empty() const { return !data; }
};
ObjText obj_text_buffer(const MeshRef& m, int precision = 4, bool normals = true);
inline std::string obj_text(const Mesh& m, int precision = 4, bool normals = true) {
    return obj_text(MeshRef::of(m), precision, normals);
}
void push_fixed(std::string& buf, float x, int prec);

}  // namespace smbh
