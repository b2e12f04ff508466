// CPU oracle for the sesmesh B200 build — TEST INFRASTRUCTURE ONLY.
//
// A C++ restatement of sesmesh 1.3.2's CPU back end for the SES mesh stage:
// arrangement, exact f64 field, lattice classification, the per-sub-block
// gather and the f32 sampling kernel (scalar form of the SIMD kernel),
// marching cubes with f64 edge refinement, assembly, measurement and the OBJ
// writer.  Only the test suite, the smoke check and the CPU-baseline leg of
// the benchmark may load it, as the checker; the product never links it.
//
// Each function cites the reference file:line it follows (paths relative to
// the sesmesh repository).  Parity is pinned by the reference's own known
// answers: paper/data/analytic.csv (vertex/triangle/component counts, area,
// volume, max |F| of 20 analytic cases), tests/surface.rs obj_snapshot and
// export/fmt.rs formatting cases; see tests/golden/.
//
// Build: -O2 -ffp-contract=off, no fast-math, no -march: every f64/f32
// expression is evaluated in the reference's operation order with IEEE
// rounding and no FMA contraction.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include <array>
#include <functional>

namespace orc {

// ---- geom/vec.rs:1-99 -------------------------------------------------------
struct V3 {
    double x = 0, y = 0, z = 0;
    V3() = default;
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    double dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    V3 cross(const V3& o) const {
        return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x);
    }
    double norm2() const { return dot(*this); }
    double norm() const { return std::sqrt(norm2()); }
    V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator*(double s) const { return V3(x * s, y * s, z * s); }
    V3 operator/(double s) const { return V3(x / s, y / s, z / s); }
    double dist(const V3& o) const { return (*this - o).norm(); }
    V3 normalized() const { return *this / norm(); }
    V3 vmin(const V3& o) const { return V3(std::fmin(x, o.x), std::fmin(y, o.y), std::fmin(z, o.z)); }
    V3 vmax(const V3& o) const { return V3(std::fmax(x, o.x), std::fmax(y, o.y), std::fmax(z, o.z)); }
    bool finite() const { return std::isfinite(x) && std::isfinite(y) && std::isfinite(z); }
};

// Rust `as` casts from f64 saturate; C++ casts of out-of-range values are UB.
inline uint64_t sat_u64(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551616.0) return UINT64_MAX;
    return (uint64_t)v;
}
inline int64_t sat_i64(double v) {
    if (std::isnan(v)) return 0;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    if (v >= 9223372036854775808.0) return INT64_MAX;
    return (int64_t)v;
}

// ---- geom/cells.rs:12-146 ---------------------------------------------------
struct CellGrid {
    V3 origin;
    double cell = 1;
    size_t dims[3] = {1, 1, 1};
    std::vector<uint32_t> starts, items;
    void build(const std::vector<V3>& pts, double cell);
    void coord(const V3& p, size_t out[3]) const;
    size_t flat(size_t x, size_t y, size_t z) const { return (z * dims[1] + y) * dims[0] + x; }
    template <class F>
    void for_each_near(const V3& c, double r, F&& f) const {
        size_t lo[3], hi[3];
        coord(c - V3(r, r, r), lo);
        coord(c + V3(r, r, r), hi);
        for (size_t z = lo[2]; z <= hi[2]; z++)
            for (size_t y = lo[1]; y <= hi[1]; y++) {
                size_t row = flat(0, y, z);
                uint32_t a = starts[row + lo[0]], b = starts[row + hi[0] + 1];
                for (uint32_t i = a; i < b; i++) f(items[i]);
            }
    }
};

struct Csr {
    std::vector<uint32_t> off{0}, items;
    size_t rows() const { return off.empty() ? 0 : off.size() - 1; }
    const uint32_t* row_begin(size_t i) const { return items.data() + off[i]; }
    const uint32_t* row_end(size_t i) const { return items.data() + off[i + 1]; }
    size_t row_len(size_t i) const { return off[i + 1] - off[i]; }
};

enum Status : uint8_t { EXPOSED = 0, BURIED = 1, CONTAINED = 2 };

struct Circle {
    uint32_t i, j;
    V3 center, axis, e1;
    double radius;
    V3 e2() const { return axis.cross(e1); }
};

struct SasVertex {
    V3 position;
    uint32_t atoms[3];
};

// ---- geom/arrangement.rs:205-228 ---------------------------------------------
struct Arrangement {
    double probe = 0;
    std::vector<V3> centers;
    std::vector<double> radii, expanded;
    std::vector<uint32_t> orig;
    std::vector<uint8_t> status;
    Csr neighbors;
    std::vector<Circle> circles;
    Csr circle_blockers;
    std::vector<SasVertex> vertices;
    CellGrid cells;
    double max_expanded = 0;
    size_t n_contained = 0;
};

struct Sphere {
    double c[3];
    double r;
};

// ---- field/point.rs -----------------------------------------------------------
enum FeatKind : uint32_t { F_SOLVENT = 0, F_BEYOND = 1, F_SPHERE = 2, F_CIRCLE = 3, F_VERTEX = 4 };
struct Feature {
    uint32_t kind = F_BEYOND, id = 0;
};
struct PointEval {
    double distance;
    V3 closest;
    Feature feature;
};
struct NearEval {
    double value;
    Feature feature;
    V3 closest;
};
struct LocalCandidates {
    std::vector<uint32_t> inside, near, spheres, s_off, s_blk, circles, c_off, c_blk, vertices;
    std::vector<std::pair<double, uint32_t>> order;
    void clear();
};

// field/mod.rs:33-41: the surface a field describes.
enum Kind : int { KIND_SES = 0, KIND_SAS = 1, KIND_VDW = 2 };

struct SesField {
    Arrangement arr;
    int kind = KIND_SES;
    double probe = 0;
    CellGrid circle_cells, vertex_cells;
    double rho_max = 0, extent = 0;

    bool inside_sas(const V3& x) const;
    PointEval ses_eval(const V3& x, double cutoff) const;
    void try_sphere_with(const V3& x, uint32_t i, const uint32_t* b0, const uint32_t* b1, PointEval& best) const;
    void try_circle_with(const V3& x, uint32_t ci, const uint32_t* b0, const uint32_t* b1, PointEval& best) const;
    void try_vertex(const V3& x, uint32_t vi, PointEval& best) const;
    void gather_local(const V3& b, double rho, double band, LocalCandidates& out) const;
    NearEval eval_local(const V3& x, double band, const LocalCandidates& l) const;
    std::pair<double, int64_t> sphere_eval(const V3& x, double cutoff) const;
    double clamped_value(const V3& x, double band) const;
    // Full sample (value, closest, normal) with the growing cutoff of
    // point.rs:304-349; used for max |F| and normal-angle checks.
    double value(const V3& x, V3* normal, bool* has_normal) const;
};

// Returns an error message (empty on success).
std::string build_field(const Sphere* s, size_t n, double probe, SesField& out, int kind = KIND_SES);

// ---- field/lattice.rs ---------------------------------------------------------
constexpr int64_t KEY_BIAS = int64_t(1) << 20;
constexpr double CLASSIFY_EPS = 2e-3;
struct Lattice {
    double h = 1;
    int64_t b = 10;
    int64_t frame[3] = {0, 0, 0};
    float h32 = 1;
    void init(double h_, size_t b_, const V3& fc);
    V3 point(int64_t i, int64_t j, int64_t k) const { return V3(double(i) * h, double(j) * h, double(k) * h); }
    V3 frame_origin() const { return point(frame[0], frame[1], frame[2]); }
    float local(int64_t idx, int a) const { return float(idx - frame[a]) * h32; }
    V3 brick_center(const int32_t k[3]) const;
    double brick_radius() const { return 0.5 * std::sqrt(3.0) * double(b) * h; }
    int64_t brick_of(double v) const { return sat_i64(std::floor(v / (double(b) * h))); }
};
uint64_t pack_key(const int32_t k[3]);
void unpack_key(uint64_t p, int32_t k[3]);
int uniform_sign(const SesField& f, const V3& center, double rho);  // 1 out, 0 in, -1 none

// ---- field/kernel.rs ----------------------------------------------------------
struct Gathered {
    size_t n_inside = 0;
    std::vector<float> nx, ny, nz, nr, nr2, nr2tol;
    std::vector<float> sx, sy, sz, sr;
    std::vector<uint32_t> s_off, s_blk;
    std::vector<float> cx, cy, cz, ux, uy, uz, ex, ey, ez, rho;
    std::vector<uint32_t> c_off, c_blk;
    std::vector<float> vx, vy, vz;
    // Global sphere index of each near entry (for list comparisons).
    std::vector<uint32_t> near_ids, s_ids, c_ids, v_ids;
    void clear();
};

struct Engine {
    SesField field;
    Lattice lattice;
    double band = 0;
    bool f32_ok = true;
    double coord_max = 0;
    int64_t sub, nsub;
    size_t samples_per_brick() const { size_t s = size_t(lattice.b + 1); return s * s * s; }
};
std::string make_engine(SesField&& field, double spacing, size_t brick, Engine& out);

struct BrickScratch {
    Gathered g;
    std::vector<float> xs, ys, zs, out, values;
    std::vector<uint32_t> groups[8];
    std::vector<uint32_t> local_of, touched;
    std::vector<std::pair<double, uint32_t>> order;
    void init(const Engine& e);
};

std::vector<uint64_t> touched_bricks(const Engine& e, std::string& err);
std::vector<std::array<int32_t, 3>> surface_bricks(const Engine& e, const std::vector<uint64_t>& touched);
void sub_states(const Engine& e, const int32_t key[3], int st[8]);
void evaluate(const Engine& e, const int32_t key[3], BrickScratch& s);
// Gathered lists of one sub-block (prepare_sub without the sample coordinates).
void gather_ses(const Engine& e, const V3& b, double rho, BrickScratch& s);
V3 sub_center(const Engine& e, const int32_t key[3], int sb, double* rho);

// ---- mesh/extract.rs + mesh/mod.rs ---------------------------------------------
struct BrickMesh {
    std::vector<uint32_t> edges;
    std::vector<std::array<float, 3>> positions, normals;
    std::vector<uint32_t> atoms;
    std::vector<uint8_t> patches;
    std::vector<std::array<uint32_t, 3>> tris;
    std::vector<uint32_t> vertex_end, tri_end;  // per brick
    uint64_t evals = 0;
};
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

double edge_clamp(const Engine& e);
void mesh_brick(const Engine& e, const int32_t key[3], const float* values, BrickMesh& out);
void cells_pass(size_t b, const float* values, BrickMesh& out);
std::string assemble(const std::vector<std::array<int32_t, 3>>& bricks, const BrickMesh& parts, Mesh& mesh);
void components(const Mesh& m, std::vector<uint32_t>& id, std::vector<Component>& comps);
void group_by_component(Mesh& m, const std::vector<uint32_t>& id, std::vector<Component>& comps);
size_t validate_defects(const Mesh& m);
std::string obj_bytes(const Mesh& m, int precision = 4, bool normals = true);
void push_fixed(std::string& buf, float x, int prec);

// ---- pipeline (surface.rs:1001-1300, CPU back end) ----------------------------
struct SurfaceStats {
    size_t touched = 0, surface_bricks = 0, vertices = 0, triangles = 0, components = 0;
    double area = 0, volume = 0;
    int64_t euler = 0;
    uint64_t refine_evaluations = 0;
    double t_geometry = 0, t_classify = 0, t_mesh = 0, t_assemble = 0, t_measure = 0;
};
struct SurfaceOut {
    Mesh mesh;
    std::vector<Component> comps;
    SurfaceStats stats;
};
std::string compute_surface(const Sphere* s, size_t n, double probe, double spacing, size_t brick,
                            SurfaceOut& out, int kind = KIND_SES);

// Threads used by the parallel loops (0 = hardware concurrency).
void set_threads(int n);
int threads();
void parallel_for(size_t n, const std::function<void(size_t, int)>& f);

}  // namespace orc
