// Host-side geometry of the mesh stage: the f64 3-vector, cell grids and the
// SAS arrangement in the layout the C ABI uploads (smb_arrangement_ref), plus
// a small parallel-for.  Restates crates/sesmesh/src/geom/{vec.rs,cells.rs,
// arrangement.rs}; every expression keeps the reference's operation order
// (built with -ffp-contract=off).
#pragma once
#include <cmath>
#include <cstdint>
#include <functional>
#include <string>
#include <vector>

namespace smbh {

struct V3 {
    double x = 0, y = 0, z = 0;
    V3() = default;
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    static V3 at(const double* p) { return V3(p[0], p[1], p[2]); }
    double dot(const V3& o) const { return x * o.x + y * o.y + z * o.z; }
    V3 cross(const V3& o) const { return V3(y * o.z - z * o.y, z * o.x - x * o.z, x * o.y - y * o.x); }
    double norm() const { return std::sqrt(dot(*this)); }
    V3 operator+(const V3& o) const { return V3(x + o.x, y + o.y, z + o.z); }
    V3 operator-(const V3& o) const { return V3(x - o.x, y - o.y, z - o.z); }
    V3 operator*(double s) const { return V3(x * s, y * s, z * s); }
    V3 operator/(double s) const { return V3(x / s, y / s, z / s); }
    double dist(const V3& o) const { return (*this - o).norm(); }
    V3 unit() const { return *this / norm(); }
    V3 lo(const V3& o) const { return V3(std::fmin(x, o.x), std::fmin(y, o.y), std::fmin(z, o.z)); }
    V3 hi(const V3& o) const { return V3(std::fmax(x, o.x), std::fmax(y, o.y), std::fmax(z, o.z)); }
};

// Rust's saturating float-to-int casts.
inline uint64_t to_u64(double v) {
    if (!(v > 0.0)) return 0;
    return v >= 18446744073709551616.0 ? UINT64_MAX : uint64_t(v);
}
inline int64_t to_i64(double v) {
    if (std::isnan(v)) return 0;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return v >= 9223372036854775808.0 ? INT64_MAX : int64_t(v);
}

// Points binned into a uniform grid, items of a cell contiguous and
// ascending (geom/cells.rs:12-130).
struct Grid {
    double origin[3] = {0, 0, 0};
    double cell = 1;
    uint32_t dims[3] = {1, 1, 1};
    std::vector<uint32_t> starts, items;

    void build(const double* pts, size_t n, size_t stride, double cell);
    inline uint32_t coord(double p, int a) const {
        double c = std::floor((p - origin[a]) / cell);
        if (!(c > 0.0)) return 0;
        uint64_t v = to_u64(c);
        return v >= dims[a] - 1 ? dims[a] - 1 : uint32_t(v);
    }
    template <class F>
    void near(const V3& c, double r, F&& f) const {
        uint32_t x0 = coord(c.x - r, 0), y0 = coord(c.y - r, 1), z0 = coord(c.z - r, 2);
        uint32_t x1 = coord(c.x + r, 0), y1 = coord(c.y + r, 1), z1 = coord(c.z + r, 2);
        for (uint32_t z = z0; z <= z1; z++)
            for (uint32_t y = y0; y <= y1; y++) {
                size_t row = (size_t(z) * dims[1] + y) * dims[0];
                for (uint32_t i = starts[row + x0], e = starts[row + x1 + 1]; i < e; i++) f(items[i]);
            }
    }
};

enum : uint32_t { EXPOSED = 0, BURIED = 1, CONTAINED = 2 };

// The SAS arrangement for one probe radius (geom/arrangement.rs:205-228),
// internal Morton order, flat arrays in the upload layout.
struct Arrangement {
    int kind = 0;     // SMB_KIND_SES, SMB_KIND_SAS or SMB_KIND_VDW (a sphere field: no circles or vertices)
    double probe = 0;  // the probe the spheres were expanded by (0 for the vdW surface)
    size_t n = 0, n_contained = 0;
    std::vector<double> center, expanded, radius;  // center: 3 per sphere
    std::vector<uint32_t> orig, status;
    std::vector<uint32_t> nb_off, nb_items;        // exposed rows only once built
    std::vector<double> circle;                    // 10 per circle: centre, axis, e1, radius
    std::vector<uint32_t> circle_ij;               // 2 per circle
    std::vector<uint32_t> cb_off, cb_items;
    std::vector<double> vertex;                    // 3 per SAS vertex
    std::vector<uint32_t> vertex_atoms;            // 3 per SAS vertex
    Grid cells, circle_cells, vertex_cells;
    double max_expanded = 0, rho_max = 0, extent = 0;

    V3 c(uint32_t i) const { return V3::at(&center[3 * size_t(i)]); }
    size_t n_circles() const { return circle_ij.size() / 2; }
    size_t n_vertices() const { return vertex_atoms.size() / 3; }
};

// Cooperative cancellation and progress (Control, crates/sesmesh/src/
// control.rs:54-131): a flag polled per sphere and per brick, and a
// callback told (0, total) and (total, total) of each stage.
struct Control {
    const volatile int32_t* cancel = nullptr;
    void (*progress)(void* user, int stage, uint64_t done, uint64_t total) = nullptr;
    void* user = nullptr;
    bool cancelled() const { return cancel && *cancel != 0; }
    void report(int stage, uint64_t done, uint64_t total) const {
        if (progress) progress(user, stage, done, total);
    }
};
// The error text of a computation stopped by its control.
extern const char* const CANCELLED;

// Builds the SES arrangement of n spheres (x, y, z, r rows); error text or
// "" (CANCELLED when ctl's flag was set before it finished).
std::string build_arrangement(const double* xyzr, size_t n, double probe, Arrangement& out,
                              const Control* ctl = nullptr, int kind = 0);
// The input checks of build_arrangement alone; error text or "".
std::string check_spheres(const double* xyzr, size_t n, double probe, int kind = 0);

void set_threads(int n);
int threads();
void parallel_for(size_t n, const std::function<void(size_t, int)>& f);

// While alive, parallel_for on this thread runs its loop in the calling
// thread (for work that is itself one of many parallel tasks).
struct SerialScope {
    SerialScope();
    ~SerialScope();
    bool prev;
};

}  // namespace smbh
