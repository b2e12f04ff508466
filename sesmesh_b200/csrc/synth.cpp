// Seeded synthetic sphere sets for the workloads the benchmark and tests use
// (no public dataset is involved).  Deterministic bit for bit on any x86-64
// host: IEEE double arithmetic only, built without FMA contraction.
//
// Globule: a self-avoiding, branching random walk of 1.5 A bonds confined to
// a ball, every pair more than two bonds apart at least 2.8 A apart (pairs two
// bonds apart at least 2.2 A, i.e. bond angles above ~94 degrees), elements
// C/N/O/S drawn 62/17/19/2 % with Bondi radii 1.70/1.55/1.52/1.80 A.  The
// walk steps from the last atom; after 48 rejected steps it branches from a
// random earlier atom.  The ball radius of an N-atom globule is the one of
// about one atom per 20 A^3, r = (3 * 20 N / (4 pi))^(1/3), unless given.
#include <cmath>
#include <cstdint>
#include <array>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

struct Rng {  // SplitMix64
    uint64_t s;
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ULL;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    }
    double uniform(double lo, double hi) { return lo + (hi - lo) * double(next() >> 11) / 9007199254740992.0; }
    size_t below(size_t n) { return size_t(next() % uint64_t(n)); }
    void unit(double v[3]) {
        for (;;) {
            double a = uniform(-1, 1), b = uniform(-1, 1), c = uniform(-1, 1);
            double n2 = a * a + b * b + c * c;
            if (n2 >= 0.01 && n2 <= 1.0) {
                double n = std::sqrt(n2);
                v[0] = a / n, v[1] = b / n, v[2] = c / n;
                return;
            }
        }
    }
};

struct Hash {
    double cell;
    std::unordered_map<uint64_t, std::vector<uint32_t>> m;
    static uint64_t key(int64_t x, int64_t y, int64_t z) {
        return (uint64_t(x + (1 << 20)) & 0x1fffff) | ((uint64_t(y + (1 << 20)) & 0x1fffff) << 21) |
               ((uint64_t(z + (1 << 20)) & 0x1fffff) << 42);
    }
    void add(const double* p, uint32_t i) {
        m[key(int64_t(std::floor(p[0] / cell)), int64_t(std::floor(p[1] / cell)), int64_t(std::floor(p[2] / cell)))]
            .push_back(i);
    }
};

double density_radius(size_t n) { return std::cbrt(3.0 * 20.0 * double(n) / (4.0 * M_PI)); }

void rotation_from_quat(double w, double x, double y, double z, double R[9]) {
    R[0] = 1 - 2 * (y * y + z * z), R[1] = 2 * (x * y - w * z), R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z), R[4] = 1 - 2 * (x * x + z * z), R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y), R[7] = 2 * (y * z + w * x), R[8] = 1 - 2 * (x * x + y * y);
}

void random_rotation(Rng& rng, double R[9]) {
    for (;;) {
        double q[4] = {rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1), rng.uniform(-1, 1)};
        double n2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        if (n2 > 0.01 && n2 <= 1.0) {
            double n = std::sqrt(n2);
            rotation_from_quat(q[0] / n, q[1] / n, q[2] / n, q[3] / n, R);
            return;
        }
    }
}

void mat_mul(const double A[9], const double B[9], double C[9]) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}

// Places a rotated, translated copy of globule g (xyzr rows, centred at the
// origin) into out.
void place(const std::vector<double>& g, const double R[9], const double t[3], double* out) {
    size_t n = g.size() / 4;
    for (size_t i = 0; i < n; i++) {
        const double* p = &g[4 * i];
        for (int a = 0; a < 3; a++) out[4 * i + a] = R[3 * a] * p[0] + R[3 * a + 1] * p[1] + R[3 * a + 2] * p[2] + t[a];
        out[4 * i + 3] = p[3];
    }
}

}  // namespace

extern "C" {

// Globule of n atoms (x, y, z, r rows) in a ball of the given radius
// (<= 0: the density radius).  Returns the atoms placed (n unless the walk
// jams: then the ball grows by 1 % and the walk continues).
size_t smb_synth_globule(uint64_t seed, size_t n, double radius, double* out) {
    if (n == 0) return 0;
    Rng rng{seed};
    double R = radius > 0 ? radius : density_radius(n);
    std::vector<double> pos;
    std::vector<uint32_t> parent;
    Hash hash{2.8, {}};
    double p0[3];
    for (;;) {
        p0[0] = rng.uniform(-1, 1) * 0.25 * R, p0[1] = rng.uniform(-1, 1) * 0.25 * R, p0[2] = rng.uniform(-1, 1) * 0.25 * R;
        if (p0[0] * p0[0] + p0[1] * p0[1] + p0[2] * p0[2] <= R * R) break;
    }
    pos.insert(pos.end(), p0, p0 + 3);
    parent.push_back(UINT32_MAX);
    hash.add(p0, 0);
    size_t cur = 0;
    int fails = 0;
    size_t stalls = 0;
    while (pos.size() / 3 < n) {
        double u[3], p[3];
        rng.unit(u);
        for (int a = 0; a < 3; a++) p[a] = pos[3 * cur + a] + 1.5 * u[a];
        bool ok = p[0] * p[0] + p[1] * p[1] + p[2] * p[2] <= R * R;
        if (ok) {
            int64_t c[3] = {int64_t(std::floor(p[0] / 2.8)), int64_t(std::floor(p[1] / 2.8)), int64_t(std::floor(p[2] / 2.8))};
            for (int64_t dz = -1; dz <= 1 && ok; dz++)
                for (int64_t dy = -1; dy <= 1 && ok; dy++)
                    for (int64_t dx = -1; dx <= 1 && ok; dx++) {
                        auto it = hash.m.find(Hash::key(c[0] + dx, c[1] + dy, c[2] + dz));
                        if (it == hash.m.end()) continue;
                        for (uint32_t j : it->second) {
                            if (j == cur) continue;
                            double d2 = 0;
                            for (int a = 0; a < 3; a++) d2 += (p[a] - pos[3 * j + a]) * (p[a] - pos[3 * j + a]);
                            bool one_three = j == parent[cur] || parent[j] == cur;
                            double lim = one_three ? 2.2 : 2.8;
                            if (d2 < lim * lim) {
                                ok = false;
                                break;
                            }
                        }
                    }
        }
        if (ok) {
            uint32_t id = uint32_t(pos.size() / 3);
            pos.insert(pos.end(), p, p + 3);
            parent.push_back(uint32_t(cur));
            hash.add(p, id);
            cur = id;
            fails = 0;
        } else if (++fails >= 48) {
            cur = rng.below(pos.size() / 3);
            fails = 0;
            if (++stalls % 20000 == 0) R *= 1.01;
        }
    }
    size_t m = pos.size() / 3;
    for (size_t i = 0; i < m; i++) {
        double e = rng.uniform(0, 1);
        double r = e < 0.62 ? 1.70 : (e < 0.79 ? 1.55 : (e < 0.98 ? 1.52 : 1.80));
        out[4 * i] = pos[3 * i], out[4 * i + 1] = pos[3 * i + 1], out[4 * i + 2] = pos[3 * i + 2], out[4 * i + 3] = r;
    }
    return m;
}

// Ring assembly: copies of one n-atom globule on stacked 7-fold rings.
// rings x 7 copies; ring k at height z[k], radius rad[k], angular offset
// off[k] (radians); each copy gets its own seeded random orientation.
size_t smb_synth_rings(uint64_t seed, size_t n, double radius, int rings, const double* z, const double* rad,
                       const double* off, double* out) {
    std::vector<double> g(4 * n);
    size_t m = smb_synth_globule(seed, n, radius, g.data());
    g.resize(4 * m);
    double c[3] = {0, 0, 0};
    for (size_t i = 0; i < m; i++)
        for (int a = 0; a < 3; a++) c[a] += g[4 * i + a];
    for (int a = 0; a < 3; a++) c[a] /= double(m);
    for (size_t i = 0; i < m; i++)
        for (int a = 0; a < 3; a++) g[4 * i + a] -= c[a];
    Rng rng{seed ^ 0x5eed5eed5eed5eedULL};
    size_t k = 0;
    for (int r = 0; r < rings; r++)
        for (int j = 0; j < 7; j++) {
            double ang = off[r] + 2.0 * M_PI * double(j) / 7.0;
            double t[3] = {rad[r] * std::cos(ang), rad[r] * std::sin(ang), z[r]};
            double R[9];
            random_rotation(rng, R);
            place(g, R, t, out + 4 * m * k);
            k++;
        }
    return m * k;
}

// Icosahedral shell: 60 copies of one n-atom globule, the copy of rotation
// g_k of the icosahedral group I centred at g_k * (shell * d0) and oriented
// by g_k * R0 (d0 a fixed generic direction, R0 a seeded orientation).
size_t smb_synth_icosahedral(uint64_t seed, size_t n, double radius, double shell, double* out) {
    std::vector<double> g(4 * n);
    size_t m = smb_synth_globule(seed, n, radius, g.data());
    g.resize(4 * m);
    double c[3] = {0, 0, 0};
    for (size_t i = 0; i < m; i++)
        for (int a = 0; a < 3; a++) c[a] += g[4 * i + a];
    for (int a = 0; a < 3; a++) c[a] /= double(m);
    for (size_t i = 0; i < m; i++)
        for (int a = 0; a < 3; a++) g[4 * i + a] -= c[a];
    // Group closure from a 5-fold axis (0, 1, phi) and a 3-fold axis (1, 1, 1).
    const double phi = (1.0 + std::sqrt(5.0)) / 2.0;
    auto axis_rot = [](double x, double y, double zz, double ang, double R[9]) {
        double n = std::sqrt(x * x + y * y + zz * zz);
        double h = 0.5 * ang, s = std::sin(h) / n;
        rotation_from_quat(std::cos(h), x * s, y * s, zz * s, R);
    };
    double A[9], B[9];
    axis_rot(0, 1, phi, 2.0 * M_PI / 5.0, A);
    axis_rot(1, 1, 1, 2.0 * M_PI / 3.0, B);
    std::vector<std::array<double, 9>> group;
    std::array<double, 9> I = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    group.push_back(I);
    for (size_t q = 0; q < group.size() && group.size() < 60; q++)
        for (const double* G : {A, B}) {
            std::array<double, 9> C;
            mat_mul(G, group[q].data(), C.data());
            bool seen = false;
            for (auto& H : group) {
                double d = 0;
                for (int i = 0; i < 9; i++) d += std::fabs(H[i] - C[i]);
                if (d < 1e-6) {
                    seen = true;
                    break;
                }
            }
            if (!seen) group.push_back(C);
        }
    double d0[3] = {0.3, 0.5, 0.81};
    double dn = std::sqrt(d0[0] * d0[0] + d0[1] * d0[1] + d0[2] * d0[2]);
    Rng rng{seed ^ 0x1c05a4ed1c05a4edULL};
    double R0[9];
    random_rotation(rng, R0);
    for (size_t k = 0; k < group.size(); k++) {
        const double* G = group[k].data();
        double p[3] = {shell * d0[0] / dn, shell * d0[1] / dn, shell * d0[2] / dn};
        double t[3];
        for (int a = 0; a < 3; a++) t[a] = G[3 * a] * p[0] + G[3 * a + 1] * p[1] + G[3 * a + 2] * p[2];
        double R[9];
        mat_mul(G, R0, R);
        place(g, R, t, out + 4 * m * k);
    }
    return m * group.size();
}

size_t smb_synth_group_size(void) { return 60; }

}  // extern "C"
