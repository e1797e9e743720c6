// scene_io.cpp — host-only helpers behind the C ABI: the .sphs snapshot file
// format and the scene builders (lattice, seeded jitter/velocities, box-wall
// and triangle-mesh boundary sampling).
#include "scene_io.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>
#include <vector>

namespace wcsph_host {

// ---------------------------------------------------------------- .sphs v1 --
// Layout of Snapshot::Header (src/cuda/SPH/snapshot.cuh:22-27, 76 bytes):
//   char magic[4] = "SPHS"; u32 version = 1; char app_name[64]; u32 fluid_n;
// then float4 positions[fluid_n], float4 velocities[fluid_n] (little endian).
struct SnapshotHeader {
    char magic[4];
    uint32_t version;
    char app_name[kAppNameMax];
    uint32_t fluid_n;
};
static_assert(sizeof(SnapshotHeader) == 76, "snapshot header must be 76 bytes");
static const char kMagic[4] = {'S', 'P', 'H', 'S'};

Status snapshot_read_header(const std::string& path, std::string* app_name, uint32_t* fluid_n,
                            std::ifstream* keep_open) {
    std::ifstream local;
    std::ifstream& f = keep_open ? *keep_open : local;
    f.open(path, std::ios::binary);
    if (!f) return {WCSPH_ERR_IO, "Snapshot::load: cannot open " + path};
    SnapshotHeader h{};
    f.read(reinterpret_cast<char*>(&h), sizeof(h));
    if (!f) return {WCSPH_ERR_SNAPSHOT_TRUNCATED, "Snapshot::load: header read failed for " + path};
    if (std::memcmp(h.magic, kMagic, 4) != 0) return {WCSPH_ERR_SNAPSHOT_MAGIC, "Snapshot::load: bad magic in " + path};
    if (h.version != kSnapshotVersion)
        return {WCSPH_ERR_SNAPSHOT_VERSION, "Snapshot::load: version mismatch (file=" + std::to_string(h.version) +
                                                ", expected=" + std::to_string(kSnapshotVersion) + ")"};
    h.app_name[kAppNameMax - 1] = '\0';  // guard against corrupt files (snapshot.cu:73)
    if (app_name) *app_name = h.app_name;
    if (fluid_n) *fluid_n = h.fluid_n;
    return {};
}

// Snapshot::load (snapshot.cu:54-106): same checks in the same order.
Status snapshot_read(const std::string& path, const std::string& app_name, uint32_t fluid_n, float* pos,
                     float* vel) {
    std::ifstream f;
    std::string name;
    uint32_t n = 0;
    Status s = snapshot_read_header(path, &name, &n, &f);
    if (!s.ok()) return s;
    if (app_name != name)
        return {WCSPH_ERR_SNAPSHOT_APP_NAME,
                "Snapshot::load: app_name mismatch (file='" + name + "', expected='" + app_name + "')"};
    if (n != fluid_n)
        return {WCSPH_ERR_SNAPSHOT_COUNT, "Snapshot::load: fluid count mismatch (file=" + std::to_string(n) +
                                              ", expected=" + std::to_string(fluid_n) + ")"};
    std::vector<float> p(4ull * n), v(4ull * n);
    f.read(reinterpret_cast<char*>(p.data()), sizeof(float) * 4 * n);
    f.read(reinterpret_cast<char*>(v.data()), sizeof(float) * 4 * n);
    if (!f) return {WCSPH_ERR_SNAPSHOT_TRUNCATED, "Snapshot::load: body read failed for " + path};
    if (pos) std::memcpy(pos, p.data(), sizeof(float) * 4 * n);
    if (vel) std::memcpy(vel, v.data(), sizeof(float) * 4 * n);
    return {};
}

// Snapshot::save (snapshot.cu:10-52).
Status snapshot_write(const std::string& path, const std::string& app_name, uint32_t fluid_n, const float* pos,
                      const float* vel) {
    if (app_name.size() >= kAppNameMax)
        return {WCSPH_ERR_SNAPSHOT_APP_NAME,
                "Snapshot::save: app_name too long (max " + std::to_string(kAppNameMax - 1) + " chars)"};
    SnapshotHeader h{};
    std::memcpy(h.magic, kMagic, 4);
    h.version = kSnapshotVersion;
    h.fluid_n = fluid_n;
    std::memcpy(h.app_name, app_name.data(), app_name.size());
    std::ofstream f(path, std::ios::binary);
    if (!f) return {WCSPH_ERR_IO, "Snapshot::save: cannot open " + path};
    f.write(reinterpret_cast<const char*>(&h), sizeof(h));
    f.write(reinterpret_cast<const char*>(pos), sizeof(float) * 4 * fluid_n);
    f.write(reinterpret_cast<const char*>(vel), sizeof(float) * 4 * fluid_n);
    if (!f) return {WCSPH_ERR_IO, "Snapshot::save: write failed for " + path};
    return {};
}

// --------------------------------------------------------------- RNG --------
// splitmix64 stream; portable and seedable (std distributions are not
// reproducible across standard libraries).
struct SplitMix64 {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform01() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }  // [0,1)
};

// FluidSimulator::init_positions (fluid_simulator.cpp:24-54): x-outer, y,
// z-inner; start = origin - (dims-1)*r; step = 2r; w = 1. Optional seeded
// jitter U(-jitter, jitter) per axis, drawn in lattice order x, y, z.
void make_lattice(const float origin[3], const uint32_t dims[3], float r, float jitter, uint64_t seed, float* out) {
    const float spacing = 2.f * r;
    const float sx = origin[0] - static_cast<float>(dims[0] - 1) * r;
    const float sy = origin[1] - static_cast<float>(dims[1] - 1) * r;
    const float sz = origin[2] - static_cast<float>(dims[2] - 1) * r;
    SplitMix64 rng{seed};
    size_t i = 0;
    for (uint32_t x = 0; x < dims[0]; ++x)
        for (uint32_t y = 0; y < dims[1]; ++y)
            for (uint32_t z = 0; z < dims[2]; ++z) {
                float px = sx + static_cast<float>(x) * spacing;
                float py = sy + static_cast<float>(y) * spacing;
                float pz = sz + static_cast<float>(z) * spacing;
                if (jitter > 0.f) {
                    px += static_cast<float>((2.0 * rng.uniform01() - 1.0) * jitter);
                    py += static_cast<float>((2.0 * rng.uniform01() - 1.0) * jitter);
                    pz += static_cast<float>((2.0 * rng.uniform01() - 1.0) * jitter);
                }
                out[4 * i + 0] = px;
                out[4 * i + 1] = py;
                out[4 * i + 2] = pz;
                out[4 * i + 3] = 1.f;
                ++i;
            }
}

// N(0, sigma) per component by the Box-Muller transform.
void make_velocities(uint32_t n, float sigma, uint64_t seed, float* out) {
    SplitMix64 rng{seed ^ 0xA5A5A5A5A5A5A5A5ull};
    auto normal = [&]() {
        double u1 = rng.uniform01();
        if (u1 < 1e-300) u1 = 1e-300;
        const double u2 = rng.uniform01();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    for (uint32_t i = 0; i < n; ++i) {
        out[4 * i + 0] = static_cast<float>(sigma * normal());
        out[4 * i + 1] = static_cast<float>(sigma * normal());
        out[4 * i + 2] = static_cast<float>(sigma * normal());
        out[4 * i + 3] = 0.f;
    }
}

// Single-layer walls: lattice points min + (i,j,k)*spacing of the box that lie
// on one of its six faces.
uint32_t sample_box_walls(const float mn[3], const float mx[3], float spacing, float* out) {
    uint32_t cnt[3];
    for (int d = 0; d < 3; ++d)
        cnt[d] = static_cast<uint32_t>(std::lround(static_cast<double>(mx[d] - mn[d]) / spacing));
    uint32_t k = 0;
    for (uint32_t i = 0; i <= cnt[0]; ++i)
        for (uint32_t j = 0; j <= cnt[1]; ++j)
            for (uint32_t l = 0; l <= cnt[2]; ++l) {
                const bool surface = i == 0 || i == cnt[0] || j == 0 || j == cnt[1] || l == 0 || l == cnt[2];
                if (!surface) continue;
                if (out) {
                    out[4 * k + 0] = mn[0] + static_cast<float>(i) * spacing;
                    out[4 * k + 1] = mn[1] + static_cast<float>(j) * spacing;
                    out[4 * k + 2] = mn[2] + static_cast<float>(l) * spacing;
                    out[4 * k + 3] = 1.f;
                }
                ++k;
            }
    return k;
}

// ------------------------------------------------ triangle-box overlap (SAT) --
// Separating-axis test of a triangle against an axis-aligned box (Akenine-
// Moeller, "Fast 3D Triangle-Box Overlap Testing", 2001): 3 box normals, the
// triangle normal and the 9 edge cross products.
namespace {
using V3 = std::array<double, 3>;
V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
V3 cross(const V3& a, const V3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
double dotv(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

bool tri_box_overlap(const V3& c, double hs, const V3& a0, const V3& a1, const V3& a2) {
    const V3 v0 = sub(a0, c), v1 = sub(a1, c), v2 = sub(a2, c);
    const V3 e[3] = {sub(v1, v0), sub(v2, v1), sub(v0, v2)};
    // 9 edge axes
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            V3 unit{0, 0, 0};
            unit[k] = 1;
            const V3 ax = cross(unit, e[i]);
            const double p0 = dotv(ax, v0), p1 = dotv(ax, v1), p2 = dotv(ax, v2);
            const double r = hs * (std::fabs(ax[0]) + std::fabs(ax[1]) + std::fabs(ax[2]));
            if (std::min({p0, p1, p2}) > r || std::max({p0, p1, p2}) < -r) return false;
        }
    // box face normals
    for (int k = 0; k < 3; ++k) {
        if (std::min({v0[k], v1[k], v2[k]}) > hs || std::max({v0[k], v1[k], v2[k]}) < -hs) return false;
    }
    // triangle plane
    const V3 nrm = cross(e[0], e[1]);
    const double d = dotv(nrm, v0);
    const double r = hs * (std::fabs(nrm[0]) + std::fabs(nrm[1]) + std::fabs(nrm[2]));
    return std::fabs(d) <= r;
}
}  // namespace

// Surface voxelisation with the semantics of a voxel grid built from a
// triangle mesh: grid origin = mesh min bound - voxel/2, a voxel is kept when
// any triangle overlaps its cube, the particle sits at the voxel centre
// (the role Open3D's VoxelGrid::CreateFromTriangleMesh plays in
// src/simulation/SPH/boundary.cpp:27-32). Output is in (i, j, k) order.
uint32_t sample_triangles(const float* verts, uint32_t ntri, float voxel, float* out) {
    if (ntri == 0) return 0;
    V3 mn{1e300, 1e300, 1e300};
    for (uint32_t t = 0; t < 3 * ntri; ++t)
        for (int d = 0; d < 3; ++d) mn[d] = std::min(mn[d], static_cast<double>(verts[3 * t + d]));
    const double vs = voxel;
    const V3 origin{mn[0] - 0.5 * vs, mn[1] - 0.5 * vs, mn[2] - 0.5 * vs};
    std::vector<std::array<int64_t, 3>> cells;
    for (uint32_t t = 0; t < ntri; ++t) {
        V3 p[3];
        for (int k = 0; k < 3; ++k)
            for (int d = 0; d < 3; ++d) p[k][d] = verts[9 * t + 3 * k + d];
        int64_t lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            const double a = std::min({p[0][d], p[1][d], p[2][d]}), b = std::max({p[0][d], p[1][d], p[2][d]});
            lo[d] = static_cast<int64_t>(std::floor((a - origin[d]) / vs)) - 1;
            hi[d] = static_cast<int64_t>(std::floor((b - origin[d]) / vs)) + 1;
        }
        for (int64_t i = lo[0]; i <= hi[0]; ++i)
            for (int64_t j = lo[1]; j <= hi[1]; ++j)
                for (int64_t k = lo[2]; k <= hi[2]; ++k) {
                    const V3 c{origin[0] + (i + 0.5) * vs, origin[1] + (j + 0.5) * vs, origin[2] + (k + 0.5) * vs};
                    if (tri_box_overlap(c, 0.5 * vs, p[0], p[1], p[2])) cells.push_back({i, j, k});
                }
    }
    std::sort(cells.begin(), cells.end());
    cells.erase(std::unique(cells.begin(), cells.end()), cells.end());
    if (out) {
        for (size_t q = 0; q < cells.size(); ++q) {
            for (int d = 0; d < 3; ++d)
                out[4 * q + d] = static_cast<float>(origin[d] + (static_cast<double>(cells[q][d]) + 0.5) * vs);
            out[4 * q + 3] = 1.f;
        }
    }
    return static_cast<uint32_t>(cells.size());
}

// Icosphere: icosahedron subdivided `level` times (each triangle split into
// four, midpoints projected to the sphere): 20 * 4^level triangles.
std::vector<float> icosphere_triangles(const float center[3], float radius, int level) {
    const double t = (1.0 + std::sqrt(5.0)) / 2.0;
    std::vector<V3> v = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                         {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    for (auto& p : v) {
        const double l = std::sqrt(dotv(p, p));
        for (auto& c : p) c /= l;
    }
    std::vector<std::array<int, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
                                         {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                         {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
                                         {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    for (int s = 0; s < level; ++s) {
        std::vector<std::array<int, 3>> nf;
        nf.reserve(f.size() * 4);
        std::vector<std::pair<std::pair<int, int>, int>> cache;
        auto mid = [&](int a, int b) {
            const auto key = std::make_pair(std::min(a, b), std::max(a, b));
            for (const auto& e : cache)
                if (e.first == key) return e.second;
            V3 m{(v[a][0] + v[b][0]) / 2, (v[a][1] + v[b][1]) / 2, (v[a][2] + v[b][2]) / 2};
            const double l = std::sqrt(dotv(m, m));
            for (auto& c : m) c /= l;
            v.push_back(m);
            cache.push_back({key, static_cast<int>(v.size()) - 1});
            return static_cast<int>(v.size()) - 1;
        };
        for (const auto& tr : f) {
            const int a = mid(tr[0], tr[1]), b = mid(tr[1], tr[2]), c = mid(tr[2], tr[0]);
            nf.push_back({tr[0], a, c});
            nf.push_back({tr[1], b, a});
            nf.push_back({tr[2], c, b});
            nf.push_back({a, b, c});
        }
        f.swap(nf);
    }
    std::vector<float> out;
    out.reserve(f.size() * 9);
    for (const auto& tr : f)
        for (int k = 0; k < 3; ++k)
            for (int d = 0; d < 3; ++d) out.push_back(static_cast<float>(center[d] + radius * v[tr[k]][d]));
    return out;
}

// ----------------------------------------------------------- .obj meshes --
// Geometry::from_file (src/render/geometry.cpp:50-140, tinyobjloader) and
// Geometry::load_triangles (geometry.cpp:185-207): vertex positions of the
// first shape's faces in file order, faces of more than three vertices
// rejected with the reference's message, optional normalisation into a unit
// box around the origin (with the reference's starting maximum of
// numeric_limits<float>::min()), then model * (x, y, z, 1). A new shape
// starts at an `o` or `g` line that follows faces; later shapes are ignored.
// Face vertices may be written v, v/vt, v//vn or v/vt/vn, with negative
// indices counting back from the last vertex.
std::vector<float> load_obj_triangles(const std::string& path, bool normalize, const float* model, Status* status) {
    auto fail = [&](int code, const std::string& msg) {
        if (status) *status = Status{code, msg};
        return std::vector<float>{};
    };
    std::ifstream in(path);
    if (!in) return fail(WCSPH_ERR_IO, "failed to load " + path);
    std::vector<float> v;    // x, y, z per vertex
    std::vector<float> out;  // 9 floats per triangle
    std::string line;
    bool faces_seen = false;
    size_t face = 0;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string tag;
        if (!(ls >> tag)) continue;
        if (tag == "v") {
            float x = 0.f, y = 0.f, z = 0.f;
            if (!(ls >> x >> y >> z)) return fail(WCSPH_ERR_IO, "failed to load " + path + ": bad vertex line");
            v.insert(v.end(), {x, y, z});
        } else if (tag == "o" || tag == "g") {
            if (faces_seen) break;   // the first shape ends here
        } else if (tag == "f") {
            std::vector<long> idx;
            std::string tok;
            while (ls >> tok) {
                const long k = std::strtol(tok.c_str(), nullptr, 10);   // vertex index before any '/'
                const long nv = static_cast<long>(v.size() / 3);
                const long i = k > 0 ? k - 1 : nv + k;
                if (k == 0 || i < 0 || i >= nv)
                    return fail(WCSPH_ERR_IO, "failed to load " + path + ": face " + std::to_string(face) +
                                                  " refers to a missing vertex");
                idx.push_back(i);
            }
            if (idx.size() > 3)
                return fail(WCSPH_ERR_INVALID_ARGUMENT, "In " + path + ": face " + std::to_string(face) + " has " +
                                                            std::to_string(idx.size()) + " vertices (not a triangle)");
            if (idx.size() == 3)
                for (long i : idx) out.insert(out.end(), {v[3 * i], v[3 * i + 1], v[3 * i + 2]});
            faces_seen = true;
            ++face;
        }
    }
    if (normalize && !out.empty()) {
        float mn[3], mx[3];
        for (int d = 0; d < 3; ++d) {
            mn[d] = std::numeric_limits<float>::max();
            mx[d] = std::numeric_limits<float>::min();
        }
        for (size_t k = 0; k < out.size(); k += 3)
            for (int d = 0; d < 3; ++d) {
                mn[d] = std::min(mn[d], out[k + d]);
                mx[d] = std::max(mx[d], out[k + d]);
            }
        float c[3], diff[3];
        for (int d = 0; d < 3; ++d) {
            c[d] = (mn[d] + mx[d]) * 0.5f;
            diff[d] = mx[d] - mn[d];
        }
        const float md = std::max(std::max(diff[0], diff[1]), diff[2]);
        for (size_t k = 0; k < out.size(); k += 3)
            for (int d = 0; d < 3; ++d) out[k + d] = (out[k + d] - c[d]) / md;
    }
    if (model) {
        for (size_t k = 0; k < out.size(); k += 3) {
            const float x = out[k], y = out[k + 1], z = out[k + 2];
            for (int d = 0; d < 3; ++d)
                out[k + d] = model[d] * x + model[4 + d] * y + model[8 + d] * z + model[12 + d];
        }
    }
    if (status) *status = Status{};
    return out;
}

}  // namespace wcsph_host
