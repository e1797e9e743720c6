// presets.cpp — named scenes: the reference's headless apps that need no
// missing asset, and the benchmark workloads. One definition shared by the
// CLI, the Python binding, the tests and bench.py.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wcsph.h"
#include "scene_io.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uni() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// glm-style rotation about z, column-major, plus inverse (transpose).
void rotz_box(float angle, const float mn[3], const float mx[3], wcsph_box* b) {
    wcsph_identity_box(mn, mx, b);
    const float c = std::cos(angle), s = std::sin(angle);
    // column 0 = (c, s, 0, 0), column 1 = (-s, c, 0, 0)
    b->model[0] = c; b->model[1] = s; b->model[4] = -s; b->model[5] = c;
    b->model_inv[0] = c; b->model_inv[1] = -s; b->model_inv[4] = s; b->model_inv[5] = c;
}

struct Built {
    wcsph_preset_info info{};
    std::vector<float> pos, vel, bpos;
};

// Lattice whose min-corner particle centre sits at `corner`
// (FluidSimulator::init_positions takes the lattice centre as origin).
std::vector<float> lattice_at_corner(const float corner[3], const uint32_t dims[3], float r, float jitter,
                                     uint64_t seed) {
    const float origin[3] = {corner[0] + static_cast<float>(dims[0] - 1) * r,
                             corner[1] + static_cast<float>(dims[1] - 1) * r,
                             corner[2] + static_cast<float>(dims[2] - 1) * r};
    std::vector<float> pos(4ull * dims[0] * dims[1] * dims[2]);
    wcsph_host::make_lattice(origin, dims, r, jitter, seed, pos.data());
    return pos;
}

void base_params(wcsph_params* p, float r) {
    wcsph_default_params(p);
    p->particle_radius = r;
}

// Tait stiffness 1000 in the textbook normalisation of the spiky gradient,
// -45/(pi h^6) (h - r)^2, expressed in the reference's normalisation
// -45/(pi h^9) (1 - q)^2 / (h r) (kernel.cuh:43-51), which is h^-6 times
// stronger: k_ref = 1000 * h^6. A literal k = 1000 with the reference's
// kernel accelerates particles to ~1e8 m/s in the first step.
float textbook_stiffness(float k, float r) {
    return static_cast<float>(static_cast<double>(k) * std::pow(4.0 * static_cast<double>(r), 6.0));
}

// Benchmark physics shared by the dam-break family: rho0 1000, Tait k 1000
// (textbook normalisation), gamma 7, viscosity 0.01, gravity -9.81 y, fixed dt.
void dam_break_physics(wcsph_params* p, float r, float dt) {
    base_params(p, r);
    p->stiffness = textbook_stiffness(1000.f, r);
    p->viscosity = 0.01f;
    p->cfl_factor = 0.f;
    p->max_time_step = dt;
    p->min_time_step = std::min(1e-5f, dt);
}

bool build(const std::string& name, uint64_t seed, Built& out) {
    wcsph_preset_info& I = out.info;
    std::memset(&I, 0, sizeof(I));
    if (name == "dam_break" || name == "rollout_block") {
        // 32^3 (or 32x32x16) lattice, r = 0.01, corner at the origin, jitter
        // +-0.1 r, tank 1.0 x 0.6 x 0.6 walled by boundary particles on a 2r grid.
        const float r = 0.01f;
        dam_break_physics(&I.params, r, 1e-3f);
        const uint32_t dims[3] = {32, 32, name == "dam_break" ? 32u : 16u};
        const float corner[3] = {r, r, r};
        out.pos = lattice_at_corner(corner, dims, r, 0.1f * r, seed);
        const float mn[3] = {0.f, 0.f, 0.f}, mx[3] = {1.0f, 0.6f, 0.6f};
        wcsph_identity_box(mn, mx, &I.box);
        const uint32_t nb = wcsph_host::sample_box_walls(mn, mx, 2 * r, nullptr);
        out.bpos.resize(4ull * nb);
        wcsph_host::sample_box_walls(mn, mx, 2 * r, out.bpos.data());
        I.delta = 1e-3f;
        if (name == "dam_break") {
            I.steps = 1000;
        } else {
            I.steps = 200;
            I.params.surface_tension = 0.f;  // the adjoint covers no surface tension
        }
    } else if (name == "mesh_obstacle") {
        // 64x96x64 block (r = 0.005) over a level-4 icosphere (R = 0.15) centred
        // in a 1 m cube; walls and sphere sampled at 2r; CFL 0.4, dt cap 1e-3, 2 s.
        const float r = 0.005f;
        dam_break_physics(&I.params, r, 1e-3f);
        I.params.cfl_factor = 0.4f;
        const uint32_t dims[3] = {64, 96, 64};
        const float corner[3] = {(1.f - 0.64f) / 2 + r, 1.f - 0.96f + r - 0.005f, (1.f - 0.64f) / 2 + r};
        out.pos = lattice_at_corner(corner, dims, r, 0.1f * r, seed);
        const float mn[3] = {0.f, 0.f, 0.f}, mx[3] = {1.f, 1.f, 1.f};
        wcsph_identity_box(mn, mx, &I.box);
        const uint32_t nw = wcsph_host::sample_box_walls(mn, mx, 2 * r, nullptr);
        out.bpos.resize(4ull * nw);
        wcsph_host::sample_box_walls(mn, mx, 2 * r, out.bpos.data());
        const float c[3] = {0.5f, 0.5f, 0.5f};
        const std::vector<float> tris = wcsph_host::icosphere_triangles(c, 0.15f, 4);
        const uint32_t ns = wcsph_host::sample_triangles(tris.data(), static_cast<uint32_t>(tris.size() / 9), 2 * r,
                                                         nullptr);
        std::vector<float> sp(4ull * ns);
        wcsph_host::sample_triangles(tris.data(), static_cast<uint32_t>(tris.size() / 9), 2 * r, sp.data());
        out.bpos.insert(out.bpos.end(), sp.begin(), sp.end());
        I.delta = 1e-3f;
        I.sim_time = 2.f;
    } else if (name == "large_tilting") {
        // 1,048,576 particles (128 x 128 x 64 lattice: a 128^3 lattice would
        // hold 2,097,152), r = 0.004, jitter +-0.2 r, velocities N(0, 0.1) per
        // component, box 2 x 1 x 1 tilting 0 -> 15 deg about z over 1 s, fixed
        // dt 5e-4, 2000 steps, no boundary particles.
        const float r = 0.004f;
        dam_break_physics(&I.params, r, 5e-4f);
        const uint32_t dims[3] = {128, 128, 64};
        const float corner[3] = {-1.f + r, -0.5f + r, -0.5f + r};
        out.pos = lattice_at_corner(corner, dims, r, 0.2f * r, seed);
        out.vel.resize(out.pos.size());
        wcsph_host::make_velocities(dims[0] * dims[1] * dims[2], 0.1f, seed + 1, out.vel.data());
        const float mn[3] = {-1.f, -0.5f, -0.5f}, mx[3] = {1.f, 0.5f, 0.5f};
        wcsph_identity_box(mn, mx, &I.box);
        I.delta = 5e-4f;
        I.steps = 2000;
        I.moving_box = 1;
    } else if (name == "surface_tension") {
        // app/surface_tension/application.cu:10-25: box half 0.8, 30^3 lattice
        // centred at the origin, external force (0, 9.81, 0), reference constants.
        wcsph_default_params(&I.params);
        I.params.external_force = WCSPH_FORCE_CONSTANT;
        I.params.external_force_param[1] = 9.81f;
        const uint32_t dims[3] = {30, 30, 30};
        const float origin[3] = {0.f, 0.f, 0.f};
        out.pos.resize(4ull * 27000);
        wcsph_host::make_lattice(origin, dims, I.params.particle_radius, 0.f, 0, out.pos.data());
        const float mn[3] = {-0.8f, -0.8f, -0.8f}, mx[3] = {0.8f, 0.8f, 0.8f};
        wcsph_identity_box(mn, mx, &I.box);
        I.delta = 0.01f;
    } else if (name == "tilting_box") {
        // app/tilting_box/application.cu:10-46: box half (2.3, 0.7, 0.6), 30^3
        // lattice at the origin, model = rotate_z(sin(t/5)/5) with
        // t += min(delta, 1/30) per update.
        wcsph_default_params(&I.params);
        const uint32_t dims[3] = {30, 30, 30};
        const float origin[3] = {0.f, 0.f, 0.f};
        out.pos.resize(4ull * 27000);
        wcsph_host::make_lattice(origin, dims, I.params.particle_radius, 0.f, 0, out.pos.data());
        const float mn[3] = {-2.3f, -0.7f, -0.6f}, mx[3] = {2.3f, 0.7f, 0.6f};
        wcsph_identity_box(mn, mx, &I.box);
        I.delta = 0.01f;
        I.moving_box = 1;
    } else {
        return false;
    }
    I.fluid_n = static_cast<uint32_t>(out.pos.size() / 4);
    I.boundary_n = static_cast<uint32_t>(out.bpos.size() / 4);
    return true;
}

void emit(const Built& b, wcsph_preset_info* info, float* pos, float* vel, float* bpos) {
    *info = b.info;
    if (pos) std::memcpy(pos, b.pos.data(), sizeof(float) * b.pos.size());
    if (vel) {
        if (b.vel.empty()) std::memset(vel, 0, sizeof(float) * b.pos.size());
        else std::memcpy(vel, b.vel.data(), sizeof(float) * b.vel.size());
    }
    if (bpos && !b.bpos.empty()) std::memcpy(bpos, b.bpos.data(), sizeof(float) * b.bpos.size());
}

}  // namespace

extern "C" {

int wcsph_preset(const char* name, uint64_t seed, wcsph_preset_info* info, float* pos, float* vel, float* bpos) {
    if (!name || !info) return WCSPH_ERR_INVALID_ARGUMENT;
    Built b;
    if (!build(name, seed, b)) return WCSPH_ERR_NOT_SUPPORTED;
    emit(b, info, pos, vel, bpos);
    return WCSPH_OK;
}

int wcsph_preset_box(const char* name, int64_t updates, float delta, wcsph_box* out) {
    if (!name || !out) return WCSPH_ERR_INVALID_ARGUMENT;
    const std::string n = name;
    if (n == "tilting_box") {
        // TiltingBoxApp::update_objects: update_time += min(delta, 1/30) before
        // each update; angle = sin(update_time / 5) / 5.
        float t = 0.f;
        for (int64_t k = 0; k < updates; ++k) t += std::min(delta, 1.f / 30.f);
        const float mn[3] = {-2.3f, -0.7f, -0.6f}, mx[3] = {2.3f, 0.7f, 0.6f};
        rotz_box(std::sin(t / 5.f) / 5.f, mn, mx, out);
        return WCSPH_OK;
    }
    if (n == "large_tilting") {
        const double t = static_cast<double>(updates) * delta;
        const double a = (15.0 * kPi / 180.0) * std::min(t / 1.0, 1.0);
        const float mn[3] = {-1.f, -0.5f, -0.5f}, mx[3] = {1.f, 0.5f, 0.5f};
        rotz_box(static_cast<float>(a), mn, mx, out);
        return WCSPH_OK;
    }
    Built b;
    if (!build(n, 0, b)) return WCSPH_ERR_NOT_SUPPORTED;
    *out = b.info.box;
    return WCSPH_OK;
}

int wcsph_preset_ensemble(uint64_t seed, uint32_t k, wcsph_preset_info* info, float* pos, float* vel, float* bpos) {
    if (!info) return WCSPH_ERR_INVALID_ARGUMENT;
    Rng rng{seed * 0x100000001B3ull + k * 0x9E3779B97F4A7C15ull + 17};
    const float r = 0.01f;
    Built b;
    wcsph_preset_info& I = b.info;
    std::memset(&I, 0, sizeof(I));
    dam_break_physics(&I.params, r, 1e-3f);
    const double ntarget = std::exp(std::log(2048.0) + rng.uni() * (std::log(65536.0) - std::log(2048.0)));
    double ext[3];
    for (double& e : ext) e = 0.3 + 0.7 * rng.uni();
    // keep the fluid block at most 40% of the box volume (scale the box up)
    const double fluid_vol = ntarget * std::pow(2.0 * r, 3.0);
    const double box_vol = ext[0] * ext[1] * ext[2];
    if (fluid_vol > 0.4 * box_vol) {
        const double s = std::cbrt(fluid_vol / (0.4 * box_vol));
        for (double& e : ext) e *= s;
    }
    const double tilt = (20.0 * kPi / 180.0) * rng.uni();
    I.params.gravity[0] = static_cast<float>(9.81 * std::sin(tilt));
    I.params.gravity[1] = static_cast<float>(-9.81 * std::cos(tilt));
    I.params.gravity[2] = 0.f;
    I.params.viscosity = static_cast<float>(0.005 + 0.045 * rng.uni());
    // dam-break block: half the box width in x, full depth in z, stacked in y
    uint32_t dims[3];
    dims[0] = std::max<uint32_t>(2, static_cast<uint32_t>(0.5 * ext[0] / (2 * r)));
    dims[2] = std::max<uint32_t>(2, static_cast<uint32_t>(ext[2] / (2 * r)) - 1);
    dims[1] = std::max<uint32_t>(2, static_cast<uint32_t>(std::ceil(ntarget / (dims[0] * dims[2]))));
    const float corner[3] = {r, r, r};
    b.pos = lattice_at_corner(corner, dims, r, 0.1f * r, seed + k);
    const float mn[3] = {0.f, 0.f, 0.f};
    const float mx[3] = {static_cast<float>(ext[0]), static_cast<float>(ext[1]), static_cast<float>(ext[2])};
    wcsph_identity_box(mn, mx, &I.box);
    const uint32_t nb = wcsph_host::sample_box_walls(mn, mx, 2 * r, nullptr);
    b.bpos.resize(4ull * nb);
    wcsph_host::sample_box_walls(mn, mx, 2 * r, b.bpos.data());
    I.delta = 1e-3f;
    I.steps = 500;
    I.fluid_n = static_cast<uint32_t>(b.pos.size() / 4);
    I.boundary_n = nb;
    emit(b, info, pos, vel, bpos);
    return WCSPH_OK;
}

}  // extern "C"
