// capi.cu — extern "C" entry points of include/wcsph.h. Every call catches
// internal exceptions and turns them into a status code + last-error text.
#include <cstring>
#include <string>

#include "batch.cuh"
#include "scene_io.h"
#include "simulator.cuh"
#include "static_sort.cuh"

struct wcsph_ctx {
    std::unique_ptr<wcsph::CUDASPHSimulator> sim;
    std::string last_error;
};

namespace {
thread_local std::string g_last_error;

template <class F>
int guarded(wcsph_ctx* ctx, F&& f) {
    try {
        f();
        return WCSPH_OK;
    } catch (const wcsph::Error& e) {
        (ctx ? ctx->last_error : g_last_error) = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        (ctx ? ctx->last_error : g_last_error) = "host allocation failed";
        return WCSPH_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        (ctx ? ctx->last_error : g_last_error) = e.what();
        return WCSPH_ERR_CUDA;
    }
}

int host_status(wcsph_ctx* ctx, const wcsph_host::Status& s) {
    if (!s.ok()) (ctx ? ctx->last_error : g_last_error) = s.message;
    return s.code;
}

#define CHECK_CTX(c) \
    do { if (!(c) || !(c)->sim) return WCSPH_ERR_INVALID_ARGUMENT; } while (0)
}  // namespace

extern "C" {

int wcsph_abi_version(void) { return WCSPH_ABI_VERSION; }

void wcsph_default_params(wcsph_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    // reference constants: common.cuh:18-23, compute_rho_p.cu:10-12,
    // compute_non_pressure_accel.cu:14-16, update_positions.cu:10-12, sph.cuh:19-32
    p->particle_radius = 0.02f;
    p->rest_density = 1000.f;
    p->stiffness = 0.1f;
    p->exponent = 7.f;
    p->max_density_ratio = 1.5f;
    p->viscosity = 0.001f;
    p->surface_tension = 0.13f;
    p->gravity[0] = 0.f; p->gravity[1] = -9.81f; p->gravity[2] = 0.f;
    p->cfl_factor = 0.4f;
    p->max_time_step = 0.0005f;
    p->min_time_step = 0.00001f;
    p->non_pressure_max_time_step = 0.015f;
    p->collision_buffer_mult = 0.75f;
    p->elasticity = 0.5f;
    p->cell_size_mult = 1.f;
    p->table_size_mult = 4;
    p->external_force = WCSPH_FORCE_NONE;
}

void wcsph_identity_box(const float mn[3], const float mx[3], wcsph_box* out) {
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    for (int d = 0; d < 3; ++d) { out->min[d] = mn[d]; out->max[d] = mx[d]; }
    for (int c = 0; c < 4; ++c) { out->model[5 * c] = 1.f; out->model_inv[5 * c] = 1.f; }
}

const char* wcsph_status_string(int s) {
    switch (s) {
    case WCSPH_OK: return "ok";
    case WCSPH_ERR_INVALID_ARGUMENT: return "invalid argument";
    case WCSPH_ERR_CUDA: return "CUDA error";
    case WCSPH_ERR_OUT_OF_MEMORY: return "out of memory";
    case WCSPH_ERR_IO: return "I/O error";
    case WCSPH_ERR_SNAPSHOT_MAGIC: return "snapshot: bad magic";
    case WCSPH_ERR_SNAPSHOT_VERSION: return "snapshot: version mismatch";
    case WCSPH_ERR_SNAPSHOT_APP_NAME: return "snapshot: app_name mismatch";
    case WCSPH_ERR_SNAPSHOT_COUNT: return "snapshot: fluid count mismatch";
    case WCSPH_ERR_SNAPSHOT_TRUNCATED: return "snapshot: truncated file";
    case WCSPH_ERR_HASH_FULL: return "spatial hash full";
    case WCSPH_ERR_NEIGHBOR_OVERFLOW: return "neighbour capacity exceeded";
    case WCSPH_ERR_DEVICE_TIMEOUT: return "device wait timed out";
    case WCSPH_ERR_NO_DEVICE: return "no CUDA device";
    case WCSPH_ERR_CONFIG: return "bad tuning configuration";
    case WCSPH_ERR_NOT_SUPPORTED: return "not supported";
    case WCSPH_ERR_STATE: return "invalid state";
    case WCSPH_ERR_BOUNDS: return "device index out of bounds (bounds-checked build)";
    default: return "unknown status";
    }
}

int wcsph_create(const wcsph_params* params, const wcsph_scene* scene, int device, wcsph_ctx** out) {
    if (!params || !scene || !out) return WCSPH_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto ctx = std::make_unique<wcsph_ctx>();
    const int s = guarded(nullptr, [&] { ctx->sim = std::make_unique<wcsph::CUDASPHSimulator>(*params, *scene, device); });
    if (s == WCSPH_OK) *out = ctx.release();
    return s;
}

int wcsph_destroy(wcsph_ctx* ctx) {
    delete ctx;
    return WCSPH_OK;
}

const char* wcsph_last_error(const wcsph_ctx* ctx) { return ctx ? ctx->last_error.c_str() : g_last_error.c_str(); }

int wcsph_step(wcsph_ctx* ctx, float delta) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->update(delta); });
}

int wcsph_step_n(wcsph_ctx* ctx, int n, float delta) {
    CHECK_CTX(ctx);
    if (n < 0) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { ctx->sim->step_n(n, delta); });
}

int wcsph_synchronize(wcsph_ctx* ctx) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->synchronize(); });
}

int wcsph_reset(wcsph_ctx* ctx) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->reset(); });
}

int wcsph_set_box(wcsph_ctx* ctx, const wcsph_box* box) {
    CHECK_CTX(ctx);
    if (!box) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { ctx->sim->set_box(*box); });
}

int wcsph_set_params(wcsph_ctx* ctx, const wcsph_params* p) {
    CHECK_CTX(ctx);
    if (!p) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { ctx->sim->set_params(*p); });
}

int wcsph_get_params(const wcsph_ctx* ctx, wcsph_params* out) {
    if (!ctx || !ctx->sim || !out) return WCSPH_ERR_INVALID_ARGUMENT;
    *out = ctx->sim->params();
    return WCSPH_OK;
}

int wcsph_get_state(wcsph_ctx* ctx, float* pos, float* vel) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->get_state(pos, vel); });
}

int wcsph_set_state(wcsph_ctx* ctx, const float* pos, const float* vel) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->set_state(pos, vel); });
}

int wcsph_snapshot_save(wcsph_ctx* ctx, const char* path, const char* app_name) {
    CHECK_CTX(ctx);
    if (!path || !app_name) return WCSPH_ERR_INVALID_ARGUMENT;
    if (std::strlen(app_name) >= wcsph_host::kAppNameMax)
        return host_status(ctx, {WCSPH_ERR_SNAPSHOT_APP_NAME, "Snapshot::save: app_name too long (max 63 chars)"});
    const uint32_t n = ctx->sim->get_fluid_particles();
    std::vector<float> pos(4ull * n), vel(4ull * n);
    const int s = guarded(ctx, [&] { ctx->sim->get_state(pos.data(), vel.data()); });
    if (s != WCSPH_OK) return s;
    return host_status(ctx, wcsph_host::snapshot_write(path, app_name, n, pos.data(), vel.data()));
}

int wcsph_snapshot_load(wcsph_ctx* ctx, const char* path, const char* app_name) {
    CHECK_CTX(ctx);
    if (!path || !app_name) return WCSPH_ERR_INVALID_ARGUMENT;
    const uint32_t n = ctx->sim->get_fluid_particles();
    std::vector<float> pos(4ull * n), vel(4ull * n);
    const int s = host_status(ctx, wcsph_host::snapshot_read(path, app_name, n, pos.data(), vel.data()));
    if (s != WCSPH_OK) return s;
    return guarded(ctx, [&] { ctx->sim->set_state(pos.data(), vel.data()); });
}

int wcsph_snapshot_read_header(const char* path, char app_name_out[64], uint32_t* fluid_n_out) {
    if (!path) return WCSPH_ERR_INVALID_ARGUMENT;
    std::string name;
    uint32_t n = 0;
    const int s = host_status(nullptr, wcsph_host::snapshot_read_header(path, &name, &n));
    if (s != WCSPH_OK) return s;
    if (app_name_out) {
        std::memset(app_name_out, 0, 64);
        std::memcpy(app_name_out, name.data(), std::min<size_t>(name.size(), 63));
    }
    if (fluid_n_out) *fluid_n_out = n;
    return WCSPH_OK;
}

int wcsph_snapshot_read(const char* path, const char* app_name, uint32_t fluid_n, float* pos, float* vel) {
    if (!path || !app_name) return WCSPH_ERR_INVALID_ARGUMENT;
    return host_status(nullptr, wcsph_host::snapshot_read(path, app_name, fluid_n, pos, vel));
}

int wcsph_snapshot_write(const char* path, const char* app_name, uint32_t fluid_n, const float* pos,
                         const float* vel) {
    if (!path || !app_name || (fluid_n && (!pos || !vel))) return WCSPH_ERR_INVALID_ARGUMENT;
    return host_status(nullptr, wcsph_host::snapshot_write(path, app_name, fluid_n, pos, vel));
}

int wcsph_metrics(wcsph_ctx* ctx, float* mean_speed, float* ke) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->metrics(mean_speed, ke); });
}

int wcsph_last_dt(wcsph_ctx* ctx, float* dt_p, float* np_dt) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->last_dt(dt_p, np_dt); });
}

int wcsph_field_size(const wcsph_ctx* ctx, int field, uint64_t* elems, uint32_t* elem_bytes) {
    if (!ctx || !ctx->sim) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(const_cast<wcsph_ctx*>(ctx), [&] {
        if (elems) *elems = ctx->sim->field_elems(field);
        if (elem_bytes) *elem_bytes = ctx->sim->field_elem_bytes(field);
    });
}

int wcsph_get_field(wcsph_ctx* ctx, int field, void* dst, uint64_t bytes) {
    CHECK_CTX(ctx);
    if (!dst) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { ctx->sim->get_field(field, dst, bytes); });
}

int wcsph_get_device_field(wcsph_ctx* ctx, int field, void** dev_ptr) {
    CHECK_CTX(ctx);
    if (!dev_ptr) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { *dev_ptr = ctx->sim->device_field(field); });
}

int wcsph_get_neighbors(wcsph_ctx* ctx, uint32_t* counts, uint32_t* offsets, uint32_t* neighbors, uint64_t capacity,
                        uint64_t* total_out) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->get_neighbors(counts, offsets, neighbors, capacity, total_out); });
}

int wcsph_get_stream(wcsph_ctx* ctx, void** stream_out) {
    CHECK_CTX(ctx);
    if (!stream_out) return WCSPH_ERR_INVALID_ARGUMENT;
    *stream_out = static_cast<void*>(ctx->sim->stream());
    return WCSPH_OK;
}

int wcsph_time_steps(wcsph_ctx* ctx, int n, float delta, float* ms_out) {
    CHECK_CTX(ctx);
    if (n < 0 || !ms_out) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { *ms_out = ctx->sim->time_steps(n, delta); });
}

int wcsph_kernel_timings(wcsph_ctx* ctx, const char** names, float* ms, int cap) {
    CHECK_CTX(ctx);
    int k = 0;
    const int s = guarded(ctx, [&] { k = ctx->sim->kernel_timings(names, ms, cap); });
    return s == WCSPH_OK ? k : -s;
}

int wcsph_launches_per_step(wcsph_ctx* ctx, int* out) {
    CHECK_CTX(ctx);
    if (!out) return WCSPH_ERR_INVALID_ARGUMENT;
    *out = ctx->sim->launches_per_step();
    return WCSPH_OK;
}

int wcsph_set_tuning(wcsph_ctx* ctx, int searcher, float budget, const char* frozen_json) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->set_tuning(searcher, budget, frozen_json); });
}

int wcsph_was_tuning_step(wcsph_ctx* ctx, int* out) {
    CHECK_CTX(ctx);
    if (!out) return WCSPH_ERR_INVALID_ARGUMENT;
    *out = ctx->sim->was_tuning_step() ? 1 : 0;
    return WCSPH_OK;
}

int wcsph_save_config(wcsph_ctx* ctx, const char* path) {
    CHECK_CTX(ctx);
    if (!path) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { ctx->sim->save_config(path); });
}

int wcsph_save_tuning_results(wcsph_ctx* ctx, const char* path) {
    CHECK_CTX(ctx);
    if (!path) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { ctx->sim->save_tuning_results(path); });
}

int wcsph_reset_tuning(wcsph_ctx* ctx) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->reset_tuning(); });
}

// ---- scene builders -------------------------------------------------------
int wcsph_make_lattice(const float origin[3], const uint32_t dims[3], float radius, float jitter, uint64_t seed,
                       float* pos_out) {
    if (!origin || !dims || !pos_out || !(radius > 0.f)) return WCSPH_ERR_INVALID_ARGUMENT;
    wcsph_host::make_lattice(origin, dims, radius, jitter, seed, pos_out);
    return WCSPH_OK;
}

int wcsph_make_velocities(uint32_t n, float sigma, uint64_t seed, float* vel_out) {
    if (!vel_out && n) return WCSPH_ERR_INVALID_ARGUMENT;
    wcsph_host::make_velocities(n, sigma, seed, vel_out);
    return WCSPH_OK;
}

int wcsph_sample_box_walls(const float mn[3], const float mx[3], float spacing, float* pos_out, uint32_t* n_out) {
    if (!mn || !mx || !n_out || !(spacing > 0.f)) return WCSPH_ERR_INVALID_ARGUMENT;
    *n_out = wcsph_host::sample_box_walls(mn, mx, spacing, pos_out);
    return WCSPH_OK;
}

int wcsph_sample_icosphere(const float center[3], float radius, int level, float voxel, float* pos_out,
                           uint32_t* n_out) {
    if (!center || !n_out || !(radius > 0.f) || !(voxel > 0.f) || level < 0 || level > 7)
        return WCSPH_ERR_INVALID_ARGUMENT;
    const std::vector<float> tris = wcsph_host::icosphere_triangles(center, radius, level);
    *n_out = wcsph_host::sample_triangles(tris.data(), static_cast<uint32_t>(tris.size() / 9), voxel, pos_out);
    return WCSPH_OK;
}

int wcsph_load_obj(const char* path, int normalize, const float model[16], float* vertices_out,
                   uint32_t* n_triangles) {
    if (!path || !n_triangles) return WCSPH_ERR_INVALID_ARGUMENT;
    wcsph_host::Status st;
    const std::vector<float> t = wcsph_host::load_obj_triangles(path, normalize != 0, model, &st);
    if (!st.ok()) {
        g_last_error = st.message;
        return st.code;
    }
    *n_triangles = static_cast<uint32_t>(t.size() / 9);
    if (vertices_out) std::memcpy(vertices_out, t.data(), sizeof(float) * t.size());
    return WCSPH_OK;
}

int wcsph_sample_triangles(const float* vertices, uint32_t n_triangles, float voxel, float* pos_out,
                           uint32_t* n_out) {
    if ((!vertices && n_triangles) || !n_out || !(voxel > 0.f)) return WCSPH_ERR_INVALID_ARGUMENT;
    *n_out = wcsph_host::sample_triangles(vertices, n_triangles, voxel, pos_out);
    return WCSPH_OK;
}

// ---- differentiable rollout ------------------------------------------------
int wcsph_rollout_forward(wcsph_ctx* ctx, int steps, float dt, int checkpoint_every, const float* target_pos,
                          float* loss_out) {
    CHECK_CTX(ctx);
    if (steps <= 0 || checkpoint_every <= 0 || !target_pos || !(dt > 0.f)) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] {
        const float l = ctx->sim->rollout_forward(steps, dt, checkpoint_every, target_pos);
        if (loss_out) *loss_out = l;
    });
}

int wcsph_rollout_backward(wcsph_ctx* ctx, float* grad_v0, float* grad_viscosity, float* grad_stiffness) {
    CHECK_CTX(ctx);
    return guarded(ctx, [&] { ctx->sim->rollout_backward(grad_v0, grad_viscosity, grad_stiffness); });
}

// ---- headless rendering --------------------------------------------------------
int wcsph_render(wcsph_ctx* ctx, const wcsph_camera* cam, const wcsph_render_opts* opts, uint8_t* rgba,
                 float* depth) {
    CHECK_CTX(ctx);
    if (!cam || !opts) return WCSPH_ERR_INVALID_ARGUMENT;
    return guarded(ctx, [&] { ctx->sim->render(*cam, *opts, rgba, depth); });
}

// ---- allocation-free key sort ------------------------------------------------
// No counterpart in the reference; for callers that cannot allocate device
// memory while they run (see include/wcsph.h). Errors go to wcsph_last_error(NULL).
int wcsph_sort_keys_static(const uint64_t* keys, uint32_t n, uint32_t* perm, void* stream) {
    return guarded(nullptr, [&] {
        wcsph::static_sort_permutation(keys, n, perm, static_cast<cudaStream_t>(stream));
    });
}

// Error-path test hook: see include/wcsph.h.
int wcsph_test_stall_sort(int enable) {
    wcsph::set_sort_stall_test(enable != 0);
    return WCSPH_OK;
}

}  // extern "C"
