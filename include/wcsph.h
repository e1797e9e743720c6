/*
 * wcsph.h — C ABI of the B200-native WCSPH time step.
 *
 * This is the drop-in boundary for the reference's solver path
 * (petbab/fluid-simulation):
 *
 *   reference interface                                   replaced by
 *   ---------------------------------------------------  ----------------------------
 *   FluidSimulator ctor + opts_t                          wcsph_create
 *     src/simulation/fluid_simulator.h:22-30
 *   CUDASPHSimulator::CUDASPHSimulator                    wcsph_create
 *     src/cuda/SPH/sph.cu:9-23, init_boundary sph.cu:84-96
 *   FluidSimulator::update / CUDASPHSimulator::update     wcsph_step, wcsph_step_n
 *     src/simulation/fluid_simulator.h:33, sph.cu:31-60
 *   StepTuner::run (raw device pointers, dt, np_dt, bb)   wcsph_step (+ wcsph_get_device_fields)
 *     src/cuda/tuning/step_tuner.cuh:146-244
 *   CUDASPHSimulator::reset  sph.cu:73-82                 wcsph_reset
 *   Snapshot::save / Snapshot::load                       wcsph_snapshot_save / _load
 *     src/cuda/SPH/snapshot.cu:10-106
 *   CUDASPHSimulator::compute_state_metrics sph.cu:180-197 wcsph_metrics
 *   Box::set_model (moving/tilting box) src/render/box.cpp:19-23   wcsph_set_box
 *   Tuner::set_searcher / set_frozen_config /             wcsph_set_tuning
 *     CUDASPHSimulator::set_tuning_budget
 *     src/cuda/tuning/tuner.cpp:48-94, sph.cu:150-160
 *   ParticleData accessors (density(), pressure(), ...)   wcsph_get_field
 *     src/cuda/SPH/particle_data.cuh:140-170
 *   NSearchHost::copy_from_device nsearch.cuh:61-92       wcsph_get_field (HASH_* fields)
 *
 * Conventions: every call returns an int status (WCSPH_OK == 0); no C++
 * exception crosses the ABI. Host pointers passed in are copied before the
 * call returns. A context is bound to one CUDA device and one stream and must
 * be driven from one host thread at a time. float4 arrays are packed as
 * 4 floats per particle (x, y, z, w) exactly like the reference's float4
 * buffers; w is 1 for positions and 0 for velocities.
 */
#ifndef WCSPH_H
#define WCSPH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WCSPH_ABI_VERSION 1

/* ---- status codes -------------------------------------------------------- */
enum wcsph_status {
    WCSPH_OK = 0,
    WCSPH_ERR_INVALID_ARGUMENT = 1,
    WCSPH_ERR_CUDA = 2,
    WCSPH_ERR_OUT_OF_MEMORY = 3,
    WCSPH_ERR_IO = 4,
    WCSPH_ERR_SNAPSHOT_MAGIC = 5,      /* Snapshot::load "bad magic"            */
    WCSPH_ERR_SNAPSHOT_VERSION = 6,    /* "version mismatch"                    */
    WCSPH_ERR_SNAPSHOT_APP_NAME = 7,   /* "app_name mismatch" / name too long   */
    WCSPH_ERR_SNAPSHOT_COUNT = 8,      /* "fluid count mismatch"                */
    WCSPH_ERR_SNAPSHOT_TRUNCATED = 9,  /* header or body read failed            */
    WCSPH_ERR_HASH_FULL = 10,          /* spatial hash has no free slot         */
    WCSPH_ERR_NEIGHBOR_OVERFLOW = 11,  /* neighbour list capacity exceeded      */
    WCSPH_ERR_DEVICE_TIMEOUT = 12,     /* a bounded device-side wait gave up    */
    WCSPH_ERR_NO_DEVICE = 13,          /* no CUDA device / extension unusable   */
    WCSPH_ERR_CONFIG = 14,             /* bad tuning config / frozen JSON       */
    WCSPH_ERR_NOT_SUPPORTED = 15,
    WCSPH_ERR_STATE = 16,              /* call not valid in the current state   */
    WCSPH_ERR_BOUNDS = 17              /* bounds-checked build (libwcsph_checked.so):
                                          a device index guard fired            */
};

/* ---- external force fields --------------------------------------------
 * The reference compiles a C++ lambda string per scene (EXTERNAL_FORCE,
 * src/cuda/tuning/kernels/compute_non_pressure_accel.cu:9-11). Here the same
 * scene forces are a fixed device-side table selected at run time.        */
enum wcsph_force_field {
    WCSPH_FORCE_NONE = 0,      /* ([](float4){ return make_float4(0.f); })              */
    WCSPH_FORCE_CONSTANT = 1,  /* constant vector (param[0..2]); surface_tension app    */
    WCSPH_FORCE_FOUNTAIN = 2,  /* app/fountain/application.cu:36-42 (params unused)     */
    WCSPH_FORCE_VORTEX = 3     /* app/vortex/application.cu:45 (params unused)          */
};

/* ---- physical + numerical parameters (run-time; compile-time constexpr in
 * the reference: src/cuda/tuning/kernels/common.cuh:18-23, compute_rho_p.cu:10-12,
 * compute_non_pressure_accel.cu:14-16, update_positions.cu:10-12,
 * src/cuda/SPH/sph.cuh:19-32). wcsph_default_params() fills the reference's
 * values. Derived exactly like the reference: spacing = 2r, support h = 2*spacing,
 * volume = spacing^3 * 0.8, mass = rest_density * volume.                   */
typedef struct wcsph_params {
    float particle_radius;            /* r; ref 0.02                              */
    float rest_density;               /* rho0; ref 1000                           */
    float stiffness;                  /* Tait k; ref 0.1                          */
    float exponent;                   /* Tait gamma; ref 7                        */
    float max_density_ratio;          /* EOS clamp; ref 1.5                       */
    float viscosity;                  /* nu; ref 0.001                            */
    float surface_tension;            /* alpha; ref 0.13                          */
    float gravity[3];                 /* ref (0,-9.81,0)                          */
    float cfl_factor;                 /* ref 0.4; <= 0 disables the CFL bound     */
    float max_time_step;              /* ref 5e-4                                 */
    float min_time_step;              /* ref 1e-5                                 */
    float non_pressure_max_time_step; /* ref 0.015                                */
    float collision_buffer_mult;      /* ref 0.75                                 */
    float elasticity;                 /* ref 0.5                                  */
    float cell_size_mult;             /* CELL_SIZE_MULT; ref tuned {0.5,2/3,1,1.5,2} */
    uint32_t table_size_mult;         /* TABLE_SIZE_MULT; power of two 1..32      */
    int32_t external_force;           /* enum wcsph_force_field                   */
    float external_force_param[4];
} wcsph_params;

/* Collision box (reference BoundingBoxGPU, src/cuda/util.cuh:9-16): min/max in
 * model space and a column-major 4x4 model matrix + its inverse (glm layout). */
typedef struct wcsph_box {
    float min[3];
    float max[3];
    float model[16];
    float model_inv[16];
} wcsph_box;

/* Scene description. Boundary particles are sampled once from the scene's
 * collision meshes (reference: generate_boundary_particles,
 * src/simulation/SPH/boundary.cpp:8-35); wcsph_sample_* below builds them.  */
typedef struct wcsph_scene {
    uint32_t fluid_n;
    const float* fluid_pos;     /* float4[fluid_n], host                      */
    const float* fluid_vel;     /* float4[fluid_n], host; NULL = zero         */
    uint32_t boundary_n;
    const float* boundary_pos;  /* float4[boundary_n], host; may be NULL if 0 */
    wcsph_box box;
} wcsph_scene;

typedef struct wcsph_ctx wcsph_ctx;

/* ---- lifecycle -------------------------------------------------------- */
int  wcsph_abi_version(void);
void wcsph_default_params(wcsph_params* out);
void wcsph_identity_box(const float min[3], const float max[3], wcsph_box* out);
const char* wcsph_status_string(int status);

/* Creates a simulator on `device` (-1 = current device). Sorts the boundary
 * once, builds its hash and computes the boundary masses (Akinci), like
 * CUDASPHSimulator::init_boundary (sph.cu:84-96).                           */
int wcsph_create(const wcsph_params* params, const wcsph_scene* scene,
                 int device, wcsph_ctx** out);
int wcsph_destroy(wcsph_ctx* ctx);
/* Thread-local text of the last error of this context (never NULL).        */
const char* wcsph_last_error(const wcsph_ctx* ctx);

/* ---- stepping ---------------------------------------------------------
 * One FluidSimulator::update(delta): np_dt = min(delta, non_pressure_max),
 * dt = min(clamp(delta, min, max), cfl*spacing/max|v|) (sph.cu:39-40,115-130),
 * then sort, neighbourhood search, density, pressure, non-pressure force,
 * integrate + box collision. The CFL max-speed comes from a device-side
 * reduction fused into the previous step: no host synchronisation.         */
int wcsph_step(wcsph_ctx* ctx, float delta);
/* n steps with the same delta; replays a captured CUDA graph of the step.  */
int wcsph_step_n(wcsph_ctx* ctx, int n, float delta);
int wcsph_synchronize(wcsph_ctx* ctx);
/* Restores the initial fluid positions, zero velocities and derived fields
 * (CUDASPHSimulator::reset, sph.cu:73-82).                                  */
int wcsph_reset(wcsph_ctx* ctx);
/* Replaces the collision box (moving/tilting box of app/tilting_box).       */
int wcsph_set_box(wcsph_ctx* ctx, const wcsph_box* box);
/* Changes viscosity / stiffness / surface tension / gravity at run time.    */
int wcsph_set_params(wcsph_ctx* ctx, const wcsph_params* params);
int wcsph_get_params(const wcsph_ctx* ctx, wcsph_params* out);

/* ---- state I/O --------------------------------------------------------- */
/* Current fluid state in the current (sorted) particle order, float4 each.  */
int wcsph_get_state(wcsph_ctx* ctx, float* pos_out, float* vel_out);
/* Overwrites the fluid state (positions to both buffers, like Snapshot::load). */
int wcsph_set_state(wcsph_ctx* ctx, const float* pos, const float* vel);
/* Byte-exact .sphs v1 (76-byte header 'SPHS', u32 version, char[64] app_name,
 * u32 fluid_n; then float4 pos[n], float4 vel[n]); same validation order and
 * messages as Snapshot::load (snapshot.cu:54-106).                           */
int wcsph_snapshot_save(wcsph_ctx* ctx, const char* path, const char* app_name);
int wcsph_snapshot_load(wcsph_ctx* ctx, const char* path, const char* app_name);
/* File-only helpers (no context): header read, and full read into host arrays. */
int wcsph_snapshot_read_header(const char* path, char app_name_out[64], uint32_t* fluid_n_out);
int wcsph_snapshot_read(const char* path, const char* app_name, uint32_t fluid_n,
                        float* pos_out, float* vel_out);
int wcsph_snapshot_write(const char* path, const char* app_name, uint32_t fluid_n,
                         const float* pos, const float* vel);

/* mean_speed = sum|v|/N, ke = sum 0.5 m |v|^2 (sph.cu:180-197).            */
int wcsph_metrics(wcsph_ctx* ctx, float* mean_speed, float* ke);
/* Time step (dt_p) and np_dt actually used by the last step.                */
int wcsph_last_dt(wcsph_ctx* ctx, float* dt_p, float* np_dt);

/* ---- field access for parity checks ------------------------------------- */
enum wcsph_field {
    WCSPH_FIELD_POSITION = 0,        /* float4[fluid_n], sorted order            */
    WCSPH_FIELD_VELOCITY = 1,        /* float4[fluid_n]                          */
    WCSPH_FIELD_DENSITY = 2,         /* float[fluid_n]                           */
    WCSPH_FIELD_PRESSURE = 3,        /* float[fluid_n]                           */
    WCSPH_FIELD_PRESSURE_ACCEL = 4,  /* float4[fluid_n]                          */
    WCSPH_FIELD_NON_PRESSURE_ACCEL = 5, /* float4[fluid_n]                       */
    WCSPH_FIELD_NORMAL = 6,          /* float4[fluid_n]                          */
    WCSPH_FIELD_MORTON_KEYS = 7,     /* u64[fluid_n]: keys of the last sort, in
                                        pre-sort (input) order                   */
    WCSPH_FIELD_PERMUTATION = 8,     /* u32[fluid_n]: sorted -> input index      */
    WCSPH_FIELD_HASH_TABLE = 9,      /* u64[table_size]                          */
    WCSPH_FIELD_HASH_CELL_START = 10,/* u32[table_size]                          */
    WCSPH_FIELD_HASH_CELL_END = 11,  /* u32[table_size]                          */
    WCSPH_FIELD_BOUNDARY_POSITION = 12, /* float4[boundary_n], sorted            */
    WCSPH_FIELD_BOUNDARY_MASS = 13,  /* float[boundary_n]                        */
    WCSPH_FIELD_COUNT_ = 14
};
/* Number of elements of a field (table_size for HASH_*).                   */
int wcsph_field_size(const wcsph_ctx* ctx, int field, uint64_t* elems, uint32_t* elem_bytes);
int wcsph_get_field(wcsph_ctx* ctx, int field, void* host_dst, uint64_t dst_bytes);
/* Device pointers of the live fields (borrowed; valid until the next call). */
int wcsph_get_device_field(wcsph_ctx* ctx, int field, void** dev_ptr);

/* Per-particle fluid neighbour sets of the last step as CSR in the reference's
 * traversal order (count_neighbors / fill_neighbors,
 * src/cuda/tuning/kernels/compute_neighbor_list.cu:10-44). counts/offsets
 * u32[fluid_n]; neighbours u32[capacity]. *total_out gets the neighbour count;
 * WCSPH_ERR_NEIGHBOR_OVERFLOW if it exceeds capacity (nothing is written past). */
int wcsph_get_neighbors(wcsph_ctx* ctx, uint32_t* counts, uint32_t* offsets,
                        uint32_t* neighbors, uint64_t capacity, uint64_t* total_out);

/* ---- timing (CUDA events on the context's stream) ----------------------- */
/* The context's CUDA stream (cudaStream_t), for callers that time or order
 * their own work against the step.                                          */
int wcsph_get_stream(wcsph_ctx* ctx, void** stream_out);
/* Runs `n` steps and returns their device time in milliseconds.            */
int wcsph_time_steps(wcsph_ctx* ctx, int n, float delta, float* ms_out);
/* Per-kernel average device time of the last timed step set; names are
 * static strings. Returns the number of entries written (<= cap).          */
int wcsph_kernel_timings(wcsph_ctx* ctx, const char** names, float* ms, int cap);
/* Number of kernel launches one step issues (for launch accounting).       */
int wcsph_launches_per_step(wcsph_ctx* ctx, int* out);

/* ---- autotuner (replaces KTT; src/cuda/tuning/tuner.cpp) -----------------*/
enum wcsph_searcher { WCSPH_SEARCH_MCMC = 0, WCSPH_SEARCH_RANDOM = 1, WCSPH_SEARCH_FULL = 2 };
/* budget = tuning iterations per step (TuningScheduler semantics,
 * src/cuda/tuning/tuning_scheduler.h:12-26); frozen_json = path of a
 * [{"Name","Value","ValueType"}] config (config_loader.cpp:8-54) or NULL.   */
int wcsph_set_tuning(wcsph_ctx* ctx, int searcher, float budget, const char* frozen_json);
/* Whether the last wcsph_step was a tuning iteration (was_scheduled_step). */
int wcsph_was_tuning_step(wcsph_ctx* ctx, int* out);
/* Writes the best (or frozen) configuration as KTT-schema JSON.            */
int wcsph_save_config(wcsph_ctx* ctx, const char* path);
/* Writes KTT-compatible results JSON (TotalDuration, ComputationResults).  */
int wcsph_save_tuning_results(wcsph_ctx* ctx, const char* path);
/* Clears searched configurations (CUDASPHSimulator::reset_tuning).         */
int wcsph_reset_tuning(wcsph_ctx* ctx);

/* ---- scene builders (host only) ----------------------------------------- */
/* Lattice of FluidSimulator::init_positions (fluid_simulator.cpp:24-54):
 * x-outer, y, z-inner; start = origin - (dims-1)*r; spacing 2r; w = 1.
 * jitter > 0 adds a seeded uniform offset in [-jitter, jitter] per axis.   */
int wcsph_make_lattice(const float origin[3], const uint32_t dims[3], float radius,
                       float jitter, uint64_t seed, float* pos_out);
/* Seeded N(0, sigma) per component velocities (w = 0).                      */
int wcsph_make_velocities(uint32_t n, float sigma, uint64_t seed, float* vel_out);
/* Single-layer wall particles of an axis-aligned box (spacing = grid step).
 * Returns the count in *n_out; pass pos_out = NULL to only count.          */
int wcsph_sample_box_walls(const float min[3], const float max[3], float spacing,
                           float* pos_out, uint32_t* n_out);
/* Surface sampling of a level-`level` subdivided icosphere (20*4^level tris)
 * by surface voxelisation at `voxel` (replaces Open3D's
 * VoxelGrid::CreateFromTriangleMesh, boundary.cpp:27-32).                    */
int wcsph_sample_icosphere(const float center[3], float radius, int level, float voxel,
                           float* pos_out, uint32_t* n_out);
/* Surface voxelisation of an arbitrary triangle soup (float3 per vertex).   */
int wcsph_sample_triangles(const float* vertices, uint32_t n_triangles, float voxel,
                           float* pos_out, uint32_t* n_out);
/* Triangles of a Wavefront .obj mesh, for wcsph_sample_triangles: replaces
 * Geometry::from_file + Geometry::load_triangles (src/render/geometry.cpp:50-140,
 * 185-207; tinyobjloader). The first shape's faces in file order; a face of
 * more than three vertices is rejected as there (WCSPH_ERR_INVALID_ARGUMENT,
 * "In <path>: face f has N vertices (not a triangle)"); normalize != 0 scales
 * the mesh into a unit box around the origin; model (column-major 4x4, NULL =
 * identity) is applied last. Call with vertices_out = NULL for the count.   */
int wcsph_load_obj(const char* path, int normalize, const float model[16], float* vertices_out,
                   uint32_t* n_triangles);

/* ---- workload presets -------------------------------------------------------
 * Scenes of the reference's headless apps that need no missing asset
 * ("surface_tension" app/surface_tension/application.cu:10-25, "tilting_box"
 * app/tilting_box/application.cu:10-46) and the benchmark workloads
 * ("dam_break", "mesh_obstacle", "large_tilting", "rollout_block").
 * Two-call pattern: pass NULL arrays to get the counts in *info first.      */
typedef struct wcsph_preset_info {
    wcsph_params params;
    wcsph_box box;          /* box at t = 0                                   */
    uint32_t fluid_n;
    uint32_t boundary_n;
    float delta;            /* requested step per update (--fixed-dt)         */
    int32_t steps;          /* workload length in steps (0 = by sim_time)      */
    float sim_time;         /* workload length in simulated seconds (0 = steps) */
    int32_t moving_box;     /* 1 if the box model changes over time           */
} wcsph_preset_info;
int wcsph_preset(const char* name, uint64_t seed, wcsph_preset_info* info,
                 float* fluid_pos, float* fluid_vel, float* boundary_pos);
/* Box of a moving-box preset after `updates` updates of `delta` each.       */
int wcsph_preset_box(const char* name, int64_t updates, float delta, wcsph_box* out);
/* Scene k of the seeded ensemble (log-uniform particle counts 2048..65536,
 * box extents U[0.3,1], gravity tilt U[0,20 deg], viscosity U[0.005,0.05]). */
int wcsph_preset_ensemble(uint64_t seed, uint32_t k, wcsph_preset_info* info,
                          float* fluid_pos, float* fluid_vel, float* boundary_pos);

/* ---- batched ensemble: many independent scenes, one launch per kernel ----
 * Scenes keep their own box, gravity and viscosity; particles of all scenes
 * live in one SoA with per-scene offsets.                                   */
typedef struct wcsph_batch wcsph_batch;
typedef struct wcsph_batch_scene {
    uint32_t fluid_n;
    const float* fluid_pos;
    const float* fluid_vel;      /* NULL = zero */
    uint32_t boundary_n;
    const float* boundary_pos;
    wcsph_box box;
    float gravity[3];
    float viscosity;
} wcsph_batch_scene;
int wcsph_batch_create(const wcsph_params* params, const wcsph_batch_scene* scenes,
                       uint32_t n_scenes, int device, wcsph_batch** out);
int wcsph_batch_destroy(wcsph_batch* b);
/* Chooses how wcsph_batch_step_n / _time_steps run n steps (both give the
 * same results, bit for bit): enable != 0 (the default) advances every scene
 * n steps in ONE persistent cooperative launch whose phases are separated by
 * bounded grid barriers (captured in a CUDA graph where the driver allows);
 * 0 launches each stage of each step separately from a per-step CUDA graph.
 * No counterpart in the reference (it has no batched ensembles).          */
int wcsph_batch_set_persistent(wcsph_batch* b, int enable);
int wcsph_batch_step_n(wcsph_batch* b, int n, float delta);
int wcsph_batch_time_steps(wcsph_batch* b, int n, float delta, float* ms_out);
/* Per-scene state in each scene's current (sorted) order.                  */
int wcsph_batch_get_state(wcsph_batch* b, uint32_t scene, float* pos_out, float* vel_out);
int wcsph_batch_metrics(wcsph_batch* b, float* mean_speed, float* ke);  /* per scene arrays */
const char* wcsph_batch_last_error(const wcsph_batch* b);

/* ---- differentiable rollout (adjoint) -------------------------------------
 * Fixed dt (CFL off), surface tension must be 0. Forward stores positions and
 * velocities every `checkpoint_every` steps; backward recomputes each segment
 * (sort + neighbourhood search again from the checkpoint) and runs the
 * hand-written adjoint kernels in reverse.
 * Loss = mean_i |x_T,i - target_i|^2 (targets indexed by initial particle id).
 * Outputs: dL/dv0 (float4 per initial particle id), dL/dnu, dL/dk.          */
int wcsph_rollout_forward(wcsph_ctx* ctx, int steps, float dt, int checkpoint_every,
                          const float* target_pos, float* loss_out);
int wcsph_rollout_backward(wcsph_ctx* ctx, float* grad_v0, float* grad_viscosity,
                           float* grad_stiffness);

/* ---- headless particle rendering ------------------------------------------
 * The reference's particle view (shaders/instanced_ball.vert:20-32 and
 * instanced_ball.frag: camera-facing quads shaded as spheres, fluid blue,
 * boundary orange, optional field visualisation) computed by CUDA kernels
 * into an RGBA8 image, without a graphics stack. Matrices are column-major
 * (glm layout); image row 0 is the top row.                                 */
typedef struct wcsph_camera {
    float projection[16];
    float view[16];
    float eye[3];
} wcsph_camera;
/* Camera(position, yaw, pitch, width, height) of src/render/camera.cpp:7-33:
 * perspective 45 deg, near 0.1, far 100, world up (0, 1, 0). The reference's
 * start view is position (0, 0, 2.5), yaw 270 deg, pitch 0 (angles in radians). */
void wcsph_camera_look(const float position[3], float yaw, float pitch, uint32_t width, uint32_t height,
                       wcsph_camera* out);
typedef struct wcsph_render_opts {
    uint32_t width, height;
    float radius;            /* sphere radius (the shaders' RADIUS 0.02)         */
    int show_boundary;       /* draw boundary particles                          */
    int field;               /* -1: plain colours; WCSPH_FIELD_DENSITY or _PRESSURE
                                (grey = value); WCSPH_FIELD_VELOCITY, _PRESSURE_ACCEL,
                                _NON_PRESSURE_ACCEL or _NORMAL (colour * dot(v, n)),
                                on fluid particles                               */
    int normalize;           /* map [min_value, max_value] to [0, 1]             */
    float min_value, max_value;
    float background[3];
    int max_pixels;          /* skip particles whose quad covers more pixels     */
} wcsph_render_opts;
void wcsph_default_render_opts(wcsph_render_opts* o);
/* Renders the current state: rgba (width*height*4 bytes) and, if not NULL,
 * depth (width*height floats, window depth in [0, 1], 1 = background).     */
int wcsph_render(wcsph_ctx* ctx, const wcsph_camera* cam, const wcsph_render_opts* opts, uint8_t* rgba,
                 float* depth);

/* ---- allocation-free key sort ---------------------------------------------
 * No counterpart in the reference (its sort is thrust::sort_by_key, which
 * allocates temporary storage on every call).
 *
 * For callers that cannot call cudaMalloc/cudaFree while they run: a render
 * or control loop that must not take the device-wide synchronisation that
 * freeing device memory implies, or a host that works inside a device memory
 * budget reserved up front. Writes to perm (device array of n uint32) the
 * stable sort permutation of the n device-resident 64-bit keys (perm[i] = index
 * of the key of rank i, equal keys in input order): the same permutation the
 * step's sort produces (WCSPH_FIELD_PERMUTATION for WCSPH_FIELD_MORTON_KEYS).
 * keys is only read. Nothing is allocated: the scratch is a device array of the
 * library image, about 1.8 MiB, that every GPU loading the library holds until
 * the process exits.
 *   - n above WCSPH_STATIC_SORT_MAX_KEYS returns WCSPH_ERR_INVALID_ARGUMENT
 *     (text via wcsph_last_error(NULL)); n == 0 does nothing.
 *   - The work is enqueued on `stream` (a cudaStream_t; NULL = the default
 *     stream) of the current device and the call returns without waiting.
 *   - The first call on a device looks up the scratch's device address (set-up
 *     done once per device); make that first call before any stream capture.
 *   - Every call on a device shares the one scratch: calls whose work overlaps
 *     on the GPU (other streams, other host threads) race and corrupt each
 *     other's results. Order them on one stream or synchronise between them.
 *   - The sort's waits between its tiles are bounded (about a second). If one
 *     runs out, the call cannot tell the host without waiting for the GPU, so
 *     it marks its output instead: every perm entry is then
 *     WCSPH_STATIC_SORT_FAILED, an index no key has. Check perm[0] < n after
 *     the stream work completes when this matters.
 *   - The scratch address is looked up again when the device's current
 *     context changes (after cudaDeviceReset, or under a driver-API context
 *     of the caller's own). */
#define WCSPH_STATIC_SORT_MAX_KEYS 65536u
#define WCSPH_STATIC_SORT_FAILED 0xFFFFFFFFu
int wcsph_sort_keys_static(const uint64_t* keys, uint32_t n, uint32_t* perm, void* stream);

/* ---- error-path test hook ---------------------------------------------------
 * No counterpart in the reference. While `enable` is non-zero, every radix sort
 * enqueued afterwards (the step's, the boundary set-up's, the batch's and
 * wcsph_sort_keys_static) withholds its first tile's look-back flags and bounds
 * each look-back wait to 4096 polls, so that the waits of the later tiles run
 * out within milliseconds. The step then reports WCSPH_ERR_DEVICE_TIMEOUT at
 * its next synchronising call and leaves the particle state as it was; the
 * static sort fills perm with WCSPH_STATIC_SORT_FAILED. Steps already captured
 * in a CUDA graph keep the setting they were captured with. Nothing faults or
 * hangs: it exists only to test these error paths. Returns WCSPH_OK.          */
int wcsph_test_stall_sort(int enable);

#ifdef __cplusplus
}
#endif
#endif /* WCSPH_H */
