// refpath_host.cu — replays the reference's CUDA step with its own kernels.
//
// TEST/BASELINE INFRASTRUCTURE (oracle/_ref only, never in the product).
// Host orchestration of CUDASPHSimulator::update (src/cuda/SPH/sph.cu:31-60)
// with the frozen-config path of StepTuner::launch
// (src/cuda/tuning/step_tuner.cuh:259-295): adapt_time_step via
// thrust::transform_reduce + host readback, ParticleData::sort via
// thrust sequence/transform/sort_by_key/gather (particle_data.cuh:112-133),
// clear + H2D shallow copy of the NSearch struct (nsearch.cuh:26-30,56-59),
// rebuild_n_search, count_neighbors -> thrust::exclusive_scan ->
// fill_neighbors, compute_rho_p, compute_pressure_accel_n_normal,
// compute_non_pressure_accel, update_positions. Boundary init follows
// sort_boundary / build_boundary_n_search / compute_boundary_mass
// (particle_data.cuh:84-110, sph.cu:84-103).
//
// Physics constants are the variant's (variant_config.h): the reference has
// them as constexpr, so each variant is a separate build.
#include <cuda_runtime.h>
#include <thrust/device_ptr.h>
#include <thrust/device_vector.h>
#include <thrust/execution_policy.h>
#include <thrust/functional.h>
#include <thrust/gather.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/transform_reduce.h>

#include <algorithm>
#include <bit>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "morton.cuh"  // shim copy of src/cuda/nsearch/morton.cuh

extern "C" {
void refk_rebuild_fluid(void* ns, const float4* pos, unsigned n, unsigned block, cudaStream_t s);
void refk_rebuild_boundary(void* ns, const float4* pos, unsigned n, cudaStream_t s);
void refk_count_neighbors(const float4* pos, unsigned* counts, unsigned n, const void* ns, unsigned block,
                          cudaStream_t s);
void refk_fill_neighbors(const float4* pos, const unsigned* offsets, unsigned* nbrs, unsigned n, const void* ns,
                         unsigned block, cudaStream_t s);
void refk_rho_p(const float4* pos, float* rho, float* prs, unsigned n, const void* ns, const unsigned* off,
                const unsigned* cnt, const unsigned* nbr, const float* bmass, const void* bns, cudaStream_t s);
void refk_pressure(const float4* pos, const float* rho, const float* prs, float4* ap, float4* normal, unsigned n,
                   const void* ns, const unsigned* off, const unsigned* cnt, const unsigned* nbr, const float* bmass,
                   const void* bns, cudaStream_t s);
void refk_non_pressure(const float4* pos, const float* rho, const float4* vel, const float4* normal, float4* anp,
                       unsigned n, const void* ns, const unsigned* off, const unsigned* cnt, const unsigned* nbr,
                       cudaStream_t s);
struct RefBox;
void refk_update_positions(float4* pos, float4* vel, const float4* ap, const float4* anp, unsigned n, float delta,
                           float np_delta, const RefBox* box, unsigned block, cudaStream_t s);
void refk_boundary_mass(const float4* bpos, float* mass, unsigned nb, const void* bns, cudaStream_t s);
}

namespace {

// Layout of the reference's NSearch (common.cuh:183-190 / nsearch.cuh:7-24).
struct NSearchView {
    unsigned long long* table;
    unsigned table_size;
    unsigned *cell_start, *cell_end;
    float cell_size;
};

struct BoxHost {
    float4 min, max;
    float4 model[4], model_inv[4];
};

struct Ctx {
    unsigned n = 0, nb = 0;
    cudaStream_t stream = nullptr;  // legacy default stream semantics: Thrust + kernels serialised
    // DoubleBuffer / DoubleGLBuffer (particle_data.cuh:14-50)
    thrust::device_vector<float4> pos[2];  // [n + nb]
    thrust::device_vector<float4> vel[2];
    int pos_src = 0, vel_src = 0;
    thrust::device_vector<unsigned long long> keys, bkeys;
    thrust::device_vector<unsigned> idx, bidx;
    thrust::device_vector<float> rho, prs, bmass;
    thrust::device_vector<float4> ap, anp, normal;
    // neighbour list (neighbor_list.cuh:6-45), capacity n * 96
    thrust::device_vector<unsigned> nl_counts, nl_offsets, nl_neighbors;
    // hash tables
    NSearchView host_fluid{}, host_boundary{};
    NSearchView* dev_fluid = nullptr;
    NSearchView* dev_boundary = nullptr;
    BoxHost box{};
    BoxHost* dev_box = nullptr;  // staged copy passed by value to update_positions
    float last_dt = 0.f, last_np_dt = 0.f;
};

Ctx* g = nullptr;

constexpr float kSpacing = 2.f * REF_PARTICLE_RADIUS;
constexpr float kSupport = 2.f * kSpacing;

struct Len2 {
    __host__ __device__ float operator()(const float4& v) const { return v.x * v.x + v.y * v.y + v.z * v.z; }
};

struct KeyOf {
    float cs;
    __device__ morton_t operator()(float4 p) const {
        int3 c{static_cast<int>(floorf(p.x / cs)), static_cast<int>(floorf(p.y / cs)),
               static_cast<int>(floorf(p.z / cs))};
        return encode_morton(c);
    }
};

void alloc_nsearch(NSearchView& h, NSearchView*& dev, unsigned table_size, float cell_size) {
    cudaMalloc(&dev, sizeof(NSearchView));
    h.table_size = table_size;
    cudaMalloc(&h.table, sizeof(unsigned long long) * table_size);
    cudaMalloc(&h.cell_start, sizeof(unsigned) * table_size);
    cudaMalloc(&h.cell_end, sizeof(unsigned) * table_size);
    h.cell_size = cell_size;
    cudaMemcpy(dev, &h, sizeof(NSearchView), cudaMemcpyHostToDevice);
}

void clear_nsearch(const NSearchView& h) {
    cudaMemset(h.table, 0xff, sizeof(unsigned long long) * h.table_size);
    cudaMemset(h.cell_start, 0, sizeof(unsigned) * h.table_size);
    cudaMemset(h.cell_end, 0, sizeof(unsigned) * h.table_size);
}

template <class T>
T* raw(thrust::device_vector<T>& v) { return thrust::raw_pointer_cast(v.data()); }

// adapt_time_step (sph.cu:115-130) with the variant's bounds; a CFL factor <= 0
// means a fixed step (the bounds alone decide).
float adapt_time_step(float delta) {
    const float vmax = std::sqrt(thrust::transform_reduce(g->vel[g->vel_src].begin(), g->vel[g->vel_src].end(),
                                                          Len2(), 0.0f, thrust::maximum<float>()));
    const float lo = REF_MIN_TIME_STEP, hi = REF_MAX_TIME_STEP;
    const float clamped = std::clamp(delta, lo, hi);
    if (REF_CFL_FACTOR <= 0.f) return clamped;
    if (vmax < 1.e-9) return hi;
    const float cfl = REF_CFL_FACTOR * kSpacing / vmax;
    return std::min(clamped, cfl);
}

void step(float delta) {
    const float np_delta = std::min(delta, static_cast<float>(REF_NP_MAX_TIME_STEP));
    delta = adapt_time_step(delta);
    g->last_dt = delta;
    g->last_np_dt = np_delta;
    const unsigned n = g->n;
    float4* pos_src = raw(g->pos[g->pos_src]);
    float4* pos_dst = raw(g->pos[1 - g->pos_src]);
    float4* vel_dst = raw(g->vel[1 - g->vel_src]);
    // ParticleData::sort (particle_data.cuh:112-133)
    thrust::sequence(g->idx.begin(), g->idx.end());
    const float cs = kSupport * static_cast<float>(REF_CELL_SIZE_MULT);
    thrust::transform(thrust::device_pointer_cast(pos_src), thrust::device_pointer_cast(pos_src) + n, g->keys.begin(),
                      KeyOf{cs});
    thrust::sort_by_key(g->keys.begin(), g->keys.end(), g->idx.begin());
    thrust::gather(g->idx.begin(), g->idx.end(), thrust::device_pointer_cast(pos_src),
                   thrust::device_pointer_cast(pos_dst));
    thrust::gather(g->idx.begin(), g->idx.end(), g->vel[g->vel_src].begin(), g->vel[1 - g->vel_src].begin());
    g->vel_src = 1 - g->vel_src;
    g->pos_src = 1 - g->pos_src;
    // StepTuner::launch (step_tuner.cuh:276-294)
    clear_nsearch(g->host_fluid);
    cudaMemcpy(g->dev_fluid, &g->host_fluid, sizeof(NSearchView), cudaMemcpyHostToDevice);
    refk_rebuild_fluid(g->dev_fluid, pos_dst, n, REF_BLOCK, 0);
    refk_count_neighbors(pos_dst, raw(g->nl_counts), n, g->dev_fluid, REF_BLOCK, 0);
    thrust::exclusive_scan(g->nl_counts.begin(), g->nl_counts.end(), g->nl_offsets.begin());
    refk_fill_neighbors(pos_dst, raw(g->nl_offsets), raw(g->nl_neighbors), n, g->dev_fluid, REF_BLOCK, 0);
    const void* bns = g->nb ? g->dev_boundary : nullptr;
    const float* bm = g->nb ? raw(g->bmass) : nullptr;
    refk_rho_p(pos_dst, raw(g->rho), raw(g->prs), n, g->dev_fluid, raw(g->nl_offsets), raw(g->nl_counts),
               raw(g->nl_neighbors), bm, bns, 0);
    refk_pressure(pos_dst, raw(g->rho), raw(g->prs), raw(g->ap), raw(g->normal), n, g->dev_fluid, raw(g->nl_offsets),
                  raw(g->nl_counts), raw(g->nl_neighbors), bm, bns, 0);
    refk_non_pressure(pos_dst, raw(g->rho), vel_dst, raw(g->normal), raw(g->anp), n, g->dev_fluid,
                      raw(g->nl_offsets), raw(g->nl_counts), raw(g->nl_neighbors), 0);
    refk_update_positions(pos_dst, vel_dst, raw(g->ap), raw(g->anp), n, delta, np_delta,
                          reinterpret_cast<const RefBox*>(&g->box), REF_BLOCK, 0);
}

}  // namespace

extern "C" {

// box: min[3], max[3], model[16], model_inv[16] (column-major)
int ref_set_box(const float* b) {
    if (!g) return 1;
    g->box.min = make_float4(b[0], b[1], b[2], 1.f);
    g->box.max = make_float4(b[3], b[4], b[5], 1.f);
    for (int c = 0; c < 4; ++c) {
        g->box.model[c] = make_float4(b[6 + 4 * c], b[7 + 4 * c], b[8 + 4 * c], b[9 + 4 * c]);
        g->box.model_inv[c] = make_float4(b[22 + 4 * c], b[23 + 4 * c], b[24 + 4 * c], b[25 + 4 * c]);
    }
    return 0;
}

int ref_create(const float* pos, const float* vel, unsigned n, const float* bpos, unsigned nb, const float* box,
               int device) {
    if (g) return 1;
    if (device >= 0) cudaSetDevice(device);
    if (n != REF_FLUID_N || nb != REF_BOUNDARY_N) return 2;  // tables were compiled for these sizes
    g = new Ctx();
    g->n = n;
    g->nb = nb;
    for (int k = 0; k < 2; ++k) {
        g->pos[k].resize(n + nb);
        g->vel[k].resize(n);
    }
    cudaMemcpy(raw(g->pos[0]), pos, sizeof(float4) * n, cudaMemcpyHostToDevice);
    cudaMemcpy(raw(g->pos[1]), pos, sizeof(float4) * n, cudaMemcpyHostToDevice);
    if (vel) cudaMemcpy(raw(g->vel[0]), vel, sizeof(float4) * n, cudaMemcpyHostToDevice);
    else thrust::fill(g->vel[0].begin(), g->vel[0].end(), make_float4(0.f, 0.f, 0.f, 0.f));
    g->keys.resize(n);
    g->idx.resize(n);
    g->rho.resize(n);
    g->prs.resize(n);
    g->ap.resize(n);
    g->anp.resize(n);
    g->normal.resize(n);
    g->nl_counts.resize(n);
    g->nl_offsets.resize(n);
    g->nl_neighbors.resize(static_cast<size_t>(n) * 96);
    ref_set_box(box);
    alloc_nsearch(g->host_fluid, g->dev_fluid, REF_TABLE_SIZE_MULT * REF_MIN_TABLE_SIZE, kSupport);
    if (nb) {
        // CUDASPHSimulator::init_boundary (sph.cu:84-96)
        float4* src = raw(g->pos[0]) + n;
        float4* dst = raw(g->pos[1]) + n;
        cudaMemcpy(src, bpos, sizeof(float4) * nb, cudaMemcpyHostToDevice);
        g->bkeys.resize(nb);
        g->bidx.resize(nb);
        thrust::sequence(g->bidx.begin(), g->bidx.end());
        thrust::transform(thrust::device_pointer_cast(src), thrust::device_pointer_cast(src) + nb, g->bkeys.begin(),
                          KeyOf{kSupport});
        thrust::sort_by_key(g->bkeys.begin(), g->bkeys.end(), g->bidx.begin());
        thrust::gather(g->bidx.begin(), g->bidx.end(), thrust::device_pointer_cast(src),
                       thrust::device_pointer_cast(dst));
        cudaMemcpy(src, dst, sizeof(float4) * nb, cudaMemcpyDeviceToDevice);
        alloc_nsearch(g->host_boundary, g->dev_boundary, static_cast<unsigned>(std::bit_ceil(nb)), kSupport);
        clear_nsearch(g->host_boundary);
        refk_rebuild_boundary(g->dev_boundary, dst, nb, 0);
        g->bmass.resize(nb);
        refk_boundary_mass(dst, raw(g->bmass), nb, g->dev_boundary, 0);
    }
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 3;
}

int ref_step(float delta) {
    if (!g) return 1;
    step(delta);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

int ref_synchronize() { return cudaDeviceSynchronize() == cudaSuccess ? 0 : 3; }

// Replaces the fluid state (n positions and velocities, float4) in the
// current buffers: the next step starts from it, as after a snapshot load.
int ref_set_state(const float* pos, const float* vel) {
    if (!g) return 1;
    cudaMemcpy(raw(g->pos[g->pos_src]), pos, sizeof(float4) * g->n, cudaMemcpyHostToDevice);
    cudaMemcpy(raw(g->vel[g->vel_src]), vel, sizeof(float4) * g->n, cudaMemcpyHostToDevice);
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 3;
}

// Times `k` steps with CUDA events on the default stream; boxes = NULL or
// k boxes of 38 floats (set before each step).
float ref_time_steps(int k, float delta, const float* boxes) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaDeviceSynchronize();
    cudaEventRecord(e0, 0);
    for (int s = 0; s < k; ++s) {
        if (boxes) ref_set_box(boxes + 38 * s);
        step(delta);
    }
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms;
}

// Fields of the last step in sorted order (the reference's buffers).
int ref_get_fields(float* pos, float* vel, float* rho, float* prs, float* ap, float* anp, float* normal,
                   unsigned long long* keys, unsigned* perm, unsigned* nl_counts, unsigned* nl_offsets,
                   unsigned* nl_neighbors, unsigned long long cap, unsigned long long* total, float* dt2) {
    if (!g) return 1;
    cudaDeviceSynchronize();
    const unsigned n = g->n;
    auto d2h = [](void* dst, const void* src, size_t bytes) {
        if (dst) cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
    };
    d2h(pos, raw(g->pos[g->pos_src]), sizeof(float4) * n);
    d2h(vel, raw(g->vel[g->vel_src]), sizeof(float4) * n);
    d2h(rho, raw(g->rho), sizeof(float) * n);
    d2h(prs, raw(g->prs), sizeof(float) * n);
    d2h(ap, raw(g->ap), sizeof(float4) * n);
    d2h(anp, raw(g->anp), sizeof(float4) * n);
    d2h(normal, raw(g->normal), sizeof(float4) * n);
    d2h(keys, raw(g->keys), sizeof(unsigned long long) * n);  // sorted keys
    d2h(perm, raw(g->idx), sizeof(unsigned) * n);
    d2h(nl_counts, raw(g->nl_counts), sizeof(unsigned) * n);
    d2h(nl_offsets, raw(g->nl_offsets), sizeof(unsigned) * n);
    std::vector<unsigned> c(n), o(n);
    cudaMemcpy(c.data(), raw(g->nl_counts), sizeof(unsigned) * n, cudaMemcpyDeviceToHost);
    cudaMemcpy(o.data(), raw(g->nl_offsets), sizeof(unsigned) * n, cudaMemcpyDeviceToHost);
    const unsigned long long t = n ? static_cast<unsigned long long>(o[n - 1]) + c[n - 1] : 0;
    if (total) *total = t;
    if (nl_neighbors && t <= cap) d2h(nl_neighbors, raw(g->nl_neighbors), sizeof(unsigned) * t);
    if (dt2) { dt2[0] = g->last_dt; dt2[1] = g->last_np_dt; }
    return 0;
}

int ref_get_hash(unsigned long long* table, unsigned* cstart, unsigned* cend, unsigned* table_size) {
    if (!g) return 1;
    const unsigned T = g->host_fluid.table_size;
    if (table_size) *table_size = T;
    if (table) cudaMemcpy(table, g->host_fluid.table, sizeof(unsigned long long) * T, cudaMemcpyDeviceToHost);
    if (cstart) cudaMemcpy(cstart, g->host_fluid.cell_start, sizeof(unsigned) * T, cudaMemcpyDeviceToHost);
    if (cend) cudaMemcpy(cend, g->host_fluid.cell_end, sizeof(unsigned) * T, cudaMemcpyDeviceToHost);
    return 0;
}

int ref_get_boundary(float* bpos, float* bmass) {
    if (!g) return 1;
    if (!g->nb) return 0;
    if (bpos) cudaMemcpy(bpos, raw(g->pos[g->pos_src]) + g->n, sizeof(float4) * g->nb, cudaMemcpyDeviceToHost);
    if (bmass) cudaMemcpy(bmass, raw(g->bmass), sizeof(float) * g->nb, cudaMemcpyDeviceToHost);
    return 0;
}

int ref_launches_per_step() {
    // thrust: sequence, transform, sort_by_key (~4 onesweep kernels + histogram),
    // 2 gathers, transform_reduce (2), exclusive_scan (2); memsets 3; kernels 7
    return 0;
}

void ref_destroy() {
    if (!g) return;
    cudaDeviceSynchronize();
    cudaFree(g->host_fluid.table);
    cudaFree(g->host_fluid.cell_start);
    cudaFree(g->host_fluid.cell_end);
    cudaFree(g->dev_fluid);
    if (g->dev_boundary) {
        cudaFree(g->host_boundary.table);
        cudaFree(g->host_boundary.cell_start);
        cudaFree(g->host_boundary.cell_end);
        cudaFree(g->dev_boundary);
    }
    delete g;
    g = nullptr;
}

}  // extern "C"
