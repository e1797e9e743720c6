// simulator.cuh — C++20 host side of the WCSPH step.
//
// FluidSimulator mirrors the reference's abstract solver interface
// (src/simulation/fluid_simulator.h:6-54: update(delta), reset(),
// get_fluid_particles()); CUDASPHSimulator mirrors the reference's CUDA
// solver (src/cuda/SPH/sph.cuh:14-86) and owns every device buffer of the
// step. The C ABI (capi.cu) is a thin exception-free wrapper over it.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/wcsph.h"
#include "radix_sort.cuh"
#include "step_kernels.cuh"

namespace wcsph {

// Internal error carrying an ABI status code.
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& msg) : std::runtime_error(msg), status(s) {}
};

void cuda_check(cudaError_t e, const char* what);
#define WCSPH_CUDA(call) ::wcsph::cuda_check((call), #call)

// Named NVTX range for the scope of the object (host side: the enqueue or
// launch of a stage; a profiler attached to the process shows them, and they
// cost nothing without one).
struct NvtxRange {
    explicit NvtxRange(const char* name);
    ~NvtxRange();
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Device buffer with RAII.
template <class T>
struct DevBuf {
    T* ptr = nullptr;
    size_t count = 0;
    DevBuf() = default;
    explicit DevBuf(size_t n) { alloc(n); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), count(o.count) { o.ptr = nullptr; o.count = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); ptr = o.ptr; count = o.count; o.ptr = nullptr; o.count = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t n) {
        release();
        if (n == 0) return;
        const cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
        if (e != cudaSuccess) {
            ptr = nullptr;
            throw Error(e == cudaErrorMemoryAllocation ? WCSPH_ERR_OUT_OF_MEMORY : WCSPH_ERR_CUDA,
                        std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
        }
        count = n;
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        count = 0;
    }
    size_t bytes() const { return count * sizeof(T); }
};

// Boundary candidates per cell (boundary_cells.cu): for every cell within one
// cell of an occupied boundary cell (cell size h), the boundary particles of
// its 27 neighbour cells in the (dx, dy, dz) order of the boundary loops, as
// (x, y, z, mass) runs [start, end) of x, found through the hash `table`.
struct BoundaryCells {
    DevBuf<u64> table;
    DevBuf<u32> start, end;
    DevBuf<float4> x;
    u32 size = 0;   // 0: not built (the passes then look the 27 cells up themselves)
    HashView view() const { return HashView{table.ptr, start.ptr, end.ptr, size ? size - 1 : 0}; }
};
// Builds bc from the boundary hash bh (bsize slots) of nb sorted boundary
// particles; batch: keys are (scene, cell). Leaves bc empty where the 32-bit
// run offsets would not suffice. Synchronises the stream.
void build_boundary_cells(BoundaryCells& bc, const HashView& bh, u32 bsize, u32 nb, const float4* bpos,
                          const float* bmass, bool batch, DevState* st, cudaStream_t s);

DevParams make_dev_params(const wcsph_params& p);
DevBox make_dev_box(const wcsph_box& b);
void validate_params(const wcsph_params& p);
// Host-side PARTICLE_MASS of sph.cuh:20-21 (volume computed through double).
float metric_mass(const wcsph_params& p);

// Tunable launch configuration of the step (the autotuner's search space).
struct StepConfig {
    int warps_density = 2;
    int warps_force = 4;
    int warps_surface = 2;
    int mask_words = 12;        // neighbour bit-matrix words per particle (cap = 32*words)
    int chunk = 0;              // sorted particles per warp: 8, 16, 32; 0 = by scene size
    int nbr_width = 64;         // neighbour-list slots per particle; 0 = walk the bit matrix
    float cell_size_mult = 1.f;
    uint32_t table_size_mult = 1;
    bool operator==(const StepConfig&) const = default;
};
// Particles per warp chunk of the traversal passes: the configured value, or
// 8 below 2^18 particles (more warps for small scenes) and 16 above. The
// list kernels take 32 particles per warp unless the chunk is 8.
uint32_t effective_chunk(const StepConfig& c, uint32_t n);


class FluidSimulator {
public:
    virtual ~FluidSimulator() = default;
    virtual void update(float delta) = 0;
    virtual void reset() = 0;
    virtual uint32_t get_fluid_particles() const = 0;
};

class Tuner;  // tuner.cuh
void destroy_adjoint(void* adjoint);  // adjoint.cu

class CUDASPHSimulator final : public FluidSimulator {
public:
    CUDASPHSimulator(const wcsph_params& params, const wcsph_scene& scene, int device);
    ~CUDASPHSimulator() override;

    void update(float delta) override;      // one step (graph replay when possible)
    void reset() override;
    uint32_t get_fluid_particles() const override { return n_; }
    uint32_t get_boundary_particles() const { return nb_; }

    void step_n(int n, float delta);
    float time_steps(int n, float delta);
    void synchronize();
    void set_box(const wcsph_box& box);
    void set_params(const wcsph_params& p);
    const wcsph_params& params() const { return params_; }

    void get_state(float* pos, float* vel);
    void set_state(const float* pos, const float* vel);
    void metrics(float* mean_speed, float* ke);
    void last_dt(float* dt_p, float* np_dt);

    uint64_t field_elems(int field) const;
    uint32_t field_elem_bytes(int field) const;
    void get_field(int field, void* dst, uint64_t bytes);
    void* device_field(int field);
    void get_neighbors(uint32_t* counts, uint32_t* offsets, uint32_t* nbrs, uint64_t cap, uint64_t* total);

    int kernel_timings(const char** names, float* ms, int cap);
    int launches_per_step() const;
    void render(const wcsph_camera& cam, const wcsph_render_opts& o, uint8_t* rgba, float* depth);
    // Full Morton keys (field), cell bounds and the compressed keys + histograms.
    void enqueue_keys();

    // tuning
    const StepConfig& config() const { return cfg_; }
    void apply_config(const StepConfig& c);
    void set_tuning(int searcher, float budget, const char* frozen_json);
    bool was_tuning_step() const { return was_tuning_step_; }
    void save_config(const char* path);
    void save_tuning_results(const char* path);
    void reset_tuning();

    // differentiable rollout (adjoint.cu)
    float rollout_forward(int steps, float dt, int checkpoint_every, const float* target);
    void rollout_backward(float* grad_v0, float* grad_visc, float* grad_stiff);

    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }

    // Enqueues one step without graph capture (also used inside capture).
    void enqueue_step(float delta);
    // Enqueues sort + neighbourhood search of one step on the current state.
    void enqueue_search(bool keys_from_state);
    // Traversal arguments with a fixed time step (CFL off): dt_p = dt.
    TravArgs fixed_args(float dt);
    // One step with a fixed time step (the differentiable rollout's forward).
    void enqueue_fixed_step(float dt);

private:
    void allocate();
    void init_boundary(const float* bpos);
    void upload_state(const float* pos, const float* vel);
    void check_device_errors();
    void invalidate_graph();
    TravArgs trav_args(float delta);
    u32 fluid_table_size() const;
    void ensure_tables();

    friend class Tuner;
    friend struct Adjoint;

    wcsph_params params_{};
    DevParams dp_{};
    DevBox box_host_{};
    StepConfig cfg_{};
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    uint32_t n_ = 0, nb_ = 0;
    float metric_mass_ = 0.f;

    std::vector<float> init_pos_;   // for reset()
    // fluid state: A = current state, B = sorted scratch of the running step
    DevBuf<float4> pos_a_, pos_b_, vel_a_, vel_b_;
    DevBuf<u64> keys_[3];
    DevBuf<u32> vals_[3];
    DevBuf<u32> hist_, offsets_, lookback_;
    DevBuf<u32> perm_;
    DevBuf<u64> ckey_;
    DevBuf<u64> table_;
    DevBuf<u32> cstart_, cend_;
    uint32_t table_size_ = 0;
    DevBuf<u32> mask_;
    DevBuf<u32> nbr_, nbr_cnt_;  // neighbour lists (nbr_width_ slots per particle) and counts
    u32 nbr_width_ = 0;          // list slots in use: cfg_.nbr_width, capped so n * slots < 2^32
    DevBuf<float> rho_, prs_;
    DevBuf<float4> recf_, recs_;   // neighbour records, two float4 per particle
    DevBuf<u64> ckeys_;         // order-equivalent short sort keys (radix_sort.cuh)
    DevBuf<float4> ap_, normal_, vlap_, anp_;
    DevBuf<float> partials_;
    DevBuf<unsigned long long> render_z_;
    DevBuf<u32> render_rgba_;
    DevBuf<float> render_depth_;
    DevBuf<u32> group_done_;
    DevBuf<double> group_partials_;
    DevBuf<DevState> st_;
    DevBuf<DevBox> box_dev_;
    // Box uploads between steps go through a small pinned ring so that the
    // copy is truly asynchronous (a pageable source may make the driver wait
    // for the stream); slot k is reused only after its last copy completed.
    static constexpr int kBoxSlots = 16;
    DevBox* box_pinned_ = nullptr;
    cudaEvent_t box_done_[kBoxSlots] = {};
    int box_slot_ = 0;
    float* metrics_pinned_ = nullptr;   // 2 floats: the metrics read-back
    DevBuf<float> metrics_dev_;
    // boundary
    DevBuf<float4> bpos_;
    DevBuf<float> bmass_;
    DevBuf<u64> btable_;
    DevBuf<u32> bcstart_, bcend_;
    uint32_t btable_size_ = 0;
    BoundaryCells bcells_;
    DevBuf<uint4> bmask_;   // boundary hit masks (per-cell runs)

    // CUDA graph of one step, keyed by the requested delta
    cudaGraphExec_t graph_exec_ = nullptr;
    float graph_delta_ = 0.f;
    bool graph_valid_ = false;
    bool stepped_since_state_ = false;
    bool was_tuning_step_ = false;

    std::unique_ptr<Tuner> tuner_;
    std::vector<std::pair<const char*, float>> kernel_times_;
    void* adjoint_ = nullptr;  // Adjoint*, owned
};

}  // namespace wcsph
