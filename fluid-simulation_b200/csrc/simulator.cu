// simulator.cu — CUDASPHSimulator: buffers, the step sequence, graph replay,
// parity field export. Reference orchestration: CUDASPHSimulator::update
// (src/cuda/SPH/sph.cu:31-60) -> StepTuner::launch (step_tuner.cuh:259-295).
#include "simulator.cuh"
#include "render.cuh"

#include <algorithm>
#include <bit>
#include <cmath>
#include <cstring>

#include <nvtx3/nvToolsExt.h>

#include "tuner.cuh"

namespace wcsph {

NvtxRange::NvtxRange(const char* name) { nvtxRangePushA(name); }
NvtxRange::~NvtxRange() { nvtxRangePop(); }

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? WCSPH_ERR_OUT_OF_MEMORY
                         : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? WCSPH_ERR_NO_DEVICE
                                                                                        : WCSPH_ERR_CUDA;
        throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}

void validate_params(const wcsph_params& p) {
    auto bad = [](const char* m) { throw Error(WCSPH_ERR_INVALID_ARGUMENT, m); };
    if (!(p.particle_radius > 0.f) || !std::isfinite(p.particle_radius)) bad("particle_radius must be > 0");
    if (!(p.rest_density > 0.f)) bad("rest_density must be > 0");
    if (!(p.max_density_ratio >= 1.f)) bad("max_density_ratio must be >= 1");
    if (!(p.max_time_step > 0.f) || !(p.min_time_step > 0.f) || p.min_time_step > p.max_time_step)
        bad("time step bounds must satisfy 0 < min <= max");
    const float m = p.cell_size_mult;
    if (!(m >= 0.5f && m <= 2.f)) bad("cell_size_mult must be in [0.5, 2] (neighbour range R <= 2)");
    const uint32_t t = p.table_size_mult;
    if (t == 0 || t > 64 || (t & (t - 1)) != 0) bad("table_size_mult must be a power of two in [1, 64]");
    if (p.external_force < WCSPH_FORCE_NONE || p.external_force > WCSPH_FORCE_VORTEX) bad("unknown external_force");
}

DevParams make_dev_params(const wcsph_params& p) {
    DevParams d{};
    d.radius = p.particle_radius;
    d.spacing = 2.f * d.radius;            // PARTICLE_SPACING (common.cuh:19)
    d.h = 2.f * d.spacing;                 // SUPPORT_RADIUS (common.cuh:20)
    d.h2 = d.h * d.h;
    d.inv_h = 1.f / d.h;
    d.cell_size = d.h * p.cell_size_mult;  // cell_size * cell_size_mult (particle_data.cuh:116)
    const float volume = d.spacing * d.spacing * d.spacing * 0.8f;  // common.cuh:22
    d.mass = p.rest_density * volume;      // common.cuh:23
    d.rest_density = p.rest_density;
    d.stiffness = p.stiffness;
    d.exponent = p.exponent;
    d.max_density_ratio = p.max_density_ratio;
    d.viscosity = p.viscosity;
    d.surface_tension = p.surface_tension;
    for (int k = 0; k < 3; ++k) d.gravity[k] = p.gravity[k];
    d.collision_buffer = d.radius * p.collision_buffer_mult;  // update_positions.cu:20
    d.elasticity = p.elasticity;
    const float h3 = PI_F * d.h * d.h * d.h;  // PI * h * h * h (kernel.cuh:13)
    d.cubic_factor = 8.f / h3;
    d.w0 = d.cubic_factor;                  // cubic_spline(0, h) = factor * 1
    d.cubic_grad_factor = 48.f / h3;        // kernel.cuh:26
    d.spiky_grad_factor = -45.f / (PI_F * std::pow(d.h, 9.f));  // kernel.cuh:47
    d.cohesion_factor = 32.f / h3;          // kernel.cuh:54
    d.visc_eps = 0.01f * d.h * d.h;         // compute_non_pressure_accel.cu:142
    d.visc_scale = p.viscosity * 10.f * d.mass;
    d.st_scale = p.surface_tension * 2.f * p.rest_density;
    d.rest_density2 = p.rest_density * p.rest_density;
    d.range = static_cast<int>(d.h / d.cell_size + .5f);  // common.cuh:131
    d.force_field = p.external_force;
    for (int k = 0; k < 4; ++k) d.force_param[k] = p.external_force_param[k];
    return d;
}

uint32_t effective_chunk(const StepConfig& c, uint32_t n) {
    if (c.chunk == 8 || c.chunk == 16 || c.chunk == 32) return static_cast<uint32_t>(c.chunk);
    return n < (1u << 18) ? 8u : 16u;
}

float metric_mass(const wcsph_params& p) {
    const float s = 2.f * p.particle_radius;
    const float volume = static_cast<float>(static_cast<double>(s * s * s) * 0.8);  // sph.cuh:20
    return p.rest_density * volume;
}

DevBox make_dev_box(const wcsph_box& b) {
    DevBox d{};
    d.min = make_float4(b.min[0], b.min[1], b.min[2], 1.f);
    d.max = make_float4(b.max[0], b.max[1], b.max[2], 1.f);
    for (int c = 0; c < 4; ++c) {
        d.model[c] = make_float4(b.model[4 * c], b.model[4 * c + 1], b.model[4 * c + 2], b.model[4 * c + 3]);
        d.model_inv[c] =
            make_float4(b.model_inv[4 * c], b.model_inv[4 * c + 1], b.model_inv[4 * c + 2], b.model_inv[4 * c + 3]);
    }
    return d;
}

// --------------------------------------------------------------------------
CUDASPHSimulator::CUDASPHSimulator(const wcsph_params& params, const wcsph_scene& scene, int device) {
    validate_params(params);
    if (scene.fluid_n == 0 || scene.fluid_pos == nullptr)
        throw Error(WCSPH_ERR_INVALID_ARGUMENT, "scene needs fluid_n > 0 and fluid_pos");
    if (scene.fluid_n >= (1u << 30)) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "fluid_n must be < 2^30");
    if (scene.boundary_n > 0 && scene.boundary_pos == nullptr)
        throw Error(WCSPH_ERR_INVALID_ARGUMENT, "boundary_n > 0 needs boundary_pos");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        throw Error(WCSPH_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0) WCSPH_CUDA(cudaGetDevice(&device));
    if (device >= count) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "device index out of range");
    device_ = device;
    WCSPH_CUDA(cudaSetDevice(device_));
    WCSPH_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));

    params_ = params;
    dp_ = make_dev_params(params_);
    metric_mass_ = metric_mass(params_);
    box_host_ = make_dev_box(scene.box);
    cfg_.cell_size_mult = params_.cell_size_mult;
    cfg_.table_size_mult = params_.table_size_mult;
    n_ = scene.fluid_n;
    nb_ = scene.boundary_n;
    init_pos_.assign(scene.fluid_pos, scene.fluid_pos + 4ull * n_);

    allocate();
    if (nb_ > 0) init_boundary(scene.boundary_pos);
    upload_state(scene.fluid_pos, scene.fluid_vel);
    WCSPH_CUDA(cudaStreamSynchronize(stream_));
    tuner_ = std::make_unique<Tuner>(this);
}

CUDASPHSimulator::~CUDASPHSimulator() {
    destroy_adjoint(adjoint_);
    adjoint_ = nullptr;
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (stream_) {
        cudaStreamSynchronize(stream_);
        cudaStreamDestroy(stream_);
    }
    for (cudaEvent_t e : box_done_)
        if (e) cudaEventDestroy(e);
    if (box_pinned_) cudaFreeHost(box_pinned_);
    if (metrics_pinned_) cudaFreeHost(metrics_pinned_);
    tuner_.reset();
}

u32 CUDASPHSimulator::fluid_table_size() const {
    // MIN_TABLE_SIZE = bit_ceil(N)/4 (step_tuner.cuh:20) times TABLE_SIZE_MULT.
    const uint64_t min_size = std::max<uint64_t>(std::bit_ceil(static_cast<uint64_t>(n_)) / 4, 64);
    return static_cast<u32>(min_size * cfg_.table_size_mult);
}

void CUDASPHSimulator::allocate() {
    const size_t n = n_;
    pos_a_.alloc(n); pos_b_.alloc(n); vel_a_.alloc(n); vel_b_.alloc(n);
    for (auto& k : keys_) k.alloc(n);
    vals_[1].alloc(n); vals_[2].alloc(n);
    hist_.alloc(SORT_DIGITS * 256);
    offsets_.alloc(SORT_DIGITS * 256);
    lookback_.alloc(static_cast<size_t>(SORT_DIGITS) * sort_tiles(n_) * 256);
    perm_.alloc(n); ckey_.alloc(n); ckeys_.alloc(n);
    rho_.alloc(n); prs_.alloc(n); recf_.alloc(2 * n); recs_.alloc(2 * n);
    ap_.alloc(n); normal_.alloc(n); vlap_.alloc(n); anp_.alloc(n);
    st_.alloc(1); box_dev_.alloc(1); metrics_dev_.alloc(2);
    partials_.alloc(2ull * pass_max_warps(n_));
    group_done_.alloc(pass_max_warps(n_) / 32u + 1u);
    group_partials_.alloc(2ull * (pass_max_warps(n_) / 32u + 1u));
    WCSPH_CUDA(cudaMemsetAsync(group_done_.ptr, 0, group_done_.bytes(), stream_));
    // Index buffers start as zeros (valid indices): a step whose sort fails
    // leaves them as they were, and nothing may then read an index past n.
    WCSPH_CUDA(cudaMemsetAsync(vals_[1].ptr, 0, vals_[1].bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(vals_[2].ptr, 0, vals_[2].bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(perm_.ptr, 0, perm_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(ckey_.ptr, 0, ckey_.bytes(), stream_));
    ensure_tables();
    WCSPH_CUDA(cudaMemsetAsync(hist_.ptr, 0, hist_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(st_.ptr, 0, sizeof(DevState), stream_));
    WCSPH_CUDA(cudaMemsetAsync(rho_.ptr, 0, rho_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(prs_.ptr, 0, prs_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(ap_.ptr, 0, ap_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(anp_.ptr, 0, anp_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(normal_.ptr, 0, normal_.bytes(), stream_));
    WCSPH_CUDA(cudaMemcpyAsync(box_dev_.ptr, &box_host_, sizeof(DevBox), cudaMemcpyHostToDevice, stream_));
}

void CUDASPHSimulator::ensure_tables() {
    const u32 t = fluid_table_size();
    if (t != table_size_) {
        table_.alloc(t); cstart_.alloc(t); cend_.alloc(t);
        table_size_ = t;
        WCSPH_CUDA(cudaMemsetAsync(table_.ptr, 0xff, table_.bytes(), stream_));
        WCSPH_CUDA(cudaMemsetAsync(cstart_.ptr, 0, cstart_.bytes(), stream_));
        WCSPH_CUDA(cudaMemsetAsync(cend_.ptr, 0, cend_.bytes(), stream_));
    }
    const size_t words = static_cast<size_t>(n_) * static_cast<size_t>(cfg_.mask_words);
    if (mask_.count != words) {
        mask_.alloc(words);
        WCSPH_CUDA(cudaMemsetAsync(mask_.ptr, 0, mask_.bytes(), stream_));
    }
    // list slots are addressed with 32-bit indices: very large scenes get
    // fewer slots (rows that do not fit are recomputed), or none below 8
    uint64_t width = static_cast<uint64_t>(cfg_.nbr_width);
    if (n_ > 0) width = std::min<uint64_t>(width, ((1ull << 32) - 1) / n_);
    nbr_width_ = width >= 8 ? static_cast<u32>(width) : 0u;
    const size_t slots = static_cast<size_t>(n_) * nbr_width_;
    if (nbr_.count != slots) {
        nbr_.alloc(slots);
        WCSPH_CUDA(cudaMemsetAsync(nbr_.ptr, 0, nbr_.bytes(), stream_));
    }
    const size_t counts = nbr_width_ > 0 ? n_ : 0;
    if (nbr_cnt_.count != counts) {
        nbr_cnt_.alloc(counts);
        WCSPH_CUDA(cudaMemsetAsync(nbr_cnt_.ptr, 0, nbr_cnt_.bytes(), stream_));
    }
}

// Boundary: Morton-sort once, hash (cell = h) and Akinci masses
// (sort_boundary particle_data.cuh:84-110, build_boundary_n_search
// sph.cu:98-103, compute_boundary_mass.cu:10-30).
void CUDASPHSimulator::init_boundary(const float* bpos_host) {
    const u32 nb = nb_;
    DevBuf<float4> tmp(nb);
    WCSPH_CUDA(cudaMemcpyAsync(tmp.ptr, bpos_host, sizeof(float4) * nb, cudaMemcpyHostToDevice, stream_));
    SortBuffers sb{};
    DevBuf<u64> k[3];
    DevBuf<u32> v[3];
    for (auto& x : k) x.alloc(nb);
    v[1].alloc(nb); v[2].alloc(nb);
    DevBuf<u32> lb(static_cast<size_t>(SORT_DIGITS) * sort_tiles(nb) * 256);
    for (int i = 0; i < 3; ++i) { sb.keys[i] = k[i].ptr; sb.vals[i] = v[i].ptr; }
    sb.hist = hist_.ptr; sb.offsets = offsets_.ptr; sb.lookback = lb.ptr; sb.capacity = nb;
    keys_hist_kernel<<<std::min<u32>((nb + 255) / 256, 1184), 256, 0, stream_>>>(tmp.ptr, nb, dp_.h, k[0].ptr,
                                                                                 hist_.ptr);
    WCSPH_CUDA(cudaGetLastError());
    WCSPH_CUDA(enqueue_sort_passes(sb, nb, st_.ptr, stream_));
    btable_size_ = std::max<u32>(std::bit_ceil(nb), 64u);
    btable_.alloc(btable_size_); bcstart_.alloc(btable_size_); bcend_.alloc(btable_size_);
    WCSPH_CUDA(cudaMemsetAsync(btable_.ptr, 0xff, btable_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(bcstart_.ptr, 0, bcstart_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(bcend_.ptr, 0, bcend_.bytes(), stream_));
    bpos_.alloc(nb);
    bmass_.alloc(nb);
    DevBuf<u32> bperm(nb);
    DevBuf<u64> bckey(nb);
    launch_reorder_cells(tmp.ptr, nullptr, v[1].ptr, v[2].ptr, st_.ptr, nb, dp_.h, bpos_.ptr, nullptr, bperm.ptr,
                         bckey.ptr, btable_.ptr, bcstart_.ptr, bcend_.ptr, btable_size_ - 1, st_.ptr, stream_);
    WCSPH_CUDA(cudaGetLastError());
    HashView bh{btable_.ptr, bcstart_.ptr, bcend_.ptr, btable_size_ - 1};
    launch_boundary_mass(dp_, bpos_.ptr, nb, bh, bmass_.ptr, stream_);
    WCSPH_CUDA(cudaGetLastError());
    build_boundary_cells(bcells_, bh, btable_size_, nb, bpos_.ptr, bmass_.ptr, false, st_.ptr, stream_);
    if (bcells_.size) bmask_.alloc(n_);
    WCSPH_CUDA(cudaStreamSynchronize(stream_));
    check_device_errors();
}

void CUDASPHSimulator::upload_state(const float* pos, const float* vel) {
    WCSPH_CUDA(cudaMemcpyAsync(pos_a_.ptr, pos, sizeof(float4) * n_, cudaMemcpyHostToDevice, stream_));
    WCSPH_CUDA(cudaMemcpyAsync(pos_b_.ptr, pos, sizeof(float4) * n_, cudaMemcpyHostToDevice, stream_));
    if (vel) WCSPH_CUDA(cudaMemcpyAsync(vel_a_.ptr, vel, sizeof(float4) * n_, cudaMemcpyHostToDevice, stream_));
    else WCSPH_CUDA(cudaMemsetAsync(vel_a_.ptr, 0, sizeof(float4) * n_, stream_));
    // fresh CFL maximum of the new state
    DevState* st = st_.ptr;
    WCSPH_CUDA(cudaMemsetAsync(&st->vmax2_bits[0], 0, sizeof(u32) * 2, stream_));
    launch_init_cfl(vel_a_.ptr, n_, st, stream_);
    WCSPH_CUDA(cudaGetLastError());
    stepped_since_state_ = false;
}

void CUDASPHSimulator::check_device_errors() {
    u32 flags = 0;
    WCSPH_CUDA(cudaMemcpy(&flags, &st_.ptr->error_flags, sizeof(u32), cudaMemcpyDeviceToHost));
    if (flags) {
        WCSPH_CUDA(cudaMemset(&st_.ptr->error_flags, 0, sizeof(u32)));
        if (flags & ERR_HASH_FULL) throw Error(WCSPH_ERR_HASH_FULL, "spatial hash table is full (raise table_size_mult)");
        if (flags & ERR_LOOKBACK_TIMEOUT) throw Error(WCSPH_ERR_DEVICE_TIMEOUT, "radix sort look-back wait timed out");
        if (flags & ERR_CAND_OVERFLOW) throw Error(WCSPH_ERR_NEIGHBOR_OVERFLOW, "boundary candidate cells exceed capacity");
        if (flags & ERR_BOUNDS) throw Error(WCSPH_ERR_BOUNDS, "device index out of bounds (bounds-checked build)");
    }
}

TravArgs CUDASPHSimulator::trav_args(float delta) {
    TravArgs a{};
    a.n = n_;
    a.pos = pos_b_.ptr;
    a.vel = vel_b_.ptr;
    a.ckey = ckey_.ptr;
    a.fluid = HashView{table_.ptr, cstart_.ptr, cend_.ptr, table_size_ - 1};
    a.range = dp_.range;
    a.nb = nb_;
    a.bpos = bpos_.ptr;
    a.bmass = bmass_.ptr;
    a.boundary = HashView{btable_.ptr, bcstart_.ptr, bcend_.ptr, btable_size_ ? btable_size_ - 1 : 0};
    a.bcell = bcells_.view();
    a.bcx = bcells_.x.ptr;
    a.bcx_n = static_cast<u32>(bcells_.x.count);
    // the density pass writes the masks where it reads the runs (cell size h);
    // they are built in its bit-matrix scratch (4 words per row)
    a.bmask = (bcells_.size && cfg_.mask_words >= 4 && dp_.cell_size == dp_.h) ? bmask_.ptr : nullptr;
    a.mask = mask_.ptr;
    a.mask_words = static_cast<u32>(cfg_.mask_words);
    a.chunk = effective_chunk(cfg_, n_);
    a.nbr = nbr_width_ > 0 ? nbr_.ptr : nullptr;
    a.pair_cells = a.nbr != nullptr ? 1u : 0u;   // the lists replace the kept bit matrix
    a.matrix_valid = 0u;
    a.nbr_cnt = nbr_cnt_.ptr;
    a.nbr_width = nbr_width_;
    a.rho = rho_.ptr; a.prs = prs_.ptr;
    a.recf = recf_.ptr; a.recs = recs_.ptr;
    a.ap = ap_.ptr; a.normal = normal_.ptr; a.vlap = vlap_.ptr; a.anp = anp_.ptr;
    a.pos_out = pos_a_.ptr; a.vel_out = vel_a_.ptr;
    a.box = box_dev_.ptr;
    a.st = st_.ptr;
    a.delta = delta;
    a.cfl_factor = params_.cfl_factor;
    a.max_dt = params_.max_time_step;
    a.min_dt = params_.min_time_step;
    a.np_max_dt = params_.non_pressure_max_time_step;
    a.metric_mass = metric_mass_;
    a.block_partials = partials_.ptr;
    a.group_done = group_done_.ptr;
    a.group_partials = group_partials_.ptr;
    return a;
}

void CUDASPHSimulator::enqueue_search(bool keys_from_state) {
    NvtxRange r("wcsph sort + neighbourhood search");
    const u32 n = n_;
    WCSPH_CUDA(cudaMemsetAsync(table_.ptr, 0xff, table_.bytes(), stream_));
    if (keys_from_state) enqueue_keys();
    SortBuffers sb{};
    for (int i = 0; i < 3; ++i) { sb.keys[i] = keys_[i].ptr; sb.vals[i] = vals_[i].ptr; }
    sb.keys[0] = ckeys_.ptr;   // the sort reads the compressed keys; keys_[0] keeps the field
    sb.hist = hist_.ptr; sb.offsets = offsets_.ptr; sb.lookback = lookback_.ptr; sb.capacity = n;
    WCSPH_CUDA(enqueue_sort_passes(sb, n, st_.ptr, stream_));
    launch_reorder_cells(pos_a_.ptr, vel_a_.ptr, vals_[1].ptr, vals_[2].ptr, st_.ptr, n, dp_.cell_size, pos_b_.ptr,
                         vel_b_.ptr, perm_.ptr, ckey_.ptr, table_.ptr, cstart_.ptr, cend_.ptr, table_size_ - 1,
                         st_.ptr, stream_);
}

void CUDASPHSimulator::enqueue_keys() {
    const u32 n = n_;
    // four blocks per SM: each flushes its histograms / bounds with global
    // atomics on shared addresses, so fewer blocks mean fewer atomics, more
    // blocks more loads in flight (two per SM: 4 us more for the histograms)
    const u32 blocks = std::min<u32>((n + 255) / 256, 592);
    keys_bounds_kernel<<<blocks, 256, 0, stream_>>>(pos_a_.ptr, n, dp_.cell_size, keys_[0].ptr, st_.ptr);
    compressed_keys_hist_kernel<<<blocks, 256, 0, stream_>>>(pos_a_.ptr, n, dp_.cell_size, st_.ptr, ckeys_.ptr,
                                                             hist_.ptr);
}

TravArgs CUDASPHSimulator::fixed_args(float dt) {
    TravArgs a = trav_args(dt);
    a.cfl_factor = 0.f;
    a.max_dt = dt;
    a.min_dt = dt;
    a.pair_cells = 0u;   // the adjoint passes walk each step's kept bit matrix
    return a;
}

void CUDASPHSimulator::enqueue_fixed_step(float dt) {
    enqueue_search(true);
    const TravArgs a = fixed_args(dt);
    launch_pass(PASS_DENSITY, dp_, a, stream_, cfg_.warps_density);
    launch_pass(PASS_FORCE, dp_, a, stream_, cfg_.warps_force);
    launch_pass(PASS_SURFACE, dp_, a, stream_, cfg_.warps_surface);
}

void CUDASPHSimulator::enqueue_step(float delta) {
    NvtxRange r("wcsph step");
    enqueue_search(true);
    const TravArgs a = trav_args(delta);
    {
        NvtxRange rd("wcsph density pass");
        launch_pass(PASS_DENSITY, dp_, a, stream_, cfg_.warps_density);
    }
    {
        NvtxRange rf("wcsph force pass");
        launch_pass(PASS_FORCE, dp_, a, stream_, cfg_.warps_force);
    }
    {
        NvtxRange rs("wcsph surface + integrate pass");
        launch_pass(PASS_SURFACE, dp_, a, stream_, cfg_.warps_surface);
    }
}

int CUDASPHSimulator::launches_per_step() const {
    // keys_bounds + compressed_keys_hist + sort_plan + 8 onesweep + reorder_cells + 3 cell passes
    return 2 + 1 + SORT_DIGITS + 1 + 3;
}

void CUDASPHSimulator::invalidate_graph() {
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    graph_exec_ = nullptr;
    graph_valid_ = false;
}

void CUDASPHSimulator::update(float delta) {
    was_tuning_step_ = false;
    if (tuner_ && tuner_->active()) {
        was_tuning_step_ = tuner_->before_step();
    }
    if (was_tuning_step_) {
        tuner_->timed_step(delta);
    } else {
        step_n(1, delta);
    }
    stepped_since_state_ = true;
}

void CUDASPHSimulator::step_n(int n, float delta) {
    NvtxRange r("wcsph step_n (graph replay)");
    if (n <= 0) return;
    if (!graph_valid_ || graph_delta_ != delta) {
        invalidate_graph();
        cudaGraph_t g = nullptr;
        WCSPH_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_step(delta);
        } catch (...) {
            cudaStreamEndCapture(stream_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        WCSPH_CUDA(cudaStreamEndCapture(stream_, &g));
        const cudaError_t e = cudaGraphInstantiate(&graph_exec_, g, 0);
        cudaGraphDestroy(g);
        WCSPH_CUDA(e);
        graph_delta_ = delta;
        graph_valid_ = true;
    }
    for (int i = 0; i < n; ++i) WCSPH_CUDA(cudaGraphLaunch(graph_exec_, stream_));
    stepped_since_state_ = true;
}

float CUDASPHSimulator::time_steps(int n, float delta) {
    step_n(0, delta);
    cudaEvent_t e0, e1;
    WCSPH_CUDA(cudaEventCreate(&e0));
    WCSPH_CUDA(cudaEventCreate(&e1));
    // make sure the graph exists before the timed region
    if (!graph_valid_ || graph_delta_ != delta) { step_n(1, delta); }
    WCSPH_CUDA(cudaEventRecord(e0, stream_));
    step_n(n, delta);
    WCSPH_CUDA(cudaEventRecord(e1, stream_));
    WCSPH_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    WCSPH_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_device_errors();
    return ms;
}

void CUDASPHSimulator::synchronize() {
    WCSPH_CUDA(cudaStreamSynchronize(stream_));
    check_device_errors();
}

void CUDASPHSimulator::set_box(const wcsph_box& box) {
    box_host_ = make_dev_box(box);
    if (!box_pinned_) {
        WCSPH_CUDA(cudaMallocHost(&box_pinned_, sizeof(DevBox) * kBoxSlots));
        for (cudaEvent_t& e : box_done_) WCSPH_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const int k = box_slot_;
    box_slot_ = (box_slot_ + 1) % kBoxSlots;
    WCSPH_CUDA(cudaEventSynchronize(box_done_[k]));   // returns at once for a never-recorded event
    box_pinned_[k] = box_host_;
    WCSPH_CUDA(cudaMemcpyAsync(box_dev_.ptr, box_pinned_ + k, sizeof(DevBox), cudaMemcpyHostToDevice, stream_));
    WCSPH_CUDA(cudaEventRecord(box_done_[k], stream_));
}

void CUDASPHSimulator::set_params(const wcsph_params& p) {
    validate_params(p);
    if (p.particle_radius != params_.particle_radius)
        throw Error(WCSPH_ERR_INVALID_ARGUMENT, "particle_radius cannot change after creation");
    params_ = p;
    dp_ = make_dev_params(params_);
    metric_mass_ = metric_mass(params_);
    if (p.cell_size_mult != cfg_.cell_size_mult || p.table_size_mult != cfg_.table_size_mult) {
        StepConfig c = cfg_;
        c.cell_size_mult = p.cell_size_mult;
        c.table_size_mult = p.table_size_mult;
        apply_config(c);
    }
    invalidate_graph();
    if (nb_ > 0) {  // boundary masses depend on rest density
        HashView bh{btable_.ptr, bcstart_.ptr, bcend_.ptr, btable_size_ - 1};
        launch_boundary_mass(dp_, bpos_.ptr, nb_, bh, bmass_.ptr, stream_);
        WCSPH_CUDA(cudaGetLastError());
        // the per-cell candidate runs carry copies of the masses
        build_boundary_cells(bcells_, bh, btable_size_, nb_, bpos_.ptr, bmass_.ptr, false, st_.ptr, stream_);
    }
}

void CUDASPHSimulator::apply_config(const StepConfig& c) {
    if (c == cfg_) return;
    if (c.mask_words < 1 || c.mask_words > 16) throw Error(WCSPH_ERR_CONFIG, "mask_words must be in [1, 16]");
    if (c.chunk != 0 && c.chunk != 8 && c.chunk != 16 && c.chunk != 32)
        throw Error(WCSPH_ERR_CONFIG, "particles_per_warp must be 8, 16 or 32");
    if (c.nbr_width < 0 || c.nbr_width > 1024)
        throw Error(WCSPH_ERR_CONFIG, "neighbour_list_width must be in [0, 1024]");
    cfg_ = c;
    params_.cell_size_mult = c.cell_size_mult;
    params_.table_size_mult = c.table_size_mult;
    dp_ = make_dev_params(params_);
    ensure_tables();
    invalidate_graph();
}

void CUDASPHSimulator::get_state(float* pos, float* vel) {
    if (pos) WCSPH_CUDA(cudaMemcpyAsync(pos, pos_a_.ptr, sizeof(float4) * n_, cudaMemcpyDeviceToHost, stream_));
    if (vel) WCSPH_CUDA(cudaMemcpyAsync(vel, vel_a_.ptr, sizeof(float4) * n_, cudaMemcpyDeviceToHost, stream_));
    synchronize();
}

void CUDASPHSimulator::set_state(const float* pos, const float* vel) {
    if (!pos) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "set_state needs positions");
    upload_state(pos, vel);
    synchronize();
}

void CUDASPHSimulator::reset() {
    // CUDASPHSimulator::reset (sph.cu:73-82): initial lattice, zero velocity,
    // zero density / pressure / non-pressure accel / normals.
    upload_state(init_pos_.data(), nullptr);
    WCSPH_CUDA(cudaMemsetAsync(rho_.ptr, 0, rho_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(prs_.ptr, 0, prs_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(anp_.ptr, 0, anp_.bytes(), stream_));
    WCSPH_CUDA(cudaMemsetAsync(normal_.ptr, 0, normal_.bytes(), stream_));
    synchronize();
}

void CUDASPHSimulator::metrics(float* mean_speed, float* ke) {
    // read back through a small pinned buffer: a pageable destination would
    // be staged by the driver on every call (this is read once per step)
    if (!metrics_pinned_) WCSPH_CUDA(cudaMallocHost(&metrics_pinned_, sizeof(float) * 2));
    float* host = metrics_pinned_;
    if (stepped_since_state_) {
        WCSPH_CUDA(cudaMemcpyAsync(host, &st_.ptr->last_mean_speed, sizeof(float) * 2, cudaMemcpyDeviceToHost,
                                   stream_));
    } else {
        launch_metrics(vel_a_.ptr, n_, metric_mass_, metrics_dev_.ptr, stream_);
        WCSPH_CUDA(cudaGetLastError());
        WCSPH_CUDA(cudaMemcpyAsync(host, metrics_dev_.ptr, sizeof(float) * 2, cudaMemcpyDeviceToHost, stream_));
    }
    synchronize();
    if (mean_speed) *mean_speed = host[0];
    if (ke) *ke = host[1];
}

void CUDASPHSimulator::last_dt(float* dt_p, float* np_dt) {
    float host[2];
    WCSPH_CUDA(cudaMemcpyAsync(host, &st_.ptr->last_dt_p, sizeof(float) * 2, cudaMemcpyDeviceToHost, stream_));
    synchronize();
    if (dt_p) *dt_p = host[0];
    if (np_dt) *np_dt = host[1];
}

uint64_t CUDASPHSimulator::field_elems(int f) const {
    switch (f) {
    case WCSPH_FIELD_HASH_TABLE: case WCSPH_FIELD_HASH_CELL_START: case WCSPH_FIELD_HASH_CELL_END:
        return table_size_;
    case WCSPH_FIELD_BOUNDARY_POSITION: case WCSPH_FIELD_BOUNDARY_MASS:
        return nb_;
    default:
        if (f < 0 || f >= WCSPH_FIELD_COUNT_) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "unknown field");
        return n_;
    }
}

uint32_t CUDASPHSimulator::field_elem_bytes(int f) const {
    switch (f) {
    case WCSPH_FIELD_POSITION: case WCSPH_FIELD_VELOCITY: case WCSPH_FIELD_PRESSURE_ACCEL:
    case WCSPH_FIELD_NON_PRESSURE_ACCEL: case WCSPH_FIELD_NORMAL: case WCSPH_FIELD_BOUNDARY_POSITION:
        return 16;
    case WCSPH_FIELD_MORTON_KEYS: case WCSPH_FIELD_HASH_TABLE:
        return 8;
    case WCSPH_FIELD_DENSITY: case WCSPH_FIELD_PRESSURE: case WCSPH_FIELD_PERMUTATION:
    case WCSPH_FIELD_HASH_CELL_START: case WCSPH_FIELD_HASH_CELL_END: case WCSPH_FIELD_BOUNDARY_MASS:
        return 4;
    default:
        throw Error(WCSPH_ERR_INVALID_ARGUMENT, "unknown field");
    }
}

void* CUDASPHSimulator::device_field(int f) {
    switch (f) {
    case WCSPH_FIELD_POSITION: return pos_a_.ptr;
    case WCSPH_FIELD_VELOCITY: return vel_a_.ptr;
    case WCSPH_FIELD_DENSITY: return rho_.ptr;
    case WCSPH_FIELD_PRESSURE: return prs_.ptr;
    case WCSPH_FIELD_PRESSURE_ACCEL: return ap_.ptr;
    case WCSPH_FIELD_NON_PRESSURE_ACCEL: return anp_.ptr;
    case WCSPH_FIELD_NORMAL: return normal_.ptr;
    case WCSPH_FIELD_MORTON_KEYS: return keys_[0].ptr;
    case WCSPH_FIELD_PERMUTATION: return perm_.ptr;
    case WCSPH_FIELD_HASH_TABLE: return table_.ptr;
    case WCSPH_FIELD_HASH_CELL_START: return cstart_.ptr;
    case WCSPH_FIELD_HASH_CELL_END: return cend_.ptr;
    case WCSPH_FIELD_BOUNDARY_POSITION: return bpos_.ptr;
    case WCSPH_FIELD_BOUNDARY_MASS: return bmass_.ptr;
    default: throw Error(WCSPH_ERR_INVALID_ARGUMENT, "unknown field");
    }
}

void CUDASPHSimulator::get_field(int f, void* dst, uint64_t bytes) {
    const uint64_t need = field_elems(f) * field_elem_bytes(f);
    if (bytes < need) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "destination buffer too small");
    if (need == 0) return;
    WCSPH_CUDA(cudaMemcpyAsync(dst, device_field(f), need, cudaMemcpyDeviceToHost, stream_));
    synchronize();
    if (f == WCSPH_FIELD_HASH_CELL_START || f == WCSPH_FIELD_HASH_CELL_END) {
        // empty slots read 0 as after clear_n_search (nsearch.cuh:26-30)
        std::vector<u64> t(table_size_);
        WCSPH_CUDA(cudaMemcpy(t.data(), table_.ptr, sizeof(u64) * table_size_, cudaMemcpyDeviceToHost));
        u32* out = static_cast<u32*>(dst);
        for (u32 s = 0; s < table_size_; ++s)
            if (t[s] == EMPTY_HASH) out[s] = 0;
    }
}

void CUDASPHSimulator::get_neighbors(uint32_t* counts, uint32_t* offsets, uint32_t* nbrs, uint64_t cap,
                                     uint64_t* total) {
    if (!stepped_since_state_) throw Error(WCSPH_ERR_STATE, "no step has run since the state was set");
    DevBuf<u32> dcounts(n_), doffsets(n_);
    DevBuf<u32> dn(std::max<uint64_t>(cap, 1));
    TravArgs a = trav_args(0.f);
    a.counts = dcounts.ptr;
    launch_pass(PASS_COUNT, dp_, a, stream_, 4);
    WCSPH_CUDA(cudaGetLastError());
    std::vector<u32> hc(n_), ho(n_);
    WCSPH_CUDA(cudaMemcpyAsync(hc.data(), dcounts.ptr, sizeof(u32) * n_, cudaMemcpyDeviceToHost, stream_));
    synchronize();
    uint64_t run = 0;
    for (u32 i = 0; i < n_; ++i) { ho[i] = static_cast<u32>(run); run += hc[i]; }
    if (total) *total = run;
    if (counts) std::memcpy(counts, hc.data(), sizeof(u32) * n_);
    if (offsets) std::memcpy(offsets, ho.data(), sizeof(u32) * n_);
    if (run > cap) throw Error(WCSPH_ERR_NEIGHBOR_OVERFLOW, "neighbour capacity exceeded");
    if (!nbrs) return;
    WCSPH_CUDA(cudaMemcpyAsync(doffsets.ptr, ho.data(), sizeof(u32) * n_, cudaMemcpyHostToDevice, stream_));
    a.offsets = doffsets.ptr;
    a.nbr_out = dn.ptr;
    a.nbr_capacity = cap;
    launch_pass(PASS_FILL, dp_, a, stream_, 4);
    WCSPH_CUDA(cudaGetLastError());
    if (run) WCSPH_CUDA(cudaMemcpyAsync(nbrs, dn.ptr, sizeof(u32) * run, cudaMemcpyDeviceToHost, stream_));
    synchronize();
}

int CUDASPHSimulator::kernel_timings(const char** names, float* ms, int cap) {
    // One step launched stage by stage with events between stages.
    static const char* kStages[] = {"keys_hist", "radix_sort", "reorder_cells", "density_pass", "force_pass",
                                    "surface_integrate_pass"};
    constexpr int NS = 6;
    cudaEvent_t ev[NS + 1];
    for (auto& e : ev) WCSPH_CUDA(cudaEventCreate(&e));
    const float delta = graph_valid_ ? graph_delta_ : params_.max_time_step;
    const u32 n = n_;
    WCSPH_CUDA(cudaEventRecord(ev[0], stream_));
    WCSPH_CUDA(cudaMemsetAsync(table_.ptr, 0xff, table_.bytes(), stream_));
    enqueue_keys();
    WCSPH_CUDA(cudaEventRecord(ev[1], stream_));
    SortBuffers sb{};
    for (int i = 0; i < 3; ++i) { sb.keys[i] = keys_[i].ptr; sb.vals[i] = vals_[i].ptr; }
    sb.keys[0] = ckeys_.ptr;
    sb.hist = hist_.ptr; sb.offsets = offsets_.ptr; sb.lookback = lookback_.ptr; sb.capacity = n;
    WCSPH_CUDA(enqueue_sort_passes(sb, n, st_.ptr, stream_));
    WCSPH_CUDA(cudaEventRecord(ev[2], stream_));
    launch_reorder_cells(pos_a_.ptr, vel_a_.ptr, vals_[1].ptr, vals_[2].ptr, st_.ptr, n, dp_.cell_size, pos_b_.ptr,
                         vel_b_.ptr, perm_.ptr, ckey_.ptr, table_.ptr, cstart_.ptr, cend_.ptr, table_size_ - 1,
                         st_.ptr, stream_);
    WCSPH_CUDA(cudaEventRecord(ev[3], stream_));
    const TravArgs a = trav_args(delta);
    launch_pass(PASS_DENSITY, dp_, a, stream_, cfg_.warps_density);
    WCSPH_CUDA(cudaEventRecord(ev[4], stream_));
    launch_pass(PASS_FORCE, dp_, a, stream_, cfg_.warps_force);
    WCSPH_CUDA(cudaEventRecord(ev[5], stream_));
    launch_pass(PASS_SURFACE, dp_, a, stream_, cfg_.warps_surface);
    WCSPH_CUDA(cudaEventRecord(ev[6], stream_));
    WCSPH_CUDA(cudaEventSynchronize(ev[NS]));
    kernel_times_.clear();
    for (int s = 0; s < NS; ++s) {
        float t = 0.f;
        WCSPH_CUDA(cudaEventElapsedTime(&t, ev[s], ev[s + 1]));
        kernel_times_.emplace_back(kStages[s], t);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    stepped_since_state_ = true;
    check_device_errors();
    const int k = std::min(cap, NS);
    for (int s = 0; s < k; ++s) {
        if (names) names[s] = kernel_times_[s].first;
        if (ms) ms[s] = kernel_times_[s].second;
    }
    return k;
}

}  // namespace wcsph

namespace wcsph {

void CUDASPHSimulator::render(const wcsph_camera& cam, const wcsph_render_opts& o, uint8_t* rgba, float* depth) {
    if (o.width == 0 || o.height == 0 || o.width > 16384 || o.height > 16384)
        throw Error(WCSPH_ERR_INVALID_ARGUMENT, "render size must be 1..16384 per side");
    if (!(o.radius > 0.f)) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "render radius must be positive");
    if (!rgba) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "render needs an rgba buffer");
    RenderArgs r{};
    std::memcpy(r.proj, cam.projection, sizeof(r.proj));
    std::memcpy(r.view, cam.view, sizeof(r.view));
    mat4_mul(r.proj, r.view, r.vp);
    if (!mat4_inverse(r.vp, r.inv_vp)) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "camera matrices are singular");
    std::memcpy(r.eye, cam.eye, sizeof(r.eye));
    r.width = o.width;
    r.height = o.height;
    r.radius = o.radius;
    r.show_boundary = o.show_boundary ? 1 : 0;
    r.normalize = o.normalize ? 1 : 0;
    r.min_value = o.min_value;
    r.max_value = o.max_value;
    std::memcpy(r.background, o.background, sizeof(r.background));
    r.max_pixels = o.max_pixels > 0 ? o.max_pixels : (1 << 16);
    const float* scalar = nullptr;
    const float4* vec = nullptr;
    switch (o.field) {
    case -1: r.mode = RENDER_PLAIN; break;
    case WCSPH_FIELD_DENSITY: case WCSPH_FIELD_PRESSURE:
        r.mode = RENDER_SCALAR; scalar = static_cast<const float*>(device_field(o.field)); break;
    case WCSPH_FIELD_VELOCITY: case WCSPH_FIELD_PRESSURE_ACCEL: case WCSPH_FIELD_NON_PRESSURE_ACCEL:
    case WCSPH_FIELD_NORMAL:
        r.mode = RENDER_VECTOR; vec = static_cast<const float4*>(device_field(o.field)); break;
    default: throw Error(WCSPH_ERR_INVALID_ARGUMENT, "field cannot be visualised");
    }
    if (r.normalize && !(r.max_value != r.min_value)) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "min_value == max_value");
    const size_t npix = static_cast<size_t>(o.width) * o.height;
    if (render_z_.count != npix) { render_z_.alloc(npix); render_rgba_.alloc(npix); render_depth_.alloc(npix); }
    enqueue_render(r, pos_a_.ptr, n_, bpos_.ptr, nb_, scalar, vec, render_z_.ptr, render_rgba_.ptr,
                   depth ? render_depth_.ptr : nullptr, stream_);
    WCSPH_CUDA(cudaGetLastError());
    WCSPH_CUDA(cudaMemcpyAsync(rgba, render_rgba_.ptr, npix * 4, cudaMemcpyDeviceToHost, stream_));
    if (depth) WCSPH_CUDA(cudaMemcpyAsync(depth, render_depth_.ptr, npix * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    synchronize();
}

}  // namespace wcsph
