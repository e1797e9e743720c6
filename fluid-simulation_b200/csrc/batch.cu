// batch.cu — batched ensemble: many independent scenes of uneven particle
// counts advanced together.
//
// All scenes share one particle SoA. The sort key carries the scene id above
// the low 48 bits of the reference's Morton key, so one stable radix sort
// keeps every scene contiguous and, inside a scene, reproduces the
// reference's Morton order for that scene alone. Cells are hashed by
// (scene, cell) so neighbourhoods never cross scenes; the integrate pass
// reads each scene's box, gravity and viscosity from a per-scene table. The
// time step is fixed (CFL off), as in the ensemble workload.
//
// Two ways to run k steps, with identical results:
//  * persistent (default): one cooperative launch of batch_persistent.cu
//    advances every scene k steps, its phases separated by grid barriers; the
//    launch is captured in a CUDA graph (or issued directly where the driver
//    does not capture cooperative launches);
//  * per stage: one launch per stage and step (keys, sort plan, 8 digit
//    passes, reorder, 3 passes), the step captured in a CUDA graph.
#include <algorithm>
#include <bit>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "batch.cuh"
#include "radix_sort.cuh"
#include "step_kernels.cuh"

namespace wcsph {

namespace {
// Per-scene mean |v| and sum |v|^2 of the state: block k reduces scene k's
// contiguous range in a fixed order (double accumulators, fixed tree), so the
// metrics do not depend on scheduling.
__global__ void batch_metrics_kernel(const float4* __restrict__ vel, const u32* __restrict__ offsets,
                                     double* __restrict__ sums /* [S][2] */) {
    __shared__ double s1[256], s2[256];
    const u32 k = blockIdx.x;
    double a = 0.0, b = 0.0;
    for (u32 i = offsets[k] + threadIdx.x; i < offsets[k + 1]; i += blockDim.x) {
        const float4 v = vel[i];
        const float d = dot3(v, v);
        a += static_cast<double>(sqrtf(d));
        b += static_cast<double>(d);
    }
    s1[threadIdx.x] = a;
    s2[threadIdx.x] = b;
    __syncthreads();
    for (u32 o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s1[threadIdx.x] += s1[threadIdx.x + o];
            s2[threadIdx.x] += s2[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        sums[2 * k] = s1[0];
        sums[2 * k + 1] = s2[0];
    }
}
}  // namespace

struct BatchSim {
    wcsph_params params{};
    DevParams dp{};
    cudaStream_t stream = nullptr;
    int device = 0;
    u32 n = 0, nb = 0, S = 0;
    std::vector<u32> offsets, counts;   // fluid ranges per scene
    std::vector<u32> scene_first;       // offsets plus the total (uploaded to scene_offsets)
    float metric_mass = 0.f;

    DevBuf<float4> pos_a, pos_b, vel_a, vel_b;
    DevBuf<u32> scene_a;
    DevBuf<u64> keys[3];
    DevBuf<u32> vals[3];
    DevBuf<u32> hist, offs, lookback, perm;
    DevBuf<u64> ckey, table;
    DevBuf<u32> cstart, cend, mask;
    DevBuf<u32> nbr, nbr_cnt;          // neighbour lists, nbr_width slots per particle
    u32 table_size = 0;
    DevBuf<float> rho, prs, partials;
    DevBuf<double> metric_sums;
    DevBuf<u32> scene_offsets;          // [S + 1] first particle of each scene (device copy of offsets)
    DevBuf<u32> barrier;                // persistent kernel: grid-barrier arrivals and generation
    bool persistent = true;
    u32 p_blocks = 0;
    size_t p_smem = 0;
    cudaGraphExec_t pgraph = nullptr;   // persistent launch of pgraph_steps steps
    float pgraph_delta = -1.f;
    int pgraph_steps = 0;
    bool coop_capture = true;           // the driver captures cooperative launches
    DevBuf<u32> group_done;
    DevBuf<double> group_partials;
    DevBuf<float4> recf, recs;
    DevBuf<float4> ap, normal, vlap, anp;
    DevBuf<DevState> st;
    DevBuf<DevScene> scenes;
    DevBuf<float4> bpos;
    DevBuf<float> bmass;
    DevBuf<u64> btable, bckey;
    DevBuf<u32> bcstart, bcend;
    BoundaryCells bcells;               // per-cell boundary candidate runs
    DevBuf<uint4> bmask;                // boundary hit masks
    u32 btable_size = 0;
    int mask_words = 12;
    int nbr_width = 64;

    cudaGraphExec_t graph = nullptr;
    float graph_delta = -1.f;
    std::string last_error;

    ~BatchSim() {
        if (graph) cudaGraphExecDestroy(graph);
        if (pgraph) cudaGraphExecDestroy(pgraph);
        if (stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }

    // persistent: the persistent kernel's traversal phases (16 particles per
    // warp chunk; the per-stage passes take 32, 3 % faster on the 256-scene
    // ensemble, where 32 slows the persistent launch). Results do not depend
    // on the chunk: a cell is handled whole by the warp of its first particle.
    TravArgs args(float delta, bool persistent = false) {
        TravArgs a{};
        a.n = n;
        a.pos = pos_b.ptr;
        a.vel = vel_b.ptr;
        a.ckey = ckey.ptr;
        a.fluid = HashView{table.ptr, cstart.ptr, cend.ptr, table_size - 1};
        a.range = dp.range;
        a.nb = nb;
        a.bpos = bpos.ptr;
        a.bmass = bmass.ptr;
        a.boundary = HashView{btable.ptr, bcstart.ptr, bcend.ptr, btable_size ? btable_size - 1 : 0};
        a.bcell = bcells.view();
        a.bcx = bcells.x.ptr;
        a.bcx_n = static_cast<u32>(bcells.x.count);
        a.bmask = (bcells.size && mask_words >= 4 && dp.cell_size == dp.h) ? bmask.ptr : nullptr;
        a.mask = mask.ptr;
        a.mask_words = static_cast<u32>(mask_words);
        a.chunk = n < (1u << 18) ? 8u : (persistent ? 16u : 32u);
        a.nbr = nbr_width > 0 ? nbr.ptr : nullptr;
        a.pair_cells = a.nbr != nullptr ? 1u : 0u;
        a.nbr_cnt = nbr_cnt.ptr;
        a.nbr_width = static_cast<u32>(nbr_width);
        a.rho = rho.ptr; a.prs = prs.ptr;
        a.recf = recf.ptr; a.recs = recs.ptr;
        a.ap = ap.ptr; a.normal = normal.ptr; a.vlap = vlap.ptr; a.anp = anp.ptr;
        a.pos_out = pos_a.ptr; a.vel_out = vel_a.ptr;
        a.box = nullptr;
        a.scenes = scenes.ptr;
        a.scene_state = scene_a.ptr;
        a.st = st.ptr;
        a.delta = delta;
        a.cfl_factor = 0.f;
        a.max_dt = params.max_time_step;
        a.min_dt = params.min_time_step;
        a.np_max_dt = params.non_pressure_max_time_step;
        a.metric_mass = metric_mass;
        a.block_partials = partials.ptr;
        a.group_done = group_done.ptr;
        a.group_partials = group_partials.ptr;
        return a;
    }

    void enqueue_step(float delta) {
        WCSPH_CUDA(cudaMemsetAsync(table.ptr, 0xff, table.bytes(), stream));
        keys_hist_kernel<<<std::min<u32>((n + 255) / 256, 1184), 256, 0, stream>>>(pos_a.ptr, n, dp.cell_size,
                                                                                   keys[0].ptr, hist.ptr, scene_a.ptr);
        SortBuffers sb{};
        for (int i = 0; i < 3; ++i) { sb.keys[i] = keys[i].ptr; sb.vals[i] = vals[i].ptr; }
        sb.hist = hist.ptr; sb.offsets = offs.ptr; sb.lookback = lookback.ptr; sb.capacity = n;
        WCSPH_CUDA(enqueue_sort_passes(sb, n, st.ptr, stream));
        launch_reorder_cells(pos_a.ptr, vel_a.ptr, vals[1].ptr, vals[2].ptr, st.ptr, n, dp.cell_size, pos_b.ptr,
                             vel_b.ptr, perm.ptr, ckey.ptr, table.ptr, cstart.ptr, cend.ptr, table_size - 1, st.ptr,
                             stream, scene_a.ptr);
        const TravArgs a = args(delta);
        launch_pass(PASS_DENSITY, dp, a, stream, 2, true);
        launch_pass(PASS_FORCE, dp, a, stream, 2, true);
        launch_pass(PASS_SURFACE, dp, a, stream, 2, true);
    }

    PersistentStep persistent_args(float delta, int steps) {
        PersistentStep ps{};
        ps.P = dp;
        ps.a = args(delta, true);
        ps.pos_state = pos_a.ptr;
        ps.vel_state = vel_a.ptr;
        ps.scene_state = scene_a.ptr;
        for (int i = 0; i < 3; ++i) { ps.keys[i] = keys[i].ptr; ps.vals[i] = vals[i].ptr; }
        ps.hist = hist.ptr;
        ps.offsets = offs.ptr;
        ps.lookback = lookback.ptr;
        ps.tiles = sort_tiles(n);
        ps.perm = perm.ptr;
        ps.table = table.ptr;
        ps.table_size = table_size;
        ps.cs = dp.cell_size;
        ps.barrier = barrier.ptr;
        ps.steps = steps;
        ps.spin_limit = LB_SPIN_LIMIT;
        ps.barrier_limit = 1u << 24;   // polls 64 ns apart: about a second
        return ps;
    }

    // Captures the cooperative launch of k steps into a graph (once per
    // (delta, k)); where the driver refuses, later calls launch directly.
    void prepare_persistent(int k, float delta) {
        if (k <= 0) return;
        if (p_blocks == 0) persistent_grid(args(delta, true), device, &p_blocks, &p_smem);
        const PersistentStep ps = persistent_args(delta, k);
        if (coop_capture && (!pgraph || pgraph_delta != delta || pgraph_steps != k)) {
            if (pgraph) cudaGraphExecDestroy(pgraph);
            pgraph = nullptr;
            cudaGraph_t g = nullptr;
            WCSPH_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            bool launched = true;
            try {
                launch_persistent(ps, p_blocks, p_smem, stream);
            } catch (const Error&) {
                launched = false;
            }
            const cudaError_t ec = cudaStreamEndCapture(stream, &g);
            cudaError_t ei = cudaErrorUnknown;
            if (launched && ec == cudaSuccess && g) ei = cudaGraphInstantiate(&pgraph, g, 0);
            if (g) cudaGraphDestroy(g);
            if (ei != cudaSuccess) {   // no capture of cooperative launches: launch directly from now on
                pgraph = nullptr;
                coop_capture = false;
                cudaGetLastError();
            } else {
                pgraph_delta = delta;
                pgraph_steps = k;
            }
        }
    }

    // k steps in one cooperative launch (graph replay when captured)
    void persistent_steps(int k, float delta) {
        if (k <= 0) return;
        NvtxRange r("wcsph ensemble: persistent launch");
        prepare_persistent(k, delta);
        if (pgraph && pgraph_delta == delta && pgraph_steps == k) WCSPH_CUDA(cudaGraphLaunch(pgraph, stream));
        else launch_persistent(persistent_args(delta, k), p_blocks, p_smem, stream);
    }

    void step_n(int k, float delta) {
        if (persistent) {
            persistent_steps(k, delta);
            return;
        }
        if (!graph || graph_delta != delta) {
            if (graph) cudaGraphExecDestroy(graph);
            graph = nullptr;
            cudaGraph_t g = nullptr;
            WCSPH_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_step(delta);
            } catch (...) {
                cudaStreamEndCapture(stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            WCSPH_CUDA(cudaStreamEndCapture(stream, &g));
            const cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
            cudaGraphDestroy(g);
            WCSPH_CUDA(e);
            graph_delta = delta;
        }
        for (int i = 0; i < k; ++i) WCSPH_CUDA(cudaGraphLaunch(graph, stream));
    }

    void check_errors() {
        WCSPH_CUDA(cudaStreamSynchronize(stream));
        u32 flags = 0;
        WCSPH_CUDA(cudaMemcpy(&flags, &st.ptr->error_flags, sizeof(u32), cudaMemcpyDeviceToHost));
        if (flags) {
            WCSPH_CUDA(cudaMemset(&st.ptr->error_flags, 0, sizeof(u32)));
            if (flags & ERR_HASH_FULL) throw Error(WCSPH_ERR_HASH_FULL, "spatial hash table is full");
            if (flags & ERR_LOOKBACK_TIMEOUT) throw Error(WCSPH_ERR_DEVICE_TIMEOUT, "radix sort look-back timed out");
            if (flags & ERR_BARRIER_TIMEOUT)
                throw Error(WCSPH_ERR_DEVICE_TIMEOUT, "persistent ensemble kernel: grid barrier timed out");
            if (flags & ERR_BOUNDS) throw Error(WCSPH_ERR_BOUNDS, "device index out of bounds (bounds-checked build)");
            throw Error(WCSPH_ERR_NEIGHBOR_OVERFLOW, "boundary candidate cells exceed capacity");
        }
    }
};

static void build_batch(BatchSim& B, const wcsph_params& p, const wcsph_batch_scene* sc, u32 S, int device) {
    validate_params(p);
    if (p.cfl_factor > 0.f)
        throw Error(WCSPH_ERR_NOT_SUPPORTED, "batched ensembles step with a fixed dt: set cfl_factor <= 0");
    if (S == 0 || S >= (1u << 15)) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "scene count must be in [1, 32767]");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) throw Error(WCSPH_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0) WCSPH_CUDA(cudaGetDevice(&device));
    B.device = device;
    WCSPH_CUDA(cudaSetDevice(device));
    WCSPH_CUDA(cudaStreamCreateWithFlags(&B.stream, cudaStreamNonBlocking));
    B.params = p;
    B.dp = make_dev_params(p);
    B.metric_mass = metric_mass(p);
    B.S = S;
    const float cs = B.dp.cell_size;
    // batched cell coordinates must lie in [-2^15, 2^15) (16-bit batch keys),
    // with a margin for the neighbour cells of the outermost particles
    const double lim = static_cast<double>(BATCH_CELL_LIMIT - 4) * cs;
    std::vector<float> pos, vel, bp;
    std::vector<u32> sid, bsid;
    std::vector<DevScene> ds(S);
    u64 total = 0, btotal = 0;
    for (u32 k = 0; k < S; ++k) {
        if (sc[k].fluid_n == 0 || !sc[k].fluid_pos) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "empty scene");
        total += sc[k].fluid_n;
        btotal += sc[k].boundary_n;
    }
    if (total >= (1ull << 30) || btotal >= (1ull << 30)) throw Error(WCSPH_ERR_INVALID_ARGUMENT, "too many particles");
    pos.reserve(4 * total);
    vel.reserve(4 * total);
    for (u32 k = 0; k < S; ++k) {
        const wcsph_batch_scene& s = sc[k];
        // the box's corners in world space (the model matrix of its frame)
        for (int c = 0; c < 8; ++c) {
            const float m[3] = {(c & 1) ? s.box.max[0] : s.box.min[0], (c & 2) ? s.box.max[1] : s.box.min[1],
                                (c & 4) ? s.box.max[2] : s.box.min[2]};
            for (int d = 0; d < 3; ++d) {
                const double w = static_cast<double>(s.box.model[d]) * m[0] + s.box.model[4 + d] * m[1] +
                                 s.box.model[8 + d] * m[2] + s.box.model[12 + d];
                if (!(std::fabs(w) < lim))
                    throw Error(WCSPH_ERR_NOT_SUPPORTED,
                                "batched scene boxes must lie within 32,764 cells of the origin per axis");
            }
        }
        B.offsets.push_back(static_cast<u32>(pos.size() / 4));
        B.counts.push_back(s.fluid_n);
        pos.insert(pos.end(), s.fluid_pos, s.fluid_pos + 4ull * s.fluid_n);
        if (s.fluid_vel) vel.insert(vel.end(), s.fluid_vel, s.fluid_vel + 4ull * s.fluid_n);
        else vel.insert(vel.end(), 4ull * s.fluid_n, 0.f);
        sid.insert(sid.end(), s.fluid_n, k);
        if (s.boundary_n) {
            bp.insert(bp.end(), s.boundary_pos, s.boundary_pos + 4ull * s.boundary_n);
            bsid.insert(bsid.end(), s.boundary_n, k);
        }
        ds[k].box = make_dev_box(s.box);
        wcsph_params q = p;
        q.viscosity = s.viscosity;
        const DevParams dq = make_dev_params(q);
        ds[k].gravity_visc = make_float4(s.gravity[0], s.gravity[1], s.gravity[2], dq.visc_scale);
    }
    for (size_t i = 0; i < pos.size() / 4; ++i)
        for (int d = 0; d < 3; ++d)
            if (!(std::fabs(static_cast<double>(pos[4 * i + d])) < lim))
                throw Error(WCSPH_ERR_NOT_SUPPORTED, "batched particles must lie within 32,764 cells of the origin per axis");
    B.n = static_cast<u32>(total);
    B.nb = static_cast<u32>(btotal);
    const size_t n = B.n;
    B.pos_a.alloc(n); B.pos_b.alloc(n); B.vel_a.alloc(n); B.vel_b.alloc(n); B.scene_a.alloc(n);
    for (auto& k : B.keys) k.alloc(n);
    B.vals[1].alloc(n); B.vals[2].alloc(n);
    B.hist.alloc(SORT_DIGITS * 256); B.offs.alloc(SORT_DIGITS * 256);
    B.lookback.alloc(static_cast<size_t>(SORT_DIGITS) * sort_tiles(B.n) * 256);
    B.perm.alloc(n); B.ckey.alloc(n);
    B.table_size = static_cast<u32>(std::max<u64>(std::bit_ceil(static_cast<u64>(n)) / 4, 64) * p.table_size_mult);
    B.table.alloc(B.table_size); B.cstart.alloc(B.table_size); B.cend.alloc(B.table_size);
    B.mask.alloc(n * static_cast<size_t>(B.mask_words));
    // 32-bit list slot indices: fewer slots for very large ensembles, none below 8
    if (n > 0) B.nbr_width = static_cast<int>(std::min<size_t>(static_cast<size_t>(B.nbr_width), ((1ull << 32) - 1) / n));
    if (B.nbr_width < 8) B.nbr_width = 0;
    B.nbr.alloc(n * static_cast<size_t>(B.nbr_width));
    B.nbr_cnt.alloc(n);
    B.rho.alloc(n); B.prs.alloc(n); B.recf.alloc(2 * n); B.recs.alloc(2 * n); B.ap.alloc(n); B.normal.alloc(n); B.vlap.alloc(n); B.anp.alloc(n);
    B.partials.alloc(2ull * pass_max_warps(B.n));
    B.group_done.alloc(pass_max_warps(B.n) / 32u + 1u);
    B.group_partials.alloc(2ull * (pass_max_warps(B.n) / 32u + 1u));
    WCSPH_CUDA(cudaMemsetAsync(B.group_done.ptr, 0, B.group_done.bytes(), B.stream));
    B.metric_sums.alloc(2ull * S);
    B.scene_offsets.alloc(S + 1ull);
    B.scene_first = B.offsets;
    B.scene_first.push_back(B.n);
    WCSPH_CUDA(cudaMemcpyAsync(B.scene_offsets.ptr, B.scene_first.data(), sizeof(u32) * (S + 1ull),
                               cudaMemcpyHostToDevice, B.stream));
    B.barrier.alloc(8);   // grid-barrier words and the persistent kernel's work counters
    WCSPH_CUDA(cudaMemsetAsync(B.barrier.ptr, 0, B.barrier.bytes(), B.stream));
    B.st.alloc(1);
    B.scenes.alloc(S);
    cudaStream_t s = B.stream;
    WCSPH_CUDA(cudaMemsetAsync(B.hist.ptr, 0, B.hist.bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.st.ptr, 0, sizeof(DevState), s));
    WCSPH_CUDA(cudaMemsetAsync(B.table.ptr, 0xff, B.table.bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.cstart.ptr, 0, B.cstart.bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.cend.ptr, 0, B.cend.bytes(), s));
    // index buffers start as valid indices (zeros): see CUDASPHSimulator::allocate
    WCSPH_CUDA(cudaMemsetAsync(B.vals[1].ptr, 0, B.vals[1].bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.vals[2].ptr, 0, B.vals[2].bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.perm.ptr, 0, B.perm.bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.ckey.ptr, 0, B.ckey.bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.mask.ptr, 0, B.mask.bytes(), s));
    if (B.nbr.ptr) WCSPH_CUDA(cudaMemsetAsync(B.nbr.ptr, 0, B.nbr.bytes(), s));
    WCSPH_CUDA(cudaMemsetAsync(B.nbr_cnt.ptr, 0, B.nbr_cnt.bytes(), s));
    WCSPH_CUDA(cudaMemcpyAsync(B.pos_a.ptr, pos.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s));
    WCSPH_CUDA(cudaMemcpyAsync(B.vel_a.ptr, vel.data(), sizeof(float4) * n, cudaMemcpyHostToDevice, s));
    WCSPH_CUDA(cudaMemcpyAsync(B.scene_a.ptr, sid.data(), sizeof(u32) * n, cudaMemcpyHostToDevice, s));
    WCSPH_CUDA(cudaMemcpyAsync(B.scenes.ptr, ds.data(), sizeof(DevScene) * S, cudaMemcpyHostToDevice, s));
    if (B.nb) {
        const u32 nbb = B.nb;
        DevBuf<float4> tmp(nbb);
        DevBuf<u32> tsid(nbb), bperm(nbb), v1(nbb), v2(nbb);
        DevBuf<u64> k0(nbb), k1(nbb), k2(nbb);
        DevBuf<u32> lb(static_cast<size_t>(SORT_DIGITS) * sort_tiles(nbb) * 256);
        WCSPH_CUDA(cudaMemcpyAsync(tmp.ptr, bp.data(), sizeof(float4) * nbb, cudaMemcpyHostToDevice, s));
        WCSPH_CUDA(cudaMemcpyAsync(tsid.ptr, bsid.data(), sizeof(u32) * nbb, cudaMemcpyHostToDevice, s));
        keys_hist_kernel<<<std::min<u32>((nbb + 255) / 256, 1184), 256, 0, s>>>(tmp.ptr, nbb, B.dp.h, k0.ptr,
                                                                                 B.hist.ptr, tsid.ptr);
        SortBuffers sb{};
        sb.keys[0] = k0.ptr; sb.keys[1] = k1.ptr; sb.keys[2] = k2.ptr;
        sb.vals[1] = v1.ptr; sb.vals[2] = v2.ptr;
        sb.hist = B.hist.ptr; sb.offsets = B.offs.ptr; sb.lookback = lb.ptr; sb.capacity = nbb;
        WCSPH_CUDA(enqueue_sort_passes(sb, nbb, B.st.ptr, s));
        B.btable_size = std::max<u32>(std::bit_ceil(nbb), 64u);
        B.btable.alloc(B.btable_size); B.bcstart.alloc(B.btable_size); B.bcend.alloc(B.btable_size);
        WCSPH_CUDA(cudaMemsetAsync(B.btable.ptr, 0xff, B.btable.bytes(), s));
        WCSPH_CUDA(cudaMemsetAsync(B.bcstart.ptr, 0, B.bcstart.bytes(), s));
        WCSPH_CUDA(cudaMemsetAsync(B.bcend.ptr, 0, B.bcend.bytes(), s));
        B.bpos.alloc(nbb); B.bmass.alloc(nbb); B.bckey.alloc(nbb);
        launch_reorder_cells(tmp.ptr, nullptr, v1.ptr, v2.ptr, B.st.ptr, nbb, B.dp.h, B.bpos.ptr, nullptr, bperm.ptr,
                             B.bckey.ptr, B.btable.ptr, B.bcstart.ptr, B.bcend.ptr, B.btable_size - 1, B.st.ptr, s,
                             tsid.ptr);
        HashView bh{B.btable.ptr, B.bcstart.ptr, B.bcend.ptr, B.btable_size - 1};
        launch_boundary_mass(B.dp, B.bpos.ptr, nbb, bh, B.bmass.ptr, s, B.bckey.ptr);
        WCSPH_CUDA(cudaGetLastError());
        build_boundary_cells(B.bcells, bh, B.btable_size, nbb, B.bpos.ptr, B.bmass.ptr, true, B.st.ptr, s);
        if (B.bcells.size) B.bmask.alloc(B.n);
        WCSPH_CUDA(cudaStreamSynchronize(s));
    }
    B.check_errors();
}

}  // namespace wcsph

struct wcsph_batch {
    wcsph::BatchSim sim;
};

namespace {
thread_local std::string g_batch_error;

template <class F>
int bguard(wcsph_batch* b, F&& f) {
    try {
        f();
        return WCSPH_OK;
    } catch (const wcsph::Error& e) {
        (b ? b->sim.last_error : g_batch_error) = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        (b ? b->sim.last_error : g_batch_error) = "host allocation failed";
        return WCSPH_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        (b ? b->sim.last_error : g_batch_error) = e.what();
        return WCSPH_ERR_CUDA;
    }
}
}  // namespace

extern "C" {

int wcsph_batch_create(const wcsph_params* params, const wcsph_batch_scene* scenes, uint32_t n_scenes, int device,
                       wcsph_batch** out) {
    if (!params || !scenes || !out) return WCSPH_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    auto b = std::make_unique<wcsph_batch>();
    const int s = bguard(nullptr, [&] { wcsph::build_batch(b->sim, *params, scenes, n_scenes, device); });
    if (s == WCSPH_OK) *out = b.release();
    return s;
}

int wcsph_batch_destroy(wcsph_batch* b) {
    delete b;
    return WCSPH_OK;
}

int wcsph_batch_set_persistent(wcsph_batch* b, int enable) {
    if (!b) return WCSPH_ERR_INVALID_ARGUMENT;
    return bguard(b, [&] {
        WCSPH_CUDA(cudaStreamSynchronize(b->sim.stream));
        b->sim.persistent = enable != 0;
    });
}

int wcsph_batch_step_n(wcsph_batch* b, int n, float delta) {
    if (!b || n < 0) return WCSPH_ERR_INVALID_ARGUMENT;
    return bguard(b, [&] { b->sim.step_n(n, delta); });
}

int wcsph_batch_time_steps(wcsph_batch* b, int n, float delta, float* ms_out) {
    if (!b || n < 0 || !ms_out) return WCSPH_ERR_INVALID_ARGUMENT;
    return bguard(b, [&] {
        // graphs and launch set-up happen before the timed region
        if (b->sim.persistent) {
            b->sim.prepare_persistent(n, delta);
        } else if (!b->sim.graph || b->sim.graph_delta != delta) {
            b->sim.step_n(1, delta);
        }
        cudaEvent_t e0, e1;
        WCSPH_CUDA(cudaEventCreate(&e0));
        WCSPH_CUDA(cudaEventCreate(&e1));
        WCSPH_CUDA(cudaEventRecord(e0, b->sim.stream));
        b->sim.step_n(n, delta);
        WCSPH_CUDA(cudaEventRecord(e1, b->sim.stream));
        WCSPH_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        WCSPH_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms_out = ms;
        b->sim.check_errors();
    });
}

int wcsph_batch_get_state(wcsph_batch* b, uint32_t scene, float* pos_out, float* vel_out) {
    if (!b || scene >= b->sim.S) return WCSPH_ERR_INVALID_ARGUMENT;
    return bguard(b, [&] {
        wcsph::BatchSim& B = b->sim;
        const size_t off = B.offsets[scene], cnt = B.counts[scene];
        if (pos_out)
            WCSPH_CUDA(cudaMemcpyAsync(pos_out, B.pos_a.ptr + off, sizeof(float4) * cnt, cudaMemcpyDeviceToHost,
                                       B.stream));
        if (vel_out)
            WCSPH_CUDA(cudaMemcpyAsync(vel_out, B.vel_a.ptr + off, sizeof(float4) * cnt, cudaMemcpyDeviceToHost,
                                       B.stream));
        B.check_errors();
    });
}

int wcsph_batch_metrics(wcsph_batch* b, float* mean_speed, float* ke) {
    if (!b) return WCSPH_ERR_INVALID_ARGUMENT;
    return bguard(b, [&] {
        wcsph::BatchSim& B = b->sim;
        wcsph::batch_metrics_kernel<<<B.S, 256, 0, B.stream>>>(B.vel_a.ptr, B.scene_offsets.ptr, B.metric_sums.ptr);
        WCSPH_CUDA(cudaGetLastError());
        std::vector<double> sums(2ull * B.S);
        WCSPH_CUDA(cudaMemcpyAsync(sums.data(), B.metric_sums.ptr, sizeof(double) * sums.size(),
                                   cudaMemcpyDeviceToHost, B.stream));
        B.check_errors();
        for (uint32_t k = 0; k < B.S; ++k) {
            if (mean_speed) mean_speed[k] = static_cast<float>(sums[2 * k] / static_cast<double>(B.counts[k]));
            if (ke) ke[k] = static_cast<float>(0.5 * static_cast<double>(B.metric_mass) * sums[2 * k + 1]);
        }
    });
}

const char* wcsph_batch_last_error(const wcsph_batch* b) {
    return b ? b->sim.last_error.c_str() : g_batch_error.c_str();
}

}  // extern "C"
