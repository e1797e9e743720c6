// batch_persistent.cu — the batched ensemble advanced by one persistent,
// cooperative launch for any number of steps.
//
// Every block stays resident for the whole launch (the cooperative launch
// refuses a grid that does not fit at once). A step runs the phases of the
// per-stage path (batch.cu) over the whole ensemble, separated by grid
// barriers instead of kernel boundaries:
//   keys + digit histograms | sort plan | the active digit passes (tiles
//   claimed in increasing order, so each look-back waits only on tiles that
//   running blocks already hold) | reorder + hash | density | force | surface
//   and integrate.
// The phases call the same device code as the per-pass kernels, so every
// scene matches its own single-scene step bit for bit. Buffers rewritten
// inside the launch (hash, sorted state, records, lists) are read with
// ordinary coherent loads (WCSPH_COHERENT_LOADS), not the read-only path.
//
// Every wait is bounded: a grid barrier gives up after barrier_limit polls and
// a look-back after spin_limit polls; either sets an error flag, after which
// the blocks leave the launch at their next barrier, and the host reports
// WCSPH_ERR_DEVICE_TIMEOUT.
#define WCSPH_COHERENT_LOADS 1
#include "batch.cuh"
#include "radix_sort_dev.cuh"
#include "step_device.cuh"

namespace wcsph {

namespace {

constexpr int PWARPS = 8;                  // warps per block: one 256-thread sort tile per block
constexpr int PTHREADS = PWARPS * 32;
constexpr u32 STOP_FLAGS = ERR_LOOKBACK_TIMEOUT | ERR_BARRIER_TIMEOUT;

__device__ __forceinline__ u32 ld_volatile(const u32* p) { return *reinterpret_cast<const volatile u32*>(p); }

// Work counters of the traversal phases (after the barrier words): warps take
// CLAIM chunks at a time, so that no block idles at a barrier while others
// still hold a long queue. Block 0 clears them with the sort plan of each step.
enum : u32 { WORK_DENSITY = 2, WORK_FORCE = 3, WORK_SURFACE = 4, BARRIER_WORDS = 5 };
constexpr u32 CLAIM = 4;

__device__ __forceinline__ u32 claim(u32* ctr) {
    u32 v = 0;
    if ((threadIdx.x & 31u) == 0) v = atomicAdd(ctr, CLAIM);
    return __shfl_sync(0xffffffffu, v, 0);
}

// Grid-wide barrier of the cooperative launch. bar[0] counts arrivals, bar[1]
// is the generation: the last arriving block resets the count and advances
// the generation, the others poll it (bounded). Writes of every block before
// the barrier are visible to every block after it (fences on both sides, as
// a cooperative-groups grid sync). Returns false once an error stops the step.
__device__ __forceinline__ bool grid_barrier(u32* bar, DevState* st, u32 limit) {
    __shared__ u32 s_go;   // the block's decision, the same for all its threads
    __syncthreads();
    if (threadIdx.x == 0) {
        const u32 gen = ld_volatile(bar + 1);
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            u32 polls = 0;
            while (ld_volatile(bar + 1) == gen) {
                if (++polls > limit) {
                    atomicOr(&st->error_flags, ERR_BARRIER_TIMEOUT);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_go = (ld_volatile(&st->error_flags) & STOP_FLAGS) == 0u ? 1u : 0u;
    }
    __syncthreads();
    return s_go != 0u;
}

size_t persistent_smem(const TravArgs& a) {
    const u32 cap = a.mask_words * 32u;
    const u32 ncell = static_cast<u32>((2 * a.range + 1) * (2 * a.range + 1) * (2 * a.range + 1));
    const bool wb = a.nb > 0;
    size_t b = sizeof(u32) * SORT_DIGITS * 256;                  // digit histograms
    b = std::max(b, sizeof(u32) * (PWARPS * 256 + 256));          // onesweep ranks and bases
    b = std::max(b, PWARPS * warp_smem_bytes<PASS_DENSITY>(cap, ncell, wb));
    if (a.nbr == nullptr) {                                       // force and surface walk the bit matrix
        b = std::max(b, PWARPS * warp_smem_bytes<PASS_FORCE>(cap, ncell, wb));
        b = std::max(b, PWARPS * warp_smem_bytes<PASS_SURFACE>(cap, ncell, wb));
    }
    return b;
}

__global__ void __launch_bounds__(PTHREADS, 3) persistent_ensemble_kernel(const PersistentStep ps) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ u32 s_tile;
    __shared__ u32 s_active[SORT_DIGITS];
    const TravArgs& a = ps.a;
    const DevParams& P = ps.P;
    DevState* st = a.st;
    const u32 n = a.n;
    const u32 tid = threadIdx.x;
    const u32 warp = tid >> 5;
    const u32 nthreads = gridDim.x * PTHREADS;
    const size_t first = static_cast<size_t>(blockIdx.x) * PTHREADS + tid;
    const size_t nlb = static_cast<size_t>(SORT_DIGITS) * ps.tiles * 256u;
    const float np_dt = a.delta < a.np_max_dt ? a.delta : a.np_max_dt;
    float rm = 0.f, rs = 0.f, rs2 = 0.f;   // unused reductions of the pass code

    for (int step = 0; step < ps.steps; ++step) {
        // keys of the state and their digit histograms; clear hash and look-back flags
        for (size_t t = first; t < ps.table_size; t += nthreads) ps.table[t] = EMPTY_HASH;
        for (size_t t = first; t < nlb; t += nthreads) ps.lookback[t] = 0u;
        sortdev::keys_hist_block(ps.pos_state, n, ps.cs, ps.keys[0], ps.hist, ps.scene_state,
                                 reinterpret_cast<u32(*)[256]>(smem), blockIdx.x * PTHREADS, nthreads);
        if (!grid_barrier(ps.barrier, st, ps.barrier_limit)) return;
        if (blockIdx.x == 0) {
            sortdev::sort_plan_block(n, ps.hist, ps.offsets, st, s_active);
            if (tid < 3) ps.barrier[WORK_DENSITY + tid] = 0u;
        }
        if (!grid_barrier(ps.barrier, st, ps.barrier_limit)) return;
        for (int p = 0; p < SORT_DIGITS; ++p) {
            if (!ld_volatile(&st->sort_active[p])) continue;   // the same for every block
            for (;;) {
                if (tid == 0) s_tile = atomicAdd(&st->sort_tile_counter[p], 1u);
                __syncthreads();
                const u32 tile = s_tile;
                if (tile >= ps.tiles) break;
                sortdev::onesweep_tile(n, p, ps.keys[0], ps.keys[1], ps.keys[2], ps.vals[1], ps.vals[2], ps.offsets,
                                       ps.lookback, ps.tiles, st, ps.spin_limit, 0u, tile,
                                       reinterpret_cast<u32(*)[256]>(smem),
                                       reinterpret_cast<u32*>(smem) + PWARPS * 256);
                __syncthreads();
            }
            if (!grid_barrier(ps.barrier, st, ps.barrier_limit)) return;
        }
        // sorted scratch, cell keys, hash
        for (u32 base = blockIdx.x * PTHREADS; base < n; base += nthreads)
            reorder_cell_item<true>(ps.pos_state, ps.vel_state, ps.vals[1], ps.vals[2], st, n, ps.cs,
                                    const_cast<float4*>(a.pos), const_cast<float4*>(a.vel), ps.perm,
                                    const_cast<u64*>(a.ckey), ps.table, const_cast<u32*>(a.fluid.cstart),
                                    const_cast<u32*>(a.fluid.cend), a.fluid.tmask, st, ps.scene_state, base + tid);
        if (!grid_barrier(ps.barrier, st, ps.barrier_limit)) return;
        const u32 nchunks = (n + a.chunk - 1) / a.chunk;
        {
            const WarpView<PASS_DENSITY> S = warp_view<PASS_DENSITY>(a, smem, warp);
            for (u32 c0 = claim(ps.barrier + WORK_DENSITY); c0 < nchunks; c0 = claim(ps.barrier + WORK_DENSITY))
                for (u32 c = c0; c < min(c0 + CLAIM, nchunks); ++c)
                    cell_pass_chunk<PASS_DENSITY, true>(P, a, S, c, 0.f, 0.f, rm, rs, rs2);
        }
        if (!grid_barrier(ps.barrier, st, ps.barrier_limit)) return;
        const u32 rows = list_rows_per_warp(a.chunk);
        const u32 ngroups = (n + rows - 1) / rows;
        if (a.nbr) {
            for (u32 g0 = claim(ps.barrier + WORK_FORCE); g0 < ngroups; g0 = claim(ps.barrier + WORK_FORCE))
                for (u32 g = g0; g < min(g0 + CLAIM, ngroups); ++g)
                    list_rows<PASS_FORCE, true, 1>(P, a, g * rows, min(rows, n - g * rows), 0.f, 0.f, rm, rs, rs2);
        } else {
            const WarpView<PASS_FORCE> S = warp_view<PASS_FORCE>(a, smem, warp);
            for (u32 c0 = claim(ps.barrier + WORK_FORCE); c0 < nchunks; c0 = claim(ps.barrier + WORK_FORCE))
                for (u32 c = c0; c < min(c0 + CLAIM, nchunks); ++c)
                    cell_pass_chunk<PASS_FORCE, true>(P, a, S, c, 0.f, 0.f, rm, rs, rs2);
        }
        if (!grid_barrier(ps.barrier, st, ps.barrier_limit)) return;
        const float dt = cfl_time_step(a, P);   // fixed step: the bounds alone decide
        if (a.nbr) {
            for (u32 g0 = claim(ps.barrier + WORK_SURFACE); g0 < ngroups; g0 = claim(ps.barrier + WORK_SURFACE))
                for (u32 g = g0; g < min(g0 + CLAIM, ngroups); ++g)
                    list_rows<PASS_SURFACE, true, 2>(P, a, g * rows, min(rows, n - g * rows), dt, np_dt, rm, rs, rs2);
        } else {
            const WarpView<PASS_SURFACE> S = warp_view<PASS_SURFACE>(a, smem, warp);
            for (u32 c0 = claim(ps.barrier + WORK_SURFACE); c0 < nchunks; c0 = claim(ps.barrier + WORK_SURFACE))
                for (u32 c = c0; c < min(c0 + CLAIM, nchunks); ++c)
                    cell_pass_chunk<PASS_SURFACE, true>(P, a, S, c, dt, np_dt, rm, rs, rs2);
        }
        if (!grid_barrier(ps.barrier, st, ps.barrier_limit)) return;
    }
}

}  // namespace

void persistent_grid(const TravArgs& a, int device, u32* blocks, size_t* smem) {
    const size_t bytes = persistent_smem(a);
    WCSPH_CUDA(cudaFuncSetAttribute(persistent_ensemble_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(bytes)));
    int per_sm = 0, sms = 0;
    WCSPH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_ensemble_kernel, PTHREADS, bytes));
    WCSPH_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    if (per_sm < 1) throw Error(WCSPH_ERR_NOT_SUPPORTED, "persistent ensemble kernel does not fit on an SM");
    *blocks = static_cast<u32>(per_sm * sms);
    *smem = bytes;
}

void launch_persistent(const PersistentStep& ps, u32 blocks, size_t smem, cudaStream_t stream) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(PTHREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    WCSPH_CUDA(cudaLaunchKernelEx(&cfg, persistent_ensemble_kernel, ps));
}

}  // namespace wcsph
