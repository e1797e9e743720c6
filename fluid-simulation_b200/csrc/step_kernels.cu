// step_kernels.cu — see step_kernels.cuh for the decomposition.
#include "step_kernels.cuh"

#include <algorithm>
#include <climits>

#include "step_device.cuh"

namespace wcsph {

namespace {

template <int KIND, int WPB, bool BATCH>
__global__ void __launch_bounds__(WPB * 32, KindCfg<KIND>::min_warps / WPB) cell_pass_kernel(const DevParams P, const TravArgs a) {
    if (a.st->error_flags & ERR_LOOKBACK_TIMEOUT) return;   // no sorted state this step (reorder skipped)
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const u32 lane = lane_id();
    const u32 warp = threadIdx.x >> 5;
    const WarpView<KIND> S = warp_view<KIND>(a, dyn_smem, warp);

    float dt = 0.f, np_dt = 0.f;
    if constexpr (KIND == PASS_SURFACE) {
        // every warp reads the CFL step itself (no block barrier); the flip of
        // the max-speed parity happens only after every warp has finished
        float t = 0.f;
        if (lane == 0) t = cfl_time_step(a, P);
        dt = __shfl_sync(FULL, t, 0);
        np_dt = a.delta < a.np_max_dt ? a.delta : a.np_max_dt;
    }
    float red_max = 0.f, red_speed = 0.f, red_speed2 = 0.f;
    cell_pass_chunk<KIND, BATCH>(P, a, S, blockIdx.x * WPB + warp, dt, np_dt, red_max, red_speed, red_speed2);

    if constexpr (KIND == PASS_ADJ_FORCE) {
        double v = static_cast<double>(red_speed);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
        if (lane == 0 && v != 0.0) atomicAdd(a.adj_accum, v);
    }
    if constexpr (KIND == PASS_SURFACE) surface_reduce<WPB>(a, dt, np_dt, red_max, red_speed, red_speed2);
}


// Resident warps per SM the register allocation of the list kernels must
// allow (36 -> 56 registers, 44 -> 46, 48 -> 42). Both passes wait on
// neighbour gathers, so resident warps pay while spills stay small: the
// force pass fits 56 registers (36 warps; at 48 it spills), the single-scene
// surface pass 40 (50 warps with two-warp blocks, against 40 at the 47 it
// takes when allowed 48). The batched passes carry the scene lookups: 56
// registers cost the force pass 4 bytes of spills and still gain (ensemble
// step 5.34 -> 5.27 ms); the batched surface pass runs at a 44-warp cap.
template <int KIND, bool BATCH>
struct ListCfg {
    static constexpr int min_warps = KIND == PASS_FORCE ? 36 : (BATCH ? 44 : 48);
};

// Force / surface pass over the neighbour lists written by the density pass.
template <int KIND, int WPB, bool BATCH>
__global__ void __launch_bounds__(WPB * 32, ListCfg<KIND, BATCH>::min_warps / WPB) list_pass_kernel(const DevParams P,
                                                                                          const TravArgs a) {
    if (a.st->error_flags & ERR_LOOKBACK_TIMEOUT) return;   // no sorted state this step (reorder skipped)
    const u32 lane = lane_id();
    const u32 warp = threadIdx.x >> 5;
    float dt = 0.f, np_dt = 0.f;
    if constexpr (KIND == PASS_SURFACE) {
        float t = 0.f;
        if (lane == 0) t = cfl_time_step(a, P);
        dt = __shfl_sync(FULL, t, 0);
        np_dt = a.delta < a.np_max_dt ? a.delta : a.np_max_dt;
    }
    float red_max = 0.f, red_speed = 0.f, red_speed2 = 0.f;
    const u32 rows = list_rows_per_warp(a.chunk);
    const u32 base = (blockIdx.x * WPB + warp) * rows;
    if (base < a.n)
        list_rows<KIND, BATCH>(P, a, base, min(rows, a.n - base), dt, np_dt, red_max, red_speed, red_speed2);
    if constexpr (KIND == PASS_SURFACE) surface_reduce<WPB>(a, dt, np_dt, red_max, red_speed, red_speed2);
}

template <bool BATCH>
__global__ void reorder_cells_kernel(const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                                     const u32* __restrict__ v1, const u32* __restrict__ v2,
                                     const DevState* st, u32 n, float cs, float4* __restrict__ pos_out,
                                     float4* __restrict__ vel_out, u32* __restrict__ perm_out,
                                     u64* __restrict__ ckey_out, u64* table, u32* cstart, u32* cend,
                                     u32 tmask, DevState* st_err, const u32* __restrict__ scene_in) {
    // a sort whose look-back wait ran out left no permutation: keep the
    // previous sorted state and hash (every later pass returns at once too)
    if (st->error_flags & ERR_LOOKBACK_TIMEOUT) return;
    reorder_cell_item<BATCH>(pos_in, vel_in, v1, v2, st, n, cs, pos_out, vel_out, perm_out, ckey_out, table, cstart,
                             cend, tmask, st_err, scene_in, blockIdx.x * blockDim.x + threadIdx.x);
}

__global__ void init_cfl_kernel(const float4* __restrict__ vel, u32 n, DevState* st) {
    float m = 0.f;
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 v = vel[i];
        m = fmaxf(m, dot3(v, v));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
    if ((threadIdx.x & 31u) == 0) atomicMax(&st->vmax2_bits[st->parity], __float_as_uint(m));
}

__global__ void metrics_kernel(const float4* __restrict__ vel, u32 n, float mass, float* out2) {
    // single block, deterministic order (used outside the step)
    __shared__ double s1[32], s2[32];
    double a = 0.0, b = 0.0;
    for (u32 i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 v = vel[i];
        const float d = dot3(v, v);
        a += static_cast<double>(sqrtf(d));
        b += static_cast<double>(d);
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(FULL, a, o);
        b += __shfl_xor_sync(FULL, b, o);
    }
    if ((threadIdx.x & 31u) == 0) { s1[threadIdx.x >> 5] = a; s2[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t1 = 0.0, t2 = 0.0;
        for (u32 w = 0; w < blockDim.x / 32; ++w) { t1 += s1[w]; t2 += s2[w]; }
        out2[0] = n ? static_cast<float>(t1 / static_cast<double>(n)) : 0.f;
        out2[1] = static_cast<float>(0.5 * static_cast<double>(mass) * t2);
    }
}

template <bool BATCH>
__global__ void boundary_mass_kernel(const DevParams P, const float4* __restrict__ bpos, u32 nb, HashView bh,
                                     float* __restrict__ bmass, const u64* __restrict__ bckey) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nb) return;
    const float4 xi = bpos[i];
    const int3 c = cell_of(xi, P.h);
    const u32 scene = BATCH ? static_cast<u32>(bckey[i] >> 48) : 0u;
    float sum = P.w0;  // cubic_spline(0, h)
    for (int x = -1; x <= 1; ++x)
        for (int y = -1; y <= 1; ++y)
            for (int z = -1; z <= 1; ++z) {
                u64 pk;
                if constexpr (BATCH)
                    pk = pack_cell_batch(scene, offset_coord(c.x) + x, offset_coord(c.y) + y, offset_coord(c.z) + z);
                else
                    pk = pack_cell(offset_coord(c.x) + x, offset_coord(c.y) + y, offset_coord(c.z) + z);
                const u32 slot = hash_find<BATCH>(bh.table, bh.tmask, pk);
                if (slot == EMPTY_CELL) continue;
                const u32 s = bh.cstart[slot], e = bh.cend[slot];
                for (u32 j = s; j < e; ++j) {
                    const float4 xj = bpos[j];
                    const float r2 = dist2(xi, xj);
                    if (j != i && r2 <= P.h2) sum += cubic_w(sqrtf(r2) * P.inv_h, P);
                }
            }
    bmass[i] = P.rest_density / sum;
}

}  // namespace

u32 pass_grid(u32 n, int wpb, u32 chunk) {
    const u32 chunks = (n + chunk - 1) / chunk;
    return (chunks + wpb - 1) / wpb;
}

void launch_reorder_cells(const float4* pos_in, const float4* vel_in, const u32* perm_src1, const u32* perm_src2,
                          const DevState* st, u32 n, float cs, float4* pos_out, float4* vel_out, u32* perm_out,
                          u64* ckey_out, u64* table, u32* cstart, u32* cend, u32 tmask, DevState* st_err,
                          cudaStream_t stream, const u32* scene_in) {
    if (n == 0) return;
    const u32 threads = 256;
    const u32 grid = (n + threads - 1) / threads;
    if (scene_in)
        reorder_cells_kernel<true><<<grid, threads, 0, stream>>>(pos_in, vel_in, perm_src1, perm_src2, st, n, cs,
                                                                 pos_out, vel_out, perm_out, ckey_out, table, cstart,
                                                                 cend, tmask, st_err, scene_in);
    else
        reorder_cells_kernel<false><<<grid, threads, 0, stream>>>(pos_in, vel_in, perm_src1, perm_src2, st, n, cs,
                                                                  pos_out, vel_out, perm_out, ckey_out, table, cstart,
                                                                  cend, tmask, st_err, nullptr);
}

template <int KIND, int WPB, bool BATCH>
static void launch_wpb(const DevParams& P, const TravArgs& a, cudaStream_t stream, u32 grid) {
    // per-warp candidate staging sized by the bit-matrix capacity 32 * mask_words
    if constexpr (KIND == PASS_FORCE || KIND == PASS_SURFACE) {
        if (a.nbr) {   // the list kernels use no shared memory (all of it serves as L1)
            list_pass_kernel<KIND, WPB, BATCH><<<grid, WPB * 32, 0, stream>>>(P, a);
            return;
        }
    }
    const u32 ncell = static_cast<u32>((2 * a.range + 1) * (2 * a.range + 1) * (2 * a.range + 1));
    const size_t bytes = warp_smem_bytes<KIND>(a.mask_words * 32u, ncell, a.nb > 0) * WPB;
    static bool configured = false;  // per instantiation; the attribute is per device function
    if (!configured) {
        cudaFuncSetAttribute(cell_pass_kernel<KIND, WPB, BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(warp_smem_bytes<KIND>(32u * MAX_MASK_WORDS, MAX_RANGE_CELLS, true) * WPB));
        configured = true;
    }
    cell_pass_kernel<KIND, WPB, BATCH><<<grid, WPB * 32, bytes, stream>>>(P, a);
}

template <int KIND, bool BATCH>
static void launch_kind(const DevParams& P, const TravArgs& a, cudaStream_t stream, int wpb) {
    const bool listed = (KIND == PASS_FORCE || KIND == PASS_SURFACE) && a.nbr != nullptr;
    const u32 grid = pass_grid(a.n, wpb, listed ? list_rows_per_warp(a.chunk) : a.chunk);
    if (grid == 0) return;
    switch (wpb) {
    case 2: launch_wpb<KIND, 2, BATCH>(P, a, stream, grid); break;
    case 8: launch_wpb<KIND, 8, BATCH>(P, a, stream, grid); break;
    default: launch_wpb<KIND, 4, BATCH>(P, a, stream, grid); break;
    }
}

template <bool BATCH>
static void launch_pass_t(int kind, const DevParams& P, const TravArgs& a, cudaStream_t stream, int wpb) {
    switch (kind) {
    case PASS_DENSITY: launch_kind<PASS_DENSITY, BATCH>(P, a, stream, wpb); break;
    case PASS_FORCE: launch_kind<PASS_FORCE, BATCH>(P, a, stream, wpb); break;
    case PASS_SURFACE: launch_kind<PASS_SURFACE, BATCH>(P, a, stream, wpb); break;
    case PASS_COUNT: launch_kind<PASS_COUNT, BATCH>(P, a, stream, wpb); break;
    case PASS_FILL: launch_kind<PASS_FILL, BATCH>(P, a, stream, wpb); break;
    case PASS_ADJ_FORCE: launch_kind<PASS_ADJ_FORCE, BATCH>(P, a, stream, wpb); break;
    case PASS_ADJ_DENSITY: launch_kind<PASS_ADJ_DENSITY, BATCH>(P, a, stream, wpb); break;
    default: break;
    }
}

void launch_pass(int kind, const DevParams& P, const TravArgs& a, cudaStream_t stream, int wpb, bool batch) {
    if (wpb != 2 && wpb != 8) wpb = 4;
    if (batch) launch_pass_t<true>(kind, P, a, stream, wpb);
    else launch_pass_t<false>(kind, P, a, stream, wpb);
}

void launch_init_cfl(const float4* vel, u32 n, DevState* st, cudaStream_t stream) {
    if (n == 0) return;
    const u32 blocks = std::min<u32>((n + 255) / 256, 1184);
    init_cfl_kernel<<<blocks, 256, 0, stream>>>(vel, n, st);
}

void launch_boundary_mass(const DevParams& P, const float4* bpos, u32 nb, HashView bh, float* bmass,
                          cudaStream_t stream, const u64* bckey) {
    if (nb == 0) return;
    if (bckey) boundary_mass_kernel<true><<<(nb + 127) / 128, 128, 0, stream>>>(P, bpos, nb, bh, bmass, bckey);
    else boundary_mass_kernel<false><<<(nb + 127) / 128, 128, 0, stream>>>(P, bpos, nb, bh, bmass, nullptr);
}

void launch_metrics(const float4* vel, u32 n, float mass, float* out2, cudaStream_t stream) {
    metrics_kernel<<<1, 1024, 0, stream>>>(vel, n, mass, out2);
}

}  // namespace wcsph
