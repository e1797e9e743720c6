// radix_sort.cu — see radix_sort.cuh for the design.
#include "radix_sort.cuh"
#include "radix_sort_dev.cuh"

#include <atomic>


namespace wcsph {

namespace {
std::atomic<bool> g_sort_stall_test{false};
}

void set_sort_stall_test(bool on) { g_sort_stall_test.store(on); }


__global__ void keys_hist_kernel(const float4* __restrict__ pos, u32 n, float cs,
                                 u64* __restrict__ keys_out, u32* __restrict__ hist,
                                 const u32* __restrict__ scene) {
    __shared__ u32 s_hist[SORT_DIGITS][256];
    sortdev::keys_hist_block(pos, n, cs, keys_out, hist, scene, s_hist, blockIdx.x * blockDim.x,
                             gridDim.x * blockDim.x);
}

__global__ void keys_bounds_kernel(const float4* __restrict__ pos, u32 n, float cs, u64* __restrict__ keys_out,
                                   DevState* __restrict__ st) {
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    auto take = [&](float4 x, u32 i) {
        const int3 c = cell_of(x, cs);
        keys_out[i] = morton_key(c);
        lo[0] = min(lo[0], c.x); hi[0] = max(hi[0], c.x);
        lo[1] = min(lo[1], c.y); hi[1] = max(hi[1], c.y);
        lo[2] = min(lo[2], c.z); hi[2] = max(hi[2], c.z);
    };
    const u32 stride = gridDim.x * blockDim.x;
    u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {   // four loads in flight per thread
        float4 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) x[u] = pos[i + u * stride];
#pragma unroll
        for (int u = 0; u < 4; ++u) take(x[u], i + u * stride);
    }
    for (; i < n; i += stride) take(pos[i], i);
    // warp, then block, then one atomic per axis and block
    __shared__ int s_lo[3], s_hi[3];
    if (threadIdx.x < 3) { s_lo[threadIdx.x] = 0; s_hi[threadIdx.x] = 0; }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        lo[d] = __reduce_min_sync(0xffffffffu, lo[d]);
        hi[d] = __reduce_max_sync(0xffffffffu, hi[d]);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            atomicMin(&s_lo[d], lo[d]);
            atomicMax(&s_hi[d], hi[d]);
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        if (s_lo[threadIdx.x] < 0) atomicMin(&st->cell_lo[threadIdx.x], s_lo[threadIdx.x]);
        if (s_hi[threadIdx.x] > 0) atomicMax(&st->cell_hi[threadIdx.x], s_hi[threadIdx.x]);
    }
}

__global__ void compressed_keys_hist_kernel(const float4* __restrict__ pos, u32 n, float cs,
                                            const DevState* __restrict__ st, u64* __restrict__ ckeys,
                                            u32* __restrict__ hist) {
    __shared__ u32 s_hist[SORT_DIGITS][256];
    for (int t = threadIdx.x; t < SORT_DIGITS * 256; t += blockDim.x) (&s_hist[0][0])[t] = 0;
    // smallest B with every cell coordinate in [-2^B, 2^B); B = 20 is the full key
    const int lo = min(st->cell_lo[0], min(st->cell_lo[1], st->cell_lo[2]));
    const int hi = max(st->cell_hi[0], max(st->cell_hi[1], st->cell_hi[2]));
    int B = 0;
    while (B < 20 && !(lo >= -(1 << B) && hi < (1 << B))) ++B;
    const int ndigits = (3 * (B + 1) + 7) / 8;   // digits above are 0 for every key
    u32 valid_keys = 0;
    __syncthreads();
    const u32 stride = gridDim.x * blockDim.x;
    // uniform trip count per warp (match.any); four loads in flight per thread
    for (u32 base = blockIdx.x * blockDim.x; base < n; base += 4 * stride) {
        float4 x[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const u32 i = base + u * stride + threadIdx.x;
            if (i < n) x[u] = pos[i];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const u32 i = base + u * stride + threadIdx.x;
            const bool valid = i < n;
            u64 key = 0;
            if (valid) {
                const int3 c = cell_of(x[u], cs);
                key = part_by_3(static_cast<u32>(c.x + (1 << B))) |
                      (part_by_3(static_cast<u32>(c.y + (1 << B))) << 1) |
                      (part_by_3(static_cast<u32>(c.z + (1 << B))) << 2);
                ckeys[i] = key;
                ++valid_keys;
            }
            sortdev::hist_add_key(s_hist, key, valid, ndigits);
        }
    }
    // the digits above ndigits: every key in bucket 0
    for (int o = 16; o > 0; o >>= 1) valid_keys += __shfl_xor_sync(0xffffffffu, valid_keys, o);
    if ((threadIdx.x & 31) == 0 && valid_keys)
        for (int p = ndigits; p < SORT_DIGITS; ++p) atomicAdd(&s_hist[p][0], valid_keys);
    __syncthreads();
    sortdev::flush_hist(s_hist, hist);
}

__global__ void hist_only_kernel(const u64* __restrict__ keys, u32 n, u32* __restrict__ hist) {
    __shared__ u32 s_hist[SORT_DIGITS][256];
    for (int t = threadIdx.x; t < SORT_DIGITS * 256; t += blockDim.x) (&s_hist[0][0])[t] = 0;
    __syncthreads();
    const u32 stride = gridDim.x * blockDim.x;
    for (u32 base = blockIdx.x * blockDim.x; base < n; base += stride) {
        const u32 i = base + threadIdx.x;
        const bool valid = i < n;
        const u64 key = valid ? keys[i] : 0ull;
        sortdev::hist_add_key(s_hist, key, valid);
    }
    __syncthreads();
    sortdev::flush_hist(s_hist, hist);
}

// One CTA of 256 threads (8 warps): digit offsets of every pass, and which
// passes are trivial.
__global__ void sort_plan_kernel(u32 n, u32* __restrict__ hist, u32* __restrict__ offsets,
                                 DevState* __restrict__ st) {
    __shared__ u32 s_active[SORT_DIGITS];
    sortdev::sort_plan_block(n, hist, offsets, st, s_active);
}

__global__ void __launch_bounds__(SORT_THREADS)
onesweep_kernel(u32 n, int pass, u64* __restrict__ k0, u64* __restrict__ k1, u64* __restrict__ k2,
                u32* __restrict__ v1, u32* __restrict__ v2, const u32* __restrict__ offsets,
                u32* __restrict__ lookback, u32 tiles, DevState* __restrict__ st, u32 spin_limit,
                u32 stall_first_tile) {
    if (!st->sort_active[pass]) return;
    __shared__ u32 s_tile;
    __shared__ u32 s_wcnt[SORT_THREADS / 32][256];
    __shared__ u32 s_base[256];
    if (threadIdx.x == 0) s_tile = atomicAdd(&st->sort_tile_counter[pass], 1u);
    __syncthreads();
    const u32 tile = s_tile;
    if (tile >= tiles) return;  // cannot happen: grid == tiles
    sortdev::onesweep_tile(n, pass, k0, k1, k2, v1, v2, offsets, lookback, tiles, st, spin_limit,
                           stall_first_tile, tile, s_wcnt, s_base);
}

cudaError_t enqueue_sort_passes(const SortBuffers& b, u32 n, DevState* st, cudaStream_t stream) {
    const u32 tiles = sort_tiles(n);
    if (n == 0) return cudaSuccess;
    const bool stall = g_sort_stall_test.load();
    const u32 spin_limit = stall ? LB_SPIN_LIMIT_STALLED : LB_SPIN_LIMIT;
    sort_plan_kernel<<<1, 256, 0, stream>>>(n, b.hist, b.offsets, st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(b.lookback, 0, sizeof(u32) * SORT_DIGITS * static_cast<size_t>(tiles) * 256u, stream);
    if (e != cudaSuccess) return e;
    for (int p = 0; p < SORT_DIGITS; ++p) {
        onesweep_kernel<<<tiles, SORT_THREADS, 0, stream>>>(n, p, b.keys[0], b.keys[1], b.keys[2],
                                                            b.vals[1], b.vals[2], b.offsets, b.lookback,
                                                            tiles, st, spin_limit, stall ? 1u : 0u);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace wcsph
