// radix_sort_dev.cuh — device-side building blocks of the onesweep radix sort
// (radix_sort.cuh has the design). The sort's kernels wrap them, and the
// persistent batched-ensemble kernel calls them between its grid barriers;
// both therefore sort with the same code and produce the same permutation.
#pragma once
#include <cuda/atomic>

#include "radix_sort.cuh"

// The persistent ensemble kernel rewrites the sort buffers within one launch
// and includes this file with WCSPH_COHERENT_LOADS 1: pointer arguments then
// carry no __restrict__, so that no load takes the non-coherent read-only path.
#ifndef WCSPH_COHERENT_LOADS
#define WCSPH_COHERENT_LOADS 0
#endif
#if WCSPH_COHERENT_LOADS
#define WCSPH_SORT_RESTRICT
#else
#define WCSPH_SORT_RESTRICT __restrict__
#endif

namespace wcsph {
namespace {   // internal linkage: each translation unit has its own flavour
namespace sortdev {

__device__ __forceinline__ u32 lanemask_lt() {
    u32 m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Warp-aggregated shared-memory increment of 8 digit histograms for one key
// per lane. Many lanes share digits (keys arrive nearly sorted), so each
// distinct digit value gets one atomic.
__device__ __forceinline__ void hist_add_key(u32 (*s_hist)[256], u64 key, bool valid, int ndigits = SORT_DIGITS) {
    const u32 lane = threadIdx.x & 31;
#pragma unroll
    for (int p = 0; p < SORT_DIGITS; ++p) {
        if (p >= ndigits) break;   // uniform across the grid
        const u32 d = valid ? static_cast<u32>((key >> (8 * p)) & 255u) : 256u;
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const u32 leader = __ffs(peers) - 1;
        if (valid && lane == leader) atomicAdd(&s_hist[p][d], static_cast<u32>(__popc(peers)));
    }
}

__device__ __forceinline__ void flush_hist(u32 (*s_hist)[256], u32* hist) {
    for (int t = threadIdx.x; t < SORT_DIGITS * 256; t += blockDim.x) {
        const u32 c = (&s_hist[0][0])[t];
        if (c) atomicAdd(hist + t, c);
    }
}

// One block: keys of particles base + threadIdx.x for base = first, first +
// stride, ... (< n) into keys_out, and their 8 digit histograms added to hist.
// With `scene` (batched ensembles) the key is batch_key(scene[i], cell).
__device__ __forceinline__ void keys_hist_block(const float4* WCSPH_SORT_RESTRICT pos, u32 n, float cs,
                                                u64* WCSPH_SORT_RESTRICT keys_out, u32* WCSPH_SORT_RESTRICT hist,
                                                const u32* WCSPH_SORT_RESTRICT scene, u32 (*s_hist)[256], u32 first,
                                                u32 stride) {
    for (int t = threadIdx.x; t < SORT_DIGITS * 256; t += blockDim.x) (&s_hist[0][0])[t] = 0;
    __syncthreads();
    // The loop trip count is uniform across the warp (match.any needs all lanes).
    for (u32 base = first; base < n; base += stride) {
        const u32 i = base + threadIdx.x;
        const bool valid = i < n;
        u64 key = 0;
        if (valid) {
            const int3 c = cell_of(pos[i], cs);
            key = scene ? batch_key(scene[i], c) : morton_key(c);
            keys_out[i] = key;
        }
        hist_add_key(s_hist, key, valid);
    }
    __syncthreads();
    flush_hist(s_hist, hist);
}

// One block of at least 256 threads: exclusive digit offsets of every pass
// (and the histograms cleared for the next sort), which passes are trivial,
// and the ping-pong buffer plan.
__device__ __forceinline__ void sort_plan_block(u32 n, u32* WCSPH_SORT_RESTRICT hist, u32* WCSPH_SORT_RESTRICT offsets,
                                                DevState* WCSPH_SORT_RESTRICT st, u32* s_active) {
    // one warp per digit pass: lane l scans buckets 8l .. 8l + 7 serially,
    // then the lanes' totals are scanned across the warp (no block barriers)
    const u32 t = threadIdx.x;
    const u32 pass = t >> 5;
    const u32 lane = t & 31u;
    if (pass < SORT_DIGITS) {
        uint4* h = reinterpret_cast<uint4*>(hist + pass * 256 + lane * 8);
        const uint4 h0 = h[0], h1 = h[1];
        h[0] = make_uint4(0u, 0u, 0u, 0u);   // ready for the next sort
        h[1] = make_uint4(0u, 0u, 0u, 0u);
        const u32 c[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
        u32 ex[8];
        u32 run = 0, mx = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            ex[k] = run;
            run += c[k];
            mx = max(mx, c[k]);
        }
        u32 incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const u32 v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= static_cast<u32>(o)) incl += v;
        }
        const u32 base = incl - run;
        uint4* out = reinterpret_cast<uint4*>(offsets + pass * 256 + lane * 8);
        out[0] = make_uint4(base + ex[0], base + ex[1], base + ex[2], base + ex[3]);
        out[1] = make_uint4(base + ex[4], base + ex[5], base + ex[6], base + ex[7]);
        // a pass is trivial when one bucket holds every key
        mx = __reduce_max_sync(0xffffffffu, mx);
        if (lane == 0) s_active[pass] = (n > 0 && mx < n) ? 1u : 0u;
    }
    __syncthreads();
    if (t == 0) {
        u32 sel = 0;
        u32 first = SORT_DIGITS;
        for (int p = 0; p < SORT_DIGITS; ++p) {
            st->sort_active[p] = s_active[p];
            st->sort_sel[p] = sel;
            st->sort_tile_counter[p] = 0;
            if (s_active[p]) {
                if (first == SORT_DIGITS) first = p;
                sel = (sel == 1u) ? 2u : 1u;
            }
        }
        st->sort_sel[SORT_DIGITS] = sel;
        st->first_active = first;
        for (int d = 0; d < 3; ++d) st->cell_lo[d] = st->cell_hi[d] = 0;   // for the next sort
    }
}

// One 2048-key tile of digit pass `pass`, by a block of SORT_THREADS threads:
// warp-level match.any ranking, decoupled look-back over the earlier tiles
// (bounded by spin_limit), scatter. Tiles must be claimed in increasing order
// by running blocks (an atomic counter), so that every tile a look-back waits
// for is already being processed.
__device__ __forceinline__ void onesweep_tile(u32 n, int pass, u64* WCSPH_SORT_RESTRICT k0, u64* WCSPH_SORT_RESTRICT k1,
                                              u64* WCSPH_SORT_RESTRICT k2, u32* WCSPH_SORT_RESTRICT v1, u32* WCSPH_SORT_RESTRICT v2,
                                              const u32* WCSPH_SORT_RESTRICT offsets, u32* WCSPH_SORT_RESTRICT lookback, u32 tiles,
                                              DevState* WCSPH_SORT_RESTRICT st, u32 spin_limit, u32 stall_first_tile,
                                              u32 tile, u32 (*s_wcnt)[256], u32* s_base) {
    constexpr int NW = SORT_THREADS / 32;
    const u32 sel_in = st->sort_sel[pass];
    const u32 sel_out = (sel_in == 1u) ? 2u : 1u;
    const u64* keys_in = sel_in == 0 ? k0 : (sel_in == 1 ? k1 : k2);
    const u32* vals_in = sel_in == 0 ? nullptr : (sel_in == 1 ? v1 : v2);
    u64* keys_out = sel_out == 1 ? k1 : k2;
    u32* vals_out = sel_out == 1 ? v1 : v2;
    const int shift = 8 * pass;

    const u32 tid = threadIdx.x;
    const u32 lane = tid & 31;
    const u32 warp = tid >> 5;
    for (int t = tid; t < NW * 256; t += SORT_THREADS) (&s_wcnt[0][0])[t] = 0;
    __syncthreads();

    u64 key[SORT_IPT];
    u32 val[SORT_IPT];
    u32 dig[SORT_IPT];
    u32 rank[SORT_IPT];
    const u32 wbase = tile * SORT_TILE + warp * (32 * SORT_IPT);
#pragma unroll
    for (int k = 0; k < SORT_IPT; ++k) {
        const u32 idx = wbase + k * 32 + lane;
        if (idx < n) {
            key[k] = keys_in[idx];
            val[k] = vals_in ? vals_in[idx] : idx;
            dig[k] = static_cast<u32>((key[k] >> shift) & 255u);
        } else {
            key[k] = 0;
            val[k] = 0;
            dig[k] = 256u;
        }
    }
    // Stable warp-level ranking: items are warp-striped so (k, lane) order is
    // the input order within the warp's 256-key segment.
    const u32 lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < SORT_IPT; ++k) {
        const u32 d = dig[k];
        const u32 peers = __match_any_sync(0xffffffffu, d);
        const u32 before = __popc(peers & lt);
        u32 base = 0;
        if (d < 256u) base = s_wcnt[warp][d];
        rank[k] = base + before;
        __syncwarp();
        if (d < 256u && (peers >> lane) == 1u)  // highest lane of the peer group
            s_wcnt[warp][d] = base + __popc(peers);
        __syncwarp();
    }
    __syncthreads();

    // Thread t = digit t: exclusive prefix over warps, tile total, look-back.
    {
        const u32 d = tid;
        u32 running = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const u32 c = s_wcnt[w][d];
            s_wcnt[w][d] = running;
            running += c;
        }
        const u32 count = running;
        u32* lb = lookback + (static_cast<size_t>(pass) * tiles) * 256u;
        cuda::atomic_ref<u32, cuda::thread_scope_device> mine(lb[static_cast<size_t>(tile) * 256u + d]);
        u32 excl = 0;
        if (tile == 0) {
            if (!stall_first_tile) mine.store(LB_FLAG_INC | count, cuda::memory_order_relaxed);
        } else {
            mine.store(LB_FLAG_AGG | count, cuda::memory_order_relaxed);
            int pred = static_cast<int>(tile) - 1;
            u32 spins = 0;
            while (pred >= 0) {
                cuda::atomic_ref<u32, cuda::thread_scope_device> other(
                    lb[static_cast<size_t>(pred) * 256u + d]);
                const u32 v = other.load(cuda::memory_order_relaxed);
                const u32 flag = v & ~LB_VALUE_MASK;
                if (flag == 0u) {
                    if (++spins > spin_limit) {  // bounded wait: flag the error, never hang
                        atomicOr(&st->error_flags, ERR_LOOKBACK_TIMEOUT);
                        break;
                    }
                    continue;
                }
                excl += v & LB_VALUE_MASK;
                if (flag == LB_FLAG_INC) break;
                --pred;
            }
            mine.store(LB_FLAG_INC | (excl + count), cuda::memory_order_relaxed);
        }
        s_base[d] = offsets[pass * 256 + d] + excl;
    }
    __syncthreads();

#pragma unroll
    for (int k = 0; k < SORT_IPT; ++k) {
        const u32 d = dig[k];
        if (d < 256u) {
            const u32 dst = s_base[d] + s_wcnt[warp][d] + rank[k];
            if (dst < n) {  // always true unless a look-back wait gave up
                keys_out[dst] = key[k];
                vals_out[dst] = val[k];
            }
        }
    }
}

}  // namespace sortdev
}  // namespace
}  // namespace wcsph
