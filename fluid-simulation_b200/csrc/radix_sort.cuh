// radix_sort.cuh — stable onesweep LSD radix sort of (u64 Morton key, u32
// particle index) pairs with digit skipping.
//
// Replaces thrust::sort_by_key in ParticleData::sort
// (src/cuda/SPH/particle_data.cuh:127). Any stable sort of the same keys gives
// the same permutation, which is what the parity tests check bit-exactly.
//
// Design (one launch per 8-bit digit, no separate upsweep):
//   keys_hist   : keys from positions + 8 digit histograms in one read
//   sort_plan   : 1 CTA — exclusive digit offsets; a digit whose histogram
//                 has a single non-empty bucket is constant over all keys and
//                 its pass is skipped (the reference's 63-bit keys usually
//                 vary in only 2-3 of the 8 digits); ping-pong buffer plan.
//   onesweep    : per 2048-key tile: warp-level match.any ranking, per-digit
//                 decoupled look-back across tiles (bounded spin), scatter.
// Buffers: keys[0] holds the input-order keys and is never overwritten (it is
// the MORTON_KEYS parity field); passes alternate between keys[1]/keys[2]
// and vals[1]/vals[2]. The first active pass generates the iota values.
#pragma once
#include "sph_common.cuh"

namespace wcsph {

constexpr int SORT_THREADS = 256;
constexpr int SORT_IPT = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_IPT;  // 2048 keys per tile
constexpr int SORT_DIGITS = 8;                      // 8 x 8-bit digits = 64 bits
constexpr u32 LB_FLAG_AGG = 1u << 30;
constexpr u32 LB_FLAG_INC = 2u << 30;
constexpr u32 LB_VALUE_MASK = (1u << 30) - 1u;
constexpr u32 LB_SPIN_LIMIT = 1u << 22;        // polls of one look-back wait (about a second)
constexpr u32 LB_SPIN_LIMIT_STALLED = 1u << 12; // with the stall test hook on (a few milliseconds)

inline u32 sort_tiles(u32 n) { return (n + SORT_TILE - 1) / SORT_TILE; }

struct SortBuffers {
    u64* keys[3];     // [0] input order (preserved), [1],[2] ping-pong
    u32* vals[3];     // [0] unused, [1],[2] ping-pong
    u32* hist;        // [8][256] digit histograms (kept zero between sorts)
    u32* offsets;     // [8][256] exclusive digit offsets
    u32* lookback;    // [8][tiles][256]
    u32 capacity;     // max keys
};

// Computes Morton keys of `pos` (cell = floorf(p / cs), particle_data.cuh:117-125)
// into keys[0] and accumulates the 8 digit histograms.
// With `scene` (batched ensembles) the key is batch_key(scene[i], cell).
__global__ void keys_hist_kernel(const float4* __restrict__ pos, u32 n, float cs,
                                 u64* __restrict__ keys_out, u32* __restrict__ hist,
                                 const u32* __restrict__ scene = nullptr);
// The per-step keys of a single scene, in two arrays:
//  * keys_bounds_kernel writes the reference's 63-bit Morton keys (the
//    MORTON_KEYS field) and folds the cell-coordinate bounds into st;
//  * compressed_keys_hist_kernel writes order-equivalent short keys for the
//    sort and their digit histograms. With every cell coordinate c in
//    [-2^B, 2^B), the offset coordinate u = c + 2^20 has bits B..19 equal to
//    NOT bit 20, so those bits never decide a Morton comparison; v = c + 2^B
//    keeps exactly bits 0..B-1 and bit 20 (as bit B), and Morton(v) orders any
//    two particles as Morton(u) does. A scene of 125 x 63 x 63 cells around
//    the origin needs 24 bits (3 digit passes) instead of 63 (8 passes); the
//    stable sort gives the same permutation.
__global__ void keys_bounds_kernel(const float4* __restrict__ pos, u32 n, float cs, u64* __restrict__ keys_out,
                                   DevState* __restrict__ st);
__global__ void compressed_keys_hist_kernel(const float4* __restrict__ pos, u32 n, float cs,
                                            const DevState* __restrict__ st, u64* __restrict__ ckeys,
                                            u32* __restrict__ hist);
// Histograms of already-computed keys (boundary sort, re-sorts).
__global__ void hist_only_kernel(const u64* __restrict__ keys, u32 n, u32* __restrict__ hist);
__global__ void sort_plan_kernel(u32 n, u32* __restrict__ hist, u32* __restrict__ offsets,
                                 DevState* __restrict__ st);
// spin_limit bounds every look-back wait; stall_first_tile makes tile 0
// withhold its look-back flags (the error-path test hook below), so that the
// waits of the later tiles run out and set ERR_LOOKBACK_TIMEOUT.
__global__ void onesweep_kernel(u32 n, int pass, u64* __restrict__ k0, u64* __restrict__ k1,
                                u64* __restrict__ k2, u32* __restrict__ v1, u32* __restrict__ v2,
                                const u32* __restrict__ offsets, u32* __restrict__ lookback,
                                u32 tiles, DevState* __restrict__ st, u32 spin_limit, u32 stall_first_tile);

// Enqueues the complete sort (after keys[0] and hist are filled) on `stream`.
// Returns the first enqueue error (cudaSuccess when every call was accepted).
// A pass whose look-back wait ran out sets ERR_LOOKBACK_TIMEOUT in
// st->error_flags; its permutation is then not a permutation, and every
// kernel that would read it (reorder, the traversal passes) leaves its
// outputs untouched instead.
cudaError_t enqueue_sort_passes(const SortBuffers& b, u32 n, DevState* st, cudaStream_t stream);

// Error-path test hook: while on, sorts enqueued afterwards stall tile 0's
// look-back flags and wait at most LB_SPIN_LIMIT_STALLED polls.
void set_sort_stall_test(bool on);

}  // namespace wcsph
