// boundary_cells.cu — per-cell boundary candidate lists.
//
// Boundary particles do not move, so the candidates a fluid particle in cell c
// tests against them — the boundary particles of the 27 cells around c, in the
// (dx, dy, dz) nesting order of for_boundary_neighbors (common.cuh:153-178) —
// depend on c alone. They are gathered once, when the boundary is set, for
// every cell within one cell of an occupied boundary cell ("near" cells),
// into one contiguous run per near cell of (x, y, z, mass). A pass then
// finds a particle's boundary candidates with one hash lookup and reads them
// as a contiguous array, instead of 27 lookups and a gather per candidate;
// a particle outside every near cell has no boundary neighbour, and its one
// lookup finds nothing. The candidate order, and with it the order of the
// boundary sums, is the reference's.
//
// Build (stream-ordered, once per boundary):
//   1. count the occupied boundary cells (slots of the boundary hash);
//   2. insert the 27 neighbours of each into a key-only hash sized for 27
//      per occupied cell at half load (so it cannot fill up), count the
//      distinct near cells, and move them into the near-cell hash proper,
//      sized for them at a quarter load (walls have 3-5 near cells per
//      occupied cell, so this table is several times smaller; at half load
//      the longer probe chains cost 0.5 % of the ensemble step);
//   3. per near cell, the candidate count (27 lookups in the boundary hash);
//   4. exclusive scan of the counts (CUB) -> run starts; total read back;
//   5. per near cell, copy its candidates into its run.
#include <cub/cub.cuh>

#include <algorithm>
#include <bit>

#include "simulator.cuh"

namespace wcsph {
namespace {

// Packed key of the neighbour (dx, dy, dz) of the cell with packed key pk.
template <bool BATCH>
__device__ __forceinline__ u64 neighbour_key(u64 pk, int q) {
    const int dx = q / 9 - 1, dy = (q / 3) % 3 - 1, dz = q % 3 - 1;
    if constexpr (BATCH) {
        const u32 scene = static_cast<u32>(pk >> 48);
        return pack_cell_batch(scene, static_cast<u32>(pk & 0xFFFFull) + dx,
                               static_cast<u32>((pk >> 16) & 0xFFFFull) + dy,
                               static_cast<u32>((pk >> 32) & 0xFFFFull) + dz);
    } else {
        return pack_cell(static_cast<u32>(pk & 0x1FFFFFull) + dx, static_cast<u32>((pk >> 21) & 0x1FFFFFull) + dy,
                         static_cast<u32>((pk >> 42) & 0x1FFFFFull) + dz);
    }
}

__global__ void count_cells_kernel(const u64* __restrict__ table, u32 size, u32* __restrict__ count) {
    u32 c = 0;
    for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < size; t += gridDim.x * blockDim.x)
        c += table[t] != EMPTY_HASH ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31u) == 0 && c) atomicAdd(count, c);
}

template <bool BATCH>
__global__ void near_insert_kernel(const u64* __restrict__ btable, u32 bsize, u64* near, u32 nmask,
                                   DevState* st) {
    for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < bsize; t += gridDim.x * blockDim.x) {
        const u64 pk = btable[t];
        if (pk == EMPTY_HASH) continue;
        for (int q = 0; q < 27; ++q)
            if (hash_insert<BATCH>(near, nmask, neighbour_key<BATCH>(pk, q)) == EMPTY_CELL)
                atomicOr(&st->error_flags, ERR_HASH_FULL);
    }
}

template <bool BATCH>
__global__ void rehash_kernel(const u64* __restrict__ from, u32 fsize, u64* to, u32 tmask, DevState* st) {
    for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < fsize; t += gridDim.x * blockDim.x) {
        const u64 pk = from[t];
        if (pk != EMPTY_HASH && hash_insert<BATCH>(to, tmask, pk) == EMPTY_CELL) atomicOr(&st->error_flags, ERR_HASH_FULL);
    }
}

template <bool BATCH>
__global__ void near_count_kernel(HashView bh, const u64* __restrict__ near, u32 nsize, u32* __restrict__ count) {
    for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < nsize; t += gridDim.x * blockDim.x) {
        const u64 pk = near[t];
        u32 c = 0;
        if (pk != EMPTY_HASH) {
            for (int q = 0; q < 27; ++q) {
                const u32 s = hash_find<BATCH>(bh.table, bh.tmask, neighbour_key<BATCH>(pk, q));
                if (s != EMPTY_CELL) c += bh.cend[s] - bh.cstart[s];
            }
        }
        count[t] = c;
    }
}

template <bool BATCH>
__global__ void near_fill_kernel(HashView bh, const u64* __restrict__ near, u32 nsize, const u32* __restrict__ start,
                                 u32* __restrict__ end, const float4* __restrict__ bpos,
                                 const float* __restrict__ bmass, float4* __restrict__ out) {
    for (u32 t = blockIdx.x * blockDim.x + threadIdx.x; t < nsize; t += gridDim.x * blockDim.x) {
        const u64 pk = near[t];
        u32 o = start[t];
        if (pk != EMPTY_HASH) {
            for (int q = 0; q < 27; ++q) {
                const u32 s = hash_find<BATCH>(bh.table, bh.tmask, neighbour_key<BATCH>(pk, q));
                if (s == EMPTY_CELL) continue;
                const u32 e = bh.cend[s];
                for (u32 b = bh.cstart[s]; b < e; ++b) {
                    const float4 x = bpos[b];
                    out[o++] = make_float4(x.x, x.y, x.z, bmass[b]);
                }
            }
        }
        end[t] = o;
    }
}

u32 grid_for(u32 n) { return std::max<u32>(1u, std::min<u32>((n + 255) / 256, 4096)); }

}  // namespace

void build_boundary_cells(BoundaryCells& bc, const HashView& bh, u32 bsize, u32 nb, const float4* bpos,
                          const float* bmass, bool batch, DevState* st, cudaStream_t s) {
    bc = BoundaryCells{};
    // run offsets are 32-bit: every boundary particle appears in at most 27 runs
    if (bsize == 0 || nb == 0 || 27ull * nb >= (1ull << 32)) return;
    DevBuf<u32> counter(1);
    WCSPH_CUDA(cudaMemsetAsync(counter.ptr, 0, sizeof(u32), s));
    count_cells_kernel<<<grid_for(bsize), 256, 0, s>>>(bh.table, bsize, counter.ptr);
    WCSPH_CUDA(cudaGetLastError());
    u32 cells = 0;
    WCSPH_CUDA(cudaMemcpyAsync(&cells, counter.ptr, sizeof(u32), cudaMemcpyDeviceToHost, s));
    WCSPH_CUDA(cudaStreamSynchronize(s));
    if (cells == 0 || 54ull * cells > (1ull << 31)) return;
    u32 nsize = 0;
    {
        const u32 wsize = static_cast<u32>(std::bit_ceil(std::max<u64>(64, 54ull * cells)));
        DevBuf<u64> wide(wsize);
        WCSPH_CUDA(cudaMemsetAsync(wide.ptr, 0xff, wide.bytes(), s));
        if (batch) near_insert_kernel<true><<<grid_for(bsize), 256, 0, s>>>(bh.table, bsize, wide.ptr, wsize - 1, st);
        else near_insert_kernel<false><<<grid_for(bsize), 256, 0, s>>>(bh.table, bsize, wide.ptr, wsize - 1, st);
        WCSPH_CUDA(cudaGetLastError());
        WCSPH_CUDA(cudaMemsetAsync(counter.ptr, 0, sizeof(u32), s));
        count_cells_kernel<<<grid_for(wsize), 256, 0, s>>>(wide.ptr, wsize, counter.ptr);
        WCSPH_CUDA(cudaGetLastError());
        u32 near = 0;
        WCSPH_CUDA(cudaMemcpyAsync(&near, counter.ptr, sizeof(u32), cudaMemcpyDeviceToHost, s));
        WCSPH_CUDA(cudaStreamSynchronize(s));
        nsize = static_cast<u32>(std::bit_ceil(std::max<u64>(64, 4ull * near)));
        bc.table.alloc(nsize);
        WCSPH_CUDA(cudaMemsetAsync(bc.table.ptr, 0xff, bc.table.bytes(), s));
        if (batch) rehash_kernel<true><<<grid_for(wsize), 256, 0, s>>>(wide.ptr, wsize, bc.table.ptr, nsize - 1, st);
        else rehash_kernel<false><<<grid_for(wsize), 256, 0, s>>>(wide.ptr, wsize, bc.table.ptr, nsize - 1, st);
        WCSPH_CUDA(cudaGetLastError());
        WCSPH_CUDA(cudaStreamSynchronize(s));   // before the wide table is freed
    }
    bc.start.alloc(nsize);
    bc.end.alloc(nsize);
    bc.size = nsize;
    DevBuf<u32> count(nsize);
    if (batch) near_count_kernel<true><<<grid_for(nsize), 256, 0, s>>>(bh, bc.table.ptr, nsize, count.ptr);
    else near_count_kernel<false><<<grid_for(nsize), 256, 0, s>>>(bh, bc.table.ptr, nsize, count.ptr);
    WCSPH_CUDA(cudaGetLastError());
    size_t temp = 0;
    WCSPH_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, count.ptr, bc.start.ptr, nsize, s));
    DevBuf<unsigned char> tmp(std::max<size_t>(temp, 1));
    WCSPH_CUDA(cub::DeviceScan::ExclusiveSum(tmp.ptr, temp, count.ptr, bc.start.ptr, nsize, s));
    u32 last[2] = {0, 0};
    WCSPH_CUDA(cudaMemcpyAsync(&last[0], bc.start.ptr + (nsize - 1), sizeof(u32), cudaMemcpyDeviceToHost, s));
    WCSPH_CUDA(cudaMemcpyAsync(&last[1], count.ptr + (nsize - 1), sizeof(u32), cudaMemcpyDeviceToHost, s));
    WCSPH_CUDA(cudaStreamSynchronize(s));
    const u64 total = static_cast<u64>(last[0]) + last[1];
    bc.x.alloc(std::max<u64>(total, 1));
    if (batch)
        near_fill_kernel<true><<<grid_for(nsize), 256, 0, s>>>(bh, bc.table.ptr, nsize, bc.start.ptr, bc.end.ptr, bpos,
                                                               bmass, bc.x.ptr);
    else
        near_fill_kernel<false><<<grid_for(nsize), 256, 0, s>>>(bh, bc.table.ptr, nsize, bc.start.ptr, bc.end.ptr,
                                                                bpos, bmass, bc.x.ptr);
    WCSPH_CUDA(cudaGetLastError());
    WCSPH_CUDA(cudaStreamSynchronize(s));
}

}  // namespace wcsph
