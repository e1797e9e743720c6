// batch.cuh — batched ensemble of independent scenes (batch.cu) and its
// persistent kernel (batch_persistent.cu).
#pragma once
#include "simulator.cuh"

namespace wcsph {

// Everything one launch of the persistent ensemble kernel needs: the
// traversal arguments of the whole ensemble plus the sort and hash buffers.
struct PersistentStep {
    DevParams P;
    TravArgs a;              // pos/vel = sorted scratch (B), pos_out/vel_out = state (A)
    const float4* pos_state; // state positions and velocities read by the keys and the reorder
    const float4* vel_state;
    u32* scene_state;        // scene id of each state particle
    u64* keys[3];
    u32* vals[3];
    u32* hist;
    u32* offsets;
    u32* lookback;
    u32 tiles;
    u32* perm;
    u64* table;
    u32 table_size;
    float cs;
    u32* barrier;            // [arrivals, generation] (zero between launches), then work counters
    int steps;
    u32 spin_limit;          // look-back polls
    u32 barrier_limit;       // grid-barrier polls (64 ns apart)
};

// Blocks of the persistent kernel that fit on the device at once (the grid of
// its cooperative launch) and the dynamic shared memory per block.
void persistent_grid(const TravArgs& a, int device, u32* blocks, size_t* smem);
// Enqueues `steps` steps of the whole ensemble as one cooperative launch.
void launch_persistent(const PersistentStep& ps, u32 blocks, size_t smem, cudaStream_t stream);

}  // namespace wcsph
