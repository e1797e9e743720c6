// step_kernels.cuh — the neighbourhood search and SPH force kernels of one
// WCSPH step (everything after the sort).
//
//   reorder_cells   gather pos/vel into sorted order + mark cell runs + insert
//                   cells into the linear-probed hash (cell_start/cell_end)
//                   (particle_data.cuh:130-131 + rebuild_n_search.cu:10-36)
//   density pass    rho, Tait p (+boundary), the cell's neighbour bit matrix
//                   over its candidate list, each particle's neighbour list
//                   and the 32-byte neighbour records of the force pass
//                   (compute_rho_p[_with_boundary], compute_rho_p.cu:192-318)
//   force pass      pressure accel (+boundary), normals, viscosity Laplacian
//                   (compute_pressure_accel_n_normal.cu:240-366 and the
//                   viscosity half of compute_non_pressure_accel.cu:114-144)
//   surface pass    surface tension, a_np, symplectic Euler + box collision,
//                   CFL max |v|^2 and metric reductions
//                   (compute_non_pressure_accel.cu + update_positions.cu:14-68)
//
// Work decomposition (the density pass, and every pass when the lists are
// off): one warp per chunk of 8, 16 or 32 particles of the sorted array
// (small scenes use small chunks so that more warps run); for every cell
// that starts inside the chunk, the warp looks
// up the (2R+1)^3 neighbour cells once (lane-parallel hash probes) and
// stages their particles (the candidates, in the reference's cell order)
// into shared memory. The home particles are taken in blocks of up to 32.
// Every lane does the same amount of work whatever the home count:
//   density pass   phase 1: each lane builds whole words of the block's
//                  neighbour bit matrix (row = home particle, bit =
//                  candidate; rows padded to whole words), testing two
//                  candidates per packed-FP32 step; phase 2 sums W over the
//                  set bits. The matrix is kept row-major in the cell's
//                  mask_words * n_home words of the mask buffer;
//   later passes   walk the set bits of that matrix (neighbours only).
// With neighbour lists on (nbr != nullptr), the density pass also writes each
// particle's neighbours, in candidate order, to its nbr_width list slots
// (slot-major, so that a warp's rows read one slot coalesced), and the force
// and surface passes no longer look at cells: lane k of a warp takes
// particle k of the warp's 32 consecutive particles (8 when the density
// chunk is 8) and sums its list in order, then its boundary
// cells, gathering each neighbour's 32-byte record with one 256-bit load.
// Rows whose neighbours did not fit (count > nbr_width, or a cell beyond
// the bit-matrix capacity) carry NBR_SPILL and are recomputed from their
// cell neighbourhood by the whole warp.
// The bit-matrix walks split the block's neighbours into 32 contiguous lane
// runs; each lane keeps one partial sum per home row it crosses and the
// partials are added per home in lane order, so results are deterministic.
#pragma once
#include "sph_common.cuh"

namespace wcsph {

constexpr int MAX_RANGE_CELLS = 125;     // (2R+1)^3 with R <= 2
constexpr int MAX_BOUNDARY_CELLS = 125;
constexpr u32 MAX_MASK_WORDS = 16;      // bit-matrix words per particle (candidate cap = 32 * words)
constexpr u32 NBR_SPILL = 0xFFFFFFFFu;  // neighbour count of a row whose list is not usable

struct HashView {
    const u64* table;
    const u32* cstart;
    const u32* cend;
    u32 tmask;
};

struct TravArgs {
    u32 n;                    // fluid particles
    const float4* pos;        // sorted positions
    const float4* vel;        // sorted velocities
    const u64* ckey;          // packed cell key per sorted particle
    HashView fluid;
    int range;                // R
    // boundary
    u32 nb;
    const float4* bpos;
    const float* bmass;
    HashView boundary;
    // per-cell boundary candidates (runs of (x, y, z, mass) in bcx; table
    // nullptr: not built, the passes look the 27 boundary cells up)
    HashView bcell;
    const float4* bcx;
    u32 bcx_n;                // entries of bcx
    // per sorted particle: bit m set when candidate m (< 128) of its cell's
    // run is within h; written by the density pass, read by the force pass
    // (nullptr: the force pass tests the whole run)
    uint4* bmask;
    // neighbour bitmasks
    u32* mask;
    u32 mask_words;           // words per particle (candidate cap = 32*mask_words)
    u32 pair_cells;           // density with lists: x-pairs of cells share one traversal; the bit
                              // matrix is then not kept (nothing reads it: the lists carry the sets)
    u32 matrix_valid;         // neighbour export: the mask buffer holds the last density pass's matrix
    u32 chunk;                // sorted particles per warp chunk: 8, 16 or 32
    // neighbour lists (nullptr: the force and surface passes walk the bit matrix)
    u32* nbr;                 // slot t of particle i at nbr[t * n + i], t < nbr_width, candidate order
    u32* nbr_cnt;             // per particle: neighbour count, or NBR_SPILL
    u32 nbr_width;
    // fields
    float* rho;
    float* prs;
    // 32-byte neighbour records (one sector per neighbour) for the gathers of
    // the force and surface passes, two float4 per particle
    float4* recf;             // [2i] (x, y, z, p / rho^2), [2i+1] (v, 1 / rho); density pass
    float4* recs;             // [2i] (x, y, z, rho), [2i+1] normal; force pass
    float4* ap;
    float4* normal;
    float4* vlap;
    float4* anp;
    // integrate outputs (state buffers)
    float4* pos_out;
    float4* vel_out;
    DevBox* box;              // device copy of the collision box
    const DevScene* scenes;   // batched ensembles: per-scene box, gravity, viscosity
    u32* scene_state;         // batched ensembles: scene id of each state particle (written by the integrate pass)
    DevState* st;
    float delta;              // requested step (host value)
    float cfl_factor;
    float max_dt, min_dt, np_max_dt;
    float metric_mass;        // host-side PARTICLE_MASS used by the ke metric
    float* block_partials;    // [warps][2] sum|v|, sum|v|^2 per warp of the surface pass
    u32* group_done;          // [ceil(warps / 32)] arrival counters (zero between launches)
    double* group_partials;   // [ceil(warps / 32)][2]
    // adjoint passes (differentiable rollout)
    const float4* adj_abar;   // dL/da_p per sorted particle
    const float4* adj_w;      // dL/d(vlap) = nu*10*m * dL/da_np
    float4* adj_xbar;         // dL/dx (sorted), accumulated
    float4* adj_vbar;         // dL/dv (sorted), accumulated
    float* adj_rhobar;        // dL/drho (complete after the adjoint force pass)
    double* adj_accum;        // [0] dL/dk
    u32* counts;              // neighbour export: counts
    const u32* offsets;       // neighbour export: offsets
    u32* nbr_out;             // neighbour export: indices
    unsigned long long nbr_capacity;
};

enum PassKind : int {
    PASS_DENSITY = 0, PASS_FORCE = 1, PASS_SURFACE = 2, PASS_COUNT = 3, PASS_FILL = 4,
    PASS_ADJ_FORCE = 5,    // reverse of pressure force (+boundary), viscosity and the Tait EOS
    PASS_ADJ_DENSITY = 6   // reverse of the density sum (+boundary)
};

// scene_in != nullptr selects the batched (scene, cell) keys.
void launch_reorder_cells(const float4* pos_in, const float4* vel_in, const u32* perm_src1,
                          const u32* perm_src2, const DevState* st, u32 n, float cs, float4* pos_out,
                          float4* vel_out, u32* perm_out, u64* ckey_out, u64* table, u32* cstart,
                          u32* cend, u32 tmask, DevState* st_err, cudaStream_t stream,
                          const u32* scene_in = nullptr);

void launch_pass(int kind, const DevParams& P, const TravArgs& a, cudaStream_t stream, int warps_per_block,
                 bool batch = false);
// Blocks of a traversal pass over n particles (chunk particles per warp).
u32 pass_grid(u32 n, int warps_per_block, u32 chunk);
// Upper bound of the warps of any traversal launch over n particles (chunk >= 8,
// at most 8 warps per block): sizes the surface pass's reduction buffers.
inline u32 pass_max_warps(u32 n) { return (n + 7u) / 8u + 8u; }

// CFL max |v|^2 of a velocity array into st->vmax2_bits[st->parity].
void launch_init_cfl(const float4* vel, u32 n, DevState* st, cudaStream_t stream);
// Boundary masses (compute_boundary_mass.cu:10-30), per-thread, init only.
// bckey != nullptr (batched): packed (scene, cell) key of each sorted boundary particle.
void launch_boundary_mass(const DevParams& P, const float4* bpos, u32 nb, HashView bh, float* bmass,
                          cudaStream_t stream, const u64* bckey = nullptr);
// Metrics of an arbitrary velocity array (used after load/reset).
void launch_metrics(const float4* vel, u32 n, float mass, float* out2, cudaStream_t stream);

}  // namespace wcsph
