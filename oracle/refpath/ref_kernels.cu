// ref_kernels.cu — launchers for ONE family of the reference's kernels.
//
// TEST/BASELINE INFRASTRUCTURE: compiled only into oracle/_ref by
// oracle/build_ref.py, never into the product library.
//
// build_ref.py compiles this file once per kernel family with
// -DREF_FAMILY=<n> and `-include variant_config.h` (the KTT parameters the
// reference passes as -D macros, step_tuner.cuh:79-121). Each compilation
// includes one shimmed reference kernel file inside its own namespace, so the
// same kernel name (e.g. rebuild_n_search for fluid and boundary tables) can
// be built twice with different table sizes and linked into one library.
#include <cuda_runtime.h>

#define REF_FAMILY_REBUILD_FLUID 1
#define REF_FAMILY_REBUILD_BOUNDARY 2
#define REF_FAMILY_NLIST 3
#define REF_FAMILY_RHO 4
#define REF_FAMILY_PRESSURE 5
#define REF_FAMILY_NONPRESSURE 6
#define REF_FAMILY_UPDATE 7
#define REF_FAMILY_BMASS 8

#if REF_FAMILY != REF_FAMILY_REBUILD_BOUNDARY && REF_FAMILY != REF_FAMILY_BMASS
// KTT parameters of the fluid table and the SPH kernels (step_tuner.cuh:79-121,
// values from the frozen config of the variant).
#define CELL_SIZE_MULT REF_CELL_SIZE_MULT
#define TABLE_SIZE_MULT REF_TABLE_SIZE_MULT
#define MIN_TABLE_SIZE REF_MIN_TABLE_SIZE
#define BOUNDARY_TABLE_SIZE_MULT 1
#define MIN_BOUNDARY_TABLE_SIZE REF_BOUNDARY_TABLE_SIZE
#define compute_rho_p_block REF_BLOCK
#define compute_rho_p_nlist 1
#define compute_rho_p_shared 0
#define compute_rho_p_cache_log2 1
#define compute_pressure_accel_n_normal_block REF_BLOCK
#define compute_pressure_accel_n_normal_nlist 1
#define compute_pressure_accel_n_normal_shared 0
#define compute_pressure_accel_n_normal_cache_log2 1
#define compute_non_pressure_accel_block REF_BLOCK
#define compute_non_pressure_accel_nlist 1
#define compute_non_pressure_accel_shared 0
#define compute_non_pressure_accel_cache_log2 1
#define EXTERNAL_FORCE REF_EXTERNAL_FORCE
#endif

#if REF_FAMILY == REF_FAMILY_REBUILD_FLUID
namespace REFNS {
using ::make_float4;
#include "rebuild_n_search.cu"
}
extern "C" void refk_rebuild_fluid(void* ns, const float4* pos, unsigned n, unsigned block, cudaStream_t s) {
    REFNS::rebuild_n_search<<<(n + block - 1) / block, block, 0, s>>>(static_cast<REFNS::NSearch*>(ns), pos, n);
}

#elif REF_FAMILY == REF_FAMILY_REBUILD_BOUNDARY
// boundary hash: TABLE_SIZE = bit_ceil(B)/2 (rebuild_n_search.cuh:40-42)
#define TABLE_SIZE (REF_BOUNDARY_TABLE_SIZE)
#define BOUNDARY_TABLE_SIZE (REF_BOUNDARY_TABLE_SIZE)
#define CELL_SIZE_MULT 1.f
namespace REFNS {
using ::make_float4;
#include "rebuild_n_search.cu"
}
extern "C" void refk_rebuild_boundary(void* ns, const float4* pos, unsigned n, cudaStream_t s) {
    REFNS::rebuild_n_search<<<(n + 127) / 128, 128, 0, s>>>(static_cast<REFNS::NSearch*>(ns), pos, n);
}

#elif REF_FAMILY == REF_FAMILY_NLIST
namespace REFNS {
using ::make_float4;
constexpr unsigned count_neighbors_u_n = 1;
constexpr unsigned fill_neighbors_u_n = 1;
#include "compute_neighbor_list.cu"
}
extern "C" void refk_count_neighbors(const float4* pos, unsigned* counts, unsigned n, const void* ns, unsigned block,
                                     cudaStream_t s) {
    REFNS::count_neighbors<<<(n + block - 1) / block, block, 0, s>>>(pos, counts, n,
                                                                     static_cast<const REFNS::NSearch*>(ns));
}
extern "C" void refk_fill_neighbors(const float4* pos, const unsigned* offsets, unsigned* nbrs, unsigned n,
                                    const void* ns, unsigned block, cudaStream_t s) {
    REFNS::fill_neighbors<<<(n + block - 1) / block, block, 0, s>>>(pos, offsets, nbrs, n,
                                                                    static_cast<const REFNS::NSearch*>(ns));
}

#elif REF_FAMILY == REF_FAMILY_RHO
namespace REFNS {
using ::make_float4;
constexpr unsigned compute_rho_p_u_n = 1;
#include "compute_rho_p.cu"
}
extern "C" void refk_rho_p(const float4* pos, float* rho, float* prs, unsigned n, const void* ns, const unsigned* off,
                           const unsigned* cnt, const unsigned* nbr, const float* bmass, const void* bns,
                           cudaStream_t s) {
    const unsigned b = compute_rho_p_block;
    if (bns)
        REFNS::compute_rho_p_with_boundary<<<(n + b - 1) / b, b, 0, s>>>(
            pos, rho, prs, n, static_cast<const REFNS::NSearch*>(ns), off, cnt, nbr, bmass,
            static_cast<const REFNS::NSearch*>(bns));
    else
        REFNS::compute_rho_p<<<(n + b - 1) / b, b, 0, s>>>(pos, rho, prs, n, static_cast<const REFNS::NSearch*>(ns), off,
                                                           cnt, nbr);
}

#elif REF_FAMILY == REF_FAMILY_PRESSURE
namespace REFNS {
using ::make_float4;
constexpr unsigned compute_pressure_accel_n_normal_u_n = 1;
#include "compute_pressure_accel_n_normal.cu"
}
extern "C" void refk_pressure(const float4* pos, const float* rho, const float* prs, float4* ap, float4* normal,
                              unsigned n, const void* ns, const unsigned* off, const unsigned* cnt, const unsigned* nbr,
                              const float* bmass, const void* bns, cudaStream_t s) {
    const unsigned b = compute_pressure_accel_n_normal_block;
    if (bns)
        REFNS::compute_pressure_accel_n_normal_with_boundary<<<(n + b - 1) / b, b, 0, s>>>(
            pos, rho, prs, ap, normal, n, static_cast<const REFNS::NSearch*>(ns), off, cnt, nbr, bmass,
            static_cast<const REFNS::NSearch*>(bns));
    else
        REFNS::compute_pressure_accel_n_normal<<<(n + b - 1) / b, b, 0, s>>>(
            pos, rho, prs, ap, normal, n, static_cast<const REFNS::NSearch*>(ns), off, cnt, nbr);
}

#elif REF_FAMILY == REF_FAMILY_NONPRESSURE
namespace REFNS {
using ::make_float4;
constexpr unsigned compute_non_pressure_accel_u_n = 1;
#include "compute_non_pressure_accel.cu"
}
extern "C" void refk_non_pressure(const float4* pos, const float* rho, const float4* vel, const float4* normal,
                                  float4* anp, unsigned n, const void* ns, const unsigned* off, const unsigned* cnt,
                                  const unsigned* nbr, cudaStream_t s) {
    const unsigned b = compute_non_pressure_accel_block;
    REFNS::compute_non_pressure_accel<<<(n + b - 1) / b, b, 0, s>>>(pos, rho, vel, normal, anp, n,
                                                                    static_cast<const REFNS::NSearch*>(ns), off, cnt,
                                                                    nbr);
}

#elif REF_FAMILY == REF_FAMILY_UPDATE
namespace REFNS {
using ::make_float4;
#include "update_positions.cu"
}
struct RefBox {
    float4 min, max;
    float4 model[4], model_inv[4];
};
extern "C" void refk_update_positions(float4* pos, float4* vel, const float4* ap, const float4* anp, unsigned n,
                                      float delta, float np_delta, const RefBox* box, unsigned block, cudaStream_t s) {
    REFNS::BoundingBoxGPU bb;
    bb.min = box->min;
    bb.max = box->max;
    for (int c = 0; c < 4; ++c) {
        bb.model.col[c] = box->model[c];
        bb.model_inv.col[c] = box->model_inv[c];
    }
    REFNS::update_positions<<<(n + block - 1) / block, block, 0, s>>>(pos, vel, ap, anp, n, delta, np_delta, bb);
}

#elif REF_FAMILY == REF_FAMILY_BMASS
// compute_boundary_mass (compute_boundary_mass.cuh:24-30): both table sizes
// are bit_ceil(B)/2, block 128.
#define TABLE_SIZE (REF_BOUNDARY_TABLE_SIZE)
#define BOUNDARY_TABLE_SIZE (REF_BOUNDARY_TABLE_SIZE)
#define CELL_SIZE_MULT 1.f
namespace REFNS {
using ::make_float4;
#include "compute_boundary_mass.cu"
}
extern "C" void refk_boundary_mass(const float4* bpos, float* mass, unsigned nb, const void* bns, cudaStream_t s) {
    REFNS::compute_boundary_mass<<<(nb + 127) / 128, 128, 0, s>>>(bpos, mass, nb, static_cast<const REFNS::NSearch*>(bns));
}
#else
#error "REF_FAMILY not set"
#endif
