// sph_common.cuh — device-side parameters, SPH kernel functions, Morton keys
// and the linear-probed cell hash shared by every kernel of the WCSPH step.
//
// Formulas follow the reference solver (petbab/fluid-simulation):
//   SPH kernels            src/cuda/SPH/kernel.cuh:8-63
//   float4 algebra         src/cuda/math.cuh:10-64 (dot/length are 3-component)
//   Morton encoding        src/cuda/nsearch/morton.cuh:7-34
//   cell hash / probing    src/cuda/tuning/kernels/common.cuh:55-124
// Physical constants are run-time values here (compile-time constexpr there).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace wcsph {

using u32 = uint32_t;
using u64 = unsigned long long;

constexpr u64 EMPTY_HASH = ~0ull;   // NSearch::EMPTY_HASH (common.cuh:52)
constexpr u32 EMPTY_CELL = ~0u;     // NSearch::EMPTY_CELL (common.cuh:53)
constexpr float PI_F = 3.1415926535897932384626433f;  // math.cuh:8

// Derived per-scene constants. Every value is produced on the host with the
// same float operation order as the reference's constexpr chain
// (common.cuh:18-23, kernel.cuh:13,25,38,47,54) so that device arithmetic
// starts from identical constants.
struct DevParams {
    float radius;          // PARTICLE_RADIUS
    float spacing;         // 2r
    float h;               // SUPPORT_RADIUS = 2*spacing
    float h2;              // h*h (is_neighbor threshold, common.cuh:41)
    float inv_h;
    float cell_size;       // h * CELL_SIZE_MULT (sort and hash cells)
    float mass;            // rest_density * spacing^3 * 0.8f
    float rest_density;
    float stiffness;
    float exponent;
    float max_density_ratio;
    float viscosity;
    float surface_tension;
    float gravity[3];
    float collision_buffer;  // radius * COLLISION_BUFFER_MULT
    float elasticity;
    float w0;                // cubic_spline(0, h) = 8/(pi h^3)
    float cubic_factor;      // 8/(pi h^3)
    float cubic_grad_factor; // 48/(pi h^3)
    float spiky_grad_factor; // -45/(pi h^9)
    float cohesion_factor;   // 32/(pi h^3)
    float visc_eps;          // 0.01 * h * h
    float visc_scale;        // viscosity * 10 * mass
    float st_scale;          // surface_tension * 2 * rest_density
    float rest_density2;     // rho0*rho0 (boundary pressure term p/(rho0*rho0))
    int   range;             // int(h / cell + .5) (common.cuh:131)
    int   force_field;       // wcsph_force_field
    float force_param[4];
};

// Collision box, BoundingBoxGPU (src/cuda/util.cuh:9-16): column-major mat4.
struct DevBox {
    float4 min, max;
    float4 model[4];
    float4 model_inv[4];
};

// ---------------------------------------------------------------- float4 --
// 3-component dot/length as in math.cuh:51-57; the w lane is carried by the
// caller where the reference's float4 algebra touches it.
__host__ __device__ __forceinline__ float dot3(float4 a, float4 b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
__host__ __device__ __forceinline__ float4 sub4(float4 a, float4 b) {
    return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
__host__ __device__ __forceinline__ float4 mat_mul(const float4 m[4], float4 v) {
    // math.cuh:78-86: result.row = sum_c col[c].row * v[c]
    return make_float4(m[0].x * v.x + m[1].x * v.y + m[2].x * v.z + m[3].x * v.w,
                       m[0].y * v.x + m[1].y * v.y + m[2].y * v.z + m[3].y * v.w,
                       m[0].z * v.x + m[1].z * v.y + m[2].z * v.z + m[3].z * v.w,
                       m[0].w * v.x + m[1].w * v.y + m[2].w * v.z + m[3].w * v.w);
}
#ifdef __CUDACC__
// mat_mul with its rounding written out (the collision response of the step).
__device__ __forceinline__ float4 mat_mul_rn(const float4 m[4], float4 v) {
    auto row = [&](float a, float b, float c, float d) {
        return __fmaf_rn(d, v.w, __fmaf_rn(c, v.z, __fmaf_rn(b, v.y, __fmul_rn(a, v.x))));
    };
    return make_float4(row(m[0].x, m[1].x, m[2].x, m[3].x), row(m[0].y, m[1].y, m[2].y, m[3].y),
                       row(m[0].z, m[1].z, m[2].z, m[3].z), row(m[0].w, m[1].w, m[2].w, m[3].w));
}
#endif

// Squared distance used by the neighbour predicate (is_neighbor,
// common.cuh:39-47, with dot() of math.cuh:54-56). The reference's
// a.x*b.x + a.y*b.y + a.z*b.z is contracted by nvcc to
// fma(z, z, fma(x, x, y*y)): y*y is rounded first, then x and z are fused in.
// The rounding is fixed here explicitly in that order so that the CUDA path,
// the oracle (the identical fma chain) and the reference's kernels decide
// pairs at |r| = h alike; other orders differ from it by one ulp on such pairs.
__device__ __forceinline__ float dist2(float4 a, float4 b) {
    const float dx = __fsub_rn(a.x, b.x);
    const float dy = __fsub_rn(a.y, b.y);
    const float dz = __fsub_rn(a.z, b.z);
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// ------------------------------------------------------------ SPH kernels --
// cubic_spline (kernel.cuh:12-19): factor*(6q^3-6q^2+1) for q<=.5,
// factor*2*(1-q)^3 for q<=1, else 0.
__device__ __forceinline__ float cubic_w(float q, const DevParams& P) {
    if (q <= 0.5f) return P.cubic_factor * (6.f * q * q * q - 6.f * q * q + 1.f);
    if (q <= 1.f) {
        const float t = 1.f - q;
        return P.cubic_factor * 2.f * (t * t * t);
    }
    return 0.f;
}
// cubic_spline_grad (kernel.cuh:22-32): coefficient multiplying r.
__device__ __forceinline__ float cubic_grad(float q, const DevParams& P) {
    if (q < 1.e-9f || q > 1.f) return 0.f;
    const float r_len = q * P.h;
    if (q <= 0.5f) return P.cubic_grad_factor * q * (3.f * q - 2.f) / (P.h * r_len);
    return -P.cubic_grad_factor * (1.f - q) * (1.f - q) / (P.h * r_len);
}
// spiky_grad (kernel.cuh:43-51): coefficient multiplying r.
__device__ __forceinline__ float spiky_grad(float q, const DevParams& P) {
    if (q < 1.e-9f || q > 1.f) return 0.f;
    const float r_len = q * P.h;
    return P.spiky_grad_factor * (1.f - q) * (1.f - q) / (P.h * r_len);
}
// cohesion (kernel.cuh:53-63), Akinci surface tension kernel.
__device__ __forceinline__ float cohesion(float q, const DevParams& P) {
    const float t = 1.f - q;
    const float iq3 = t * t * t;
    const float q3 = q * q * q;
    if (q <= 0.5f) return P.cohesion_factor * (2.f * q3 * iq3 - 1.f / 64.f);
    if (q <= 1.f) return P.cohesion_factor * q3 * iq3;
    return 0.f;
}
// Tait EOS (compute_rho_p.cu:236-238): p = k*(clamp(rho/rho0,1,max)^gamma-1).
__device__ __forceinline__ float tait_pressure(float rho, const DevParams& P) {
    float ratio = fmaxf(rho / P.rest_density, 1.0f);
    ratio = fminf(ratio, P.max_density_ratio);
    return P.stiffness * (powf(ratio, P.exponent) - 1.f);
}

// External force table (replaces the EXTERNAL_FORCE lambda string).
__device__ __forceinline__ float4 external_force(float4 pos, const DevParams& P) {
    switch (P.force_field) {
    case 1:  // constant vector
        return make_float4(P.force_param[0], P.force_param[1], P.force_param[2], 0.f);
    case 2: {  // app/fountain/application.cu:36-42
        if (pos.x * pos.x + pos.z * pos.z < .2f && pos.y < 0.f)
            return make_float4(0.f, 25.f, 0.f, 0.f);
        if (pos.y < -0.3f) {
            const float4 d = make_float4(-pos.x, 0.f, -pos.z, 0.f);
            const float len = sqrtf(dot3(d, d));
            return make_float4(2.f * (d.x / len), 2.f * (d.y / len), 2.f * (d.z / len), 0.f);
        }
        return make_float4(0.f, 0.f, 0.f, 0.f);
    }
    case 3: {  // app/vortex/application.cu:45
        if (pos.y < -0.5f) {
            const float4 d = make_float4(pos.z, 0.f, -pos.x, 0.f);
            const float len = sqrtf(dot3(d, d));
            return make_float4(2.f * (d.x / len), 2.f * (d.y / len), 2.f * (d.z / len), 0.f);
        }
        return make_float4(0.f, 0.f, 0.f, 0.f);
    }
    default:
        return make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// ------------------------------------------------------------ Morton keys --
// part_by_3 / signed_to_unsigned / encode_morton (morton.cuh:7-34): 21 bits
// per axis after a +2^20 offset, x | y<<1 | z<<2, 63-bit key.
__host__ __device__ __forceinline__ u64 part_by_3(u64 n) {
    n &= 0x1fffffull;
    n = (n | (n << 32)) & 0x1f00000000ffffull;
    n = (n | (n << 16)) & 0x1f0000ff0000ffull;
    n = (n | (n << 8)) & 0x100f00f00f00f00full;
    n = (n | (n << 4)) & 0x10c30c30c30c30c3ull;
    n = (n | (n << 2)) & 0x1249249249249249ull;
    return n;
}
__host__ __device__ __forceinline__ u32 offset_coord(int c) {
    return static_cast<u32>(c) + (1u << 20);
}
// Cell coordinate of a position: floorf(p / cs) in IEEE float, exactly as the
// sort's key lambda (particle_data.cuh:117-125) and NSearch::cell_coord
// (common.cuh:73-79) compute it.
__device__ __forceinline__ int3 cell_of(float4 p, float cs) {
    return make_int3(static_cast<int>(floorf(__fdiv_rn(p.x, cs))),
                     static_cast<int>(floorf(__fdiv_rn(p.y, cs))),
                     static_cast<int>(floorf(__fdiv_rn(p.z, cs))));
}
__host__ __device__ __forceinline__ u64 morton_key(int3 c) {
    return part_by_3(offset_coord(c.x)) | (part_by_3(offset_coord(c.y)) << 1) |
           (part_by_3(offset_coord(c.z)) << 2);
}

// ------------------------------------------------------------- cell hash --
// NSearch::pack (common.cuh:55-57): 21-bit offset coords packed x|y<<21|z<<42.
__host__ __device__ __forceinline__ u64 pack_cell(u32 x, u32 y, u32 z) {
    return static_cast<u64>(x) | (static_cast<u64>(y) << 21) | (static_cast<u64>(z) << 42);
}
__host__ __device__ __forceinline__ u64 pack_cell(int3 c) {
    return pack_cell(offset_coord(c.x), offset_coord(c.y), offset_coord(c.z));
}
// NSearch::cell_hash (common.cuh:65-67) on the unsigned (offset) coords.
__host__ __device__ __forceinline__ u64 cell_hash(u32 x, u32 y, u32 z) {
    return 73856093ull * x ^ 19349663ull * y ^ 83492791ull * z;
}
__host__ __device__ __forceinline__ u64 cell_hash_packed(u64 pk) {
    return cell_hash(static_cast<u32>(pk & 0x1FFFFFull), static_cast<u32>((pk >> 21) & 0x1FFFFFull),
                     static_cast<u32>((pk >> 42) & 0x1FFFFFull));
}

// Batched ensembles key cells by (scene, cell): the low 16 bits per axis of
// the offset coordinates plus the scene id in bits 48..62, unique for cell
// coordinates in [-2^15, 2^15) (checked at creation).
__host__ __device__ __forceinline__ u64 pack_cell_batch(u32 scene, u32 x, u32 y, u32 z) {
    return (static_cast<u64>(scene) << 48) | static_cast<u64>(x & 0xFFFFu) |
           (static_cast<u64>(y & 0xFFFFu) << 16) | (static_cast<u64>(z & 0xFFFFu) << 32);
}
__host__ __device__ __forceinline__ u64 cell_hash_batch(u64 pk) {
    const u32 s = static_cast<u32>(pk >> 48);
    return cell_hash(static_cast<u32>(pk & 0xFFFFull), static_cast<u32>((pk >> 16) & 0xFFFFull),
                     static_cast<u32>((pk >> 32) & 0xFFFFull)) ^ (0x9E3779B97F4A7C15ull * s);
}
template <bool BATCH>
__host__ __device__ __forceinline__ u64 slot_hash(u64 pk) {
    if constexpr (BATCH) return cell_hash_batch(pk);
    else return cell_hash_packed(pk);
}
// Sort key of a batched particle: the scene id in bits 48..62 and, below, the
// Morton key of the cell coordinates offset by 2^15 (16 bits per axis). For
// cells in [-2^15, 2^15) it orders the particles of a scene exactly as the
// reference's 63-bit key of c + 2^20 does: bits 15..19 of c + 2^20 repeat the
// inverse of its bit 20 (the sign), which bit 15 of c + 2^15 carries, so the
// first differing bit of two keys sits at the same place in both. The stable
// sort therefore gives every scene the permutation of its own single step.
__host__ __device__ __forceinline__ u64 batch_key(u32 scene, int3 c) {
    return (static_cast<u64>(scene) << 48) | part_by_3(static_cast<u32>(c.x + 32768)) |
           (part_by_3(static_cast<u32>(c.y + 32768)) << 1) | (part_by_3(static_cast<u32>(c.z + 32768)) << 2);
}
constexpr int BATCH_CELL_LIMIT = 32768;   // batched cell coordinates lie in [-limit, limit)

// Linear-probed lookup (find_cell_in_table, common.cuh:89-102). table_size is
// a power of two so `% T` is a mask; the probe is bounded by T.
template <bool BATCH = false>
__device__ __forceinline__ u32 hash_find(const u64* __restrict__ table, u32 tmask, u64 pk) {
    u32 t = static_cast<u32>(slot_hash<BATCH>(pk) & tmask);
    for (u32 j = 0; j <= tmask; ++j) {
        const u64 k = __ldg(table + t);
        if (k == EMPTY_HASH) return EMPTY_CELL;
        if (k == pk) return t;
        t = (t + 1) & tmask;
    }
    return EMPTY_CELL;
}
// add_cell (common.cuh:104-114) with atomicCAS; returns EMPTY_CELL when the
// table is full (the reference returns -1 and then writes cell_start[-1]).
template <bool BATCH = false>
__device__ __forceinline__ u32 hash_insert(u64* table, u32 tmask, u64 pk) {
    u32 t = static_cast<u32>(slot_hash<BATCH>(pk) & tmask);
    for (u32 j = 0; j <= tmask; ++j) {
        const u64 old = atomicCAS(table + t, EMPTY_HASH, pk);
        if (old == EMPTY_HASH || old == pk) return t;
        t = (t + 1) & tmask;
    }
    return EMPTY_CELL;
}

// Per-scene constants of a batched ensemble (read by the integrate pass).
struct DevScene {
    DevBox box;
    float4 gravity_visc;   // gravity x, y, z and viscosity * 10 * mass
};

// Device-side step state: CFL reduction, metrics, sort bookkeeping, errors.
struct DevState {
    // CFL: max |v|^2 of the state at the start of the current step
    // (bits of a non-negative float, atomicMax-able as u32).
    u32 vmax2_bits[2];
    u32 parity;                 // which vmax2 slot is "current"
    u32 blocks_done;            // last-block detection in the integrate pass
    float sum_speed_acc;        // accumulators of the running step
    float sum_speed2_acc;
    float last_mean_speed;      // metrics of the last completed step
    float last_ke;
    float last_dt_p;
    float last_np_dt;
    u32 error_flags;            // bit 0 hash full, bit 1 lookback timeout, bit 2 overflow
    u32 pad0;
    // radix sort
    u32 sort_active[8];         // pass p sorts digit p (bits 8p..8p+7)
    u32 sort_sel[9];            // buffer read by pass p; sort_sel[8] = final
    u32 sort_tile_counter[8];
    u32 first_active;           // first active pass (generates the iota values)
    u32 pad1[2];
    // cell-coordinate bounds of the particles of the current sort (0 is always
    // included; reset to 0 by the sort plan): they choose the compressed keys
    int cell_lo[3];
    int cell_hi[3];
};

enum : u32 {
    ERR_HASH_FULL = 1u,
    ERR_LOOKBACK_TIMEOUT = 2u,
    ERR_CAND_OVERFLOW = 4u,
    ERR_BARRIER_TIMEOUT = 8u,   // a grid barrier of the persistent ensemble kernel waited too long
    ERR_BOUNDS = 16u,           // bounds-checked build: an index guard fired
};

}  // namespace wcsph
