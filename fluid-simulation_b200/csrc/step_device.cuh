// step_device.cuh — device code of the neighbourhood search and the SPH
// passes (step_kernels.cuh describes the decomposition). step_kernels.cu
// wraps it in the per-pass kernels; batch_persistent.cu calls it between the
// grid barriers of the persistent ensemble kernel.
//
// Loads of data that a pass only reads go through the read-only data path
// (ld.global.nc) in the per-pass kernels. The persistent kernel rewrites the
// same buffers within one launch (hash, sorted state, records, lists, every
// step), for which the read-only path is not coherent; it includes this file
// with WCSPH_COHERENT_LOADS 1, which makes those loads ordinary global loads
// and drops the __restrict__ of pointer arguments (through which the compiler
// may otherwise choose the read-only path by itself).
// Everything here has internal linkage, so both variants can coexist.
#pragma once
#include <climits>

#include "step_kernels.cuh"

#ifndef WCSPH_COHERENT_LOADS
#define WCSPH_COHERENT_LOADS 0
#endif
#if WCSPH_COHERENT_LOADS
#define WCSPH_RO_QUAL ""
#define WCSPH_RESTRICT
#else
#define WCSPH_RO_QUAL ".nc"
#define WCSPH_RESTRICT __restrict__
#endif

namespace wcsph {
namespace {

// Index guards of the bounds-checked build (compiled with WCSPH_CHECKS=1:
// `make checked`, lib/libwcsph_checked.so). An index at or past its bound
// raises ERR_BOUNDS in the step's error flags and is replaced by 0, so that
// the access stays inside its buffer and nothing faults; the host then
// reports WCSPH_ERR_BOUNDS. The default build compiles the guards away.
#ifndef WCSPH_CHECKS
#define WCSPH_CHECKS 0
#endif
__device__ __forceinline__ u32 guard_st(DevState* st, u32 idx, u32 bound) {
#if WCSPH_CHECKS
    if (idx >= bound) {
        atomicOr(&st->error_flags, ERR_BOUNDS);
        return 0u;
    }
#else
    (void)st;
    (void)bound;
#endif
    return idx;
}

template <class T>
__device__ __forceinline__ T ro_ld(const T* p) {
#if WCSPH_COHERENT_LOADS
    return *p;
#else
    return __ldg(p);
#endif
}

__device__ __forceinline__ u32 guard(const TravArgs& a, u32 idx, u32 bound) { return guard_st(a.st, idx, bound); }
// Cells of the staged neighbourhood ranges: (2R + 1)^3, or the 36 of an x-pair union.
__device__ __forceinline__ u32 range_cells(const TravArgs& a) {
    const u32 d = 2u * static_cast<u32>(a.range) + 1u;
    return max(d * d * d, 36u);
}

// Linear-probed lookup of a packed cell key (find_cell_in_table,
// common.cuh:89-102), with the loads of this file's flavour.
template <bool BATCH = false>
__device__ __forceinline__ u32 find_slot(const u64* WCSPH_RESTRICT table, u32 tmask, u64 pk) {
    u32 t = static_cast<u32>(slot_hash<BATCH>(pk) & tmask);
    for (u32 j = 0; j <= tmask; ++j) {
        const u64 k = ro_ld(table + t);
        if (k == EMPTY_HASH) return EMPTY_CELL;
        if (k == pk) return t;
        t = (t + 1) & tmask;
    }
    return EMPTY_CELL;
}


constexpr u32 FULL = 0xffffffffu;
constexpr u32 BCAND_CAP = 256;   // boundary candidates expanded per warp and chunk
constexpr u32 HOME_BLOCK = 32;   // home particles (bit-matrix rows) handled together
constexpr u32 SEG_SLOTS = 64;    // segment partials, slot = lane + row (both < 32)
constexpr u32 NO_HOME = 0xFFFFFFFFu;   // home rows not among the staged candidates

// Candidate index of home row k of a home block: rows [0, split) are staged
// at c1 + k, later rows at c2 + (k - split) (the second cell of an x-pair);
// c1 == NO_HOME: the home rows are not staged (read from global memory).
struct HomeMap {
    u32 split, c1, c2;
    __device__ __forceinline__ u32 cand(u32 k) const { return k < split ? c1 + k : c2 + (k - split); }
};


__device__ __forceinline__ u32 lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ u32 warp_incl_scan(u32 v) {
    const u32 lane = lane_id();
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const u32 t = __shfl_up_sync(FULL, v, o);
        if (lane >= static_cast<u32>(o)) v += t;
    }
    return v;
}

// What each pass stages per candidate in shared memory and how many floats
// it accumulates per (home, candidate-run) segment.
//   DENSITY: positions in blocks of 16 candidate pairs, each pair as
//            (x0,x1)(y0,y1)(z0,z1) float2s, one pad float2 per block (so that
//            lanes on different blocks hit different banks); the distance
//            test reads a pair per packed FP32 step; the range (cell) of
//            each candidate as a byte, from which its neighbour-list entry
//            rstart[q] + m - rpref[q] follows
//   COUNT / FILL / ADJ_*: float4 positions and particle indices
//   FORCE / SURFACE: particle indices only (they visit neighbours only and
//            read the neighbour's fields through L1)
template <int KIND>
struct KindCfg {
    static constexpr bool soa = KIND == PASS_DENSITY;
    static constexpr bool stage_sa =
        KIND == PASS_COUNT || KIND == PASS_FILL || KIND == PASS_ADJ_FORCE || KIND == PASS_ADJ_DENSITY;
    static constexpr bool stage_j = KIND != PASS_DENSITY;
    static constexpr bool stage_q = KIND == PASS_DENSITY;   // the candidate's range (neighbour lists)
    static constexpr bool boundary =
        KIND == PASS_DENSITY || KIND == PASS_FORCE || KIND == PASS_ADJ_FORCE || KIND == PASS_ADJ_DENSITY;
    static constexpr int nf = (KIND == PASS_FORCE || KIND == PASS_ADJ_FORCE) ? 9
                              : (KIND == PASS_SURFACE || KIND == PASS_ADJ_DENSITY) ? 3 : 1;
    static constexpr int nfb = KIND == PASS_ADJ_FORCE ? 4 : (KIND == PASS_DENSITY ? 1 : 3);
    // resident warps per SM the register allocation must allow (32 -> 64 registers,
    // 28 -> 72, 24 -> 80, 16 -> 128): the density pass spills a little at 72
    // registers, which costs less than fewer resident warps at 80; the force
    // pass spills below 80 and the adjoint force pass below 128
    static constexpr int min_warps = KIND == PASS_DENSITY ? 28
                                     : KIND == PASS_SURFACE ? 32 : (KIND == PASS_ADJ_FORCE ? 16 : 24);
};

__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~static_cast<size_t>(15); }

// float2 index of candidate pair pp in the density staging layout.
__host__ __device__ __forceinline__ u32 pair_slot(u32 pp) { return 3u * pp + (pp >> 4); }

// Per-warp shared memory, sized by the candidate capacity cap = 32 * mask_words.
template <int KIND>
struct WarpView {
    float4* sa;
    float2* sp;    // density: candidate pair positions (pair_slot layout)
    u32* cand;
    unsigned char* cq;   // density: range of each candidate
    u32* rstart;   // fluid cells: first particle
    u32* rpref;    // fluid cells: exclusive prefix of the cell sizes (+ total)
    u32* bcand;
    u32* bstart;
    u32* bpref;
    float* part;   // [SEG_SLOTS][nf] segment partials
    u32* aux;      // the block's bit matrix (cap words)
    u32* hoff;     // row hit offsets (HOME_BLOCK + 1)
};

// ncell = (2R + 1)^3 fluid neighbour cells.
template <int KIND>
__host__ __device__ __forceinline__ size_t warp_smem_bytes(u32 cap, u32 ncell, bool with_boundary,
                                                           WarpView<KIND>* v = nullptr, unsigned char* base = nullptr) {
    using C = KindCfg<KIND>;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = base ? base + o : nullptr;
        o += align16(bytes);
        return p;
    };
    unsigned char* sa = C::stage_sa ? take(16ull * cap) : nullptr;
    unsigned char* sp = C::soa ? take(8ull * pair_slot(cap / 2)) : nullptr;
    unsigned char* cand = C::stage_j ? take(4ull * cap) : nullptr;
    unsigned char* cq = C::stage_q ? take(cap) : nullptr;
    // density: room for the 36-cell union of an x-pair of cells (R = 1)
    const u32 nrange = (KIND == PASS_DENSITY && ncell < 36u) ? 36u : ncell;
    unsigned char* rstart = take(4ull * (nrange + 3));
    unsigned char* rpref = take(4ull * (nrange + 3));
    unsigned char *bcand = nullptr, *bstart = nullptr, *bpref = nullptr;
    if (C::boundary && with_boundary) {   // only scenes with boundary particles
        bcand = take(4ull * BCAND_CAP);
        bstart = take(4ull * (MAX_BOUNDARY_CELLS + 3));
        bpref = take(4ull * (MAX_BOUNDARY_CELLS + 3));
    }
    unsigned char* part = take(4ull * SEG_SLOTS * C::nf);
    // the block's bit matrix (density builds it here; the later passes copy it in)
    unsigned char* aux = (KIND == PASS_COUNT || KIND == PASS_FILL) ? nullptr : take(4ull * cap);
    unsigned char* hoff = take(4ull * (HOME_BLOCK + 4));
    if (v) {
        v->sa = reinterpret_cast<float4*>(sa);
        v->sp = reinterpret_cast<float2*>(sp);
        v->cand = reinterpret_cast<u32*>(cand);
        v->cq = cq;
        v->rstart = reinterpret_cast<u32*>(rstart);
        v->rpref = reinterpret_cast<u32*>(rpref);
        v->bcand = reinterpret_cast<u32*>(bcand);
        v->bstart = reinterpret_cast<u32*>(bstart);
        v->bpref = reinterpret_cast<u32*>(bpref);
        v->part = reinterpret_cast<float*>(part);
        v->aux = reinterpret_cast<u32*>(aux);
        v->hoff = reinterpret_cast<u32*>(hoff);
    }
    return o;
}

// Looks up `ncell` cells (lane-parallel) and stores their ranges as
// (start, exclusive prefix); returns the total candidate count.
template <bool BATCH, class CellFn>
__device__ __forceinline__ u32 gather_ranges(u32* rstart, u32* rpref, u32 ncell, const HashView& hv,
                                             CellFn cell_of_q) {
    const u32 lane = lane_id();
    u32 total = 0;
    for (u32 base = 0; base < ncell; base += 32) {
        const u32 q = base + lane;
        u32 s = 0, cnt = 0;
        if (q < ncell) {
            const u64 pk = cell_of_q(q);
            const u32 slot = find_slot<BATCH>(hv.table, hv.tmask, pk);
            if (slot != EMPTY_CELL) {
                s = ro_ld(hv.cstart + slot);
                cnt = ro_ld(hv.cend + slot) - s;
            }
        }
        const u32 incl = warp_incl_scan(cnt);
        if (q < ncell) {
            rstart[q] = s;
            rpref[q] = total + incl - cnt;
        }
        total += __shfl_sync(FULL, incl, 31);
    }
    if (lane == 0) rpref[ncell] = total;
    __syncwarp();
    return total;
}

// Offset (dx, dy, dz) in [-R, R]^3 of neighbour cell q (x outermost, z
// innermost: the reference's nesting order); R = 1 divides by a constant.
__device__ __forceinline__ void cell_offset(u32 q, int R, int& dx, int& dy, int& dz) {
    if (R == 1) {
        dz = static_cast<int>(q % 3u) - 1;
        dy = static_cast<int>((q / 3u) % 3u) - 1;
        dx = static_cast<int>(q / 9u) - 1;
    } else {
        const u32 D = static_cast<u32>(2 * R + 1);
        dz = static_cast<int>(q % D) - R;
        dy = static_cast<int>((q / D) % D) - R;
        dx = static_cast<int>(q / (D * D)) - R;
    }
}

// Index of the range holding candidate m (rpref[lo] <= m < rpref[lo + 1]).
__device__ __forceinline__ u32 range_of(const u32* rpref, u32 ncell, u32 m) {
    u32 lo = 0, hi = ncell;
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (rpref[mid] <= m) lo = mid; else hi = mid;
    }
    return lo;
}

// cand[m - c0] = particle index of candidate m, m in [c0, c0 + len).
__device__ __forceinline__ void expand(u32* cand, const u32* rstart, const u32* rpref, u32 ncell, u32 c0,
                                       u32 len) {
    __syncwarp();
    for (u32 ml = lane_id(); ml < len; ml += 32) {
        const u32 m = c0 + ml;
        const u32 lo = range_of(rpref, ncell, m);
        cand[ml] = rstart[lo] + (m - rpref[lo]);
    }
    __syncwarp();
}

// Stages candidates [c0, c0 + len) into shared memory: lane q walks cell q's
// particles, so the loads are independent (no per-candidate search).
// DENSITY pads the staged count up to a multiple of 32 with candidates at
// infinity (never neighbours), so bit-matrix rows fill whole words.
template <int KIND>
__device__ __forceinline__ void soa_store(const WarpView<KIND>& S, u32 m, float4 x) {
    float* f = reinterpret_cast<float*>(S.sp + pair_slot(m >> 1)) + (m & 1u);
    f[0] = x.x;
    f[2] = x.y;
    f[4] = x.z;
}

template <int KIND>
__device__ __forceinline__ void stage(const WarpView<KIND>& S, const TravArgs& a, u32 ncell, u32 c0, u32 len) {
    __syncwarp();
    const u32 lane = lane_id();
    const u32 c1 = c0 + len;
    for (u32 qb = 0; qb < ncell; qb += 32) {
        // a last round of fewer than 32 cells (the 36-cell union of an x-pair)
        // spreads each cell over 32 / cells lanes
        const u32 rem = min(32u, ncell - qb);
        const u32 lpc = rem == 32u ? 1u : 32u / rem;
        const u32 q = qb + lane / lpc;
        const u32 sub = lane - (lane / lpc) * lpc;
        u32 lo = 0, hi = 0, src = 0;
        if (lane / lpc < rem) {
            const u32 b = S.rpref[q], e = S.rpref[q + 1];
            lo = max(b, c0);
            hi = min(e, c1);
            src = S.rstart[q] + (lo - b);
        }
        for (u32 t = sub; lo + t < hi; t += lpc) {
            const u32 j = guard(a, src + t, a.n);
            const u32 ml = guard(a, lo + t - c0, a.mask_words * 32u);
            if constexpr (KindCfg<KIND>::stage_j) S.cand[ml] = j;
            if constexpr (KindCfg<KIND>::stage_q) S.cq[ml] = static_cast<unsigned char>(q);
            if constexpr (KindCfg<KIND>::stage_sa) S.sa[ml] = ro_ld(a.pos + j);
            if constexpr (KindCfg<KIND>::soa) soa_store(S, ml, ro_ld(a.pos + j));
        }
    }
    if constexpr (KindCfg<KIND>::soa) {
        const float inf = __int_as_float(0x7f800000);
        for (u32 ml = len + lane; ml < ((len + 31u) & ~31u); ml += 32) soa_store(S, ml, make_float4(inf, inf, inf, 0.f));
    }
    __syncwarp();
}

// A neighbour's data as the pair arithmetic reads it.
//   x: position; FORCE: b = (v_j, 1 / rho_j), c = p_j / rho_j^2;
//   SURFACE: b = n_j, c = rho_j; j: particle index (passes that address j).
// Force and surface read one 32-byte record per neighbour (recf / recs).
struct Nbr {
    float4 x, b;
    float c;
    u32 j;
};

// A 32-byte record (two float4) in one 256-bit read-only load; the record
// starts on a 32-byte boundary (the buffers are cudaMalloc'd, records are
// 32 bytes).
__device__ __forceinline__ void load_record(const float4* r, float4& x, float4& b) {
    asm("ld.global" WCSPH_RO_QUAL ".v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(x.x), "=f"(x.y), "=f"(x.z), "=f"(x.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(r));
}

// Neighbour records of particle j (force and surface passes).
template <int KIND>
__device__ __forceinline__ Nbr fetch_j(const TravArgs& a, u32 j) {
    Nbr d;
    j = guard(a, j, a.n);
    d.j = j;
    load_record((KIND == PASS_FORCE ? a.recf : a.recs) + 2 * static_cast<size_t>(j), d.x, d.b);
    d.c = d.x.w;
    return d;
}

template <int KIND>
__device__ __forceinline__ Nbr fetch(const WarpView<KIND>& S, const TravArgs& a, u32 m) {
    Nbr d;
    m = guard(a, m, a.mask_words * 32u);
    if constexpr (KindCfg<KIND>::soa) {
        const float* f = reinterpret_cast<const float*>(S.sp + pair_slot(m >> 1)) + (m & 1u);
        d.x = make_float4(f[0], f[2], f[4], 0.f);
    } else if constexpr (KIND == PASS_FORCE || KIND == PASS_SURFACE) {
        d = fetch_j<KIND>(a, S.cand[m]);
    } else {
        d.j = S.cand[m];
        d.x = S.sa[m];
    }
    return d;
}

__device__ __forceinline__ float4 f4(float x, float y, float z, float w = 0.f) { return make_float4(x, y, z, w); }

// Box collision (resolve_collisions, update_positions.cu:14-52).
__device__ __forceinline__ void resolve_collision(float4& x, float4& v, const DevBox& bb, const DevParams& P) {
    float4 pos = mat_mul_rn(bb.model_inv, x);
    float4 vel = mat_mul_rn(bb.model_inv, v);
    bool changed = false;
    const float buf = P.collision_buffer;
    if (pos.x - buf < bb.min.x) { pos.x = bb.min.x + P.radius; vel.x *= -P.elasticity; changed = true; }
    else if (pos.x + buf > bb.max.x) { pos.x = bb.max.x - P.radius; vel.x *= -P.elasticity; changed = true; }
    if (pos.y - buf < bb.min.y) { pos.y = bb.min.y + P.radius; vel.y *= -P.elasticity; changed = true; }
    else if (pos.y + buf > bb.max.y) { pos.y = bb.max.y - P.radius; vel.y *= -P.elasticity; changed = true; }
    if (pos.z - buf < bb.min.z) { pos.z = bb.min.z + P.radius; vel.z *= -P.elasticity; changed = true; }
    else if (pos.z + buf > bb.max.z) { pos.z = bb.max.z - P.radius; vel.z *= -P.elasticity; changed = true; }
    if (changed) {
        x = mat_mul_rn(bb.model, pos);
        v = mat_mul_rn(bb.model, vel);
    }
}

// adapt_time_step (sph.cu:115-130) evaluated on the device.
__device__ __forceinline__ float cfl_time_step(const TravArgs& a, const DevParams& P) {
    const u32 parity = a.st->parity;
    const float vmax = sqrtf(__uint_as_float(a.st->vmax2_bits[parity]));
    const float clamped = a.delta < a.min_dt ? a.min_dt : (a.max_dt < a.delta ? a.max_dt : a.delta);
    if (a.cfl_factor <= 0.f) return clamped;
    if (static_cast<double>(vmax) < 1.e-9) return a.max_dt;
    const float cfl = (a.cfl_factor * P.spacing) / vmax;
    return cfl < clamped ? cfl : clamped;
}

struct HomeData {
    float4 x, v, n, abar, w;
    float rho, prs, dpi;
    float rb;         // dL/drho of the home particle (adjoint density pass)
};

template <int KIND>
__device__ __forceinline__ HomeData load_home(const TravArgs& a, u32 i) {
    HomeData H;
    i = guard(a, i, a.n);
    if constexpr (KIND == PASS_FORCE) {
        load_record(a.recf + 2 * static_cast<size_t>(i), H.x, H.v);   // x.w = p / rho^2
        H.prs = ro_ld(a.prs + i);
        H.dpi = H.x.w;
    } else if constexpr (KIND == PASS_SURFACE) {
        load_record(a.recs + 2 * static_cast<size_t>(i), H.x, H.n);   // x.w = rho
        H.rho = H.x.w;
    } else {
        H.x = ro_ld(a.pos + i);
    }
    if constexpr (KIND == PASS_ADJ_FORCE) {
        H.v = ro_ld(a.vel + i);
        H.rho = ro_ld(a.rho + i);
        H.prs = ro_ld(a.prs + i);
        H.dpi = H.prs / (H.rho * H.rho);
    }
    if constexpr (KIND == PASS_ADJ_FORCE) {
        H.abar = ro_ld(a.adj_abar + i);
        H.w = ro_ld(a.adj_w + i);
    }
    if constexpr (KIND == PASS_ADJ_DENSITY) H.rb = ro_ld(a.adj_rhobar + i);
    return H;
}

// d/dr of the coefficient functions (as functions of r = q h):
//   spiky_grad  g_s = F (1-q)^2 / (h r)            -> -F (1-q)(1+q) / (h r^2)
//   cubic_grad  g_c = F q (3q-2) / (h r) (q <= .5) -> 3 F / h^3
//               g_c = -F (1-q)^2 / (h r) (q > .5)   ->  F (1-q)(1+q) / (h r^2)
__device__ __forceinline__ float spiky_grad_dr(float q, float r, const DevParams& P) {
    if (q < 1.e-9f || q > 1.f) return 0.f;
    return -P.spiky_grad_factor * (1.f - q) * (1.f + q) / (P.h * r * r);
}
__device__ __forceinline__ float cubic_grad_dr(float q, float r, const DevParams& P) {
    if (q < 1.e-9f || q > 1.f) return 0.f;
    if (q <= 0.5f) return 3.f * P.cubic_grad_factor / (P.h * P.h * P.h);
    return P.cubic_grad_factor * (1.f - q) * (1.f + q) / (P.h * r * r);
}

// Cubic spline divided by its factor 8/(pi h^3) (kernel.cuh:12-19), without
// branches: 6q^3 - 6q^2 + 1 (q <= 1/2), 2(1-q)^3 (q <= 1), 0 beyond.
__device__ __forceinline__ float cubic_shape(float q) {
    const float t = __fsub_rn(1.f, q);
    const float inner = __fmaf_rn(__fmul_rn(__fmul_rn(6.f, q), q), __fsub_rn(q, 1.f), 1.f);
    const float outer = __fmul_rn(__fmul_rn(__fmul_rn(2.f, t), t), t);
    return q <= 0.5f ? inner : (q <= 1.f ? outer : 0.f);
}

// |r| / h from r^2 with one reciprocal square root; 0 for coincident points.
__device__ __forceinline__ float q_of(float r2, float& rinv, const DevParams& P) {
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(rinv) : "f"(fmaxf(r2, 1e-30f)));
    return __fmul_rn(__fmul_rn(r2, rinv), P.inv_h);
}

// Fluid pair (i, candidate m of the staged chunk) contributions. v[] holds
// the segment accumulators of the pass:
//   DENSITY     v0 = sum W / cubic_factor
//   FORCE       v0..2 = -sum (p_i/rho_i^2 + p_j/rho_j^2) g_s r, v3..5 = sum g_c r / rho_j,
//               v6..8 = sum (v_ij . r) g_c r / (rho_j (r^2 + eps))
//   SURFACE     v0..2 = sum (m r/|r| C(q) + n_i - n_j) / (rho_i + rho_j)
//   ADJ_FORCE   v0..2 = dL/dx_i, v3..5 = dL/dv_i, v6 = pressure-coefficient term, v7 = viscosity rho term
//   ADJ_DENSITY v0..2 = dL/dx_i
template <int KIND>
__device__ __forceinline__ void fluid_pair(float* v, const HomeData& H, const Nbr& d, float r2, const DevParams& P,
                                           const TravArgs& a) {
    const float rx = H.x.x - d.x.x, ry = H.x.y - d.x.y, rz = H.x.z - d.x.z;
    if constexpr (KIND == PASS_DENSITY) {
        float rinv;
        v[0] = __fadd_rn(v[0], cubic_shape(q_of(r2, rinv, P)));
    } else if constexpr (KIND == PASS_FORCE) {
        // spiky_grad / cubic_grad (kernel.cuh:22-51) as coefficients of r
        // rounding written out (see finish_row): the sums must not depend on
        // which kernel this is inlined into
        float rinv;
        const float q = q_of(r2, rinv, P);
        const float t = __fsub_rn(1.f, q);
        const float t2 = __fmul_rn(t, t);
        const float kr = (q >= 1.e-9f && q <= 1.f) ? __fmul_rn(rinv, P.inv_h) : 0.f;
        const float sg = __fmul_rn(__fmul_rn(P.spiky_grad_factor, t2), kr);
        const float shape = q <= 0.5f ? __fmul_rn(q, __fmaf_rn(3.f, q, -2.f)) : -t2;
        const float cg = __fmul_rn(__fmul_rn(P.cubic_grad_factor, shape), kr);
        const float c = __fmul_rn(__fadd_rn(H.dpi, d.c), sg);
        v[0] = __fmaf_rn(-c, rx, v[0]); v[1] = __fmaf_rn(-c, ry, v[1]); v[2] = __fmaf_rn(-c, rz, v[2]);
        const float cn = __fmul_rn(cg, d.b.w);
        v[3] = __fmaf_rn(rx, cn, v[3]); v[4] = __fmaf_rn(ry, cn, v[4]); v[5] = __fmaf_rn(rz, cn, v[5]);
        const float vr = __fmaf_rn(__fsub_rn(H.v.z, d.b.z), rz,
                                   __fmaf_rn(__fsub_rn(H.v.y, d.b.y), ry, __fmul_rn(__fsub_rn(H.v.x, d.b.x), rx)));
        const float s = __fdividef(__fmul_rn(vr, cn), __fadd_rn(r2, P.visc_eps));
        v[6] = __fmaf_rn(s, rx, v[6]); v[7] = __fmaf_rn(s, ry, v[7]); v[8] = __fmaf_rn(s, rz, v[8]);
    } else if constexpr (KIND == PASS_SURFACE) {
        // cohesion (kernel.cuh:53-63); pairs closer than 1e-3 are skipped
        const float4 nj = d.b;
        const float rho_j = d.c;
        float rinv;
        const float q = q_of(r2, rinv, P);
        const float t = __fsub_rn(1.f, q);
        const float q3t3 = __fmul_rn(__fmul_rn(__fmul_rn(q, q), q), __fmul_rn(__fmul_rn(t, t), t));
        const float shape = q <= 0.5f ? __fmaf_rn(2.f, q3t3, -1.f / 64.f) : (q <= 1.f ? q3t3 : 0.f);
        const float coh = __fmul_rn(P.cohesion_factor, shape);
        const float inv = r2 > 1e-6f ? __fdividef(1.f, __fadd_rn(H.rho, rho_j)) : 0.f;
        const float cm = __fmul_rn(__fmul_rn(P.mass, coh), rinv);
        v[0] = __fmaf_rn(__fsub_rn(__fmaf_rn(cm, rx, H.n.x), nj.x), inv, v[0]);
        v[1] = __fmaf_rn(__fsub_rn(__fmaf_rn(cm, ry, H.n.y), nj.y), inv, v[1]);
        v[2] = __fmaf_rn(__fsub_rn(__fmaf_rn(cm, rz, H.n.z), nj.z), inv, v[2]);
    } else if constexpr (KIND == PASS_ADJ_FORCE) {
        // pressure: a_i = -m sum_j A_ij F(r_ij), F(r) = g_s(|r|) r, A_ij = p_i/rho_i^2 + p_j/rho_j^2
        const u32 j = d.j;
        const float rl = sqrtf(r2);
        const float q = rl * P.inv_h;
        const float dj = ro_ld(a.rho + j);
        const float pj = ro_ld(a.prs + j);
        const float4 aj = ro_ld(a.adj_abar + j);
        const float gs = spiky_grad(q, P);
        const float gsp = rl > 0.f ? spiky_grad_dr(q, rl, P) / rl : 0.f;
        const float A = H.dpi + pj / (dj * dj);
        const float dax = H.abar.x - aj.x, day = H.abar.y - aj.y, daz = H.abar.z - aj.z;
        const float rda = rx * dax + ry * day + rz * daz;
        v[6] += -P.mass * gs * rda;
        // x_i: -m A J_F(r) (abar_i - abar_j), J_F = g_s I + (g_s'/|r|) r r^T
        const float cA = -P.mass * A;
        v[0] += cA * (gs * dax + gsp * rda * rx);
        v[1] += cA * (gs * day + gsp * rda * ry);
        v[2] += cA * (gs * daz + gsp * rda * rz);
        // viscosity: vlap_i = sum_j (u.r) G(|r|) r / rho_j, u = v_i - v_j, G = g_c / (r^2 + eps)
        const float4 vj = ro_ld(a.vel + j);
        const float4 wj = ro_ld(a.adj_w + j);
        const float gc = cubic_grad(q, P);
        const float gcp = rl > 0.f ? cubic_grad_dr(q, rl, P) : 0.f;
        const float den = r2 + P.visc_eps;
        const float G = gc / den;
        const float Gp = rl > 0.f ? (gcp / den - 2.f * rl * gc / (den * den)) / rl : 0.f;  // G'/|r|
        const float ux = H.v.x - vj.x, uy = H.v.y - vj.y, uz = H.v.z - vj.z;
        const float ur = ux * rx + uy * ry + uz * rz;
        const float wir = H.w.x * rx + H.w.y * ry + H.w.z * rz;
        const float wjr = wj.x * rx + wj.y * ry + wj.z * rz;
        const float inv_dj = 1.f / dj, inv_di = 1.f / H.rho;
        const float cv = G * (wir * inv_dj - wjr * inv_di);
        v[3] += cv * rx; v[4] += cv * ry; v[5] += cv * rz;
        v[7] += ur * G * wjr;
        const float si = inv_dj, sj = inv_di;
        v[0] += si * (ux * G * wir + ur * G * H.w.x + ur * wir * Gp * rx) -
                sj * (ux * G * wjr + ur * G * wj.x + ur * wjr * Gp * rx);
        v[1] += si * (uy * G * wir + ur * G * H.w.y + ur * wir * Gp * ry) -
                sj * (uy * G * wjr + ur * G * wj.y + ur * wjr * Gp * ry);
        v[2] += si * (uz * G * wir + ur * G * H.w.z + ur * wir * Gp * rz) -
                sj * (uz * G * wjr + ur * G * wj.z + ur * wjr * Gp * rz);
    } else if constexpr (KIND == PASS_ADJ_DENSITY) {
        // rho_i = m (W(0) + sum_j W(|r_ij|)): dW/dx_i = g_c r_ij, shared by rho_i and rho_j
        const u32 j = d.j;
        const float q = sqrtf(r2) * P.inv_h;
        const float rb = ro_ld(a.adj_rhobar + j);
        const float c = P.mass * cubic_grad(q, P) * (H.rb + rb);
        v[0] += c * rx; v[1] += c * ry; v[2] += c * rz;
    }
}

// Boundary pair contributions; v[] of the pass:
//   DENSITY v0 = sum m_b W / cubic_factor; FORCE v0..2 = boundary pressure accel;
//   ADJ_FORCE v0..2 = dL/dx_i, v3 = boundary pressure-coefficient term; ADJ_DENSITY v0..2 = dL/dx_i
template <int KIND>
__device__ __forceinline__ void boundary_pair_m(float* v, const HomeData& H, float mb, float4 xb, float r2,
                                                const DevParams& P) {
    const float rx = H.x.x - xb.x, ry = H.x.y - xb.y, rz = H.x.z - xb.z;
    if constexpr (KIND == PASS_DENSITY) {
        float rinv;
        v[0] = __fmaf_rn(cubic_shape(q_of(r2, rinv, P)), mb, v[0]);
    } else if constexpr (KIND == PASS_FORCE) {
        // rounding written out (see finish_row)
        const float q = __fmul_rn(__fsqrt_rn(r2), P.inv_h);
        float sgr = 0.f;   // spiky_grad (kernel.cuh:43-51)
        if (!(q < 1.e-9f || q > 1.f)) {
            const float t = __fsub_rn(1.f, q);
            sgr = __fdiv_rn(__fmul_rn(__fmul_rn(P.spiky_grad_factor, t), t), __fmul_rn(P.h, __fmul_rn(q, P.h)));
        }
        const float c = __fmul_rn(__fmul_rn(mb, __fadd_rn(H.dpi, __fdiv_rn(H.prs, P.rest_density2))), sgr);
        v[0] = __fmaf_rn(-c, rx, v[0]); v[1] = __fmaf_rn(-c, ry, v[1]); v[2] = __fmaf_rn(-c, rz, v[2]);
    } else if constexpr (KIND == PASS_ADJ_FORCE) {
        // a_i -= m_b B_i F(r_ib), B_i = p_i/rho_i^2 + p_i/rho0^2
        const float rl = sqrtf(r2);
        const float q = rl * P.inv_h;
        const float gs = spiky_grad(q, P);
        const float gsp = rl > 0.f ? spiky_grad_dr(q, rl, P) / rl : 0.f;
        const float B = H.dpi + H.prs / P.rest_density2;
        const float ra = rx * H.abar.x + ry * H.abar.y + rz * H.abar.z;
        v[3] += -mb * gs * ra;
        const float cB = -mb * B;
        v[0] += cB * (gs * H.abar.x + gsp * ra * rx);
        v[1] += cB * (gs * H.abar.y + gsp * ra * ry);
        v[2] += cB * (gs * H.abar.z + gsp * ra * rz);
    } else if constexpr (KIND == PASS_ADJ_DENSITY) {
        const float c = mb * H.rb * cubic_grad(sqrtf(r2) * P.inv_h, P);
        v[0] += c * rx; v[1] += c * ry; v[2] += c * rz;
    }
}
template <int KIND>
__device__ __forceinline__ void boundary_pair(float* v, const HomeData& H, u32 b, float4 xb, float r2,
                                              const DevParams& P, const TravArgs& a) {
    boundary_pair_m<KIND>(v, H, ro_ld(a.bmass + guard(a, b, a.nb)), xb, r2, P);
}

// Boundary key of cell c (cell size h) of the scene.
template <bool BATCH>
__device__ __forceinline__ u64 boundary_cell_key(int3 c, u32 scene) {
    if constexpr (BATCH) return pack_cell_batch(scene, offset_coord(c.x), offset_coord(c.y), offset_coord(c.z));
    else return pack_cell(c);
}

// Run [start, end) of the per-cell boundary candidates of cell key pk
// (empty when pk is not within one cell of any boundary particle).
template <bool BATCH>
__device__ __forceinline__ void boundary_run(const TravArgs& a, u64 pk, u32& start, u32& end) {
    const u32 slot = find_slot<BATCH>(a.bcell.table, a.bcell.tmask, pk);
    start = end = 0;
    if (slot != EMPTY_CELL) {
        start = ro_ld(a.bcell.cstart + slot);
        end = ro_ld(a.bcell.cend + slot);
    }
}

// ---------------------------------------------------------------------------
// Segmented runs. A block of nh home particles (rows) is processed as one
// flat item space split into 32 contiguous runs, one per lane, so every lane
// does the same amount of work whatever the home count. A lane's run crosses
// rows in order; it stores one partial per (lane, row) segment in slot
// lane + row (unique: a later lane never reaches an earlier row), and
// combine() then adds, on lane k, the partials of row k in lane order, so
// the sums are deterministic.
// ---------------------------------------------------------------------------
template <int NF>
__device__ __forceinline__ void store_partial(float* part, u32 slot, const float* v) {
#pragma unroll
    for (int f = 0; f < NF; ++f) part[slot * NF + f] = v[f];
}

// Row k (the calling lane's row, lane - first row of the run) owns items
// [lo, hi); c = run length.
template <int NF>
__device__ __forceinline__ void combine(const float* part, float* res, bool active, u32 lo, u32 hi, u32 c,
                                        u32 k) {
    if (active && hi > lo) {
        // x / c as a multiply-high, exact for x < 2^32 / c (x <= 32 c here)
        const u32 inv = 0xFFFFFFFFu / c + 1u;
        const u32 l_lo = c == 1u ? lo : __umulhi(lo, inv);
        const u32 l_hi = c == 1u ? hi - 1 : __umulhi(hi - 1, inv);
        for (u32 l = l_lo; l <= l_hi; ++l) {
#pragma unroll
            for (int f = 0; f < NF; ++f) res[f] += part[(l + k) * NF + f];
        }
    }
    __syncwarp();
}

// Fluid pairs rows [0, nh) x staged candidates [0, len) (candidate index
// c0 + m), each tested against h^2 and the home particle itself (candidate
// index self0 + row): the path of cells whose candidates exceed the bit
// matrix capacity. Returns the run length.
template <int KIND>
__device__ __forceinline__ u32 fluid_pair_run(const WarpView<KIND>& S, const DevParams& P, const TravArgs& a,
                                              u32 nh, u32 len, u32 c0, u32 i0, u32 self0) {
    constexpr int NF = KindCfg<KIND>::nf;
    const u32 lane = lane_id();
    const u32 total = nh * len;
    const u32 c = ((total + 31u) >> 5) | 1u;  // odd: spreads the lanes' staged reads over the banks
    u32 p = lane * c;
    const u32 e = min(p + c, total);
    if (p < e) {
        u32 k = p / len;
        u32 m = p - k * len;
        HomeData H = load_home<KIND>(a, i0 + k);
        u32 self = self0 + k - c0;
        float v[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) v[f] = 0.f;
        for (;;) {
            const Nbr d = fetch<KIND>(S, a, m);
            const float r2 = dist2(H.x, d.x);
            if (r2 <= P.h2 && m != self) fluid_pair<KIND>(v, H, d, r2, P, a);
            ++p;
            if (++m == len || p == e) {
                store_partial<NF>(S.part, lane + k, v);
                if (p == e) break;
#pragma unroll
                for (int f = 0; f < NF; ++f) v[f] = 0.f;
                m = 0;
                ++k;
                H = load_home<KIND>(a, i0 + k);
                self = self0 + k - c0;
            }
        }
    }
    __syncwarp();
    return c;
}

// Position of home row k of the density pass: from the staged candidates
// (hm maps rows to candidate indices) when they hold the home cells, else
// from global memory.
__device__ __forceinline__ float4 home_x(const WarpView<PASS_DENSITY>& S, const TravArgs& a, u32 i0, HomeMap hm,
                                         u32 k) {
    if (hm.c1 != NO_HOME) {
        const u32 m = guard(a, hm.cand(k), a.mask_words * 32u);
        const float* f = reinterpret_cast<const float*>(S.sp + pair_slot(m >> 1)) + (m & 1u);
        return make_float4(f[0], f[2], f[4], 0.f);
    }
    return ro_ld(a.pos + guard(a, i0 + k, a.n));
}

// Neighbour pairs of rows [0, nh) read from the block's bit matrix in
// global memory (bits, row length M), split by hits. Returns the run length
// (0: no hits) and, for row k = lane, its hit range [lo, hi).
// lists (density pass): hit r of row k also goes to slot r of particle
// i0 + k, nbr[r * n + i0 + k], for r < nbr_width.
template <int KIND, bool SHARED_BITS = false>
__device__ __forceinline__ u32 fluid_hit_run(const WarpView<KIND>& S, const DevParams& P, const TravArgs& a,
                                             const u32* WCSPH_RESTRICT bits, u32 nh, u32 M, u32 i0, u32& lo,
                                             u32& hi, bool lists = false, HomeMap hm = HomeMap{32u, NO_HOME, 0u}) {
    auto home = [&](u32 k) -> HomeData {
        if constexpr (KIND == PASS_DENSITY) {
            if (hm.c1 != NO_HOME) {
                HomeData H;
                H.x = home_x(S, a, i0, hm, k);
                return H;
            }
        }
        return load_home<KIND>(a, i0 + k);
    };
    auto ld = [&](u32 w) -> u32 {
        if constexpr (SHARED_BITS) return bits[w];
        else return ro_ld(bits + w);
    };
    constexpr int NF = KindCfg<KIND>::nf;
    const u32 lane = lane_id();
    const u32 nwords = (nh * M + 31u) >> 5;
    u32 cnt = 0;
    if (lane < nh) {
        const u32 b0 = lane * M, b1 = b0 + M - 1;
        const u32 w0 = b0 >> 5, w1 = b1 >> 5;
        for (u32 w = w0; w <= w1; ++w) {
            u32 x = ld(w);
            if (w == w0) x &= FULL << (b0 & 31u);
            if (w == w1) x &= FULL >> (31u - (b1 & 31u));
            cnt += __popc(x);
        }
    }
    const u32 incl = warp_incl_scan(cnt);
    const u32 total = __shfl_sync(FULL, incl, 31);
    u32* hoff = S.hoff;
    lo = incl - cnt;
    hi = incl;
    if (lane < nh) hoff[lane] = lo;
    if (lane == 0) hoff[nh] = total;
    __syncwarp();
    if (total == 0) return 0;
    const u32 c = (total + 31u) >> 5;
    u32 h = lane * c;
    const u32 e = min(h + c, total);
    if (h < e) {
        u32 k = 0, kh = nh;  // the row holding hit h: largest k with hoff[k] <= h
        while (kh - k > 1) {
            const u32 mid = (k + kh) >> 1;
            if (hoff[mid] <= h) k = mid; else kh = mid;
        }
        u32 r = h - hoff[k];
        u32 row0 = k * M;
        u32 wr = row0 >> 5;
        u32 word = ld(wr) & (FULL << (row0 & 31u));
        for (;;) {
            const u32 pc = __popc(word);
            if (r < pc || wr + 1 >= nwords) break;
            r -= pc;
            word = ld(++wr);
        }
        for (; r && word; --r) word &= word - 1;
        HomeData H = home(k);
        float v[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) v[f] = 0.f;
        // density lists: list slot of hit h is h - (first hit of its row); u32
        // indices (the host caps nbr_width so that n * nbr_width < 2^32)
        u32 slot_base = hoff[k];
        while (word) {
            const u32 b = __ffs(word) - 1;
            word &= word - 1;
            const u32 p = (wr << 5) + b;
            if (p >= row0 + M) {   // the walk crossed into a later row: close row k's segment
                store_partial<NF>(S.part, lane + k, v);
#pragma unroll
                for (int f = 0; f < NF; ++f) v[f] = 0.f;
                do { ++k; row0 += M; } while (p >= row0 + M);
                H = home(k);
                slot_base = hoff[k];
            }
            if constexpr (KIND == PASS_DENSITY) {
                const u32 slot = h - slot_base;
                if (lists && slot < a.nbr_width) {
                    const u32 m = guard(a, p - row0, a.mask_words * 32u);
                    const u32 q = guard(a, S.cq[m], range_cells(a));
                    a.nbr[slot * a.n + guard(a, i0 + k, a.n)] = S.rstart[q] + (m - S.rpref[q]);
                }
            }
            const Nbr d = fetch<KIND>(S, a, p - row0);
            fluid_pair<KIND>(v, H, d, dist2(H.x, d.x), P, a);
            if (++h == e) break;
            while (word == 0 && wr + 1 < nwords) word = ld(++wr);
        }
        store_partial<NF>(S.part, lane + k, v);
    }
    __syncwarp();
    return c;
}

// Density pass, phase 1: distance test of rows [0, nh) x staged candidates
// [0, 32 wpr) (the padding candidates lie at infinity). One lane builds one
// word of the bit matrix (row-major, wpr words per row): 16 candidate pairs,
// unrolled, each tested in packed FP32 with the rounding of dist2()
// (x_i - x_j is formed as fma(x_j, -1, x_i), the same single rounding).
// The home particle's own bit is set here and cleared by the caller.
// Row windows: rows [0, hm.split) keep candidates [0, win_a) only, later rows
// [win_b, 32 wpr) only (the two cells of an x-pair, each restricted to its own
// 27 neighbour cells; a single cell passes win_a = 32 wpr).
__device__ __forceinline__ void density_test_words(const WarpView<PASS_DENSITY>& S, const DevParams& P,
                                                   const TravArgs& a, u32 nh, u32 wpr, u32 i0, HomeMap hm,
                                                   u32 win_a, u32 win_b) {
    const u32 nwords = nh * wpr;
    const float2 neg = make_float2(-1.f, -1.f);
    // w / wpr as a multiply-high: exact for w < 2^32 / wpr^2 (here w < 32 * 16)
    const u32 inv = 0xFFFFFFFFu / wpr + 1u;
    for (u32 w = lane_id(); w < nwords; w += 32) {
        const u32 k = wpr == 1u ? w : __umulhi(w, inv);
        const u32 wi = w - k * wpr;
        const float4 h = home_x(S, a, i0, hm, k);
        const float2 X = make_float2(h.x, h.x), Y = make_float2(h.y, h.y), Z = make_float2(h.z, h.z);
        const float2* base = S.sp + pair_slot(wi * 16u);
        u32 bits = 0;
#pragma unroll
        for (int t = 0; t < 16; ++t) {
            const float2 dx = __ffma2_rn(base[3 * t], neg, X);
            const float2 dy = __ffma2_rn(base[3 * t + 1], neg, Y);
            const float2 dz = __ffma2_rn(base[3 * t + 2], neg, Z);
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
            bits |= (r2.x <= P.h2 ? 1u << (2 * t) : 0u) | (r2.y <= P.h2 ? 2u << (2 * t) : 0u);
        }
        // candidates [lo, hi) of the row's window within this word
        const u32 lo = k < hm.split ? 0u : win_b, hi = k < hm.split ? win_a : 0xFFFFFFFFu;
        const u32 w0 = wi << 5;
        if (lo > w0) bits &= lo >= w0 + 32u ? 0u : FULL << (lo - w0);
        if (hi < w0 + 32u) bits &= hi <= w0 ? 0u : FULL >> (w0 + 32u - hi);
        S.aux[w] = bits;
    }
    __syncwarp();
}

// Boundary pairs rows [0, nh) x expanded boundary candidates [0, len).
template <int KIND>
__device__ __forceinline__ u32 boundary_pair_run(const WarpView<KIND>& S, const DevParams& P, const TravArgs& a,
                                                 u32 nh, u32 len, u32 i0) {
    constexpr int NFB = KindCfg<KIND>::nfb;
    const u32 lane = lane_id();
    const u32 total = nh * len;
    const u32 c = ((total + 31u) >> 5) | 1u;
    u32 p = lane * c;
    const u32 e = min(p + c, total);
    if (p < e) {
        u32 k = p / len;
        u32 m = p - k * len;
        HomeData H = load_home<KIND>(a, i0 + k);
        float v[NFB];
#pragma unroll
        for (int f = 0; f < NFB; ++f) v[f] = 0.f;
        for (;;) {
            const u32 b = guard(a, S.bcand[m], a.nb);
            const float4 xb = ro_ld(a.bpos + b);
            const float r2 = dist2(H.x, xb);
            if (r2 <= P.h2) boundary_pair<KIND>(v, H, b, xb, r2, P, a);
            ++p;
            if (++m == len || p == e) {
                store_partial<NFB>(S.part, lane + k, v);
                if (p == e) break;
#pragma unroll
                for (int f = 0; f < NFB; ++f) v[f] = 0.f;
                m = 0;
                ++k;
                H = load_home<KIND>(a, i0 + k);
            }
        }
    }
    __syncwarp();
    return c;
}

// Boundary pairs of rows [0, nh) from per-cell candidate runs: rows
// [0, split) against run A = [sa, sa + la) of bcx, later rows against run
// B = [sb, sb + lb) (the second cell of an x-pair). Segmented like
// boundary_pair_run; returns the run length and, for row k = lane, its item
// range [lo, hi).
// masks (density, a.bmask): hit m < 128 of row k also sets bit m of
// S.aux[4k .. 4k + 3], which the caller zeroes before and stores after.
template <int KIND>
__device__ __forceinline__ u32 boundary_cells_run(const WarpView<KIND>& S, const DevParams& P, const TravArgs& a,
                                                  u32 nh, u32 i0, u32 split, u32 sa, u32 la, u32 sb, u32 lb,
                                                  u32& lo, u32& hi, bool masks = false) {
    constexpr int NFB = KindCfg<KIND>::nfb;
    const u32 lane = lane_id();
    const u32 na = split * la;
    const u32 total = na + (nh - split) * lb;
    lo = lane < split ? lane * la : na + (min(lane, nh) - split) * lb;
    hi = lo + (lane < nh ? (lane < split ? la : lb) : 0u);
    if (total == 0) return 0;
    const u32 c = ((total + 31u) >> 5) | 1u;
    u32 p = lane * c;
    const u32 e = min(p + c, total);
    if (p < e) {
        u32 k, m;
        if (p < na) {
            k = p / la;
            m = p - k * la;
        } else {
            const u32 q = p - na;
            k = split + q / lb;
            m = q - (k - split) * lb;
        }
        u32 len = k < split ? la : lb;
        u32 run = k < split ? sa : sb;
        HomeData H = load_home<KIND>(a, i0 + k);
        float v[NFB];
#pragma unroll
        for (int f = 0; f < NFB; ++f) v[f] = 0.f;
        for (;;) {
            const float4 xb = ro_ld(a.bcx + guard(a, run + m, a.bcx_n));
            const float r2 = dist2(H.x, xb);
            if (r2 <= P.h2) {
                boundary_pair_m<KIND>(v, H, xb.w, xb, r2, P);
                if (masks && m < 128u) atomicOr(S.aux + 4u * k + (m >> 5), 1u << (m & 31u));
            }
            ++p;
            if (++m == len || p == e) {
                store_partial<NFB>(S.part, lane + k, v);
                if (p == e) break;
#pragma unroll
                for (int f = 0; f < NFB; ++f) v[f] = 0.f;
                m = 0;
                ++k;
                len = k < split ? la : lb;
                run = k < split ? sa : sb;
                H = load_home<KIND>(a, i0 + k);
            }
        }
    }
    __syncwarp();
    return c;
}

// Per-row epilogue of a pass: the sums res (fluid) and resb (boundary) of
// particle i become its fields; the surface pass integrates and adds to
// the warp's CFL / metric reductions. The rounding of every step is written
// out (__fmaf_rn, __fmul_rn, __fadd_rn): the compiler would otherwise choose
// which products to fuse by the surrounding code, and the per-pass kernels and
// the persistent ensemble kernel, which inline this into different code, must
// produce the same bits.
template <int KIND, bool BATCH>
__device__ __forceinline__ void finish_row(const DevParams& P, const TravArgs& a, u32 i, const float* res,
                                           const float* resb, u32 row_cnt, u32 scene, float dt, float np_dt,
                                           float& red_max, float& red_speed, float& red_speed2) {
    if constexpr (KIND == PASS_DENSITY) {
        // compute_density: (W(0) + sum W) * m, then + sum m_b W
        const float rho = __fmaf_rn(__fmaf_rn(P.cubic_factor, res[0], P.w0), P.mass, __fmul_rn(P.cubic_factor, resb[0]));
        const float prs = tait_pressure(rho, P);
        a.rho[i] = rho;
        a.prs[i] = prs;
        if (a.nbr) a.nbr_cnt[i] = row_cnt;
        // the force pass's neighbour records
        const float4 xi = a.pos[i];
        const float4 vi = a.vel[i];
        a.recf[2 * static_cast<size_t>(i)] = make_float4(xi.x, xi.y, xi.z, __fdiv_rn(prs, __fmul_rn(rho, rho)));
        a.recf[2 * static_cast<size_t>(i) + 1] = make_float4(vi.x, vi.y, vi.z, __fdiv_rn(1.f, rho));
    } else if constexpr (KIND == PASS_FORCE) {
        // compute_pressure_accel_n_normal_with_boundary: m * sum_fluid, then
        // the boundary term (compute_pressure_accel_n_normal.cu:346-364)
        a.ap[i] = f4(__fmaf_rn(P.mass, res[0], resb[0]), __fmaf_rn(P.mass, res[1], resb[1]),
                     __fmaf_rn(P.mass, res[2], resb[2]));
        const float sn = __fmul_rn(P.h, P.mass);
        const float4 ni = f4(__fmul_rn(sn, res[3]), __fmul_rn(sn, res[4]), __fmul_rn(sn, res[5]));
        a.normal[i] = ni;
        a.vlap[i] = f4(res[6], res[7], res[8]);
        // the surface pass's neighbour record
        const float4 xi = a.pos[i];
        a.recs[2 * static_cast<size_t>(i)] = make_float4(xi.x, xi.y, xi.z, a.rho[i]);
        a.recs[2 * static_cast<size_t>(i) + 1] = ni;
    } else if constexpr (KIND == PASS_SURFACE) {
        // a_np = g + F_ext + nu*10*m*vlap - alpha*2*rho0*f
        const float4 xi = a.pos[i];
        const float4 vi = a.vel[i];
        const float4 api = a.ap[i];
        const float4 vli = a.vlap[i];
        const float4 fe = external_force(xi, P);
        float4 gv = make_float4(P.gravity[0], P.gravity[1], P.gravity[2], P.visc_scale);
        const DevBox* bb = a.box;
        if constexpr (BATCH) {
            gv = a.scenes[scene].gravity_visc;
            bb = &a.scenes[scene].box;
            a.scene_state[i] = scene;
        }
        auto accel = [&](float g, float f, float vl, float st) {
            return __fmaf_rn(-P.st_scale, st, __fmaf_rn(gv.w, vl, __fadd_rn(g, f)));
        };
        float4 anp;
        anp.x = accel(gv.x, fe.x, vli.x, res[0]);
        anp.y = accel(gv.y, fe.y, vli.y, res[1]);
        anp.z = accel(gv.z, fe.z, vli.z, res[2]);
        anp.w = 0.f;
        a.anp[i] = anp;
        // update_positions.cu:64-67: v += np_dt a_np + dt a_p; x += dt v
        float4 v = vi, x = xi;
        v.x = __fadd_rn(v.x, __fmaf_rn(np_dt, anp.x, __fmul_rn(dt, api.x)));
        v.y = __fadd_rn(v.y, __fmaf_rn(np_dt, anp.y, __fmul_rn(dt, api.y)));
        v.z = __fadd_rn(v.z, __fmaf_rn(np_dt, anp.z, __fmul_rn(dt, api.z)));
        x.x = __fmaf_rn(dt, v.x, x.x);
        x.y = __fmaf_rn(dt, v.y, x.y);
        x.z = __fmaf_rn(dt, v.z, x.z);
        x.w = __fmaf_rn(dt, v.w, x.w);
        resolve_collision(x, v, *bb, P);
        a.pos_out[i] = x;
        a.vel_out[i] = v;
        const float s2 = dot3(v, v);
        red_max = fmaxf(red_max, s2);
        red_speed += sqrtf(s2);
        red_speed2 += s2;
    } else if constexpr (KIND == PASS_ADJ_FORCE) {
        const float rho_i = a.rho[i];
        const float prs_i = a.prs[i];
        const float pt = res[6], vt = res[7], bt = resb[3];
        const float inv_r2 = 1.f / (rho_i * rho_i);
        const float pbar = pt * inv_r2 + bt * (inv_r2 + 1.f / P.rest_density2);
        float rhobar = (pt + bt) * (-2.f * prs_i * inv_r2 / rho_i) + vt * inv_r2;
        // Tait EOS with the clamp of compute_rho_p.cu:236-238
        const float ratio = rho_i / P.rest_density;
        const float rc = fminf(fmaxf(ratio, 1.f), P.max_density_ratio);
        if (ratio > 1.f && ratio < P.max_density_ratio)
            rhobar += pbar * P.stiffness * P.exponent * powf(ratio, P.exponent - 1.f) / P.rest_density;
        red_speed += pbar * (powf(rc, P.exponent) - 1.f);  // dL/dk partial
        a.adj_rhobar[i] = rhobar;
        const float4 xb0 = a.adj_xbar[i], vb0 = a.adj_vbar[i];
        a.adj_xbar[i] = f4(xb0.x + res[0] + resb[0], xb0.y + res[1] + resb[1],
                           xb0.z + res[2] + resb[2]);
        a.adj_vbar[i] = f4(vb0.x + res[3], vb0.y + res[4], vb0.z + res[5]);
    } else if constexpr (KIND == PASS_ADJ_DENSITY) {
        const float4 xb0 = a.adj_xbar[i];
        a.adj_xbar[i] = f4(xb0.x + res[0] + resb[0], xb0.y + res[1] + resb[1],
                           xb0.z + res[2] + resb[2]);
    }
}

// Cell coordinates (and scene) of a packed cell key.
template <bool BATCH>
__device__ __forceinline__ void decode_cell(u64 pk, u32& ux, u32& uy, u32& uz, u32& scene) {
    if constexpr (BATCH) {
        scene = static_cast<u32>(pk >> 48);
        ux = static_cast<u32>(pk & 0xFFFFull);
        uy = static_cast<u32>((pk >> 16) & 0xFFFFull);
        uz = static_cast<u32>((pk >> 32) & 0xFFFFull);
    } else {
        scene = 0;
        ux = static_cast<u32>(pk & 0x1FFFFFull);
        uy = static_cast<u32>((pk >> 21) & 0x1FFFFFull);
        uz = static_cast<u32>((pk >> 42) & 0x1FFFFFull);
    }
}

// The fluid sums of one row (particle i) without its list: lane q walks
// neighbour cells q, q + 32, ... of i's cell (its hash probe and particles),
// testing every candidate against h^2; the lanes' partials are then added
// in a fixed butterfly order. Returns the sums on every lane.
template <int KIND, bool BATCH>
__device__ __forceinline__ void spill_row(const DevParams& P, const TravArgs& a, u32 i, float* out) {
    constexpr int NF = KindCfg<KIND>::nf;
    const u32 lane = lane_id();
    u32 ux, uy, uz, scene;
    decode_cell<BATCH>(a.ckey[i], ux, uy, uz, scene);
    const int R = a.range;
    const u32 D = static_cast<u32>(2 * R + 1);
    const u32 ncell = D * D * D;
    const HomeData H = load_home<KIND>(a, i);
    float v[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) v[f] = 0.f;
    for (u32 q = lane; q < ncell; q += 32) {
        int dx, dy, dz;
        cell_offset(q, R, dx, dy, dz);
        u64 pk;
        if constexpr (BATCH) pk = pack_cell_batch(scene, ux + dx, uy + dy, uz + dz);
        else pk = pack_cell(ux + dx, uy + dy, uz + dz);
        const u32 slot = find_slot<BATCH>(a.fluid.table, a.fluid.tmask, pk);
        if (slot == EMPTY_CELL) continue;
        const u32 e = ro_ld(a.fluid.cend + slot);
        for (u32 j = ro_ld(a.fluid.cstart + slot); j < e; ++j) {
            const Nbr d = fetch_j<KIND>(a, j);
            const float r2 = dist2(H.x, d.x);
            if (r2 <= P.h2 && j != i) fluid_pair<KIND>(v, H, d, r2, P, a);
        }
    }
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        float x = v[f];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(FULL, x, o);
        out[f] = x;
    }
}

// Boundary sums of one row (particle i, home data H): the 3x3x3 boundary
// cells around its own cell in x, y, z nesting order, as for_boundary_neighbors
// (common.cuh:153-178) visits them, one particle after the other.
template <int KIND, bool BATCH>
__device__ __forceinline__ void boundary_row(const DevParams& P, const TravArgs& a, const HomeData& H, u32 scene,
                                             float* resb, u32 i) {
    const int3 c = cell_of(H.x, P.h);
    if (a.bcell.table != nullptr) {   // the cell's candidates, gathered in the same order
        u32 t, e;
        boundary_run<BATCH>(a, boundary_cell_key<BATCH>(c, scene), t, e);
        if (a.bmask != nullptr && e - t <= 128u) {
            // the density pass of this step marked the candidates within h
            // (same positions, same predicate): visit those, in run order
            const uint4 mk = ro_ld(a.bmask + i);
            const u32 words[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
            for (u32 w = 0; w < 4; ++w) {
                for (u32 bits = words[w]; bits; bits &= bits - 1) {
                    const float4 xb = ro_ld(a.bcx + guard(a, t + 32u * w + (__ffs(bits) - 1), a.bcx_n));
                    boundary_pair_m<KIND>(resb, H, xb.w, xb, dist2(H.x, xb), P);
                }
            }
            return;
        }
        for (; t < e; ++t) {
            const float4 xb = ro_ld(a.bcx + guard(a, t, a.bcx_n));
            const float r2 = dist2(H.x, xb);
            if (r2 <= P.h2) boundary_pair_m<KIND>(resb, H, xb.w, xb, r2, P);
        }
        return;
    }
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                u64 pk;
                if constexpr (BATCH)
                    pk = pack_cell_batch(scene, offset_coord(c.x + dx), offset_coord(c.y + dy), offset_coord(c.z + dz));
                else pk = pack_cell(make_int3(c.x + dx, c.y + dy, c.z + dz));
                const u32 slot = find_slot<BATCH>(a.boundary.table, a.boundary.tmask, pk);
                if (slot == EMPTY_CELL) continue;
                const u32 e = ro_ld(a.boundary.cend + slot);
                for (u32 b = ro_ld(a.boundary.cstart + slot); b < e; ++b) {
                    const float4 xb = ro_ld(a.bpos + guard(a, b, a.nb));
                    const float r2 = dist2(H.x, xb);
                    if (r2 <= P.h2) boundary_pair<KIND>(resb, H, b, xb, r2, P, a);
                }
            }
}

// Force / surface pass over listed neighbours: the warp's rows are the
// particles [i0, i0 + nh) of its chunk, whatever their cells; lane k sums
// row k's list in order (the reference's per-particle order), so a row's
// sums do not depend on which particles share its warp.
// DEPTH: neighbour records in flight per lane while a pair is summed (1, or
// 2 where the registers are there anyway: the persistent ensemble kernel
// runs at the density pass's register budget, with fewer resident warps than
// the list kernels; its surface phase gains from the second record in flight,
// its force phase does not).
template <int KIND, bool BATCH, int DEPTH = 1>
__device__ __forceinline__ void list_rows(const DevParams& P, const TravArgs& a, u32 i0, u32 nh, float dt,
                                          float np_dt, float& red_max, float& red_speed, float& red_speed2) {
    using C = KindCfg<KIND>;
    constexpr int NF = C::nf;
    constexpr int NFB = C::nfb;
    const u32 lane = lane_id();
    const bool act = lane < nh;
    const u32 i = i0 + (act ? lane : 0u);
    const u32 cnt = act ? ro_ld(a.nbr_cnt + i) : 0u;
    const bool spill = act && cnt > a.nbr_width;
    float res[NF], resb[NFB];
#pragma unroll
    for (int f = 0; f < NF; ++f) res[f] = 0.f;
    for (u32 sp = __ballot_sync(FULL, spill); sp; sp &= sp - 1) {
        const u32 f = __ffs(sp) - 1;
        float t[NF];
        spill_row<KIND, BATCH>(P, a, i0 + f, t);
        if (lane == f) {
#pragma unroll
            for (int g = 0; g < NF; ++g) res[g] = t[g];
        }
    }
#pragma unroll
    for (int f = 0; f < NFB; ++f) resb[f] = 0.f;
    const u64 pk = act ? a.ckey[i] : 0ull;
    const u32 scene = BATCH ? static_cast<u32>(pk >> 48) : 0u;
    if (act) {
        const HomeData H = load_home<KIND>(a, i);
        if (!spill && cnt > 0) {
            // slot t of row i at nbr[t * n + i]; the next neighbour's records
            // and the index after it are in flight while a pair is summed
            const size_t stride = a.n;
            if constexpr (DEPTH == 1) {
                const u32* lst = a.nbr + i + stride;
                Nbr d = fetch_j<KIND>(a, ro_ld(a.nbr + i));
                u32 jn = cnt > 1 ? ro_ld(lst) : 0u;
                lst += stride;
                for (u32 t = 0; t < cnt; ++t) {
                    Nbr dn = d;
                    if (t + 1 < cnt) dn = fetch_j<KIND>(a, jn);
                    if (t + 2 < cnt) {
                        jn = ro_ld(lst);
                        lst += stride;
                    }
                    fluid_pair<KIND>(res, H, d, dist2(H.x, d.x), P, a);
                    d = dn;
                }
            } else {
                const u32* lst = a.nbr + i;
                Nbr d0 = fetch_j<KIND>(a, ro_ld(lst));
                Nbr d1 = d0;
                if (cnt > 1) d1 = fetch_j<KIND>(a, ro_ld(lst + stride));
                u32 jn = cnt > 2 ? ro_ld(lst + 2 * stride) : 0u;
                lst += 3 * stride;
                for (u32 t = 0; t < cnt; ++t) {
                    Nbr d2 = d1;
                    if (t + 2 < cnt) d2 = fetch_j<KIND>(a, jn);
                    if (t + 3 < cnt) {
                        jn = ro_ld(lst);
                        lst += stride;
                    }
                    fluid_pair<KIND>(res, H, d0, dist2(H.x, d0.x), P, a);
                    d0 = d1;
                    d1 = d2;
                }
            }
        }
        if constexpr (C::boundary) {
            if (a.nb > 0) boundary_row<KIND, BATCH>(P, a, H, scene, resb, i);
        }
    }
    if (act) finish_row<KIND, BATCH>(P, a, i, res, resb, 0u, scene, dt, np_dt, red_max, red_speed, red_speed2);
}

// Surface pass: CFL max |v|^2 and the metric sums without block barriers:
// warp partials -> groups of 32 warps -> whole grid; each level is finished
// by its last arriving warp and summed in index order (deterministic). The
// last warp also publishes dt and flips the max-speed parity.
template <int WPB>
__device__ __forceinline__ void surface_reduce(const TravArgs& a, float dt, float np_dt, float red_max, float red_speed,
                                               float red_speed2) {
    const u32 lane = lane_id();
    const u32 warp = threadIdx.x >> 5;
    const u32 n = a.n;
    for (int o = 16; o > 0; o >>= 1) {
        red_max = fmaxf(red_max, __shfl_xor_sync(FULL, red_max, o));
        red_speed += __shfl_xor_sync(FULL, red_speed, o);
        red_speed2 += __shfl_xor_sync(FULL, red_speed2, o);
    }
    const u32 nwarps = gridDim.x * WPB;
    const u32 gw = blockIdx.x * WPB + warp;
    const u32 group = gw >> 5;
    const u32 ngroups = (nwarps + 31u) >> 5;
    const u32 gsize = min(32u, nwarps - (group << 5));
    u32 last = 0;
    if (lane == 0) {
        a.block_partials[2 * gw] = red_speed;
        a.block_partials[2 * gw + 1] = red_speed2;
        atomicMax(&a.st->vmax2_bits[a.st->parity ^ 1u], __float_as_uint(red_max));
        __threadfence();
        last = atomicAdd(a.group_done + group, 1u) == gsize - 1 ? 1u : 0u;
    }
    if (__shfl_sync(FULL, last, 0)) {
        __threadfence();
        const u32 w = (group << 5) + lane;
        double s1 = lane < gsize ? static_cast<double>(__ldcg(a.block_partials + 2 * w)) : 0.0;
        double s2 = lane < gsize ? static_cast<double>(__ldcg(a.block_partials + 2 * w + 1)) : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_xor_sync(FULL, s1, o);
            s2 += __shfl_xor_sync(FULL, s2, o);
        }
        u32 top = 0;
        if (lane == 0) {
            a.group_partials[2 * group] = s1;
            a.group_partials[2 * group + 1] = s2;
            a.group_done[group] = 0u;
            __threadfence();
            top = atomicAdd(&a.st->blocks_done, 1u) == ngroups - 1 ? 1u : 0u;
        }
        if (__shfl_sync(FULL, top, 0)) {
            __threadfence();
            double t1 = 0.0, t2 = 0.0;
            for (u32 g = lane; g < ngroups; g += 32) {
                t1 += __ldcg(a.group_partials + 2 * g);
                t2 += __ldcg(a.group_partials + 2 * g + 1);
            }
            for (int o = 16; o > 0; o >>= 1) {
                t1 += __shfl_xor_sync(FULL, t1, o);
                t2 += __shfl_xor_sync(FULL, t2, o);
            }
            if (lane == 0) {
                DevState* st = a.st;
                st->last_mean_speed = static_cast<float>(t1 / static_cast<double>(n));
                st->last_ke = static_cast<float>(0.5 * static_cast<double>(a.metric_mass) * t2);
                st->last_dt_p = dt;
                st->last_np_dt = np_dt;
                const u32 old = st->parity;
                st->vmax2_bits[old] = 0u;
                st->parity = old ^ 1u;
                st->blocks_done = 0u;
            }
        }
    }
}

// One chunk of a traversal pass: the cells that start among the chunk's
// a.chunk sorted particles (a cell is handled whole by the warp of its first
// particle), by the calling warp, with its shared-memory view S. The pass
// kernels call it once per warp; the persistent ensemble kernel calls it for
// every chunk its warps take.
template <int KIND, bool BATCH>
__device__ __forceinline__ void cell_pass_chunk(const DevParams& P, const TravArgs& a, const WarpView<KIND>& S,
                                                u32 chunk, float dt, float np_dt, float& red_max, float& red_speed,
                                                float& red_speed2) {
    using C = KindCfg<KIND>;
    constexpr int NF = C::nf;
    constexpr int NFB = C::nfb;
    const u32 lane = lane_id();
    const u32 cap = a.mask_words * 32u;
    const u32 per_chunk = a.chunk;
    const u32 base = chunk * per_chunk;
    const u32 n = a.n;
    const int R = a.range;
    const u32 D = static_cast<u32>(2 * R + 1);
    const u32 ncell = D * D * D;
    const u32 qc = ncell >> 1;

    if (base < n) {
        const u32 i0l = base + lane;
        const bool in = lane < per_chunk && i0l < n;
        const u64 my_pk = in ? a.ckey[i0l] : 0ull;
        u64 prev_pk = __shfl_up_sync(FULL, my_pk, 1);
        if (lane == 0) prev_pk = i0l > 0 ? a.ckey[i0l - 1] : ~my_pk;
        // cells that start in this chunk (a cell is handled whole by the warp of its first particle)
        u32 starts = __ballot_sync(FULL, in && (i0l == 0 || my_pk != prev_pk));
        while (starts) {
            const u32 s = __ffs(starts) - 1;
            starts &= starts - 1;
            const u64 pk = __shfl_sync(FULL, my_pk, s);
            u32 ux, uy, uz, scene = 0;
            if constexpr (BATCH) {
                scene = static_cast<u32>(pk >> 48);
                ux = static_cast<u32>(pk & 0xFFFFull);
                uy = static_cast<u32>((pk >> 16) & 0xFFFFull);
                uz = static_cast<u32>((pk >> 32) & 0xFFFFull);
            } else {
                ux = static_cast<u32>(pk & 0x1FFFFFull);
                uy = static_cast<u32>((pk >> 21) & 0x1FFFFFull);
                uz = static_cast<u32>((pk >> 42) & 0x1FFFFFull);
            }
            // Density with lists: a cell of even x and the cell of x + 1 after
            // it (Morton-consecutive, so adjacent in sorted order whenever both
            // are occupied) form an x-pair, handled whole by the warp of the
            // first: one lookup of the union of their neighbour cells (4 x 3 x 3,
            // in the reference's x, y, z order), one staging, and twice the
            // home rows per walk. The warp of the second cell skips it.
            bool pair_try = false;
            if constexpr (KIND == PASS_DENSITY) {
                if (a.pair_cells && R == 1) {
                    if (ux & 1u) {
                        u64 apk;
                        if constexpr (BATCH) apk = pack_cell_batch(scene, ux - 1u, uy, uz);
                        else apk = pack_cell(ux - 1u, uy, uz);
                        if (__shfl_sync(FULL, prev_pk, s) == apk && base + s > 0) continue;
                    } else {
                        pair_try = true;
                    }
                }
            }
            u32 gx = ux;   // x of the cell whose neighbourhood is gathered
            auto gather = [&](u32 nc) {
                return gather_ranges<BATCH>(S.rstart, S.rpref, nc, a.fluid, [&](u32 q) {
                    int dx, dy, dz;
                    cell_offset(q, R, dx, dy, dz);   // R = 1: q < 36 gives dx in [-1, 2]
                    if constexpr (BATCH) return pack_cell_batch(scene, gx + dx, uy + dy, uz + dz);
                    else return pack_cell(gx + dx, uy + dy, uz + dz);
                });
            };
            u32 units = 1;
            for (u32 unit = 0; unit < units; ++unit) {
            // fluid neighbour cells in the reference's x, y, z nesting order
            u32 M, ncs, home_start, n_home, self_base;
            bool pair = false;
            u32 nA = 0, selfB = 0, winA = 0, winB = 0;
            if (unit == 0) {
                M = gather(pair_try ? 36u : ncell);
                ncs = ncell;
                home_start = S.rstart[qc];
                n_home = S.rpref[qc + 1] - S.rpref[qc];
                self_base = S.rpref[qc];   // candidate index of the first home particle
                if (pair_try) {
                    // union cells 0..26: the first cell's neighbourhood, 9..35: the second's
                    nA = n_home;
                    const u32 nB = S.rpref[23] - S.rpref[22];
                    const bool second = nB > 0 && S.rstart[22] == home_start + nA;
                    if (second && ((M + 31u) & ~31u) <= a.mask_words * 32u) {
                        pair = true;
                        ncs = 36;
                        n_home = nA + nB;
                        selfB = S.rpref[22];
                        winA = S.rpref[27];
                        winB = S.rpref[9];
                    } else {
                        M = S.rpref[27];   // the first cell alone (its 27 cells lead the union)
                        if (second) units = 2;
                    }
                }
            } else {
                // the second cell of a pair whose union exceeds the bit-matrix capacity
                gx = ux + 1u;
                M = gather(ncell);
                ncs = ncell;
                home_start = S.rstart[qc];
                n_home = S.rpref[qc + 1] - S.rpref[qc];
                self_base = S.rpref[qc];
            }
            const u32 Mrow = (M + 31u) & ~31u;     // bit-matrix row length (whole words)
            const bool masked = Mrow <= cap;

            // boundary neighbour cells: union of the home particles' 3x3x3
            // boundary-cell neighbourhoods (cell size h, R = 1,
            // for_boundary_neighbors common.cuh:153-178)
            u32 MB = 0, nbc = 0;
            // density with per-cell boundary candidates (cell size h): the
            // runs of the unit's home cells (A, and B of an x-pair)
            const bool use_cells = KIND == PASS_DENSITY && a.bcell.table != nullptr && P.cell_size == P.h;
            u32 bra = 0, bla = 0, brb = 0, blb = 0;
            if (use_cells && a.nb > 0) {
                u32 s0 = 0, s1 = 0;
                if (lane < (pair ? 2u : 1u)) {
                    const int3 hc = cell_of(a.pos[home_start + (lane ? nA : 0u)], P.h);
                    boundary_run<BATCH>(a, boundary_cell_key<BATCH>(hc, scene), s0, s1);
                }
                bra = __shfl_sync(FULL, s0, 0);
                bla = __shfl_sync(FULL, s1, 0) - bra;
                brb = __shfl_sync(FULL, s0, 1);
                blb = __shfl_sync(FULL, s1, 1) - brb;
            }
            if constexpr (C::boundary) {
                if (a.nb > 0 && !use_cells) {
                    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
                    for (u32 k = lane; k < n_home; k += 32) {
                        const int3 c = cell_of(a.pos[home_start + k], P.h);
                        lo[0] = min(lo[0], c.x); hi[0] = max(hi[0], c.x);
                        lo[1] = min(lo[1], c.y); hi[1] = max(hi[1], c.y);
                        lo[2] = min(lo[2], c.z); hi[2] = max(hi[2], c.z);
                    }
#pragma unroll
                    for (int d = 0; d < 3; ++d) {
                        lo[d] = __reduce_min_sync(FULL, lo[d]) - 1;
                        hi[d] = __reduce_max_sync(FULL, hi[d]) + 1;
                    }
                    const u32 bx = hi[0] - lo[0] + 1, by = hi[1] - lo[1] + 1, bz = hi[2] - lo[2] + 1;
                    nbc = bx * by * bz;
                    if (nbc > MAX_BOUNDARY_CELLS) {
                        if (lane == 0) atomicOr(&a.st->error_flags, ERR_CAND_OVERFLOW);
                        nbc = 0;
                    } else {
                        MB = gather_ranges<BATCH>(S.bstart, S.bpref, nbc, a.boundary, [&](u32 q) {
                            const int cz = lo[2] + static_cast<int>(q % bz);
                            const int cy = lo[1] + static_cast<int>((q / bz) % by);
                            const int cx = lo[0] + static_cast<int>(q / (bz * by));
                            if constexpr (BATCH)
                                return pack_cell_batch(scene, offset_coord(cx), offset_coord(cy), offset_coord(cz));
                            else return pack_cell(make_int3(cx, cy, cz));
                        });
                    }
                }
            }

            if (masked) stage<KIND>(S, a, ncs, 0, M);
            // the cell's neighbour bit matrix: row k = home particle k, bit m = candidate m
            u32* const cell_bits = a.mask + static_cast<size_t>(home_start) * a.mask_words;

            for (u32 hb = 0; hb < n_home; hb += HOME_BLOCK) {
                const u32 nh = min(HOME_BLOCK, n_home - hb);
                const u32 i0 = home_start + hb;
                const u32 self0 = self_base + hb;
                // candidate index of each home row of the block (x-pairs: the
                // rows of the second cell follow those of the first)
                const HomeMap hm = pair ? HomeMap{nA > hb ? nA - hb : 0u, self0, selfB + (hb > nA ? hb - nA : 0u)}
                                        : HomeMap{32u, self0, 0u};
                const bool act = lane < nh;
                const u32 i = i0 + (act ? lane : 0u);
                u32* const blk_bits = cell_bits + (hb >> 5) * Mrow;   // row hb starts at bit hb * Mrow
                float res[NF], resb[NFB];
#pragma unroll
                for (int f = 0; f < NF; ++f) res[f] = 0.f;
#pragma unroll
                for (int f = 0; f < NFB; ++f) resb[f] = 0.f;
                u32 row_cnt = NBR_SPILL;   // density with lists: the row's listed neighbour count

                if constexpr (KIND == PASS_COUNT || KIND == PASS_FILL) {
                    // sequential per home particle, in candidate order (the reference's order)
                    u32 cnt = 0;
                    u32 wpos = 0;
                    if constexpr (KIND == PASS_FILL) wpos = act ? a.offsets[i] : 0u;
                    if (masked && a.matrix_valid) {
                        if (act) {
                            const u32 b0 = lane * Mrow, b1 = b0 + Mrow - 1;
                            for (u32 w = b0 >> 5; w <= (b1 >> 5); ++w) {
                                u32 x = blk_bits[w];
                                if (w == (b0 >> 5)) x &= FULL << (b0 & 31u);
                                if (w == (b1 >> 5)) x &= FULL >> (31u - (b1 & 31u));
                                while (x) {
                                    const u32 bit = __ffs(x) - 1;
                                    x &= x - 1;
                                    if constexpr (KIND == PASS_FILL) {
                                        const u32 m = (w << 5) + bit - b0;
                                        if (wpos < a.nbr_capacity) a.nbr_out[wpos] = S.cand[m];
                                        ++wpos;
                                    }
                                    ++cnt;
                                }
                            }
                        }
                    } else {
                        const float4 xi = a.pos[i];
                        for (u32 c0 = 0; c0 < M; c0 += cap) {
                            const u32 len = min(cap, M - c0);
                            stage<KIND>(S, a, ncs, c0, len);
                            if (act) {
                                for (u32 ml = 0; ml < len; ++ml) {
                                    if (c0 + ml != self0 + lane && dist2(xi, S.sa[ml]) <= P.h2) {
                                        if constexpr (KIND == PASS_FILL) {
                                            if (wpos < a.nbr_capacity) a.nbr_out[wpos] = S.cand[ml];
                                            ++wpos;
                                        }
                                        ++cnt;
                                    }
                                }
                            }
                        }
                    }
                    if constexpr (KIND == PASS_COUNT) {
                        if (act) a.counts[i] = cnt;
                    }
                    continue;
                } else if constexpr (KIND == PASS_DENSITY) {
                    // phase 1 tests every candidate and builds the bit matrix in shared
                    // memory; phase 2 sums W over the neighbours only (and, with
                    // lists on, writes them to the rows' lists)
                    auto density_chunk = [&](u32 c0, u32 len, bool keep_bits) {
                        const u32 wpr = (len + 31u) >> 5;
                        const u32 len32 = wpr << 5;
                        const u32 nwords = nh * wpr;
                        // masked: the home cells are staged
                        const HomeMap hmc = keep_bits ? hm : HomeMap{32u, NO_HOME, 0u};
                        density_test_words(S, P, a, nh, wpr, i0, hmc, pair ? winA : len32, winB);
                        const u32 self = (keep_bits ? hm.cand(lane) : self0 + lane) - c0;   // the home particle itself
                        if (act && self < len) {
                            const u32 item = lane * len32 + self;
                            atomicAnd(S.aux + (item >> 5), ~(1u << (item & 31u)));
                        }
                        __syncwarp();
                        u32 lo, hi;
                        const u32 c = fluid_hit_run<KIND, true>(S, P, a, S.aux, nh, len32, i0, lo, hi,
                                                                keep_bits && a.nbr != nullptr, hmc);
                        if (c) combine<NF>(S.part, res, act, lo, hi, c, lane);
                        if (keep_bits && hi - lo <= a.nbr_width) row_cnt = hi - lo;
                        if (keep_bits && !a.pair_cells)   // kept for the neighbour export and the adjoint
                            for (u32 w = lane; w < nwords; w += 32) blk_bits[w] = S.aux[w];
                        __syncwarp();
                    };
                    if (masked) {
                        density_chunk(0, M, true);
                    } else {
                        for (u32 c0 = 0; c0 < M; c0 += cap) {
                            const u32 len = min(cap, M - c0);
                            stage<KIND>(S, a, ncs, c0, len);
                            density_chunk(c0, len, false);
                        }
                    }
                } else {
                    if (masked) {
                        // one coalesced copy of the block's bit matrix, then walks in shared memory
                        const u32 nwords = (nh * Mrow) >> 5;
                        for (u32 w = lane; w < nwords; w += 32) S.aux[w] = ro_ld(blk_bits + w);
                        __syncwarp();
                        u32 lo, hi;
                        const u32 c = fluid_hit_run<KIND, true>(S, P, a, S.aux, nh, Mrow, i0, lo, hi);
                        if (c) combine<NF>(S.part, res, act, lo, hi, c, lane);
                    } else {
                        for (u32 c0 = 0; c0 < M; c0 += cap) {
                            const u32 len = min(cap, M - c0);
                            stage<KIND>(S, a, ncs, c0, len);
                            const u32 c = fluid_pair_run<KIND>(S, P, a, nh, len, c0, i0, self0);
                            combine<NF>(S.part, res, act, lane * len, lane * len + len, c, lane);
                        }
                    }
                }

                // boundary candidates (density and pressure passes)
                if (use_cells) {
                    const bool masks = a.bmask != nullptr;
                    if (masks) {
                        for (u32 w = lane; w < 4u * nh; w += 32) S.aux[w] = 0u;
                        __syncwarp();
                    }
                    u32 blo, bhi;
                    const u32 c = boundary_cells_run<KIND>(S, P, a, nh, i0, min(hm.split, nh), bra, bla, brb, blb,
                                                           blo, bhi, masks);
                    if (c) combine<NFB>(S.part, resb, act, blo, bhi, c, lane);
                    if (masks && act)
                        a.bmask[i] = make_uint4(S.aux[4 * lane], S.aux[4 * lane + 1], S.aux[4 * lane + 2],
                                                S.aux[4 * lane + 3]);
                } else if constexpr (C::boundary) {
                    for (u32 c0 = 0; c0 < MB; c0 += BCAND_CAP) {
                        const u32 len = min(BCAND_CAP, MB - c0);
                        expand(S.bcand, S.bstart, S.bpref, nbc, c0, len);
                        const u32 c = boundary_pair_run<KIND>(S, P, a, nh, len, i0);
                        combine<NFB>(S.part, resb, act, lane * len, lane * len + len, c, lane);
                    }
                }

                if (act)
                    finish_row<KIND, BATCH>(P, a, i, res, resb, row_cnt, scene, dt, np_dt, red_max, red_speed,
                                            red_speed2);
            }
            }   // units
        }
    }

}

// Shared-memory view of the calling warp (warp slot `warp` of the block's
// dynamic shared memory) for pass KIND.
template <int KIND>
__device__ __forceinline__ WarpView<KIND> warp_view(const TravArgs& a, unsigned char* smem, u32 warp) {
    WarpView<KIND> S;
    const u32 cap = a.mask_words * 32u;
    const u32 ncell_s = static_cast<u32>((2 * a.range + 1) * (2 * a.range + 1) * (2 * a.range + 1));
    const size_t wbytes = warp_smem_bytes<KIND>(cap, ncell_s, a.nb > 0);
    warp_smem_bytes<KIND>(cap, ncell_s, a.nb > 0, &S, smem + warp * wbytes);
    return S;
}

// Particles per warp of the list kernels: one per lane, except for small
// scenes (density chunks of 8), which keep 8 so that more warps run.
__host__ __device__ inline u32 list_rows_per_warp(u32 chunk) { return chunk == 8u ? 8u : 32u; }

template <bool BATCH>
__device__ __forceinline__ u64 cell_key_of(float4 p, float cs, const u32* scene_in, u32 src) {
    const int3 c = cell_of(p, cs);
    if constexpr (BATCH) return pack_cell_batch(scene_in[src], offset_coord(c.x), offset_coord(c.y), offset_coord(c.z));
    else return pack_cell(c);
}

// Reorder + hash build for sorted index i (gather pos/vel into sorted order,
// cell keys, run starts/ends into the hash; rebuild_n_search.cu:19-34). All 32
// lanes of a warp must call it together (i >= n for the idle ones).
template <bool BATCH>
__device__ __forceinline__ void reorder_cell_item(const float4* WCSPH_RESTRICT pos_in, const float4* WCSPH_RESTRICT vel_in,
                                                  const u32* WCSPH_RESTRICT v1, const u32* WCSPH_RESTRICT v2,
                                                  const DevState* st, u32 n, float cs, float4* WCSPH_RESTRICT pos_out,
                                                  float4* WCSPH_RESTRICT vel_out, u32* WCSPH_RESTRICT perm_out,
                                                  u64* WCSPH_RESTRICT ckey_out, u64* table, u32* cstart, u32* cend,
                                                  u32 tmask, DevState* st_err, const u32* WCSPH_RESTRICT scene_in, u32 i) {
    const u32 lane = threadIdx.x & 31u;
    const u32 sel = st->sort_sel[8];
    const u32* perm = sel == 0 ? nullptr : (sel == 1 ? v1 : v2);
    const bool valid = i < n;
    u64 pk = 0;
    if (valid) {
        const u32 src = guard_st(st_err, perm ? perm[i] : i, n);
        const float4 p = pos_in[src];
        pos_out[i] = p;
        if (vel_out) vel_out[i] = vel_in[src];
        perm_out[i] = src;
        pk = cell_key_of<BATCH>(p, cs, scene_in, src);
        ckey_out[i] = pk;
    }
    u64 prev = __shfl_up_sync(FULL, pk, 1);
    u64 next = __shfl_down_sync(FULL, pk, 1);
    if (valid && lane == 0 && i > 0) {
        const u32 s2 = guard_st(st_err, perm ? perm[i - 1] : i - 1, n);
        prev = cell_key_of<BATCH>(pos_in[s2], cs, scene_in, s2);
    }
    if (valid && lane == 31 && i + 1 < n) {
        const u32 s2 = guard_st(st_err, perm ? perm[i + 1] : i + 1, n);
        next = cell_key_of<BATCH>(pos_in[s2], cs, scene_in, s2);
    }
    if (!valid) return;
    // rebuild_n_search.cu:19-34: a run of equal cells starts where the key
    // changes and ends (non-inclusive) at the next change.
    if (i == 0 || pk != prev) {
        const u32 slot = hash_insert<BATCH>(table, tmask, pk);
        if (slot == EMPTY_CELL) atomicOr(&st_err->error_flags, ERR_HASH_FULL);
        else cstart[slot] = i;
    }
    if (i == n - 1 || pk != next) {
        const u32 slot = hash_insert<BATCH>(table, tmask, pk);
        if (slot == EMPTY_CELL) atomicOr(&st_err->error_flags, ERR_HASH_FULL);
        else cend[slot] = i + 1;
    }
}


}  // namespace
}  // namespace wcsph
