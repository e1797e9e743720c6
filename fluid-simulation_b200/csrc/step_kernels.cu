// step_kernels.cu — see step_kernels.cuh for the decomposition.
#include "step_kernels.cuh"

#include <algorithm>
#include <climits>

namespace wcsph {

namespace {

constexpr u32 FULL = 0xffffffffu;
constexpr int CAND_CAP = 512;        // fluid candidates staged per warp (= 32 * max mask words)
constexpr int BCAND_CAP = 256;       // boundary candidates staged per warp and chunk

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

struct WarpSmem {
    u32 cand[CAND_CAP];
    u32 rstart[MAX_RANGE_CELLS + 3];
    u32 rpref[MAX_RANGE_CELLS + 3];
    u32 bcand[BCAND_CAP];
    u32 bstart[MAX_BOUNDARY_CELLS + 3];
    u32 bpref[MAX_BOUNDARY_CELLS + 3];
};

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
            const u32 slot = hash_find<BATCH>(hv.table, hv.tmask, pk);
            if (slot != EMPTY_CELL) {
                s = __ldg(hv.cstart + slot);
                cnt = __ldg(hv.cend + slot) - s;
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

// cand[m - c0] = particle index of candidate m, m in [c0, c0 + len).
__device__ __forceinline__ void expand(u32* cand, const u32* rstart, const u32* rpref, u32 ncell,
                                       u32 c0, u32 len) {
    __syncwarp();
    for (u32 ml = lane_id(); ml < len; ml += 32) {
        const u32 m = c0 + ml;
        u32 lo = 0, hi = ncell;
        while (hi - lo > 1) {
            const u32 mid = (lo + hi) >> 1;
            if (rpref[mid] <= m) lo = mid; else hi = mid;
        }
        cand[ml] = rstart[lo] + (m - rpref[lo]);
    }
    __syncwarp();
}

template <typename T>
__device__ __forceinline__ T group_sum(T v, u32 L);

template <>
__device__ __forceinline__ float group_sum<float>(float v, u32 L) {
    for (u32 o = L >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}
__device__ __forceinline__ float4 group_sum4(float4 v, u32 L) {
    for (u32 o = L >> 1; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(FULL, v.x, o);
        v.y += __shfl_xor_sync(FULL, v.y, o);
        v.z += __shfl_xor_sync(FULL, v.z, o);
    }
    return v;
}

__device__ __forceinline__ float4 f4(float x, float y, float z, float w = 0.f) { return make_float4(x, y, z, w); }

// Box collision (resolve_collisions, update_positions.cu:14-52).
__device__ __forceinline__ void resolve_collision(float4& x, float4& v, const DevBox& bb, const DevParams& P) {
    float4 pos = mat_mul(bb.model_inv, x);
    float4 vel = mat_mul(bb.model_inv, v);
    bool changed = false;
    const float buf = P.collision_buffer;
    if (pos.x - buf < bb.min.x) { pos.x = bb.min.x + P.radius; vel.x *= -P.elasticity; changed = true; }
    else if (pos.x + buf > bb.max.x) { pos.x = bb.max.x - P.radius; vel.x *= -P.elasticity; changed = true; }
    if (pos.y - buf < bb.min.y) { pos.y = bb.min.y + P.radius; vel.y *= -P.elasticity; changed = true; }
    else if (pos.y + buf > bb.max.y) { pos.y = bb.max.y - P.radius; vel.y *= -P.elasticity; changed = true; }
    if (pos.z - buf < bb.min.z) { pos.z = bb.min.z + P.radius; vel.z *= -P.elasticity; changed = true; }
    else if (pos.z + buf > bb.max.z) { pos.z = bb.max.z - P.radius; vel.z *= -P.elasticity; changed = true; }
    if (changed) {
        x = mat_mul(bb.model, pos);
        v = mat_mul(bb.model, vel);
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
    float4 x, v, n, ap, vl;
    float rho, prs, dpi;
    float4 abar, w;   // adjoint passes
    float rb;         // dL/drho of the home particle (adjoint density pass)
};

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

template <int KIND>
__device__ __forceinline__ constexpr bool uses_boundary() {
    return KIND == PASS_DENSITY || KIND == PASS_FORCE || KIND == PASS_ADJ_FORCE || KIND == PASS_ADJ_DENSITY;
}
template <int KIND>
__device__ __forceinline__ constexpr bool uses_masks() {
    return KIND == PASS_FORCE || KIND == PASS_SURFACE || KIND == PASS_ADJ_FORCE || KIND == PASS_ADJ_DENSITY;
}

// Per-lane accumulators of every pass (unused members are eliminated).
struct Acc {
    float w;        // density: sum W (fluid), boundary: sum m_b W
    float wb;
    float4 a;       // pressure accel (fluid part) / surface force
    float4 ab;      // boundary pressure accel (added after the fluid mass factor)
    float4 nrm;     // normal
    float4 vl;      // viscosity laplacian
    u32 cnt;
    // adjoint accumulators
    float4 xb, vb;  // dL/dx_i, dL/dv_i contributions
    float pt;       // sum_j -m (abar_i - abar_j) . F(r_ij)   (pressure coefficient sensitivity)
    float bt;       // sum_b -m_b abar_i . F(r_ib)             (boundary pressure coefficient)
    float vt;       // sum_j (v_ij . r_ij) G_ij (w_j . r_ij)   (viscosity rho_i sensitivity)
};

template <int KIND>
__device__ __forceinline__ void fluid_pair(Acc& acc, const HomeData& H, u32 j, float4 xj, float r2,
                                           const DevParams& P, const TravArgs& a) {
    const float q = sqrtf(r2) * P.inv_h;
    if constexpr (KIND == PASS_DENSITY) {
        acc.w += cubic_w(q, P);
    } else if constexpr (KIND == PASS_FORCE) {
        const float4 r = f4(H.x.x - xj.x, H.x.y - xj.y, H.x.z - xj.z);
        const float dj = __ldg(a.rho + j);
        const float pj = __ldg(a.prs + j);
        const float4 vj = __ldg(a.vel + j);
        const float sg = spiky_grad(q, P);
        const float cg = cubic_grad(q, P);
        const float dpj = pj / (dj * dj);
        const float c = (H.dpi + dpj) * sg;
        acc.a.x -= c * r.x; acc.a.y -= c * r.y; acc.a.z -= c * r.z;
        const float cn = cg / dj;
        acc.nrm.x += r.x * cn; acc.nrm.y += r.y * cn; acc.nrm.z += r.z * cn;
        const float vr = (H.v.x - vj.x) * r.x + (H.v.y - vj.y) * r.y + (H.v.z - vj.z) * r.z;
        const float s = vr * cg / (dj * (r2 + P.visc_eps));
        acc.vl.x += s * r.x; acc.vl.y += s * r.y; acc.vl.z += s * r.z;
    } else if constexpr (KIND == PASS_SURFACE) {
        if (r2 > 1e-6f) {
            const float dj = __ldg(a.rho + j);
            const float4 nj = __ldg(a.normal + j);
            const float4 r = f4(H.x.x - xj.x, H.x.y - xj.y, H.x.z - xj.z);
            const float len = sqrtf(r2);
            const float c = cohesion(q, P);
            const float inv = 1.f / (H.rho + dj);
            acc.a.x += (P.mass * (r.x / len) * c + H.n.x - nj.x) * inv;
            acc.a.y += (P.mass * (r.y / len) * c + H.n.y - nj.y) * inv;
            acc.a.z += (P.mass * (r.z / len) * c + H.n.z - nj.z) * inv;
        }
    } else if constexpr (KIND == PASS_ADJ_FORCE) {
        // pressure: a_i = -m sum_j A_ij F(r_ij), F(r) = g_s(|r|) r, A_ij = p_i/rho_i^2 + p_j/rho_j^2
        const float4 r = f4(H.x.x - xj.x, H.x.y - xj.y, H.x.z - xj.z);
        const float rl = sqrtf(r2);
        const float dj = __ldg(a.rho + j);
        const float pj = __ldg(a.prs + j);
        const float4 aj = __ldg(a.adj_abar + j);
        const float gs = spiky_grad(q, P);
        const float gsp = rl > 0.f ? spiky_grad_dr(q, rl, P) / rl : 0.f;
        const float A = H.dpi + pj / (dj * dj);
        const float dax = H.abar.x - aj.x, day = H.abar.y - aj.y, daz = H.abar.z - aj.z;
        const float rda = r.x * dax + r.y * day + r.z * daz;
        acc.pt += -P.mass * gs * rda;
        // x_i: -m A J_F(r) (abar_i - abar_j), J_F = g_s I + (g_s'/|r|) r r^T
        const float cA = -P.mass * A;
        acc.xb.x += cA * (gs * dax + gsp * rda * r.x);
        acc.xb.y += cA * (gs * day + gsp * rda * r.y);
        acc.xb.z += cA * (gs * daz + gsp * rda * r.z);
        // viscosity: vlap_i = sum_j (u.r) G(|r|) r / rho_j, u = v_i - v_j, G = g_c / (r^2 + eps)
        const float4 vj = __ldg(a.vel + j);
        const float4 wj = __ldg(a.adj_w + j);
        const float gc = cubic_grad(q, P);
        const float gcp = rl > 0.f ? cubic_grad_dr(q, rl, P) : 0.f;
        const float den = r2 + P.visc_eps;
        const float G = gc / den;
        const float Gp = rl > 0.f ? (gcp / den - 2.f * rl * gc / (den * den)) / rl : 0.f;  // G'/|r|
        const float ux = H.v.x - vj.x, uy = H.v.y - vj.y, uz = H.v.z - vj.z;
        const float ur = ux * r.x + uy * r.y + uz * r.z;
        const float wir = H.w.x * r.x + H.w.y * r.y + H.w.z * r.z;
        const float wjr = wj.x * r.x + wj.y * r.y + wj.z * r.z;
        const float inv_dj = 1.f / dj, inv_di = 1.f / H.rho;
        const float cv = G * (wir * inv_dj - wjr * inv_di);
        acc.vb.x += cv * r.x; acc.vb.y += cv * r.y; acc.vb.z += cv * r.z;
        acc.vt += ur * G * wjr;
        const float si = inv_dj, sj = inv_di;
        acc.xb.x += si * (ux * G * wir + ur * G * H.w.x + ur * wir * Gp * r.x) -
                    sj * (ux * G * wjr + ur * G * wj.x + ur * wjr * Gp * r.x);
        acc.xb.y += si * (uy * G * wir + ur * G * H.w.y + ur * wir * Gp * r.y) -
                    sj * (uy * G * wjr + ur * G * wj.y + ur * wjr * Gp * r.y);
        acc.xb.z += si * (uz * G * wir + ur * G * H.w.z + ur * wir * Gp * r.z) -
                    sj * (uz * G * wjr + ur * G * wj.z + ur * wjr * Gp * r.z);
    } else if constexpr (KIND == PASS_ADJ_DENSITY) {
        // rho_i = m (W(0) + sum_j W(|r_ij|)): dW/dx_i = g_c r_ij, shared by rho_i and rho_j
        const float rb = __ldg(a.adj_rhobar + j);
        const float c = P.mass * cubic_grad(q, P) * (H.rb + rb);
        const float4 r = f4(H.x.x - xj.x, H.x.y - xj.y, H.x.z - xj.z);
        acc.xb.x += c * r.x; acc.xb.y += c * r.y; acc.xb.z += c * r.z;
    }
}

template <int KIND>
__device__ __forceinline__ void boundary_pair(Acc& acc, const HomeData& H, u32 b, float4 xb, float r2,
                                              const DevParams& P, const TravArgs& a) {
    const float q = sqrtf(r2) * P.inv_h;
    const float mb = __ldg(a.bmass + b);
    if constexpr (KIND == PASS_DENSITY) {
        acc.wb += cubic_w(q, P) * mb;
    } else if constexpr (KIND == PASS_FORCE) {
        const float b_p_term = H.dpi + H.prs / P.rest_density2;
        const float c = mb * b_p_term * spiky_grad(q, P);
        acc.ab.x -= c * (H.x.x - xb.x);
        acc.ab.y -= c * (H.x.y - xb.y);
        acc.ab.z -= c * (H.x.z - xb.z);
    } else if constexpr (KIND == PASS_ADJ_FORCE) {
        // a_i -= m_b B_i F(r_ib), B_i = p_i/rho_i^2 + p_i/rho0^2
        const float4 r = f4(H.x.x - xb.x, H.x.y - xb.y, H.x.z - xb.z);
        const float rl = sqrtf(r2);
        const float gs = spiky_grad(q, P);
        const float gsp = rl > 0.f ? spiky_grad_dr(q, rl, P) / rl : 0.f;
        const float B = H.dpi + H.prs / P.rest_density2;
        const float ra = r.x * H.abar.x + r.y * H.abar.y + r.z * H.abar.z;
        acc.bt += -mb * gs * ra;
        const float cB = -mb * B;
        acc.xb.x += cB * (gs * H.abar.x + gsp * ra * r.x);
        acc.xb.y += cB * (gs * H.abar.y + gsp * ra * r.y);
        acc.xb.z += cB * (gs * H.abar.z + gsp * ra * r.z);
    } else if constexpr (KIND == PASS_ADJ_DENSITY) {
        const float c = mb * H.rb * cubic_grad(q, P);
        acc.xb.x += c * (H.x.x - xb.x);
        acc.xb.y += c * (H.x.y - xb.y);
        acc.xb.z += c * (H.x.z - xb.z);
    }
}

template <int KIND, int WPB, bool BATCH>
__global__ void __launch_bounds__(WPB * 32) cell_pass_kernel(const DevParams P, const TravArgs a) {
    __shared__ WarpSmem smem[WPB];
    __shared__ float s_dt, s_np_dt;
    __shared__ float s_red[WPB][3];
    __shared__ bool s_last;
    const u32 lane = lane_id();
    const u32 warp = threadIdx.x >> 5;
    WarpSmem& S = smem[warp];

    float dt = 0.f, np_dt = 0.f;
    if constexpr (KIND == PASS_SURFACE) {
        if (threadIdx.x == 0) {
            s_dt = cfl_time_step(a, P);
            s_np_dt = a.delta < a.np_max_dt ? a.delta : a.np_max_dt;
        }
        __syncthreads();
        dt = s_dt;
        np_dt = s_np_dt;
    }
    float red_max = 0.f, red_speed = 0.f, red_speed2 = 0.f;

    const u32 chunk = blockIdx.x * WPB + warp;
    const u32 base = chunk * 32u;
    const u32 n = a.n;
    const int R = a.range;
    const u32 D = static_cast<u32>(2 * R + 1);
    const u32 ncell = D * D * D;
    const u32 qc = ncell >> 1;
    const u32 cap = a.mask_words * 32u;

    if (base < n) {
        const u32 i0 = base + lane;
        const u64 my_pk = i0 < n ? a.ckey[i0] : 0ull;
        u64 prev_pk = __shfl_up_sync(FULL, my_pk, 1);
        if (lane == 0) prev_pk = i0 > 0 ? a.ckey[i0 - 1] : ~my_pk;
        u32 starts = __ballot_sync(FULL, i0 < n && (i0 == 0 || my_pk != prev_pk));
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
            // fluid neighbour cells in the reference's x, y, z nesting order
            const u32 M = gather_ranges<BATCH>(S.rstart, S.rpref, ncell, a.fluid, [&](u32 q) {
                const int dz = static_cast<int>(q % D) - R;
                const int dy = static_cast<int>((q / D) % D) - R;
                const int dx = static_cast<int>(q / (D * D)) - R;
                if constexpr (BATCH) return pack_cell_batch(scene, ux + dx, uy + dy, uz + dz);
                else return pack_cell(ux + dx, uy + dy, uz + dz);
            });
            const u32 home_start = S.rstart[qc];
            const u32 n_home = S.rpref[qc + 1] - S.rpref[qc];
            const bool masked = M <= cap;
            const u32 nwords = (M + 31) >> 5;

            // boundary neighbour cells: union of the home particles' 3x3x3
            // boundary-cell neighbourhoods (cell size h, R = 1,
            // for_boundary_neighbors common.cuh:153-178)
            u32 MB = 0, nbc = 0;
            if constexpr (uses_boundary<KIND>()) {
                if (a.nb > 0) {
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

            if (masked && M > 0) expand(S.cand, S.rstart, S.rpref, ncell, 0, M);

            for (u32 hb = 0; hb < n_home; hb += 32) {
                const u32 nh = min(32u, n_home - hb);
                const u32 lg = nh <= 1 ? 0u : 32u - __clz(nh - 1);  // ceil(log2(nh))
                const u32 L = 32u >> lg;
                const u32 g = lane >> (5u - lg);
                const u32 l = lane & (L - 1u);
                const bool hv = g < nh;
                const u32 i = home_start + hb + (hv ? g : 0u);

                HomeData H;
                H.x = a.pos[i];
                if constexpr (KIND == PASS_FORCE || KIND == PASS_SURFACE) {
                    H.v = a.vel[i];
                    H.rho = a.rho[i];
                    H.prs = a.prs[i];
                    H.dpi = H.prs / (H.rho * H.rho);
                }
                if constexpr (KIND == PASS_SURFACE) {
                    H.n = a.normal[i];
                    H.ap = a.ap[i];
                    H.vl = a.vlap[i];
                }
                if constexpr (KIND == PASS_ADJ_FORCE) {
                    H.v = a.vel[i];
                    H.rho = a.rho[i];
                    H.prs = a.prs[i];
                    H.dpi = H.prs / (H.rho * H.rho);
                    H.abar = a.adj_abar[i];
                    H.w = a.adj_w[i];
                }
                if constexpr (KIND == PASS_ADJ_DENSITY) H.rb = a.adj_rhobar[i];
                Acc acc{};

                if constexpr (KIND == PASS_DENSITY) {
                    // full candidate scan; writes the neighbour bitmasks
                    for (u32 c0 = 0; c0 < M; c0 += CAND_CAP) {
                        const u32 len = min(static_cast<u32>(CAND_CAP), M - c0);
                        if (!masked) expand(S.cand, S.rstart, S.rpref, ncell, c0, len);
                        const u32 iters = (len + L - 1) / L;
                        u32 word = 0;
                        for (u32 it = 0; it < iters; ++it) {
                            const u32 ml = it * L + l;
                            bool nb = false;
                            if (ml < len && hv) {
                                const u32 j = S.cand[ml];
                                const float4 xj = a.pos[j];
                                const float r2 = dist2(H.x, xj);
                                nb = (j != i) && (r2 <= P.h2);
                                if (nb) fluid_pair<KIND>(acc, H, j, xj, r2, P, a);
                            }
                            if (masked) {
                                const u32 bal = __ballot_sync(FULL, nb);
                                const u32 gbits = L == 32u ? bal : ((bal >> (g * L)) & ((1u << L) - 1u));
                                const u32 bitpos = (it * L) & 31u;
                                word |= gbits << bitpos;
                                if (bitpos + L == 32u || it + 1 == iters) {
                                    if (l == 0 && hv) a.mask[static_cast<size_t>(i) * a.mask_words + ((c0 + it * L) >> 5)] = word;
                                    word = 0;
                                }
                            }
                        }
                    }
                } else if constexpr (uses_masks<KIND>()) {
                    if (masked) {
                        if (hv) {
                            const u32* mrow = a.mask + static_cast<size_t>(i) * a.mask_words;
                            for (u32 w = l; w < nwords; w += L) {
                                u32 bits = mrow[w];
                                while (bits) {
                                    const u32 b = __ffs(bits) - 1;
                                    bits &= bits - 1;
                                    const u32 j = S.cand[w * 32 + b];
                                    const float4 xj = a.pos[j];
                                    fluid_pair<KIND>(acc, H, j, xj, dist2(H.x, xj), P, a);
                                }
                            }
                        }
                    } else {
                        for (u32 c0 = 0; c0 < M; c0 += CAND_CAP) {
                            const u32 len = min(static_cast<u32>(CAND_CAP), M - c0);
                            expand(S.cand, S.rstart, S.rpref, ncell, c0, len);
                            if (hv) {
                                for (u32 ml = l; ml < len; ml += L) {
                                    const u32 j = S.cand[ml];
                                    const float4 xj = a.pos[j];
                                    const float r2 = dist2(H.x, xj);
                                    if (j != i && r2 <= P.h2) fluid_pair<KIND>(acc, H, j, xj, r2, P, a);
                                }
                            }
                        }
                    }
                } else {  // PASS_COUNT / PASS_FILL: sequential in candidate order (reference order)
                    u32 wpos = 0;
                    if constexpr (KIND == PASS_FILL) wpos = hv ? a.offsets[i] : 0u;
                    for (u32 c0 = 0; c0 < M; c0 += CAND_CAP) {
                        const u32 len = min(static_cast<u32>(CAND_CAP), M - c0);
                        if (!masked) expand(S.cand, S.rstart, S.rpref, ncell, c0, len);
                        if (hv && l == 0) {
                            for (u32 ml = 0; ml < len; ++ml) {
                                const u32 j = S.cand[ml];
                                bool nb;
                                if (masked) {
                                    nb = (a.mask[static_cast<size_t>(i) * a.mask_words + (ml >> 5)] >> (ml & 31)) & 1u;
                                } else {
                                    nb = (j != i) && dist2(H.x, a.pos[j]) <= P.h2;
                                }
                                if (nb) {
                                    if constexpr (KIND == PASS_FILL) {
                                        if (wpos < a.nbr_capacity) a.nbr_out[wpos] = j;
                                        ++wpos;
                                    }
                                    ++acc.cnt;
                                }
                            }
                        }
                    }
                }

                // boundary candidates (density and pressure passes)
                if constexpr (uses_boundary<KIND>()) {
                    for (u32 c0 = 0; c0 < MB; c0 += BCAND_CAP) {
                        const u32 len = min(static_cast<u32>(BCAND_CAP), MB - c0);
                        expand(S.bcand, S.bstart, S.bpref, nbc, c0, len);
                        if (hv) {
                            for (u32 ml = l; ml < len; ml += L) {
                                const u32 b = S.bcand[ml];
                                const float4 xb = a.bpos[b];
                                const float r2 = dist2(H.x, xb);
                                if (r2 <= P.h2) boundary_pair<KIND>(acc, H, b, xb, r2, P, a);
                            }
                        }
                    }
                }

                // combine the L lanes of each group
                if constexpr (KIND == PASS_DENSITY) {
                    acc.w = group_sum<float>(acc.w, L);
                    acc.wb = group_sum<float>(acc.wb, L);
                } else if constexpr (KIND == PASS_FORCE) {
                    acc.a = group_sum4(acc.a, L);
                    acc.ab = group_sum4(acc.ab, L);
                    acc.nrm = group_sum4(acc.nrm, L);
                    acc.vl = group_sum4(acc.vl, L);
                } else if constexpr (KIND == PASS_SURFACE) {
                    acc.a = group_sum4(acc.a, L);
                } else if constexpr (KIND == PASS_ADJ_FORCE) {
                    acc.xb = group_sum4(acc.xb, L);
                    acc.vb = group_sum4(acc.vb, L);
                    acc.pt = group_sum<float>(acc.pt, L);
                    acc.bt = group_sum<float>(acc.bt, L);
                    acc.vt = group_sum<float>(acc.vt, L);
                } else if constexpr (KIND == PASS_ADJ_DENSITY) {
                    acc.xb = group_sum4(acc.xb, L);
                }

                if (hv && l == 0) {
                    if constexpr (KIND == PASS_DENSITY) {
                        // compute_density: (W(0) + sum W) * m, then + sum m_b W
                        const float rho = (P.w0 + acc.w) * P.mass + acc.wb;
                        a.rho[i] = rho;
                        a.prs[i] = tait_pressure(rho, P);
                    } else if constexpr (KIND == PASS_FORCE) {
                        // compute_pressure_accel_n_normal_with_boundary: m * sum_fluid, then
                        // the boundary term (compute_pressure_accel_n_normal.cu:346-364)
                        a.ap[i] = f4(P.mass * acc.a.x + acc.ab.x, P.mass * acc.a.y + acc.ab.y,
                                     P.mass * acc.a.z + acc.ab.z);
                        const float sn = P.h * P.mass;
                        a.normal[i] = f4(sn * acc.nrm.x, sn * acc.nrm.y, sn * acc.nrm.z);
                        a.vlap[i] = acc.vl;
                    } else if constexpr (KIND == PASS_SURFACE) {
                        // a_np = g + F_ext + nu*10*m*vlap - alpha*2*rho0*f
                        const float4 fe = external_force(H.x, P);
                        float4 gv = make_float4(P.gravity[0], P.gravity[1], P.gravity[2], P.visc_scale);
                        const DevBox* bb = a.box;
                        if constexpr (BATCH) {
                            gv = a.scenes[scene].gravity_visc;
                            bb = &a.scenes[scene].box;
                            a.scene_state[i] = scene;
                        }
                        float4 anp;
                        anp.x = gv.x + fe.x + gv.w * H.vl.x - P.st_scale * acc.a.x;
                        anp.y = gv.y + fe.y + gv.w * H.vl.y - P.st_scale * acc.a.y;
                        anp.z = gv.z + fe.z + gv.w * H.vl.z - P.st_scale * acc.a.z;
                        anp.w = 0.f;
                        a.anp[i] = anp;
                        // update_positions.cu:64-67
                        float4 v = H.v, x = H.x;
                        v.x += np_dt * anp.x + dt * H.ap.x;
                        v.y += np_dt * anp.y + dt * H.ap.y;
                        v.z += np_dt * anp.z + dt * H.ap.z;
                        x.x += dt * v.x;
                        x.y += dt * v.y;
                        x.z += dt * v.z;
                        x.w += dt * v.w;
                        resolve_collision(x, v, *bb, P);
                        a.pos_out[i] = x;
                        a.vel_out[i] = v;
                        const float s2 = dot3(v, v);
                        red_max = fmaxf(red_max, s2);
                        red_speed += sqrtf(s2);
                        red_speed2 += s2;
                    } else if constexpr (KIND == PASS_COUNT) {
                        a.counts[i] = acc.cnt;
                    } else if constexpr (KIND == PASS_ADJ_FORCE) {
                        const float inv_r2 = 1.f / (H.rho * H.rho);
                        const float pbar = acc.pt * inv_r2 + acc.bt * (inv_r2 + 1.f / P.rest_density2);
                        float rhobar = (acc.pt + acc.bt) * (-2.f * H.prs * inv_r2 / H.rho) - acc.vt * inv_r2;
                        // Tait EOS with the clamp of compute_rho_p.cu:236-238
                        const float ratio = H.rho / P.rest_density;
                        const float rc = fminf(fmaxf(ratio, 1.f), P.max_density_ratio);
                        if (ratio > 1.f && ratio < P.max_density_ratio)
                            rhobar += pbar * P.stiffness * P.exponent * powf(ratio, P.exponent - 1.f) / P.rest_density;
                        red_speed += pbar * (powf(rc, P.exponent) - 1.f);  // dL/dk partial
                        a.adj_rhobar[i] = rhobar;
                        float4 xb0 = a.adj_xbar[i], vb0 = a.adj_vbar[i];
                        a.adj_xbar[i] = f4(xb0.x + acc.xb.x, xb0.y + acc.xb.y, xb0.z + acc.xb.z);
                        a.adj_vbar[i] = f4(vb0.x + acc.vb.x, vb0.y + acc.vb.y, vb0.z + acc.vb.z);
                    } else if constexpr (KIND == PASS_ADJ_DENSITY) {
                        float4 xb0 = a.adj_xbar[i];
                        a.adj_xbar[i] = f4(xb0.x + acc.xb.x, xb0.y + acc.xb.y, xb0.z + acc.xb.z);
                    }
                }
            }
        }
    }

    if constexpr (KIND == PASS_ADJ_FORCE) {
        double v = static_cast<double>(red_speed);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
        if (lane == 0 && v != 0.0) atomicAdd(a.adj_accum, v);
    }
    if constexpr (KIND == PASS_SURFACE) {
        // block reduction -> per-block partials (deterministic final sum)
        for (int o = 16; o > 0; o >>= 1) {
            red_max = fmaxf(red_max, __shfl_xor_sync(FULL, red_max, o));
            red_speed += __shfl_xor_sync(FULL, red_speed, o);
            red_speed2 += __shfl_xor_sync(FULL, red_speed2, o);
        }
        if (lane == 0) { s_red[warp][0] = red_max; s_red[warp][1] = red_speed; s_red[warp][2] = red_speed2; }
        __syncthreads();
        if (threadIdx.x == 0) {
            float m = 0.f, s1 = 0.f, s2 = 0.f;
            for (int w = 0; w < WPB; ++w) { m = fmaxf(m, s_red[w][0]); s1 += s_red[w][1]; s2 += s_red[w][2]; }
            a.block_partials[2 * blockIdx.x] = s1;
            a.block_partials[2 * blockIdx.x + 1] = s2;
            atomicMax(&a.st->vmax2_bits[a.st->parity ^ 1u], __float_as_uint(m));
            __threadfence();
            const u32 prev = atomicAdd(&a.st->blocks_done, 1u);
            s_last = (prev == gridDim.x - 1);
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            double s1 = 0.0, s2 = 0.0;
            for (u32 b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
                s1 += static_cast<double>(__ldcg(a.block_partials + 2 * b));
                s2 += static_cast<double>(__ldcg(a.block_partials + 2 * b + 1));
            }
            for (int o = 16; o > 0; o >>= 1) {
                s1 += __shfl_xor_sync(FULL, s1, o);
                s2 += __shfl_xor_sync(FULL, s2, o);
            }
            __shared__ double s_d[WPB][2];
            if (lane == 0) { s_d[warp][0] = s1; s_d[warp][1] = s2; }
            __syncthreads();
            if (threadIdx.x == 0) {
                double t1 = 0.0, t2 = 0.0;
                for (int w = 0; w < WPB; ++w) { t1 += s_d[w][0]; t2 += s_d[w][1]; }
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

template <bool BATCH>
__device__ __forceinline__ u64 cell_key_of(float4 p, float cs, const u32* scene_in, u32 src) {
    const int3 c = cell_of(p, cs);
    if constexpr (BATCH) return pack_cell_batch(scene_in[src], offset_coord(c.x), offset_coord(c.y), offset_coord(c.z));
    else return pack_cell(c);
}

template <bool BATCH>
__global__ void reorder_cells_kernel(const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                                     const u32* __restrict__ v1, const u32* __restrict__ v2,
                                     const DevState* st, u32 n, float cs, float4* __restrict__ pos_out,
                                     float4* __restrict__ vel_out, u32* __restrict__ perm_out,
                                     u64* __restrict__ ckey_out, u64* table, u32* cstart, u32* cend,
                                     u32 tmask, DevState* st_err, const u32* __restrict__ scene_in) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 lane = threadIdx.x & 31u;
    const u32 sel = st->sort_sel[8];
    const u32* perm = sel == 0 ? nullptr : (sel == 1 ? v1 : v2);
    const bool valid = i < n;
    u64 pk = 0;
    if (valid) {
        const u32 src = perm ? perm[i] : i;
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
        const u32 s2 = perm ? perm[i - 1] : i - 1;
        prev = cell_key_of<BATCH>(pos_in[s2], cs, scene_in, s2);
    }
    if (valid && lane == 31 && i + 1 < n) {
        const u32 s2 = perm ? perm[i + 1] : i + 1;
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

u32 pass_grid(u32 n, int wpb) {
    const u32 chunks = (n + 31) / 32;
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

template <int KIND, bool BATCH>
static void launch_kind(const DevParams& P, const TravArgs& a, cudaStream_t stream, int wpb) {
    const u32 grid = pass_grid(a.n, wpb);
    if (grid == 0) return;
    switch (wpb) {
    case 2: cell_pass_kernel<KIND, 2, BATCH><<<grid, 64, 0, stream>>>(P, a); break;
    case 8: cell_pass_kernel<KIND, 8, BATCH><<<grid, 256, 0, stream>>>(P, a); break;
    default: cell_pass_kernel<KIND, 4, BATCH><<<grid, 128, 0, stream>>>(P, a); break;
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
