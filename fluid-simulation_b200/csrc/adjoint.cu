// adjoint.cu — differentiable rollout: forward with checkpoints every K
// steps, backward by hand-written adjoint kernels.
//
// Forward (fixed dt, CFL off, surface tension 0): every step is the normal
// step (sort, hash, density, pressure, viscosity, integrate + collision).
// Positions, velocities and particle ids are checkpointed every K steps.
//
// Backward, per segment (last first): the segment is re-run from its
// checkpoint, each step with its own buffer set swapped in (sorted state,
// permutation, hash and cell ranges, neighbour bit matrix, density, pressure,
// accelerations), so every step's neighbour sets are recomputed from the
// checkpoint, not stored across the rollout. Then for each step in reverse,
// with that step's set swapped in again, the adjoint kernels run:
//   adj_integrate   reverse of box collision and symplectic Euler (per particle)
//   ADJ_FORCE pass  reverse of the symmetric pressure force (+boundary term),
//                   the viscosity Laplacian and the clamped Tait EOS
//   ADJ_DENSITY pass reverse of the density sum (+boundary term)
//   unsort          dL/dx, dL/dv back through the sort permutation
// Gradients: dL/dv0 per initial particle, dL/dnu, dL/dk.
// Loss: mean_i |x_T,i - target_{id(i)}|^2.
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "simulator.cuh"

namespace wcsph {

namespace {

__global__ void iota_kernel(u32* ids, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) ids[i] = i;
}

__global__ void ids_gather_kernel(const u32* __restrict__ ids_in, const u32* __restrict__ perm,
                                  u32* __restrict__ ids_out, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const u32 j = perm[i];
        if (j < n) ids_out[i] = ids_in[j];   // always true unless the step's sort failed (reported)
    }
}

__global__ void loss_kernel(const float4* __restrict__ pos, const u32* __restrict__ ids,
                            const float4* __restrict__ target, u32 n, double* sum, float4* __restrict__ xbar) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (i < n) {
        const float4 x = pos[i];
        const float4 t = target[ids[i]];
        const double dx = static_cast<double>(x.x) - t.x, dy = static_cast<double>(x.y) - t.y,
                     dz = static_cast<double>(x.z) - t.z;
        v = dx * dx + dy * dy + dz * dz;
        if (xbar) {
            const double c = 2.0 / static_cast<double>(n);
            xbar[i] = make_float4(static_cast<float>(c * dx), static_cast<float>(c * dy), static_cast<float>(c * dz),
                                  0.f);
        }
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31u) == 0 && v != 0.0) atomicAdd(sum, v);
}

// Reverse of update_positions + resolve_collisions (update_positions.cu:14-68)
// for one particle in sorted order. Recomputes the forward integrate with the
// same float operations so that the collision branches are the forward's.
__global__ void adj_integrate_kernel(const DevParams P, const float4* __restrict__ x_s, const float4* __restrict__ v_s,
                                     const float4* __restrict__ ap, const float4* __restrict__ vlap,
                                     const DevBox* __restrict__ box, float dt, float np_dt,
                                     const float4* __restrict__ xbar_out, const float4* __restrict__ vbar_out,
                                     float4* __restrict__ xbar_s, float4* __restrict__ vbar_s,
                                     float4* __restrict__ abar, float4* __restrict__ w, u32 n, double* nubar) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    double nb = 0.0;
    if (i < n) {
        const float4 x0 = x_s[i], v0 = v_s[i], a_p = ap[i], vl = vlap[i];
        float fe[3] = {0.f, 0.f, 0.f};
        if (P.force_field == 1) { fe[0] = P.force_param[0]; fe[1] = P.force_param[1]; fe[2] = P.force_param[2]; }
        float4 anp;
        anp.x = P.gravity[0] + fe[0] + P.visc_scale * vl.x;
        anp.y = P.gravity[1] + fe[1] + P.visc_scale * vl.y;
        anp.z = P.gravity[2] + fe[2] + P.visc_scale * vl.z;
        float4 v = v0, x = x0;
        v.x += np_dt * anp.x + dt * a_p.x;
        v.y += np_dt * anp.y + dt * a_p.y;
        v.z += np_dt * anp.z + dt * a_p.z;
        x.x += dt * v.x; x.y += dt * v.y; x.z += dt * v.z; x.w += dt * v.w;
        const DevBox& bb = *box;
        const float4 p = mat_mul(bb.model_inv, x);
        int snap[3] = {0, 0, 0};
        const float buf = P.collision_buffer;
        const float pc[3] = {p.x, p.y, p.z};
        const float mn[3] = {bb.min.x, bb.min.y, bb.min.z}, mx[3] = {bb.max.x, bb.max.y, bb.max.z};
        bool changed = false;
        for (int d = 0; d < 3; ++d) {
            if (pc[d] - buf < mn[d]) { snap[d] = 1; changed = true; }
            else if (pc[d] + buf > mx[d]) { snap[d] = 1; changed = true; }
        }
        float4 xb = xbar_out[i], vb = vbar_out[i];
        if (changed) {
            // x_out = M p, v_out = M u (3x3 linear part; the translation has no gradient)
            const float4* M = bb.model;
            const float4* Mi = bb.model_inv;
            float pb[3], ub[3];
            // pb = M^T xb: pb[c] = sum_r M[c].row * xb[row]
            pb[0] = M[0].x * xb.x + M[0].y * xb.y + M[0].z * xb.z;
            pb[1] = M[1].x * xb.x + M[1].y * xb.y + M[1].z * xb.z;
            pb[2] = M[2].x * xb.x + M[2].y * xb.y + M[2].z * xb.z;
            ub[0] = M[0].x * vb.x + M[0].y * vb.y + M[0].z * vb.z;
            ub[1] = M[1].x * vb.x + M[1].y * vb.y + M[1].z * vb.z;
            ub[2] = M[2].x * vb.x + M[2].y * vb.y + M[2].z * vb.z;
            for (int d = 0; d < 3; ++d)
                if (snap[d]) { pb[d] = 0.f; ub[d] *= -P.elasticity; }
            // p = Mi x', u = Mi v'  ->  x'bar = Mi^T pb
            xb = make_float4(Mi[0].x * pb[0] + Mi[0].y * pb[1] + Mi[0].z * pb[2],
                             Mi[1].x * pb[0] + Mi[1].y * pb[1] + Mi[1].z * pb[2],
                             Mi[2].x * pb[0] + Mi[2].y * pb[1] + Mi[2].z * pb[2], 0.f);
            vb = make_float4(Mi[0].x * ub[0] + Mi[0].y * ub[1] + Mi[0].z * ub[2],
                             Mi[1].x * ub[0] + Mi[1].y * ub[1] + Mi[1].z * ub[2],
                             Mi[2].x * ub[0] + Mi[2].y * ub[1] + Mi[2].z * ub[2], 0.f);
        }
        // x' = x + dt v'  ;  v' = v + np_dt a_np + dt a_p
        const float4 vt = make_float4(vb.x + dt * xb.x, vb.y + dt * xb.y, vb.z + dt * xb.z, 0.f);
        xbar_s[i] = make_float4(xb.x, xb.y, xb.z, 0.f);
        vbar_s[i] = vt;
        abar[i] = make_float4(dt * vt.x, dt * vt.y, dt * vt.z, 0.f);
        const float4 anb = make_float4(np_dt * vt.x, np_dt * vt.y, np_dt * vt.z, 0.f);
        w[i] = make_float4(P.visc_scale * anb.x, P.visc_scale * anb.y, P.visc_scale * anb.z, 0.f);
        // a_np = g + nu*10*m*vlap: dL/dnu = 10 m (abar_np . vlap)
        nb = 10.0 * static_cast<double>(P.mass) *
             (static_cast<double>(anb.x) * vl.x + static_cast<double>(anb.y) * vl.y + static_cast<double>(anb.z) * vl.z);
    }
    for (int o = 16; o > 0; o >>= 1) nb += __shfl_xor_sync(0xffffffffu, nb, o);
    if ((threadIdx.x & 31u) == 0 && nb != 0.0) atomicAdd(nubar, nb);
}

__global__ void unsort_kernel(const u32* __restrict__ perm, const float4* __restrict__ xs, const float4* __restrict__ vs,
                              float4* __restrict__ xo, float4* __restrict__ vo, u32 n) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const u32 j = perm[i];
        if (j < n) {   // always true unless the step's sort failed (reported)
            xo[j] = xs[i];
            vo[j] = vs[i];
        }
    }
}

inline u32 blocks(u32 n) { return (n + 255) / 256; }

}  // namespace

// The step buffers that the adjoint kernels read, for one step of a segment.
struct StepSet {
    DevBuf<float4> pos_b, vel_b, ap, vlap;
    DevBuf<u32> perm, cstart, cend, mask;
    DevBuf<u64> ckey, table;
    DevBuf<float> rho, prs;
};

struct Adjoint {
    int steps = 0, every = 0;
    float dt = 0.f;
    bool have_forward = false;
    DevBuf<float4> ck_pos, ck_vel;   // [n_ckpt * n]
    DevBuf<u32> ck_ids;
    std::vector<StepSet> seg;        // one buffer set per step of a segment
    DevBuf<u32> ids_a, ids_b;
    DevBuf<float4> target;
    DevBuf<float4> final_pos, final_vel;
    DevBuf<float4> xbar, vbar, xbar_s, vbar_s, abar, w;
    DevBuf<float> rhobar;
    DevBuf<double> accum;            // [0] loss, [1] dL/dnu, [2] dL/dk
};

void destroy_adjoint(void* adjoint) { delete static_cast<Adjoint*>(adjoint); }

static Adjoint& adj_of(void*& slot) {
    if (!slot) slot = new Adjoint();
    return *static_cast<Adjoint*>(slot);
}

float CUDASPHSimulator::rollout_forward(int steps, float dt, int every, const float* target_host) {
    if (params_.surface_tension != 0.f)
        throw Error(WCSPH_ERR_NOT_SUPPORTED, "the differentiable rollout needs surface_tension = 0");
    if (params_.external_force != WCSPH_FORCE_NONE && params_.external_force != WCSPH_FORCE_CONSTANT)
        throw Error(WCSPH_ERR_NOT_SUPPORTED, "the differentiable rollout supports no or constant external force");
    Adjoint& A = adj_of(adjoint_);
    const u32 n = n_;
    const int nck = steps / every + 1;
    A.steps = steps; A.every = every; A.dt = dt;
    A.ck_pos.alloc(static_cast<size_t>(nck) * n); A.ck_vel.alloc(static_cast<size_t>(nck) * n);
    A.ck_ids.alloc(static_cast<size_t>(nck) * n);
    if (static_cast<int>(A.seg.size()) != every) A.seg = std::vector<StepSet>(every);
    for (StepSet& b : A.seg) {
        if (b.pos_b.count != n) {
            b.pos_b.alloc(n); b.vel_b.alloc(n); b.ap.alloc(n); b.vlap.alloc(n);
            b.perm.alloc(n); b.ckey.alloc(n); b.rho.alloc(n); b.prs.alloc(n);
        }
        if (b.table.count != table_size_) { b.table.alloc(table_size_); b.cstart.alloc(table_size_); b.cend.alloc(table_size_); }
        if (b.mask.count != mask_.count) b.mask.alloc(mask_.count);
    }
    A.ids_a.alloc(n); A.ids_b.alloc(n);
    A.target.alloc(n); A.final_pos.alloc(n); A.final_vel.alloc(n);
    A.xbar.alloc(n); A.vbar.alloc(n); A.xbar_s.alloc(n); A.vbar_s.alloc(n); A.abar.alloc(n); A.w.alloc(n);
    A.rhobar.alloc(n);
    A.accum.alloc(3);
    WCSPH_CUDA(cudaMemcpyAsync(A.target.ptr, target_host, sizeof(float4) * n, cudaMemcpyHostToDevice, stream_));
    invalidate_graph();
    iota_kernel<<<blocks(n), 256, 0, stream_>>>(A.ids_a.ptr, n);
    auto ckpt = [&](int c) {
        WCSPH_CUDA(cudaMemcpyAsync(A.ck_pos.ptr + static_cast<size_t>(c) * n, pos_a_.ptr, sizeof(float4) * n,
                                   cudaMemcpyDeviceToDevice, stream_));
        WCSPH_CUDA(cudaMemcpyAsync(A.ck_vel.ptr + static_cast<size_t>(c) * n, vel_a_.ptr, sizeof(float4) * n,
                                   cudaMemcpyDeviceToDevice, stream_));
        WCSPH_CUDA(cudaMemcpyAsync(A.ck_ids.ptr + static_cast<size_t>(c) * n, A.ids_a.ptr, sizeof(u32) * n,
                                   cudaMemcpyDeviceToDevice, stream_));
    };
    ckpt(0);
    for (int s = 0; s < steps; ++s) {
        enqueue_fixed_step(dt);
        ids_gather_kernel<<<blocks(n), 256, 0, stream_>>>(A.ids_a.ptr, perm_.ptr, A.ids_b.ptr, n);
        std::swap(A.ids_a, A.ids_b);
        if ((s + 1) % every == 0) ckpt((s + 1) / every);
    }
    WCSPH_CUDA(cudaMemcpyAsync(A.final_pos.ptr, pos_a_.ptr, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
    WCSPH_CUDA(cudaMemcpyAsync(A.final_vel.ptr, vel_a_.ptr, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
    WCSPH_CUDA(cudaMemsetAsync(A.accum.ptr, 0, sizeof(double) * 3, stream_));
    loss_kernel<<<blocks(n), 256, 0, stream_>>>(pos_a_.ptr, A.ids_a.ptr, A.target.ptr, n, A.accum.ptr, nullptr);
    WCSPH_CUDA(cudaGetLastError());
    double loss = 0.0;
    WCSPH_CUDA(cudaMemcpyAsync(&loss, A.accum.ptr, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    synchronize();
    A.have_forward = true;
    stepped_since_state_ = true;
    return static_cast<float>(loss / static_cast<double>(n));
}

void CUDASPHSimulator::rollout_backward(float* grad_v0, float* grad_visc, float* grad_stiff) {
    if (!adjoint_ || !static_cast<Adjoint*>(adjoint_)->have_forward)
        throw Error(WCSPH_ERR_STATE, "rollout_backward needs a rollout_forward first");
    Adjoint& A = *static_cast<Adjoint*>(adjoint_);
    const u32 n = n_;
    const float dt = A.dt;
    // exchanges the context's step buffers with a segment step's set (pointer swaps)
    auto swap_step = [this](StepSet& b) {
        std::swap(pos_b_, b.pos_b); std::swap(vel_b_, b.vel_b); std::swap(ap_, b.ap); std::swap(vlap_, b.vlap);
        std::swap(perm_, b.perm); std::swap(cstart_, b.cstart); std::swap(cend_, b.cend); std::swap(mask_, b.mask);
        std::swap(ckey_, b.ckey); std::swap(table_, b.table); std::swap(rho_, b.rho); std::swap(prs_, b.prs);
    };
    const float np_dt = dt < params_.non_pressure_max_time_step ? dt : params_.non_pressure_max_time_step;
    // dL/dx_T in the final state order, dL/dv_T = 0
    WCSPH_CUDA(cudaMemsetAsync(A.accum.ptr, 0, sizeof(double) * 3, stream_));
    loss_kernel<<<blocks(n), 256, 0, stream_>>>(A.final_pos.ptr, A.ids_a.ptr, A.target.ptr, n, A.accum.ptr,
                                                A.xbar.ptr);
    WCSPH_CUDA(cudaMemsetAsync(A.vbar.ptr, 0, sizeof(float4) * n, stream_));
    const int nseg = (A.steps + A.every - 1) / A.every;
    for (int seg = nseg - 1; seg >= 0; --seg) {
        const int s0 = seg * A.every;
        const int s1 = std::min(s0 + A.every, A.steps);
        WCSPH_CUDA(cudaMemcpyAsync(pos_a_.ptr, A.ck_pos.ptr + static_cast<size_t>(seg) * n, sizeof(float4) * n,
                                   cudaMemcpyDeviceToDevice, stream_));
        WCSPH_CUDA(cudaMemcpyAsync(vel_a_.ptr, A.ck_vel.ptr + static_cast<size_t>(seg) * n, sizeof(float4) * n,
                                   cudaMemcpyDeviceToDevice, stream_));
        for (int s = s0; s < s1; ++s) {  // re-run the segment, each step into its own buffer set
            swap_step(A.seg[s - s0]);
            enqueue_fixed_step(dt);
            swap_step(A.seg[s - s0]);
        }
        for (int s = s1 - 1; s >= s0; --s) {
            swap_step(A.seg[s - s0]);   // step s's sorted input, search and forces
            TravArgs a = fixed_args(dt);
            adj_integrate_kernel<<<blocks(n), 256, 0, stream_>>>(dp_, pos_b_.ptr, vel_b_.ptr, ap_.ptr, vlap_.ptr,
                                                                 box_dev_.ptr, dt, np_dt, A.xbar.ptr, A.vbar.ptr,
                                                                 A.xbar_s.ptr, A.vbar_s.ptr, A.abar.ptr, A.w.ptr, n,
                                                                 A.accum.ptr + 1);
            a.adj_abar = A.abar.ptr;
            a.adj_w = A.w.ptr;
            a.adj_xbar = A.xbar_s.ptr;
            a.adj_vbar = A.vbar_s.ptr;
            a.adj_rhobar = A.rhobar.ptr;
            a.adj_accum = A.accum.ptr + 2;
            launch_pass(PASS_ADJ_FORCE, dp_, a, stream_, 4);
            launch_pass(PASS_ADJ_DENSITY, dp_, a, stream_, 4);
            unsort_kernel<<<blocks(n), 256, 0, stream_>>>(perm_.ptr, A.xbar_s.ptr, A.vbar_s.ptr, A.xbar.ptr,
                                                          A.vbar.ptr, n);
            WCSPH_CUDA(cudaGetLastError());
            swap_step(A.seg[s - s0]);
        }
    }
    double acc[3];
    WCSPH_CUDA(cudaMemcpyAsync(acc, A.accum.ptr, sizeof(double) * 3, cudaMemcpyDeviceToHost, stream_));
    if (grad_v0)
        WCSPH_CUDA(cudaMemcpyAsync(grad_v0, A.vbar.ptr, sizeof(float4) * n, cudaMemcpyDeviceToHost, stream_));
    // the context returns to the state after the rollout
    WCSPH_CUDA(cudaMemcpyAsync(pos_a_.ptr, A.final_pos.ptr, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
    WCSPH_CUDA(cudaMemcpyAsync(vel_a_.ptr, A.final_vel.ptr, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream_));
    synchronize();
    if (grad_visc) *grad_visc = static_cast<float>(acc[1]);
    if (grad_stiff) *grad_stiff = static_cast<float>(acc[2]);
}

}  // namespace wcsph
