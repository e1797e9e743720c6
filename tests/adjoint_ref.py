"""FP64 host reverse-mode reference of the differentiable rollout (PyTorch
autograd, CPU). TEST INFRASTRUCTURE ONLY.

Restates one fixed-dt WCSPH step without surface tension — density
(compute_rho_p.cu:87-100,301-316), clamped Tait EOS (:236-238), symmetric
pressure force with the boundary term (compute_pressure_accel_n_normal.cu:
99-123,346-364), viscosity (compute_non_pressure_accel.cu:138-140),
symplectic Euler + box collision (update_positions.cu:14-68) — in float64
with particles kept in their initial order (the sort only permutes, so it
does not change the math). Neighbour pairs are rebuilt every step from the
positions (no gradient through the selection).
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.spatial import cKDTree
from torch.utils.checkpoint import checkpoint


class Scene:
    def __init__(self, params, box, pos, vel, bpos=None, bmass=None):
        f32 = np.float32
        self.r = float(f32(params.particle_radius))
        self.spacing = float(f32(2 * f32(self.r)))
        self.h = float(f32(2 * f32(self.spacing)))
        self.mass = float(params.rest_density) * self.spacing ** 3 * 0.8
        self.rho0 = float(params.rest_density)
        self.gamma = float(params.exponent)
        self.max_ratio = float(params.max_density_ratio)
        self.g = torch.tensor([float(x) for x in params.gravity], dtype=torch.float64)
        self.buf = float(f32(f32(self.r) * f32(params.collision_buffer_mult)))
        self.elasticity = float(params.elasticity)
        self.np_max = float(params.non_pressure_max_time_step)
        self.box_min = np.array(list(box.min), np.float64)
        self.box_max = np.array(list(box.max), np.float64)
        h = self.h
        self.cubic_f = 8.0 / (np.pi * h ** 3)
        self.cubic_grad_f = 48.0 / (np.pi * h ** 3)
        self.spiky_grad_f = -45.0 / (np.pi * h ** 9)
        self.eps = 0.01 * h * h
        self.x0 = torch.tensor(pos[:, :3], dtype=torch.float64)
        self.v0 = torch.tensor(vel[:, :3], dtype=torch.float64)
        self.bpos = None if bpos is None else torch.tensor(bpos[:, :3], dtype=torch.float64)
        self.bmass = None if bmass is None else torch.tensor(bmass, dtype=torch.float64)
        self._btree = None

    # ---- kernels as functions of q and |r| -------------------------------
    def W(self, q):
        a = self.cubic_f * (6 * q ** 3 - 6 * q ** 2 + 1)
        b = self.cubic_f * 2 * (1 - q) ** 3
        return torch.where(q <= 0.5, a, torch.where(q <= 1.0, b, torch.zeros_like(q)))

    def gc(self, q, rl):
        safe = torch.where(rl > 0, rl, torch.ones_like(rl))
        a = self.cubic_grad_f * q * (3 * q - 2) / (self.h * safe)
        b = -self.cubic_grad_f * (1 - q) ** 2 / (self.h * safe)
        v = torch.where(q <= 0.5, a, b)
        return torch.where((q < 1e-9) | (q > 1.0), torch.zeros_like(q), v)

    def gs(self, q, rl):
        safe = torch.where(rl > 0, rl, torch.ones_like(rl))
        v = self.spiky_grad_f * (1 - q) ** 2 / (self.h * safe)
        return torch.where((q < 1e-9) | (q > 1.0), torch.zeros_like(q), v)

    # ---- neighbour pairs (no gradient) --------------------------------------
    def pairs(self, x):
        # pairs at |r| ~ h contribute ~0 (every kernel vanishes there), so the
        # selection is made in float64 without the CUDA path's exact rounding
        xn = x.detach().numpy()
        h2 = float(np.float32(np.float32(self.h) * np.float32(self.h)))
        reach = np.sqrt(h2) * (1.0 + 1e-9)
        tree = cKDTree(xn)
        pr = tree.query_pairs(reach, output_type="ndarray")
        if len(pr):
            d = xn[pr[:, 0]] - xn[pr[:, 1]]
            pr = pr[(d * d).sum(1) <= h2]
        i = np.concatenate([pr[:, 0], pr[:, 1]]).astype(np.int64)
        j = np.concatenate([pr[:, 1], pr[:, 0]]).astype(np.int64)
        order = np.lexsort((j, i))
        i, j = i[order], j[order]
        bi = bj = None
        if self.bpos is not None:
            if self._btree is None:
                self._btree = cKDTree(self.bpos.numpy())
            hits = tree.query_ball_tree(self._btree, reach)
            bi = np.repeat(np.arange(len(hits)), [len(h) for h in hits]).astype(np.int64)
            bj = np.fromiter((b for h in hits for b in sorted(h)), np.int64, count=len(bi))
            if len(bi):
                db = xn[bi] - self.bpos.numpy()[bj]
                keep = (db * db).sum(1) <= h2
                bi, bj = bi[keep], bj[keep]
        return i, j, bi, bj

    def step(self, x, v, nu, k, dt):
        n = x.shape[0]
        i, j, bi, bj = self.pairs(x)
        i = torch.from_numpy(i)
        j = torch.from_numpy(j)
        r = x[i] - x[j]
        rl = torch.sqrt((r * r).sum(1))
        q = rl / self.h
        rho = self.mass * (self.cubic_f + torch.zeros(n, dtype=torch.float64).index_add(0, i, self.W(q)))
        if bi is not None and len(bi):
            bi_t, bj_t = torch.from_numpy(bi), torch.from_numpy(bj)
            rb = x[bi_t] - self.bpos[bj_t]
            rbl = torch.sqrt((rb * rb).sum(1))
            qb = rbl / self.h
            rho = rho + torch.zeros(n, dtype=torch.float64).index_add(0, bi_t, self.W(qb) * self.bmass[bj_t])
        ratio = torch.clamp(rho / self.rho0, 1.0, self.max_ratio)
        p = k * (ratio ** self.gamma - 1.0)
        dp = p / rho ** 2
        A = dp[i] + dp[j]
        ap = -self.mass * torch.zeros_like(x).index_add(0, i, (A * self.gs(q, rl))[:, None] * r)
        if bi is not None and len(bi):
            B = dp + p / self.rho0 ** 2
            ap = ap - torch.zeros_like(x).index_add(
                0, bi_t, (self.bmass[bj_t] * B[bi_t] * self.gs(qb, rbl))[:, None] * rb)
        u = v[i] - v[j]
        s = (u * r).sum(1) * self.gc(q, rl) / (rho[j] * (rl * rl + self.eps))
        vlap = torch.zeros_like(x).index_add(0, i, s[:, None] * r)
        anp = self.g[None, :] + nu * 10.0 * self.mass * vlap
        np_dt = min(dt, self.np_max)
        v1 = v + np_dt * anp + dt * ap
        x1 = x + dt * v1
        # box collision (identity model matrix)
        lo = torch.from_numpy(x1.detach().numpy() - self.buf < self.box_min[None, :])
        hi = torch.from_numpy(x1.detach().numpy() + self.buf > self.box_max[None, :]) & ~lo
        mn = torch.from_numpy(self.box_min + self.r).expand_as(x1)
        mx = torch.from_numpy(self.box_max - self.r).expand_as(x1)
        x1 = torch.where(lo, mn, torch.where(hi, mx, x1))
        v1 = torch.where(lo | hi, -self.elasticity * v1, v1)
        return x1, v1

    def rollout(self, v0, nu, k, steps, dt, target, grad=True):
        x, v = self.x0.clone(), v0
        for _ in range(steps):
            if grad:
                x, v = checkpoint(self.step, x, v, nu, k, dt, use_reentrant=False)
            else:
                x, v = self.step(x, v, nu, k, dt)
        return ((x - target) ** 2).sum(1).mean()


def reference_gradients(scene: Scene, nu: float, k: float, steps: int, dt: float, target: np.ndarray):
    """Loss and dL/dv0, dL/dnu, dL/dk by FP64 reverse mode."""
    v0 = scene.v0.clone().requires_grad_(True)
    nu_t = torch.tensor(nu, dtype=torch.float64, requires_grad=True)
    k_t = torch.tensor(k, dtype=torch.float64, requires_grad=True)
    tgt = torch.tensor(target[:, :3], dtype=torch.float64)
    loss = scene.rollout(v0, nu_t, k_t, steps, dt, tgt)
    loss.backward()
    return float(loss.detach()), v0.grad.numpy(), float(nu_t.grad), float(k_t.grad)


def fd_gradient(scene: Scene, nu: float, k: float, steps: int, dt: float, target: np.ndarray, which: str,
                index=None, step=1e-4) -> float:
    """FP64 central difference of the loss (relative step for nu, k; absolute for v0)."""
    tgt = torch.tensor(target[:, :3], dtype=torch.float64)

    def L(dnu=0.0, dk=0.0, dv=None):
        v0 = scene.v0.clone()
        if dv is not None:
            v0[index] += dv
        with torch.no_grad():
            return float(scene.rollout(v0, nu + dnu, k + dk, steps, dt, tgt, grad=False))

    if which == "nu":
        e = step * nu
        return (L(dnu=e) - L(dnu=-e)) / (2 * e)
    if which == "k":
        e = step * k
        return (L(dk=e) - L(dk=-e)) / (2 * e)
    e = step
    return (L(dv=e) - L(dv=-e)) / (2 * e)
