"""Hand-written CUDA adjoint (wcsph_rollout_forward/backward) against the
FP64 reverse-mode reference and FP64 central finite differences, on a
2048-particle copy of the differentiable-rollout workload (16x16x8 block,
r = 0.01, walls, 200 fixed 1e-3 steps, checkpoints every 20 steps,
target = initial lattice + (0.2, 0, 0.1)).

Tolerances (the 1e-3 relative of the differentiable-rollout target):
|g_cuda - g_ref| <= GRAD_TOL * |g_ref| for dL/dnu and dL/dk, and
||g_cuda - g_ref|| <= VEC_TOL * ||g_ref|| for dL/dv0, against FP64 reverse
mode and against FP64 central differences. The differences use a step that
crosses no neighbour-set change (FD_STEP, relative for nu and k, absolute in
m/s for v0): a pair entering or leaving the support radius inside the
difference makes the loss jump, which a derivative does not see. The 1e-4
step of the workload's specification crosses such a change for nu; its value
is printed beside the converged one.
"""
import numpy as np
import pytest

import oracle
import wcsph
from adjoint_ref import Scene, fd_gradient, reference_gradients

pytestmark = pytest.mark.gpu
GRAD_TOL = 1e-3
VEC_TOL = 1e-3
FD_STEP = 1e-6


def rollout_scene(dims=(16, 16, 8)):
    r = 0.01
    rd = float(np.float32(r))
    p = wcsph.default_params(particle_radius=r, stiffness=float(np.float32(1000.0 * (4 * rd) ** 6)), viscosity=0.01,
                             surface_tension=0.0, max_time_step=1e-3, cfl_factor=0.0)
    pos = wcsph.make_lattice(tuple(r + (d - 1) * r for d in dims), dims, r, 0.1 * r, 0)
    tank = (1.0, 0.6, 0.6)
    bx = wcsph.box((0, 0, 0), tank)
    walls = wcsph.sample_box_walls((0, 0, 0), tank, 2 * r)
    target = pos.copy()
    target[:, 0] += 0.2
    target[:, 2] += 0.1
    return p, bx, pos, walls, target


def cuda_gradients(p, bx, pos, walls, target, steps, dt, every):
    sim = wcsph.CUDASPHSimulator(p, pos, bx, boundary_pos=walls)
    loss = sim.rollout_forward(steps, dt, every, target)
    gv, gnu, gk = sim.rollout_backward()
    bpos = sim.field("boundary_position")
    bmass = sim.field("boundary_mass")
    sim.close()
    return loss, gv, gnu, gk, bpos, bmass


@pytest.mark.parametrize("steps", [20, 200])
def test_adjoint_matches_fp64_reverse_mode(steps):
    p, bx, pos, walls, target = rollout_scene()
    dt = 1e-3
    loss, gv, gnu, gk, bpos, bmass = cuda_gradients(p, bx, pos, walls, target, steps, dt, 20)
    sc = Scene(p, bx, pos, np.zeros_like(pos), bpos, bmass.astype(np.float64))
    rloss, rgv, rgnu, rgk = reference_gradients(sc, float(p.viscosity), float(p.stiffness), steps, dt, target)
    print(f"steps={steps} loss {loss:.6g} ref {rloss:.6g}; dL/dnu {gnu:.6g} ref {rgnu:.6g}; "
          f"dL/dk {gk:.6g} ref {rgk:.6g}; |dv0| rel err "
          f"{np.linalg.norm(gv[:, :3] - rgv) / np.linalg.norm(rgv):.3g}")
    assert abs(loss - rloss) <= 1e-4 * rloss
    assert abs(gnu - rgnu) <= GRAD_TOL * abs(rgnu)
    assert abs(gk - rgk) <= GRAD_TOL * abs(rgk)
    assert np.linalg.norm(gv[:, :3] - rgv) <= VEC_TOL * np.linalg.norm(rgv)


def test_adjoint_matches_finite_differences():
    p, bx, pos, walls, target = rollout_scene()
    steps, dt = 200, 1e-3
    loss, gv, gnu, gk, bpos, bmass = cuda_gradients(p, bx, pos, walls, target, steps, dt, 20)
    sc = Scene(p, bx, pos, np.zeros_like(pos), bpos, bmass.astype(np.float64))
    nu, k = float(p.viscosity), float(p.stiffness)
    fnu = fd_gradient(sc, nu, k, steps, dt, target, "nu", step=FD_STEP)
    fk = fd_gradient(sc, nu, k, steps, dt, target, "k", step=FD_STEP)
    fnu_spec = fd_gradient(sc, nu, k, steps, dt, target, "nu", step=1e-4)
    print(f"dL/dnu {gnu:.7g} fd({FD_STEP:g}) {fnu:.7g} (fd(1e-4) {fnu_spec:.7g}, crosses a neighbour-set change); "
          f"dL/dk {gk:.7g} fd {fk:.7g}")
    assert abs(gnu - fnu) <= GRAD_TOL * abs(fnu)
    assert abs(gk - fk) <= GRAD_TOL * abs(fk)
    # three components of dL/dv0 (particles at the corner, inside and at the far end of the block)
    got, want = [], []
    for idx in ((5, 0), (1000, 1), (2000, 2)):
        want.append(fd_gradient(sc, nu, k, steps, dt, target, "v0", index=idx, step=FD_STEP))
        got.append(float(gv[idx]))
    got, want = np.array(got), np.array(want)
    print("dL/dv0 components", got, "fd", want)
    assert np.linalg.norm(got - want) <= VEC_TOL * np.linalg.norm(want)


def test_rollout_restores_final_state_and_is_repeatable():
    p, bx, pos, walls, target = rollout_scene(dims=(8, 8, 8))
    sim = wcsph.CUDASPHSimulator(p, pos, bx, boundary_pos=walls)
    l1 = sim.rollout_forward(40, 1e-3, 10, target)
    after, _ = sim.get_state()
    g1 = sim.rollout_backward()
    after2, _ = sim.get_state()
    assert np.array_equal(after, after2)
    sim.set_state(pos)
    l2 = sim.rollout_forward(40, 1e-3, 10, target)
    g2 = sim.rollout_backward()
    sim.close()
    assert l1 == l2
    assert np.array_equal(g1[0], g2[0]) or np.allclose(g1[0], g2[0], rtol=1e-5, atol=1e-9)


def test_rollout_rejects_surface_tension():
    p, bx, pos, walls, target = rollout_scene(dims=(4, 4, 4))
    p.surface_tension = 0.13
    sim = wcsph.CUDASPHSimulator(p, pos, bx, boundary_pos=walls)
    with pytest.raises(wcsph.WcsphError) as e:
        sim.rollout_forward(5, 1e-3, 5, target)
    assert e.value.status == wcsph.ERR_NOT_SUPPORTED
    with pytest.raises(wcsph.WcsphError):
        sim.rollout_backward()
    sim.close()
