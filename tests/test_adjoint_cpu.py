"""The FP64 reverse-mode reference (adjoint_ref.py) against FP64 central finite
differences, on CPU (small scene, short rollout). Pins the math the CUDA
adjoint is compared with on the GPU (test_gpu_adjoint.py)."""
import numpy as np
import pytest

import oracle
import wcsph
from adjoint_ref import Scene, fd_gradient, reference_gradients


def small_scene(dims=(6, 6, 6), tank=(0.3, 0.3, 0.3), steps=30):
    r = 0.01
    rd = float(np.float32(r))
    p = wcsph.default_params(particle_radius=r, stiffness=float(np.float32(1000.0 * (4 * rd) ** 6)), viscosity=0.01,
                             surface_tension=0.0, max_time_step=1e-3, cfl_factor=0.0)
    pos = wcsph.make_lattice(tuple(r + (d - 1) * r for d in dims), dims, r, 0.1 * r, 21)
    vel = wcsph.make_velocities(pos.shape[0], 0.2, seed=4)
    bx = wcsph.box((0, 0, 0), tank)
    walls = wcsph.sample_box_walls((0, 0, 0), tank, 2 * r)
    bs, bm = oracle.boundary_init(p, walls)
    target = pos.copy()
    target[:, 0] += 0.2
    target[:, 2] += 0.1
    return p, bx, pos, vel, bs, bm, target, steps


def test_reverse_mode_matches_finite_differences():
    p, bx, pos, vel, bs, bm, target, steps = small_scene()
    sc = Scene(p, bx, pos, vel, bs, bm)
    nu, k, dt = float(p.viscosity), float(p.stiffness), 1e-3
    loss, gv, gnu, gk = reference_gradients(sc, nu, k, steps, dt, target)
    assert np.isfinite(loss) and loss > 0
    for which, got in (("nu", gnu), ("k", gk)):
        fd = fd_gradient(sc, nu, k, steps, dt, target, which)
        assert abs(got - fd) <= 1e-3 * abs(fd) + 1e-12, (which, got, fd)
    for idx in ((3, 0), (100, 1), (200, 2)):
        fd = fd_gradient(sc, nu, k, steps, dt, target, "v0", index=idx)
        assert abs(gv[idx] - fd) <= 1e-3 * max(abs(fd), 1e-9), (idx, gv[idx], fd)
