"""Batched ensemble vs the same scenes stepped one by one.

Inside a scene the batch reproduces the single-scene path exactly: the
scene-major sort key keeps each scene's Morton order, cells are looked up
per (scene, cell) in the same traversal order, and every per-scene constant
(box, gravity, viscosity) is the single scene's. So states must match
bit-exactly after several steps.
"""
import numpy as np
import pytest

import wcsph

pytestmark = pytest.mark.gpu


def scenes(k=5, seed=3):
    out = []
    for i in range(k):
        pre = wcsph.preset_ensemble(seed, i)
        out.append(pre)
    return out


def test_batch_matches_sequential_bit_exact():
    pres = scenes(5)
    p = pres[0].params  # shared physics; per-scene gravity and viscosity below
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box, gravity=tuple(s.params.gravity),
                                  viscosity=s.params.viscosity, fluid_vel=s.vel, boundary_pos=s.bpos) for s in pres]
    b = wcsph.BatchSimulator(p, specs)
    b.step_n(4, 1e-3)
    for k, s in enumerate(pres):
        sim = s.simulator()
        sim.step_n(4, 1e-3)
        pos, vel = sim.get_state()
        ms, ke = sim.compute_state_metrics()
        sim.close()
        bpos, bvel = b.get_state(k)
        assert np.array_equal(pos, bpos), f"scene {k}: positions differ"
        assert np.array_equal(vel, bvel), f"scene {k}: velocities differ"
    bms, bke = b.metrics()
    b.close()


def test_batch_metrics_per_scene():
    pres = scenes(3, seed=8)
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box, gravity=tuple(s.params.gravity),
                                  viscosity=s.params.viscosity, boundary_pos=s.bpos) for s in pres]
    b = wcsph.BatchSimulator(pres[0].params, specs)
    b.step_n(3, 1e-3)
    ms, ke = b.metrics()
    for k, s in enumerate(pres):
        _, vel = b.get_state(k)
        sp = np.linalg.norm(vel[:, :3].astype(np.float64), axis=1)
        assert abs(ms[k] - sp.mean()) <= 1e-4 * sp.mean()
        mass = 1000.0 * float(np.float32(np.float64(np.float32(0.02) ** 3) * 0.8))
        assert abs(ke[k] - 0.5 * mass * (sp ** 2).sum()) <= 1e-4 * 0.5 * mass * (sp ** 2).sum()
    b.close()


def test_batch_rejects_cfl_and_negative_coordinates():
    pres = scenes(2)
    p = pres[0].params
    p.cfl_factor = 0.4
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box) for s in pres]
    with pytest.raises(wcsph.WcsphError) as e:
        wcsph.BatchSimulator(p, specs)
    assert e.value.status == wcsph.ERR_NOT_SUPPORTED
    p.cfl_factor = 0.0
    moved = pres[0].pos.copy()
    moved[:, 0] -= 5.0
    specs = [wcsph.BatchSceneSpec(fluid_pos=moved, box=wcsph.box((-6, 0, 0), (1, 1, 1)))]
    with pytest.raises(wcsph.WcsphError) as e:
        wcsph.BatchSimulator(p, specs)
    assert e.value.status == wcsph.ERR_NOT_SUPPORTED
