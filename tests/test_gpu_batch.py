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


@pytest.mark.parametrize("persistent", [True, False])
def test_batch_matches_sequential_bit_exact(persistent):
    """Both ways of running the ensemble (one persistent cooperative launch for
    all steps, or one launch per stage and step) reproduce each scene's own
    single-scene steps bit for bit."""
    pres = scenes(5)
    p = pres[0].params  # shared physics; per-scene gravity and viscosity below
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box, gravity=tuple(s.params.gravity),
                                  viscosity=s.params.viscosity, fluid_vel=s.vel, boundary_pos=s.bpos) for s in pres]
    b = wcsph.BatchSimulator(p, specs)
    b.set_persistent(persistent)
    b.step_n(4, 1e-3)
    b.step_n(2, 1e-3)   # a second launch continues from the first
    for k, s in enumerate(pres):
        sim = s.simulator()
        sim.step_n(6, 1e-3)
        pos, vel = sim.get_state()
        sim.close()
        bpos, bvel = b.get_state(k)
        assert np.array_equal(pos, bpos), f"scene {k}: positions differ"
        assert np.array_equal(vel, bvel), f"scene {k}: velocities differ"
    b.close()


def test_batch_metrics_per_scene():
    """Per-scene mean speed and kinetic energy, reduced in a fixed order
    (repeatable bit for bit) and equal to the FP64 sums of the state."""
    pres = scenes(3, seed=8)
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box, gravity=tuple(s.params.gravity),
                                  viscosity=s.params.viscosity, boundary_pos=s.bpos) for s in pres]
    b = wcsph.BatchSimulator(pres[0].params, specs)
    b.step_n(3, 1e-3)
    ms, ke = b.metrics()
    ms2, ke2 = b.metrics()
    assert np.array_equal(ms, ms2) and np.array_equal(ke, ke2)
    mass = 1000.0 * float(np.float32(np.float64(np.float32(0.02) ** 3) * 0.8))
    for k, s in enumerate(pres):
        _, vel = b.get_state(k)
        sp = np.sqrt((vel[:, :3].astype(np.float32) ** 2).sum(1, dtype=np.float32)).astype(np.float64)
        assert abs(ms[k] - sp.mean()) <= 1e-6 * sp.mean()
        want = 0.5 * mass * (sp ** 2).sum()
        assert abs(ke[k] - want) <= 1e-5 * want
    b.close()


def test_batch_rejects_cfl():
    pres = scenes(2)
    p = pres[0].params
    p.cfl_factor = 0.4
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box) for s in pres]
    with pytest.raises(wcsph.WcsphError) as e:
        wcsph.BatchSimulator(p, specs)
    assert e.value.status == wcsph.ERR_NOT_SUPPORTED


def test_batch_scene_at_negative_coordinates_matches_its_own_run():
    """A scene moved to negative cell coordinates (the batch key offsets cells
    by 2^15 instead of truncating the reference's key) still reproduces its
    single-scene run bit for bit, beside a scene in the positive octant."""
    pres = scenes(2, seed=11)
    shift = np.array([-3.0, -1.0, -2.0, 0.0], np.float32)
    moved_pos = pres[0].pos + shift
    moved_bpos = pres[0].bpos + shift
    mn = np.array(list(pres[0].box.min), np.float32) + shift[:3]
    mx = np.array(list(pres[0].box.max), np.float32) + shift[:3]
    moved_box = wcsph.box(tuple(mn), tuple(mx))
    p = pres[0].params
    specs = [wcsph.BatchSceneSpec(fluid_pos=moved_pos, box=moved_box, gravity=tuple(p.gravity),
                                  viscosity=p.viscosity, boundary_pos=moved_bpos),
             wcsph.BatchSceneSpec(fluid_pos=pres[1].pos, box=pres[1].box, gravity=tuple(pres[1].params.gravity),
                                  viscosity=pres[1].params.viscosity, boundary_pos=pres[1].bpos)]
    b = wcsph.BatchSimulator(p, specs)
    b.step_n(5, 1e-3)
    sim = wcsph.CUDASPHSimulator(p, moved_pos, moved_box, boundary_pos=moved_bpos)
    sim.step_n(5, 1e-3)
    pos, vel = sim.get_state()
    sim.close()
    bpos, bvel = b.get_state(0)
    b.close()
    assert np.array_equal(pos, bpos) and np.array_equal(vel, bvel)
