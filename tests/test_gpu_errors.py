"""Error paths of the step, driven so that nothing faults or hangs.

The reference has no error reporting on these paths: `add_cell` returns -1
when the spatial hash is full and the caller then writes cell_start[-1]
(src/cuda/tuning/kernels/common.cuh:104-124, rebuild_n_search.cu:19-34), and
`fill_neighbors` has no capacity guard (compute_neighbor_list.cu:40-43).
Here a full hash sets an error flag that the next synchronising call reports,
list rows beyond their capacity are recomputed from their cells (covered by
test_gpu_parity.test_neighbour_list_widths with widths 8 and 32), and every
device wait is bounded: the test hook `wcsph.stall_sort` makes the radix
sort's look-back waits run out in milliseconds, which must surface as
ERR_DEVICE_TIMEOUT with the particle state left as it was.
"""
import numpy as np
import pytest

import wcsph
from parity import dam_break_scene, run_one_step

pytestmark = pytest.mark.gpu


def spread_scene(n_side=16, r=0.01):
    """n_side^3 particles 3h apart: every particle alone in its cell."""
    h = 4 * r
    g = np.stack(np.meshgrid(*[np.arange(n_side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    pos = np.zeros((g.shape[0], 4), np.float32)
    pos[:, :3] = (0.1 + 3 * h * g).astype(np.float32)
    pos[:, 3] = 1.0
    ext = 0.2 + 3 * h * n_side
    return pos, wcsph.box((0, 0, 0), (ext, ext, ext))


def test_full_hash_table_is_reported():
    pos, bx = spread_scene()           # 4,096 cells in a table of bit_ceil(4096) / 4 = 1,024 slots
    p = wcsph.default_params(particle_radius=0.01, max_time_step=1e-3, cfl_factor=0.0, table_size_mult=1)
    with wcsph.CUDASPHSimulator(p, pos, bx) as sim:
        sim.update(1e-3)
        with pytest.raises(wcsph.WcsphError) as e:
            sim.synchronize()
        assert e.value.status == wcsph.ERR_HASH_FULL
        assert "spatial hash table is full" in e.value.message
        sim.synchronize()                 # the flag was reported once and cleared; the context still works
    # with room for every cell the same scene steps cleanly: no particle has a neighbour
    p.table_size_mult = 8
    out = run_one_step(p, bx, pos, None, None, 1e-3)
    counts, _, _ = out["neighbors"]
    assert not counts.any()
    assert np.allclose(out["density"], out["density"][0])


def test_sort_wait_timeout_is_reported_and_keeps_the_state():
    p, bx, pos, _ = dam_break_scene(dims=(24, 24, 24), walls=False)   # 13,824 particles: 7 sort tiles
    vel = wcsph.make_velocities(pos.shape[0], 0.2, seed=4)
    with wcsph.CUDASPHSimulator(p, pos, bx, fluid_vel=vel) as sim:
        before_pos, before_vel = sim.get_state()
        with wcsph.stall_sort():
            sim.update(1e-3)              # the step's graph is captured with the stalled sort
            with pytest.raises(wcsph.WcsphError) as e:
                sim.synchronize()
        assert e.value.status == wcsph.ERR_DEVICE_TIMEOUT
        assert "look-back" in e.value.message
        after_pos, after_vel = sim.get_state()
        assert np.array_equal(after_pos, before_pos) and np.array_equal(after_vel, before_vel)
    # the device is still usable: a fresh context steps the same scene normally
    with wcsph.CUDASPHSimulator(p, pos, bx, fluid_vel=vel) as sim:
        sim.update(1e-3)
        sim.synchronize()
        x, _ = sim.get_state()
        assert np.isfinite(x).all() and not np.array_equal(x, pos)
