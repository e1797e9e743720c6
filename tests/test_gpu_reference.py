"""CUDA step vs the reference's own CUDA kernels (one step, same input).

The reference side is either a committed golden fixture
(tests/golden/ref_<name>.npz) or, where the harness was built
(oracle/_ref/<name>), a live run in a child process. Integer work must
match bit-exactly (Morton keys, stable-sort permutation, cell ranges,
neighbour lists in the reference traversal order); float fields within
REL_TOL (field-scaled, see parity.py).

Scenes: the three 2,048-particle fixtures, the 32^3 dam break with walls,
the mesh obstacle (393,216 fluid particles over a level-4 icosphere and
walls, 64,276 boundary particles, CFL-adaptive dt) and the 1,048,576-particle
tilting box. The trajectory tests replay the reference's own run step by
step: every step of the CUDA path starts from the reference's state of the
step before, so the CFL step, keys, permutation and neighbour counts are
compared bit for bit at every step of a long run with no accumulated drift.
"""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import fixtures
import refpath
import wcsph
from parity import check_fields, field_close, hash_cell_map, pressure_bounds

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"
GEN = GOLDEN / "make_ref_fixtures.py"


def reference_outputs(name, tmp_path):
    npz = GOLDEN / f"ref_{name}.npz"
    if not npz.exists():
        if not refpath.available(name):
            pytest.skip(f"no golden fixture and no reference harness for {name}")
        subprocess.run([sys.executable, str(GEN), str(tmp_path), name], check=True, timeout=600)
        npz = tmp_path / f"ref_{name}.npz"
    d = np.load(npz)
    return {k: d[k] for k in d.files}


def scene(name):
    if name in fixtures.NAMES:
        return fixtures.scene(name)
    pre = wcsph.preset(name)
    return pre.params, pre.box, pre.pos, pre.vel, pre.bpos, pre.info.delta


@pytest.mark.parametrize("name", list(fixtures.NAMES) + ["dam_break", "mesh_obstacle", "large_tilting"])
def test_cuda_path_matches_reference_kernels(name, tmp_path):
    ref = reference_outputs(name, tmp_path)
    p, bx, pos, vel, bpos, delta = scene(name)
    sim = wcsph.CUDASPHSimulator(p, pos, bx, fluid_vel=vel, boundary_pos=bpos)
    sim.update(delta)
    got = {k: sim.field(k) for k in ("position", "velocity", "density", "pressure", "pressure_accel",
                                     "non_pressure_accel", "normal", "morton_keys", "permutation", "hash_table",
                                     "hash_cell_start", "hash_cell_end", "boundary_position", "boundary_mass")}
    counts, offsets, idx = sim.neighbors()
    dt = sim.last_dt()
    sim.close()
    assert np.array_equal(np.sort(got["morton_keys"]), ref["sorted_keys"]), "Morton keys differ"
    assert np.array_equal(got["permutation"], ref["permutation"]), "sort permutation differs"
    mine = hash_cell_map(got["hash_table"], got["hash_cell_start"], got["hash_cell_end"])
    theirs = {int(k): (int(s), int(e)) for k, s, e in zip(ref["cell_keys"], ref["cell_start"], ref["cell_end"])}
    assert mine == theirs, "cell ranges differ"
    assert np.array_equal(counts, ref["nbr_counts"]), "neighbour counts differ"
    assert np.array_equal(idx, ref["nbr_idx"]), "neighbour lists differ"
    assert dt[0] == ref["dt"][0] and dt[1] == ref["dt"][1]
    if bpos is not None:
        assert np.array_equal(got["boundary_position"], ref["boundary_position"])
        ok, worst = field_close(got["boundary_mass"], ref["boundary_mass"])
        assert ok, worst
    spos = pos[ref["permutation"]]
    bounds = pressure_bounds(p, ref["density"], ref["pressure"], spos,
                             (ref["nbr_counts"], ref["nbr_offsets"], ref["nbr_idx"]),
                             ref.get("boundary_position"), ref.get("boundary_mass"), dt=float(ref["dt"][0]))
    fails = check_fields(got, ref, bounds)
    assert not fails, fails


def reference_trajectory(name, steps, full, skip, vy, tmp_path):
    if not refpath.available(name):
        pytest.skip(f"no reference harness for {name}")
    out = tmp_path / f"traj_{name}"
    subprocess.run([sys.executable, str(GEN), str(out), name, "--trajectory", str(steps), "--skip", str(skip),
                    "--vy", str(vy), *map(str, full)], check=True, timeout=1800)
    return out


@pytest.mark.parametrize("name,steps,skip,vy,full", [("mesh_obstacle", 50, 0, 0.0, (0, 1, 25, 49)),
                                                     ("mesh_obstacle", 50, 0, -8.0, (0, 24, 49)),
                                                     ("large_tilting", 10, 0, 0.0, (0, 9))])
def test_reference_trajectory_replayed_step_by_step(name, steps, skip, vy, full, tmp_path):
    """Config 1 (mesh obstacle, CFL 0.4, dt cap 1e-3) for its first 50 steps,
    in which the collapsing column stays below the 4 m/s at which the CFL
    step 0.4 * 2r / max|v| drops under the cap; the same scene thrown down at
    8 m/s onto the sphere, in which the CFL rule sets dt; and
    the 1,048,576-particle tilting box for the first 10 steps of its box
    schedule: at every
    step the CFL step (dt_p, np_dt), sorted Morton keys, permutation and
    neighbour counts equal the reference's and density is within 1e-5; at
    the `full` steps the neighbour lists are compared in reference order and
    every field is checked."""
    traj = reference_trajectory(name, steps, full, skip, vy, tmp_path)
    pre = wcsph.preset(name)
    p, delta = pre.params, pre.info.delta
    sim = wcsph.CUDASPHSimulator(p, pre.pos, pre.box, fluid_vel=pre.vel, boundary_pos=pre.bpos)
    dts = []
    try:
        for k in range(steps):
            d = traj / f"step_{k:04d}"
            ld = lambda f: np.load(d / f"{f}.npy")  # noqa: E731
            in_pos, in_vel = ld("in_pos"), ld("in_vel")
            sim.set_state(in_pos, in_vel)
            if pre.info.moving_box:
                sim.set_box(pre.box_at(skip + k + 1))
            sim.update(delta)
            dt = sim.last_dt()
            want_dt = ld("dt")
            dts.append(float(want_dt[0]))
            assert dt[0] == want_dt[0] and dt[1] == want_dt[1], f"step {k}: dt {dt} vs {tuple(want_dt)}"
            keys = sim.field("morton_keys")
            perm = sim.field("permutation")
            assert np.array_equal(np.sort(keys), ld("sorted_keys")), f"step {k}: Morton keys differ"
            assert np.array_equal(perm, ld("permutation")), f"step {k}: permutation differs"
            counts, offsets, idx = sim.neighbors()
            assert np.array_equal(counts, ld("nbr_counts")), f"step {k}: neighbour counts differ"
            got = {"density": sim.field("density")}
            rep = field_close(got["density"], ld("density"))
            assert rep[0], f"step {k}: density {rep[1]:.3g} x tolerance"
            if k in full:
                assert np.array_equal(idx, ld("nbr_idx")), f"step {k}: neighbour lists differ"
                for f in ("position", "velocity", "pressure", "pressure_accel", "non_pressure_accel", "normal"):
                    got[f] = sim.field(f)
                want = {f: ld(f) for f in ("density", "pressure", "position", "velocity", "pressure_accel",
                                           "non_pressure_accel", "normal")}
                bpos = ld("boundary_position") if pre.bpos is not None else None
                bmass = ld("boundary_mass") if pre.bpos is not None else None
                bounds = pressure_bounds(p, want["density"], want["pressure"], in_pos[ld("permutation")],
                                         (ld("nbr_counts"), ld("nbr_offsets"), ld("nbr_idx")), bpos, bmass,
                                         dt=float(want_dt[0]))
                fails = check_fields(got, want, bounds)
                assert not fails, f"step {k}: {fails}"
    finally:
        sim.close()
    capped = sum(d == float(np.float32(p.max_time_step)) for d in dts)
    print(f"{name} (vy {vy}): dt from {min(dts):.4g} to {max(dts):.4g}, {steps - capped} of {steps} steps set by CFL")
    if vy:
        assert capped <= steps // 2, dts   # the thrown scene runs mostly on the CFL step
