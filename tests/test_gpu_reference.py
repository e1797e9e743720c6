"""CUDA step vs the reference's own CUDA kernels (one step, same input).

The reference side is either a committed golden fixture
(tests/golden/ref_<name>.npz) or, where the harness was built
(oracle/_ref/<name>), a live run in a child process. Integer work must
match bit-exactly (Morton keys, stable-sort permutation, cell ranges,
neighbour lists in the reference traversal order); float fields within
REL_TOL (field-scaled, see parity.py).
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


@pytest.mark.parametrize("name", list(fixtures.NAMES) + ["dam_break"])
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
