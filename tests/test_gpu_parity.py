"""CUDA step vs the CPU oracle, one step, through the C ABI.

Bit-exact: Morton keys, stable-sort permutation, cell ranges of the hash and
per-particle neighbour lists (including the reference traversal order).
Within REL_TOL (field-scaled, see parity.py): density, pressure, pressure
acceleration, non-pressure acceleration, normals, positions, velocities.
"""
import numpy as np
import pytest

import wcsph
from parity import (check_fields, dam_break_scene, field_close, hash_cell_map, oracle_one_step,
                    packed_from_morton, pressure_bounds, run_one_step)

pytestmark = pytest.mark.gpu


def check_step(p, bx, pos, vel, bpos, delta, with_fields=True, nbr_cap=None, config=None):
    got = run_one_step(p, bx, pos, vel, bpos, delta, config=config)
    ref, bs, bm = oracle_one_step(p, bx, pos, vel, bpos, delta, nbr_cap=nbr_cap)
    n = pos.shape[0]
    # integer work: bit-exact
    assert np.array_equal(got["morton_keys"], ref.keys), "Morton keys differ"
    assert np.array_equal(got["permutation"], ref.perm), "sort permutation differs"
    cells = hash_cell_map(got["hash_table"], got["hash_cell_start"], got["hash_cell_end"])
    # oracle cell runs keyed by packed cell key
    import oracle
    spos = pos[ref.perm]
    cs = np.float32(np.float32(4 * p.particle_radius) * np.float32(p.cell_size_mult))
    okeys, ostart, oend = oracle.cell_ranges(spos, float(cs))
    want = {int(k): (int(s), int(e)) for k, s, e in zip(packed_from_morton(okeys), ostart, oend)}
    assert cells == want, "cell ranges differ"
    counts, offsets, idx = got["neighbors"]
    assert np.array_equal(counts, ref.nbr_counts), "neighbour counts differ"
    assert np.array_equal(offsets, ref.nbr_offsets)
    assert np.array_equal(idx, ref.nbr_idx), "neighbour lists (reference order) differ"
    if bpos is not None and len(bpos):
        assert np.array_equal(got["boundary_position"], bs), "boundary sort differs"
        ok, worst = field_close(got["boundary_mass"], bm)
        assert ok, f"boundary mass off by {worst:.3g} x tol"
    assert got["dt"][0] == np.float32(ref.dt_p) and got["dt"][1] == np.float32(ref.np_dt)
    if not with_fields:
        return got, ref
    want = {"density": ref.rho, "pressure": ref.prs, "pressure_accel": ref.ap, "non_pressure_accel": ref.anp,
            "normal": ref.normal, "position": ref.pos, "velocity": ref.vel}
    bounds = pressure_bounds(p, ref.rho, ref.prs, pos[ref.perm], (ref.nbr_counts, ref.nbr_offsets, ref.nbr_idx),
                             bs, bm, dt=ref.dt_p)
    fails = check_fields(got, want, bounds)
    assert not fails, fails
    ms, ke = got["metrics"]
    oms, oke = oracle.metrics(p, got["velocity"])
    assert abs(ms - oms) <= 1e-5 * max(abs(oms), 1e-12) and abs(ke - oke) <= 1e-5 * max(abs(oke), 1e-12)
    return got, ref


def test_dam_break_with_walls():
    p, bx, pos, bpos = dam_break_scene(dims=(16, 16, 16))
    check_step(p, bx, pos, np.zeros_like(pos), bpos, 1e-3)


@pytest.mark.parametrize("width", [0, 8, 32])
def test_neighbour_list_widths(width):
    # 0: the force and surface passes walk the density pass's bit matrix;
    # 8 / 32: lists too short for all / some particles, whose rows are
    # recomputed from their cell neighbourhoods (the default width fits all)
    p, bx, pos, bpos = dam_break_scene(dims=(16, 16, 16))
    vel = wcsph.make_velocities(pos.shape[0], 0.3, seed=9)
    check_step(p, bx, pos, vel, bpos, 1e-3, config={"neighbour_list_width": width})


def test_dense_cell_short_lists():
    rng = np.random.default_rng(1)
    pos = np.zeros((500, 4), np.float32)
    pos[:, :3] = (0.3 + rng.random((500, 3)) * 0.06).astype(np.float32)
    pos[:, 3] = 1.0
    p = wcsph.default_params(particle_radius=0.01, max_time_step=1e-3, cfl_factor=0.0)
    bx = wcsph.box((0, 0, 0), (1, 1, 1))
    check_step(p, bx, pos, np.zeros_like(pos), None, 1e-3, config={"neighbour_list_width": 40, "mask_words": 4})


def test_dam_break_no_walls_cfl_random_velocity():
    p, bx, pos, _ = dam_break_scene(dims=(20, 12, 14), walls=False, cfl_factor=0.4, max_time_step=5e-4)
    vel = wcsph.make_velocities(pos.shape[0], 0.5, seed=3)
    check_step(p, bx, pos, vel, None, 0.01)


@pytest.mark.parametrize("mult", [0.5, 2.0 / 3.0, 1.5, 2.0])
def test_cell_size_multipliers(mult):
    p, bx, pos, bpos = dam_break_scene(dims=(12, 14, 10), cell_size_mult=mult, table_size_mult=16)
    check_step(p, bx, pos, np.zeros_like(pos), bpos, 1e-3)


@pytest.mark.parametrize("words", [2, 3])
def test_walls_without_boundary_hit_masks(words):
    # below 4 bit-matrix words the density pass keeps no boundary hit masks:
    # the force pass scans each particle's whole per-cell boundary run (and
    # most cells take the chunked path of an over-full bit matrix)
    p, bx, pos, bpos = dam_break_scene(dims=(12, 14, 10))
    vel = wcsph.make_velocities(pos.shape[0], 0.3, seed=5)
    check_step(p, bx, pos, vel, bpos, 1e-3, config={"mask_words": words})


def test_reference_constants_origin_centred_tilted_box():
    # reference defaults (r = 0.02, k = 0.1, nu = 0.001); the lattice straddles
    # the origin so cell coordinates change sign (63-bit keys), box rotated 0.1 rad
    p = wcsph.default_params()
    pos = wcsph.make_lattice((0.0, 0.0, 0.0), (14, 14, 14), 0.02, 0.002, 11)
    bx = wcsph.box((-2.3, -0.7, -0.6), (2.3, 0.7, 0.6), model=wcsph.rotation_z(0.1))
    vel = wcsph.make_velocities(pos.shape[0], 1.0, seed=5)
    check_step(p, bx, pos, vel, None, 0.01)


@pytest.mark.parametrize("force", [wcsph.FORCE_CONSTANT, wcsph.FORCE_FOUNTAIN, wcsph.FORCE_VORTEX])
def test_external_forces(force):
    p = wcsph.default_params(external_force=force, external_force_param=(0.0, 9.81, 0.0))
    pos = wcsph.make_lattice((0.0, -0.4, 0.0), (12, 12, 12), 0.02, 0.002, 13)
    bx = wcsph.box((-0.8, -0.8, -0.8), (0.8, 0.8, 0.8))
    check_step(p, bx, pos, np.zeros_like(pos), None, 0.01)


def test_neighbour_pair_at_the_support_radius():
    """A pair whose |r| is within one ulp of h (observed in the reference's own
    run of the tilting box): neighbours for the reference, so for the CUDA
    path and the oracle too."""
    from test_oracle_cpu import edge_pair_scene

    p, bx, pos = edge_pair_scene()
    got, ref = check_step(p, bx, pos, np.zeros_like(pos), None, 5e-4)
    assert list(got["neighbors"][0]) == [1, 1]


@pytest.mark.parametrize("n", [1, 2, 33, 100])
def test_tiny_scenes(n):
    p, bx, pos, bpos = dam_break_scene(dims=(6, 6, 6))
    check_step(p, bx, pos[:n].copy(), np.zeros((n, 4), np.float32), bpos, 1e-3)


def test_dense_cell_many_home_batches():
    # 700 particles packed into few cells: exercises home batches > 32 and
    # candidate lists beyond the 512-entry bitmask capacity (rescan path)
    rng = np.random.default_rng(0)
    pos = np.zeros((700, 4), np.float32)
    pos[:, :3] = (0.3 + rng.random((700, 3)) * 0.05).astype(np.float32)
    pos[:, 3] = 1.0
    p = wcsph.default_params(particle_radius=0.01, max_time_step=1e-3, cfl_factor=0.0)
    bx = wcsph.box((0, 0, 0), (1, 1, 1))
    check_step(p, bx, pos, np.zeros_like(pos), None, 1e-3)


def test_benchmark_scene_full_size():
    """The 1,048,576-particle benchmark scene (tilting-box preset, r = 0.004,
    jitter +-0.2 r, N(0, 0.1) velocities): one step at full size, every check
    of the small scenes (33 M neighbour pairs compared bit-exact)."""
    pre = wcsph.preset("large_tilting")
    n = pre.info.fluid_n
    assert n == 1 << 20
    check_step(pre.params, pre.box, pre.pos, pre.vel, None, pre.info.delta, nbr_cap=n * 96)
