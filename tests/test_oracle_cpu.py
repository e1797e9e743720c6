"""The oracle itself: known answers derived from the reference source and,
when present, the golden fixtures produced by the reference's own CUDA
kernels (tests/golden/ref_*.npz). Runs on CPU."""
from pathlib import Path

import numpy as np
import pytest

import oracle
import wcsph
from parity import check_fields, field_close, packed_from_morton, pressure_bounds

GOLDEN = Path(__file__).resolve().parent / "golden"


def _interleave(c):
    # independent restatement of encode_morton (morton.cuh:30-34) by bit loop
    u = [(int(x) + (1 << 20)) & 0xFFFFFFFF for x in c]
    key = 0
    for b in range(21):
        for axis in range(3):
            key |= ((u[axis] >> b) & 1) << (3 * b + axis)
    return key


def test_morton_known_answers():
    # cell (0,0,0): bit 20 of each offset coordinate lands at bits 60..62
    k = oracle.morton_keys(np.zeros((1, 4), np.float32), 0.04)
    assert int(k[0]) == 0x7000000000000000
    rng = np.random.default_rng(1)
    pos = (rng.random((500, 4)) * 40 - 20).astype(np.float32)
    cs = np.float32(0.08)
    keys = oracle.morton_keys(pos, float(cs))
    for p, key in zip(pos, keys):
        c = [int(np.floor(np.float32(p[d]) / cs)) for d in range(3)]
        assert int(key) == _interleave(c)


def test_sort_is_stable():
    rng = np.random.default_rng(2)
    keys = rng.integers(0, 50, 5000).astype(np.uint64) * np.uint64(0x100000001)
    assert np.array_equal(oracle.sort_perm(keys), np.argsort(keys, kind="stable").astype(np.uint32))


def _single(p, pos, bpos=None, delta=1e-3, vel=None):
    bx = wcsph.box((-10, -10, -10), (10, 10, 10))
    vel = np.zeros_like(pos) if vel is None else vel
    if bpos is not None:
        bs, bm = oracle.boundary_init(p, bpos)
        return oracle.step(p, bx, pos, vel, bs, bm, delta=delta), bm
    return oracle.step(p, bx, pos, vel, delta=delta), None


def test_isolated_particle_density_and_boundary_mass():
    p = wcsph.default_params()
    h = 4 * np.float64(np.float32(0.02))
    w0 = 8.0 / (np.pi * h ** 3)
    mass = 1000.0 * (2 * np.float64(np.float32(0.02))) ** 3 * 0.8
    pos = np.array([[0.1, 0.2, 0.3, 1.0]], np.float32)
    r, _ = _single(p, pos)
    assert abs(r.rho[0] - mass * w0) < 1e-9 * mass * w0
    assert r.prs[0] == 0.0  # ratio clamped to 1
    far = np.array([[5.0, 5.0, 5.0, 1.0]], np.float32)
    _, bm = _single(p, pos, bpos=far)
    # m_b = rho0 / W(0) for an isolated boundary particle (compute_boundary_mass.cu:19,29)
    assert abs(bm[0] - 1000.0 / w0) < 1e-9 * 1000.0 / w0


def test_cfl_time_step_rule():
    p = wcsph.default_params()
    pos = wcsph.make_lattice((0, 0, 0), (3, 3, 3), 0.02)
    r, _ = _single(p, pos, delta=0.01)
    assert np.float32(r.dt_p) == np.float32(5e-4) and np.float32(r.np_dt) == np.float32(0.01)
    r, _ = _single(p, pos, delta=1e-4)      # v = 0 returns max_step, not delta (sph.cu:123-124)
    assert np.float32(r.dt_p) == np.float32(5e-4)
    vel = np.zeros_like(pos)
    vel[3, 0] = 100.0                       # 0.4 * 0.04 / 100 = 1.6e-4 binds
    r, _ = _single(p, pos, delta=0.01, vel=vel)
    assert np.float32(r.dt_p) == np.float32(np.float32(0.4) * np.float32(0.04) / np.float32(100.0))
    r, _ = _single(p, pos, delta=0.1)
    assert np.float32(r.np_dt) == np.float32(0.015)


def test_neighbor_sets_against_brute_force():
    p = wcsph.default_params(particle_radius=0.01)
    pos = wcsph.make_lattice((0.2, 0.2, 0.2), (9, 8, 7), 0.01, 0.003, 5)
    r, _ = _single(p, pos)
    spos = pos[r.perm].astype(np.float64)
    h2 = np.float64(np.float32(0.04) * np.float32(0.04))
    d2 = ((spos[:, None, :3] - spos[None, :, :3]) ** 2).sum(-1)
    n = pos.shape[0]
    for i in range(n):
        got = set(r.nbr_idx[r.nbr_offsets[i]:r.nbr_offsets[i] + r.nbr_counts[i]].tolist())
        clear_in = set(np.nonzero(d2[i] < h2 * (1 - 1e-6))[0].tolist()) - {i}
        clear_out = set(np.nonzero(d2[i] > h2 * (1 + 1e-6))[0].tolist())
        assert clear_in <= got and not (got & clear_out)


# Two particles of the 1,048,576-particle tilting box at step 6 of the
# reference's own run, |r| within one ulp of h = 0.016: the reference's
# kernels (dot(r, r) contracted to fma(z, z, fma(x, x, y*y))) count them as
# neighbours; the order fma(z, z, fma(y, y, x*x)) would not.
EDGE_PAIR = ((-0.043888334184885025, 0.30357417464256287, -0.3445073962211609),
             (-0.044758860021829605, 0.3195130228996277, -0.3434140682220459))


def edge_pair_scene():
    p = wcsph.default_params(particle_radius=0.004, max_time_step=5e-4, cfl_factor=0.0)
    pos = np.zeros((2, 4), np.float32)
    pos[:, :3] = np.array(EDGE_PAIR, np.float32)
    pos[:, 3] = 1.0
    return p, wcsph.box((-1, -0.5, -0.5), (1, 0.5, 0.5)), pos


def test_neighbour_predicate_rounds_like_the_reference():
    p, bx, pos = edge_pair_scene()
    r = oracle.step(p, bx, pos, np.zeros_like(pos), None, None, delta=5e-4, nbr_cap=16)
    assert list(r.nbr_counts) == [1, 1]


def test_metrics_known_answer():
    p = wcsph.default_params()
    vel = np.zeros((4, 4), np.float32)
    vel[:, 0] = [1, 2, 3, 4]
    ms, ke = oracle.metrics(p, vel)
    s = np.float32(0.04)
    mass = 1000.0 * np.float64(np.float32(np.float64(s * s * s) * 0.8))
    assert abs(ms - 2.5) < 1e-12 and abs(ke - 0.5 * mass * 30) < 1e-12


@pytest.mark.parametrize("name", ["fixture_surface", "fixture_tilting", "fixture_dambreak"])
def test_oracle_against_reference_kernel_fixtures(name):
    """Pins the oracle to the reference's own CUDA kernels (golden fixtures)."""
    path = GOLDEN / f"ref_{name}.npz"
    if not path.exists():
        pytest.skip(f"{path.name} not generated yet (tests/golden/make_ref_fixtures.py on a GPU)")
    import fixtures

    ref = fixtures.load(name)
    p, bx, pos, vel, bpos, delta = fixtures.scene(name)
    if bpos is not None:
        bs, bm = oracle.boundary_init(p, bpos)
        assert np.array_equal(bs, ref["boundary_position"])
        ok, worst = field_close(bm, ref["boundary_mass"])
        assert ok, worst
        r = oracle.step(p, bx, pos, vel, bs, bm, delta=delta)
    else:
        r = oracle.step(p, bx, pos, vel, delta=delta)
    assert np.array_equal(np.sort(r.keys), ref["sorted_keys"])
    assert np.array_equal(r.perm, ref["permutation"])
    cs = float(np.float32(4 * p.particle_radius) * np.float32(p.cell_size_mult))
    k, s, e = oracle.cell_ranges(pos[r.perm], cs)
    want = {int(a): (int(b), int(c)) for a, b, c in zip(ref["cell_keys"], ref["cell_start"], ref["cell_end"])}
    got = {int(a): (int(b), int(c)) for a, b, c in zip(packed_from_morton(k), s, e)}
    assert got == want
    assert np.array_equal(r.nbr_counts, ref["nbr_counts"])
    assert np.array_equal(r.nbr_idx, ref["nbr_idx"])
    assert np.float32(r.dt_p) == ref["dt"][0] and np.float32(r.np_dt) == ref["dt"][1]
    mine = {"density": r.rho, "pressure": r.prs, "pressure_accel": r.ap, "non_pressure_accel": r.anp,
            "normal": r.normal, "position": r.pos, "velocity": r.vel}
    bounds = pressure_bounds(p, ref["density"], ref["pressure"], pos[r.perm],
                             (ref["nbr_counts"], ref["nbr_offsets"], ref["nbr_idx"]),
                             ref.get("boundary_position"), ref.get("boundary_mass"), dt=float(ref["dt"][0]))
    fails = check_fields(mine, ref, bounds)
    assert not fails, fails
