"""C ABI checks that need no GPU: symbols, defaults, scene builders, presets."""
import ctypes as C

import numpy as np

import wcsph


def test_library_exports_every_header_symbol():
    lib = wcsph.load_library()
    syms = wcsph.header_symbols()
    assert len(syms) >= 50
    missing = [s for s in syms if not hasattr(lib, s)]
    assert missing == []
    assert lib.wcsph_abi_version() == 1


def test_checked_library_exports_every_header_symbol():
    # the bounds-checked build (`make checked`) has the same ABI
    path = wcsph.CHECKED_LIB_PATH
    if not path.exists():
        import pytest

        pytest.skip("lib/libwcsph_checked.so is not built (make -C fluid-simulation_b200 checked)")
    lib = C.CDLL(str(path))
    missing = [s for s in wcsph.header_symbols() if not hasattr(lib, s)]
    assert missing == []
    assert lib.wcsph_abi_version() == 1
    lib.wcsph_status_string.restype = C.c_char_p
    assert b"bounds" in lib.wcsph_status_string(wcsph.ERR_BOUNDS)


def test_default_params_are_the_reference_constants():
    p = wcsph.default_params()
    # common.cuh:18-23, compute_rho_p.cu:10-12, compute_non_pressure_accel.cu:14-16,
    # update_positions.cu:10-12, sph.cuh:26-32
    assert np.float32(p.particle_radius) == np.float32(0.02)
    assert p.rest_density == 1000.0 and np.float32(p.stiffness) == np.float32(0.1) and p.exponent == 7.0
    assert p.max_density_ratio == 1.5
    assert np.float32(p.viscosity) == np.float32(0.001) and np.float32(p.surface_tension) == np.float32(0.13)
    assert list(p.gravity) == [0.0, np.float32(-9.81), 0.0]
    assert np.float32(p.cfl_factor) == np.float32(0.4)
    assert np.float32(p.max_time_step) == np.float32(5e-4) and np.float32(p.min_time_step) == np.float32(1e-5)
    assert np.float32(p.non_pressure_max_time_step) == np.float32(0.015)
    assert p.collision_buffer_mult == 0.75 and p.elasticity == 0.5


def test_status_strings_and_identity_box():
    lib = wcsph.load_library()
    assert lib.wcsph_status_string(0) == b"ok"
    assert b"magic" in lib.wcsph_status_string(wcsph.ERR_SNAPSHOT_MAGIC)
    b = wcsph.box((0, 1, 2), (3, 4, 5))
    assert list(b.min) == [0, 1, 2] and list(b.max) == [3, 4, 5]
    assert np.allclose(np.array(b.model).reshape(4, 4), np.eye(4))


def test_create_without_device_fails_cleanly():
    # no CUDA device in this container: a status code, not a crash or a CPU fallback
    import conftest

    if conftest.HAS_GPU:
        return
    p = wcsph.default_params()
    pos = wcsph.make_lattice((0, 0, 0), (4, 4, 4), 0.02)
    try:
        wcsph.CUDASPHSimulator(p, pos, wcsph.box((-1, -1, -1), (1, 1, 1)))
    except wcsph.WcsphError as e:
        assert e.status in (wcsph.ERR_NO_DEVICE, wcsph.ERR_CUDA)
    else:
        raise AssertionError("create succeeded without a GPU")


def test_lattice_matches_init_positions_order():
    # fluid_simulator.cpp:24-54: start = origin - (dims-1) r; x outer, z inner; w = 1
    pos = wcsph.make_lattice((1.0, 2.0, 3.0), (3, 2, 4), 0.02)
    assert pos.shape == (24, 4)
    start = np.float32(1.0) - np.float32(2) * np.float32(0.02)
    assert pos[0, 0] == start
    assert np.allclose(pos[1, :3] - pos[0, :3], [0, 0, 0.04])       # z fastest
    assert np.allclose(pos[4, :3] - pos[0, :3], [0, 0.04, 0])        # then y
    assert np.allclose(pos[8, :3] - pos[0, :3], [0.04, 0, 0])        # x slowest
    assert np.all(pos[:, 3] == 1.0)
    assert np.allclose(pos[:, :3].mean(0), [1.0, 2.0, 3.0], atol=1e-6)


def test_jitter_and_velocities_are_seeded():
    a = wcsph.make_lattice((0, 0, 0), (8, 8, 8), 0.01, jitter=0.001, seed=3)
    b = wcsph.make_lattice((0, 0, 0), (8, 8, 8), 0.01, jitter=0.001, seed=3)
    c = wcsph.make_lattice((0, 0, 0), (8, 8, 8), 0.01, jitter=0.0, seed=3)
    assert np.array_equal(a, b)
    d = a[:, :3] - c[:, :3]
    assert np.abs(d).max() <= 0.001 + 1e-7 and np.abs(d).max() > 0.0009
    v = wcsph.make_velocities(200000, 0.1, seed=9)
    assert np.all(v[:, 3] == 0)
    assert abs(v[:, :3].std() - 0.1) < 1e-3 and abs(v[:, :3].mean()) < 1e-3


def test_box_walls_config0_count():
    walls = wcsph.sample_box_walls((0, 0, 0), (1.0, 0.6, 0.6), 0.02)
    # (51*31*31) lattice points minus the (49*29*29) interior
    assert walls.shape[0] == 51 * 31 * 31 - 49 * 29 * 29 == 7802
    on_face = ((np.isclose(walls[:, 0], 0) | np.isclose(walls[:, 0], 1.0)) |
               (np.isclose(walls[:, 1], 0) | np.isclose(walls[:, 1], 0.6)) |
               (np.isclose(walls[:, 2], 0) | np.isclose(walls[:, 2], 0.6)))
    assert on_face.all()
    assert len({tuple(x) for x in np.round(walls[:, :3], 6)}) == walls.shape[0]


def test_icosphere_surface_sampling():
    pts = wcsph.sample_icosphere((0.5, 0.5, 0.5), 0.15, 4, 0.01)
    r = np.linalg.norm(pts[:, :3] - 0.5, axis=1)
    # voxel centres of voxels touching the surface lie within half a voxel diagonal
    assert np.all(np.abs(r - 0.15) <= 0.5 * 0.01 * np.sqrt(3) + 1e-6)
    assert 3000 < pts.shape[0] < 6000
    # 20 * 4^4 = 5120 triangles; a closed shell: every direction is covered
    dirs = (pts[:, :3] - 0.5) / r[:, None]
    for axis in range(3):
        assert dirs[:, axis].max() > 0.99 and dirs[:, axis].min() < -0.99


def test_presets_match_the_workloads():
    d = wcsph.preset("dam_break")
    assert (d.info.fluid_n, d.info.boundary_n, d.info.steps) == (32768, 7802, 1000)
    # Tait k = 1000 in the textbook spiky normalisation = 1000 h^6 in the reference's
    assert np.float32(d.params.stiffness) == np.float32(1000.0 * (4.0 * float(np.float32(0.01))) ** 6)
    assert np.float32(d.params.viscosity) == np.float32(0.01)
    assert d.params.cfl_factor == 0 and np.float32(d.params.max_time_step) == np.float32(1e-3)
    t = wcsph.preset("large_tilting")
    assert t.info.fluid_n == 1048576 and t.info.boundary_n == 0 and t.info.moving_box == 1
    assert abs(t.vel[:, :3].std() - 0.1) < 2e-3
    b0, b1 = t.box_at(0), t.box_at(2000)
    assert np.allclose(np.array(b0.model).reshape(4, 4), np.eye(4))
    ang = np.arctan2(b1.model[1], b1.model[0])
    assert abs(np.degrees(ang) - 15.0) < 1e-4
    m = wcsph.preset("mesh_obstacle")
    assert m.info.fluid_n == 393216 and m.info.boundary_n > 60000
    assert np.float32(m.params.cfl_factor) == np.float32(0.4) and m.info.sim_time == 2.0
    r = wcsph.preset("rollout_block")
    assert r.info.fluid_n == 16384 and r.info.steps == 200 and r.params.surface_tension == 0.0
    s = wcsph.preset("surface_tension")
    assert s.info.fluid_n == 27000 and s.params.external_force == wcsph.FORCE_CONSTANT
    tb = wcsph.preset("tilting_box")
    bx = tb.box_at(3)
    # TiltingBoxApp::update_objects: t += min(delta, 1/30); angle = sin(t/5)/5
    t3 = np.float32(0.01) * 3
    assert abs(np.arctan2(bx.model[1], bx.model[0]) - np.sin(t3 / 5) / 5) < 1e-6


def test_ensemble_preset_distribution():
    n = [wcsph.preset_ensemble(1, k).info.fluid_n for k in range(256)]
    assert 4.0e6 < sum(n) < 5.5e6
    assert min(n) >= 2048 * 0.9 and max(n) <= 65536 * 1.2
    lg = np.log(n)
    # log-uniform between ln 2048 and ln 65536: mean near the midpoint
    assert abs(lg.mean() - 0.5 * (np.log(2048) + np.log(65536))) < 0.3
    e = wcsph.preset_ensemble(1, 5)
    assert 0.005 <= e.params.viscosity <= 0.05
    g = np.array(e.params.gravity)
    assert abs(np.linalg.norm(g) - 9.81) < 1e-4 and np.degrees(np.arctan2(g[0], -g[1])) <= 20.0 + 1e-4
