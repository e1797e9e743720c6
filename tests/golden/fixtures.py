"""The golden fixture scenes, defined once for the fixture generator and the tests.

Each fixture is one step of the reference's own CUDA path (the harness in
oracle/_ref, variant of the same name) from the stored/generated input.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "fluid-simulation_b200"))
import wcsph  # noqa: E402

NAMES = ("fixture_surface", "fixture_tilting", "fixture_dambreak")
DAMBREAK_TANK = (0.6, 0.4, 0.4)


def textbook_stiffness(k: float, r: float) -> float:
    """Tait k in the textbook spiky normalisation -> the reference's (k * (4r)^6)."""
    rd = float(np.float32(r))
    return float(np.float32(k * (4.0 * rd) ** 6))


def scene(name: str):
    """-> (params, box, pos, vel, boundary_pos or None, delta)."""
    if name == "fixture_surface":
        # app/surface_tension/application.cu:10-25
        p = wcsph.default_params(external_force=wcsph.FORCE_CONSTANT, external_force_param=(0.0, 9.81, 0.0),
                                 table_size_mult=8)
        pos, vel = wcsph.snapshot_read(HERE / "surface_settled_2048.sphs", "surface_tension", 2048)
        return p, wcsph.box((-0.8, -0.8, -0.8), (0.8, 0.8, 0.8)), pos, vel, None, 0.01
    if name == "fixture_tilting":
        # app/tilting_box/application.cu:10-46, box model rotated 0.1 rad about z
        p = wcsph.default_params(table_size_mult=16)
        pos, vel = wcsph.snapshot_read(HERE / "tilting_chaotic_2048.sphs", "tilting_box", 2048)
        bx = wcsph.box((-2.3, -0.7, -0.6), (2.3, 0.7, 0.6), model=wcsph.rotation_z(0.1))
        return p, bx, pos, vel, None, 0.01
    if name == "fixture_dambreak":
        r = 0.01
        p = wcsph.default_params(particle_radius=r, stiffness=textbook_stiffness(1000.0, r), viscosity=0.01,
                                 max_time_step=1e-3, cfl_factor=0.0, table_size_mult=4)
        dims = (16, 16, 8)
        pos = wcsph.make_lattice(tuple(r + (d - 1) * r for d in dims), dims, r, 0.1 * r, 7)
        bpos = wcsph.sample_box_walls((0, 0, 0), DAMBREAK_TANK, 2 * r)
        return p, wcsph.box((0, 0, 0), DAMBREAK_TANK), pos, np.zeros_like(pos), bpos, 1e-3
    raise KeyError(name)


def load(name: str) -> dict:
    d = np.load(HERE / f"ref_{name}.npz")
    return {k: d[k] for k in d.files}
