"""Benchmark scene generators restated in numpy (test and baseline infrastructure).

The reference arm of bench.py (`--impl reference`) times the reference's own
CUDA kernels. Its processes must not load this project's library, so the
scenes it needs are rebuilt here from the same definitions, bit for bit:

  * lattice  FluidSimulator::init_positions (src/simulation/fluid_simulator.cpp:24-54):
             x-outer, y, z-inner, start = origin - (dims - 1) r, step 2r, w = 1;
             plus a seeded U(-jitter, jitter) per axis drawn in lattice order
             from a splitmix64 stream (the library's wcsph_make_lattice);
  * velocities  N(0, sigma) per component by the Box-Muller transform from the
             same stream family (wcsph_make_velocities);
  * box walls  single-layer wall particles on a 2r grid (wcsph_sample_box_walls);
  * tilting box  rotation about z growing linearly to 15 degrees over 1 s
             (the large scene's schedule), glm column-major model matrices.

Floating-point steps follow the library's order of operations: float32 lattice
arithmetic, double jitter and Box-Muller terms rounded once to float32, and the
C library's log/cos (Python's math module) and cosf/sinf (libm through ctypes).
tests/test_scenes_cpu.py checks every array against the library, bit for bit.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)

_libm = ctypes.CDLL("libm.so.6")
_libm.cosf.restype = ctypes.c_float
_libm.cosf.argtypes = [ctypes.c_float]
_libm.sinf.restype = ctypes.c_float
_libm.sinf.argtypes = [ctypes.c_float]


def splitmix_uniform(seed: int, count: int) -> np.ndarray:
    """The first `count` draws in [0, 1) of the splitmix64 stream seeded `seed`
    (state += golden; xor-shift-multiply mix; top 53 bits / 2^53)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, count + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def make_lattice(origin, dims, r, jitter=0.0, seed=0) -> np.ndarray:
    f = np.float32
    r = f(r)
    spacing = f(2.0) * r
    dims = tuple(int(d) for d in dims)
    start = [f(origin[a]) - f(dims[a] - 1) * r for a in range(3)]
    g = np.stack(np.meshgrid(*[np.arange(d, dtype=np.float32) for d in dims], indexing="ij"), -1).reshape(-1, 3)
    out = np.empty((g.shape[0], 4), np.float32)
    for a in range(3):
        out[:, a] = start[a] + g[:, a] * spacing
    if f(jitter) > 0:
        u = splitmix_uniform(seed, 3 * g.shape[0]).reshape(-1, 3)
        out[:, :3] += ((2.0 * u - 1.0) * float(f(jitter))).astype(np.float32)
    out[:, 3] = 1.0
    return out


def make_velocities(n: int, sigma: float, seed: int) -> np.ndarray:
    u = splitmix_uniform(seed ^ 0xA5A5A5A5A5A5A5A5, 6 * n).reshape(-1, 2)
    u1 = np.maximum(u[:, 0], 1e-300)
    logs = np.fromiter((math.log(x) for x in u1.tolist()), np.float64, count=u1.size)
    coss = np.fromiter((math.cos(6.283185307179586 * x) for x in u[:, 1].tolist()), np.float64, count=u1.size)
    normal = np.sqrt(-2.0 * logs) * coss
    out = np.zeros((n, 4), np.float32)
    out[:, :3] = (float(np.float32(sigma)) * normal).reshape(n, 3).astype(np.float32)
    return out


def sample_box_walls(mn, mx, spacing) -> np.ndarray:
    f = np.float32
    spacing = f(spacing)
    cnt = [int(round(float(f(mx[d]) - f(mn[d])) / float(spacing))) for d in range(3)]
    g = np.stack(np.meshgrid(*[np.arange(c + 1) for c in cnt], indexing="ij"), -1).reshape(-1, 3)
    surf = (g == 0).any(1) | (g == np.array(cnt)).any(1)
    g = g[surf]
    out = np.empty((g.shape[0], 4), np.float32)
    for d in range(3):
        out[:, d] = f(mn[d]) + g[:, d].astype(np.float32) * spacing
    out[:, 3] = 1.0
    return out


def box_floats(mn, mx, angle=None) -> np.ndarray:
    """min[3], max[3], model[16], model_inv[16] (column-major) of a box rotated
    `angle` (float32 radians) about z; identity when angle is None."""
    model = np.eye(4, dtype=np.float32).reshape(-1)
    inv = model.copy()
    if angle is not None:
        c = _libm.cosf(float(np.float32(angle)))
        s = _libm.sinf(float(np.float32(angle)))
        model[0], model[1], model[4], model[5] = c, s, -s, c
        inv[0], inv[1], inv[4], inv[5] = c, -s, s, c
    return np.concatenate([np.asarray(mn, np.float32), np.asarray(mx, np.float32), model, inv]).astype(np.float32)


@dataclass
class Scene:
    name: str
    pos: np.ndarray
    vel: np.ndarray
    bpos: np.ndarray | None
    delta: float
    box0: np.ndarray          # 38 floats
    moving: bool

    def box_at(self, updates: int) -> np.ndarray:
        if self.name != "large_tilting":
            return self.box0
        t = float(updates) * float(np.float32(self.delta))
        a = (15.0 * math.pi / 180.0) * min(t / 1.0, 1.0)
        return box_floats((-1.0, -0.5, -0.5), (1.0, 0.5, 0.5), np.float32(a))


def scene(name: str, seed: int = 0) -> Scene:
    """The bench workloads the reference harness is built for."""
    f = np.float32
    if name == "large_tilting":
        r = f(0.004)
        dims = (128, 128, 64)
        corner = (f(-1.0) + r, f(-0.5) + r, f(-0.5) + r)
        origin = [corner[a] + f(dims[a] - 1) * r for a in range(3)]
        pos = make_lattice(origin, dims, r, f(0.2) * r, seed)
        vel = make_velocities(pos.shape[0], 0.1, seed + 1)
        return Scene(name, pos, vel, None, float(f(5e-4)), box_floats((-1.0, -0.5, -0.5), (1.0, 0.5, 0.5)), True)
    if name == "dam_break":
        r = f(0.01)
        dims = (32, 32, 32)
        origin = [r + f(d - 1) * r for d in dims]
        pos = make_lattice(origin, dims, r, f(0.1) * r, seed)
        bpos = sample_box_walls((0.0, 0.0, 0.0), (1.0, 0.6, 0.6), f(2.0) * r)
        return Scene(name, pos, np.zeros_like(pos), bpos, float(f(1e-3)),
                     box_floats((0.0, 0.0, 0.0), (1.0, 0.6, 0.6)), False)
    raise KeyError(f"no numpy restatement of scene {name!r}")
