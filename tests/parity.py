"""Shared parity helpers: scenes at oracle-friendly sizes and comparisons.

Tolerances (stated once, used by every parity test):
  * integer work (Morton keys, permutation, cell ranges, neighbour sets):
    bit-exact;
  * float fields after one step vs the FP64 oracle: field-scaled relative
    error |a - b| <= REL_TOL * max(|b|, max|b| over the field), REL_TOL = 1e-5
    (pressure and pressure acceleration cancel to ~0 in the interior, so a
    per-element relative bound would be ill-posed there).
"""
from __future__ import annotations

import numpy as np

import oracle
import wcsph

REL_TOL = 1e-5


def field_close(got, want, tol=REL_TOL, comps=3):
    got = np.asarray(got, np.float64)
    want = np.asarray(want, np.float64)
    if got.ndim == 2:
        got, want = got[:, :comps], want[:, :comps]
    scale = np.max(np.abs(want)) if want.size else 0.0
    bound = tol * np.maximum(np.abs(want), scale) + 1e-30
    err = np.abs(got - want)
    worst = float(np.max(err / bound)) if err.size else 0.0
    return worst <= 1.0, worst


def dam_break_scene(dims=(16, 16, 16), r=0.01, jitter_frac=0.1, seed=7, walls=True, tank=(1.0, 0.6, 0.6),
                    **param_overrides):
    """Dam break with the lattice corner at r from the tank's min corner."""
    kw = dict(particle_radius=r, stiffness=1000.0, viscosity=0.01, max_time_step=1e-3, cfl_factor=0.0)
    kw.update(param_overrides)
    p = wcsph.default_params(**kw)
    origin = tuple(r + (d - 1) * r for d in dims)
    pos = wcsph.make_lattice(origin, dims, r, jitter_frac * r, seed)
    bx = wcsph.box((0, 0, 0), tank)
    bpos = wcsph.sample_box_walls((0, 0, 0), tank, 2 * r) if walls else None
    return p, bx, pos, bpos


def run_one_step(p, bx, pos, vel, bpos, delta, **sim_kw):
    sim = wcsph.CUDASPHSimulator(p, pos, bx, fluid_vel=vel, boundary_pos=bpos, **sim_kw)
    sim.update(delta)
    out = {k: sim.field(k) for k in ("position", "velocity", "density", "pressure", "pressure_accel",
                                     "non_pressure_accel", "normal", "morton_keys", "permutation",
                                     "hash_table", "hash_cell_start", "hash_cell_end", "boundary_position",
                                     "boundary_mass")}
    out["neighbors"] = sim.neighbors()
    out["dt"] = sim.last_dt()
    out["metrics"] = sim.compute_state_metrics()
    sim.close()
    return out


def oracle_one_step(p, bx, pos, vel, bpos, delta):
    if bpos is not None and len(bpos):
        bs, bm = oracle.boundary_init(p, bpos)
    else:
        bs, bm = None, None
    return oracle.step(p, bx, pos, vel, bs, bm, delta=delta), bs, bm


def hash_cell_map(table, cstart, cend):
    """Slot layout depends on insertion races; compare the cell -> range map."""
    occ = table != np.uint64(0xFFFFFFFFFFFFFFFF)
    return {int(k): (int(s), int(e)) for k, s, e in zip(table[occ], cstart[occ], cend[occ])}


def packed_from_morton(keys):
    """Morton key -> NSearch::pack key (de-interleave 21-bit offset coords)."""
    keys = np.asarray(keys, np.uint64)

    def compact(v):
        v = v & np.uint64(0x1249249249249249)
        v = (v | (v >> np.uint64(2))) & np.uint64(0x10C30C30C30C30C3)
        v = (v | (v >> np.uint64(4))) & np.uint64(0x100F00F00F00F00F)
        v = (v | (v >> np.uint64(8))) & np.uint64(0x1F0000FF0000FF)
        v = (v | (v >> np.uint64(16))) & np.uint64(0x1F00000000FFFF)
        v = (v | (v >> np.uint64(32))) & np.uint64(0x1FFFFF)
        return v

    x = compact(keys)
    y = compact(keys >> np.uint64(1))
    z = compact(keys >> np.uint64(2))
    return x | (y << np.uint64(21)) | (z << np.uint64(42))


def neighbor_sets(counts, offsets, idx):
    return [np.sort(idx[o:o + c]) for c, o in zip(counts, offsets)]
