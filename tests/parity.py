"""Shared parity helpers: scenes at oracle-friendly sizes and comparisons.

Tolerances (stated once, used by every parity test):
  * integer work (Morton keys, permutation, cell ranges, neighbour sets):
    bit-exact;
  * density, normals, non-pressure acceleration: field-scaled relative error
    |a - b| <= REL_TOL * max(|b|, max|b| over the field), REL_TOL = 1e-5
    (accelerations cancel to ~0 in the interior, so a per-element relative
    bound would be ill-posed there);
  * pressure and the fields it drives (pressure acceleration, velocity,
    position): the same 1e-5 relative density tolerance propagated through
    the Tait EOS, dp = REL_TOL * k gamma (rho/rho0)^gamma (its sensitivity to
    a relative density change), and through the pressure-force sum,
    da_i = m sum_j (dp_i/rho_i^2 + dp_j/rho_j^2) |grad W_ij| (+ boundary),
    dv = dt da, dx = dt^2 da; plus REL_TOL of the field's maximum. Near rest
    density the EOS amplifies an FP32 density rounding by gamma / (1 -
    ratio^-gamma), which no per-element 1e-5 bound can absorb: the
    reference's own kernels and the FP64 oracle differ by ~9x a plain
    field-scaled 1e-5 on a settled scene.
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


def pressure_bounds(p, rho, prs, spos, nbr, bpos=None, bmass=None, dt=0.0, tol=REL_TOL):
    """Per-particle absolute bounds for pressure, a_p, velocity and position
    (see the module docstring). rho/prs/spos are the reference values in
    sorted order; nbr = (counts, offsets, idx) fluid neighbour lists."""
    rho = np.asarray(rho, np.float64)
    prs = np.asarray(prs, np.float64)
    r = float(np.float32(p.particle_radius))
    h = 4.0 * r
    mass = float(p.rest_density) * (2 * r) ** 3 * 0.8
    rho0, k, gam, mx = float(p.rest_density), float(p.stiffness), float(p.exponent), float(p.max_density_ratio)
    ratio = rho / rho0
    inside = (ratio > 1.0) & (ratio < mx)
    dp = tol * k * gam * np.clip(ratio, 1.0, mx) ** gam * inside + tol * np.abs(prs)
    spiky = -45.0 / (np.pi * h ** 9)

    def grad_norm(d):
        rl = np.sqrt((d * d).sum(-1))
        q = rl / h
        g = np.where((q >= 1e-9) & (q <= 1.0), spiky * (1 - q) ** 2 / (h * np.maximum(rl, 1e-30)), 0.0)
        return np.abs(g) * rl

    counts, offsets, idx = nbr
    i = np.repeat(np.arange(len(counts)), counts)
    x = np.asarray(spos, np.float64)[:, :3]
    gw = grad_norm(x[i] - x[idx])
    da = mass * np.bincount(i, weights=(dp[i] / rho[i] ** 2 + dp[idx] / rho[idx] ** 2) * gw, minlength=len(rho))
    if bpos is not None and len(bpos):
        from scipy.spatial import cKDTree

        b = np.asarray(bpos, np.float64)[:, :3]
        # fluid-boundary pairs within h (a superset of the kernel's support is harmless: the gradient is 0 beyond h)
        pairs = cKDTree(x).sparse_distance_matrix(cKDTree(b), h * (1 + 1e-6), output_type="coo_matrix")
        q = pairs.data / h
        g = np.where((q >= 1e-9) & (q <= 1.0), np.abs(spiky) * (1 - q) ** 2 / h, 0.0)   # |grad W| = |g| |r|
        w = np.bincount(pairs.row, weights=np.asarray(bmass, np.float64)[pairs.col] * g, minlength=len(x))
        da += dp * (1 / rho ** 2 + 1 / rho0 ** 2) * w
    return {"pressure": dp, "pressure_accel": da, "velocity": dt * da, "position": dt * dt * da}


FIELDS = ("density", "pressure", "pressure_accel", "non_pressure_accel", "normal", "position", "velocity")


def field_report(got: dict, want: dict, bounds: dict | None = None, tol=REL_TOL, fields=FIELDS) -> dict:
    """Per field: `plain` = worst |error| / (tol x field scale), the plain
    field-scaled 1e-5 test; `widened` = the same against the plain bound plus
    the propagated EOS bound (fields listed in `bounds` only)."""
    out = {}
    for f in fields:
        g = np.asarray(got[f], np.float64)
        w = np.asarray(want[f], np.float64)
        if g.ndim == 2:
            g, w = g[:, :3], w[:, :3]
        scale = np.max(np.abs(w)) if w.size else 0.0
        bound = tol * np.maximum(np.abs(w), scale) + 1e-30
        err = np.abs(g - w)
        r = {"plain": float(np.max(err / bound)) if g.size else 0.0}
        if bounds is not None and f in bounds:
            extra = np.asarray(bounds[f], np.float64)
            wide = bound + (extra[:, None] if g.ndim == 2 else extra)
            r["widened"] = float(np.max(err / wide)) if g.size else 0.0
        out[f] = r
    _append_report(out)
    return out


def check_fields(got: dict, want: dict, bounds: dict | None = None, tol=REL_TOL, fields=FIELDS):
    """-> list of failure strings (empty when every field is within tolerance).
    A field passes under the plain field-scaled bound; only a field that
    fails it and has a propagated EOS bound (pressure and what it drives) is
    then held to the widened bound."""
    fails = []
    for f, r in field_report(got, want, bounds, tol, fields).items():
        if r["plain"] <= 1.0:
            continue
        if "widened" in r and r["widened"] <= 1.0:
            continue
        fails.append(f"{f}: worst error {r['plain']:.3g} x the plain tolerance"
                     + (f", {r['widened']:.3g} x the widened one" if "widened" in r else ""))
    return fails


def _append_report(rep: dict):
    """With WCSPH_PARITY_REPORT set, every comparison is appended to that
    file as one JSON line (test id, per-field ratios) for the record."""
    import json
    import os

    path = os.environ.get("WCSPH_PARITY_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps({"test": os.environ.get("PYTEST_CURRENT_TEST", "?"), "fields": rep}) + "\n")


def dam_break_scene(dims=(16, 16, 16), r=0.01, jitter_frac=0.1, seed=7, walls=True, tank=(1.0, 0.6, 0.6),
                    **param_overrides):
    """Dam break with the lattice corner at r from the tank's min corner."""
    rd = float(np.float32(r))
    kw = dict(particle_radius=r, stiffness=float(np.float32(1000.0 * (4.0 * rd) ** 6)), viscosity=0.01,
              max_time_step=1e-3, cfl_factor=0.0)
    kw.update(param_overrides)
    p = wcsph.default_params(**kw)
    origin = tuple(r + (d - 1) * r for d in dims)
    pos = wcsph.make_lattice(origin, dims, r, jitter_frac * r, seed)
    bx = wcsph.box((0, 0, 0), tank)
    bpos = wcsph.sample_box_walls((0, 0, 0), tank, 2 * r) if walls else None
    return p, bx, pos, bpos


def run_one_step(p, bx, pos, vel, bpos, delta, config=None, **sim_kw):
    """config: {name: value} entries of a frozen traversal config (KTT schema)."""
    sim = wcsph.CUDASPHSimulator(p, pos, bx, fluid_vel=vel, boundary_pos=bpos, **sim_kw)
    if config:
        import json, os, tempfile
        fd, path = tempfile.mkstemp(suffix=".json")
        with os.fdopen(fd, "w") as f:
            json.dump([{"Name": k, "Value": v, "ValueType": "UnsignedInt"} for k, v in config.items()], f)
        try:
            sim.set_tuning(wcsph.SEARCH_MCMC, 0.0, path)
        finally:
            os.unlink(path)
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


def oracle_one_step(p, bx, pos, vel, bpos, delta, nbr_cap=None):
    if bpos is not None and len(bpos):
        bs, bm = oracle.boundary_init(p, bpos)
    else:
        bs, bm = None, None
    n = pos.shape[0]
    cap = nbr_cap if nbr_cap is not None else n * min(max(n, 1), 1024)
    return oracle.step(p, bx, pos, vel, bs, bm, delta=delta, nbr_cap=cap), bs, bm


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
