#!/usr/bin/env python3
"""Generates tests/golden/ref_<fixture>.npz by running the reference's own
CUDA kernels (oracle/_ref harness, built from the reference sources by
oracle/build_ref.py) for one step from each fixture input. Needs a GPU:

    python tests/golden/make_ref_fixtures.py [out_dir]

Each fixture runs in its own process (the harness is a per-process singleton).
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(ROOT / "oracle"))


def scene_of(name: str):
    """Fixture scenes, or any preset workload with a harness variant of its name."""
    import fixtures

    if name in fixtures.NAMES:
        return fixtures.scene(name)
    sys.path.insert(0, str(ROOT / "fluid-simulation_b200"))
    import wcsph

    pre = wcsph.preset(name)
    return pre.params, pre.box, pre.pos, pre.vel, pre.bpos, pre.info.delta


def one(name: str, out_dir: Path):
    import refpath

    p, bx, pos, vel, bpos, delta = scene_of(name)
    sim = refpath.RefSim(name, pos, vel, bpos, bx)
    sim.step(delta)
    f = sim.fields()
    sim.close()
    cnt, off, nbr = f.pop("neighbors")
    dt = f.pop("dt")
    occ = f["hash_table"] != np.uint64(0xFFFFFFFFFFFFFFFF)
    np.savez_compressed(
        out_dir / f"ref_{name}.npz", nbr_counts=cnt, nbr_offsets=off, nbr_idx=nbr, dt=np.array(dt, np.float32),
        cell_keys=f.pop("hash_table")[occ], cell_start=f.pop("hash_cell_start")[occ],
        cell_end=f.pop("hash_cell_end")[occ], **f)
    print(name, "ok", int(cnt.sum()), "neighbour pairs", flush=True)


def trajectory(name: str, out_dir: Path, steps: int, full: set[int], skip: int = 0, vy: float = 0.0):
    """The reference's own trajectory of `steps` steps, after `skip` unrecorded
    steps from the scene's initial state (with `vy` added to every fluid
    particle's initial y velocity), one directory per recorded step: the
    step's input state (in_pos, in_vel),
    its sorted keys, permutation, (dt, np_dt), density, pressure and neighbour
    counts; steps in `full` also keep every field and the neighbour lists.
    A moving box is set to the scene's schedule before each step, as bench.py
    does."""
    import refpath

    p, bx, pos, vel, bpos, delta = scene_of(name)
    if vy:
        vel = np.array(vel, np.float32, copy=True)
        vel[:, 1] += np.float32(vy)
    box_at = None
    if name not in __import__("fixtures").NAMES:
        import wcsph

        pre = wcsph.preset(name)
        box_at = pre.box_at if pre.info.moving_box else None
    sim = refpath.RefSim(name, pos, vel, bpos, bx)
    for k in range(skip):
        if box_at is not None:
            sim.set_box(box_at(k + 1))
        sim.step(delta)
    in_pos, in_vel = (pos, vel) if skip == 0 else sim.state()
    n = pos.shape[0]
    for k in range(steps):
        d = out_dir / f"step_{k:04d}"
        d.mkdir(parents=True, exist_ok=True)
        if box_at is not None:
            sim.set_box(box_at(skip + k + 1))
        sim.step(delta)
        np.save(d / "in_pos.npy", in_pos)
        np.save(d / "in_vel.npy", in_vel)
        if k in full:
            f = sim.fields()
            cnt, off, nbr = f.pop("neighbors")
            np.save(d / "nbr_offsets.npy", off)
            np.save(d / "nbr_idx.npy", nbr)
            for key in ("position", "velocity", "pressure_accel", "non_pressure_accel", "normal"):
                np.save(d / f"{key}.npy", f[key])
            if bpos is not None:
                np.save(d / "boundary_position.npy", f["boundary_position"])
                np.save(d / "boundary_mass.npy", f["boundary_mass"])
            keys, perm, rho, prs, dt = f["sorted_keys"], f["permutation"], f["density"], f["pressure"], f["dt"]
        else:
            keys = np.empty(n, np.uint64)
            perm = np.empty(n, np.uint32)
            rho = np.empty(n, np.float32)
            prs = np.empty(n, np.float32)
            cnt = np.empty(n, np.uint32)
            dt2 = np.empty(2, np.float32)
            sim._get(sorted_keys=keys, permutation=perm, density=rho, pressure=prs, nbr_counts=cnt, dt=dt2)
            dt = (float(dt2[0]), float(dt2[1]))
        np.save(d / "sorted_keys.npy", keys)
        np.save(d / "permutation.npy", perm)
        np.save(d / "density.npy", rho)
        np.save(d / "pressure.npy", prs)
        np.save(d / "nbr_counts.npy", cnt)
        np.save(d / "dt.npy", np.array(dt, np.float32))
        in_pos, in_vel = sim.state()
    sim.close()
    print(name, "trajectory ok", steps, "steps", flush=True)


def main():
    # make_ref_fixtures.py [out_dir [scene [--trajectory STEPS [--skip N] [--vy V] [FULL_STEP ...]]]]
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE
    if len(sys.argv) > 3 and sys.argv[3] == "--trajectory":
        rest = sys.argv[5:]
        opt = {"--skip": 0, "--vy": 0.0}
        while rest[:1] and rest[0] in opt:
            opt[rest[0]] = type(opt[rest[0]])(rest[1])
            rest = rest[2:]
        trajectory(sys.argv[2], out, int(sys.argv[4]), {int(x) for x in rest}, opt["--skip"], opt["--vy"])
        return
    if len(sys.argv) > 2:
        one(sys.argv[2], out)
        return
    import fixtures
    for name in fixtures.NAMES:
        subprocess.run([sys.executable, __file__, str(out), name], check=True)


if __name__ == "__main__":
    main()
