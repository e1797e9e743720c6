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


def main():
    # make_ref_fixtures.py [out_dir [scene]]
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE
    if len(sys.argv) > 2:
        one(sys.argv[2], out)
        return
    import fixtures
    for name in fixtures.NAMES:
        subprocess.run([sys.executable, __file__, str(out), name], check=True)


if __name__ == "__main__":
    main()
