"""The bounds-checked build (lib/libwcsph_checked.so, WCSPH_CHECKS=1) against
the default build: every device index guard stays silent on the dam break
with walls, the mesh obstacle, the 1 M tilting box and a small ensemble in
both modes, and the states after the steps are the same bits.

Each library runs in a process of its own (WCSPH_LIBRARY picks it), this file
being the script: `python tests/test_gpu_checked.py <out.npz>`.
"""
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
pytestmark = pytest.mark.gpu


def _scenes(out):
    sys.path.insert(0, str(ROOT / "fluid-simulation_b200"))
    import wcsph

    res = {}
    for name, steps in (("dam_break", 20), ("mesh_obstacle", 3), ("large_tilting", 2)):
        pre = wcsph.preset(name)
        sim = pre.simulator(device=0)
        for k in range(steps):
            if pre.info.moving_box:
                sim.set_box(pre.box_at(k + 1))
            sim.step_n(1, pre.info.delta)
        res[name + "_pos"], res[name + "_vel"] = sim.get_state()
        res[name + "_rho"] = sim.field("density")
        sim.close()
    pres = [wcsph.preset_ensemble(1, k) for k in range(8)]
    specs = [wcsph.BatchSceneSpec(fluid_pos=s.pos, box=s.box, gravity=tuple(s.params.gravity),
                                  viscosity=s.params.viscosity, boundary_pos=s.bpos) for s in pres]
    for persistent in (True, False):
        b = wcsph.BatchSimulator(pres[0].params, specs)
        b.set_persistent(persistent)
        b.step_n(5, 1e-3)
        for k in range(len(pres)):
            res[f"ens{int(persistent)}_{k}_pos"], res[f"ens{int(persistent)}_{k}_vel"] = b.get_state(k)
        b.close()
    # the library this process mapped (the parent checks it is the one it asked for)
    maps = Path("/proc/self/maps").read_text()
    res["mapped"] = np.array(sorted({ln.split()[-1] for ln in maps.splitlines() if "libwcsph" in ln}))
    np.savez(out, **res)


def _run(lib, out):
    env = dict(os.environ, WCSPH_LIBRARY=str(lib))
    r = subprocess.run([sys.executable, __file__, str(out)], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    d = np.load(out)
    assert [Path(m).name for m in d["mapped"]] == [Path(lib).name], d["mapped"]
    return d


def test_checked_build_is_silent_and_bit_identical(tmp_path):
    lib_dir = ROOT / "fluid-simulation_b200" / "lib"
    checked = lib_dir / "libwcsph_checked.so"
    assert checked.exists(), "bounds-checked library not built (make -C fluid-simulation_b200 checked)"
    # a guard that fired would make a step raise WcsphError(ERR_BOUNDS) in the child
    got = _run(checked, tmp_path / "checked.npz")
    want = _run(lib_dir / "libwcsph.so", tmp_path / "default.npz")
    assert sorted(got.files) == sorted(want.files)
    for k in want.files:
        if k == "mapped":
            continue
        assert np.array_equal(got[k].view(np.uint32), want[k].view(np.uint32)), k


if __name__ == "__main__":
    _scenes(sys.argv[1])
