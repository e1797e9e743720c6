"""ctypes driver of the reference-kernel harness (oracle/_ref/<variant>).

TEST AND BASELINE INFRASTRUCTURE: runs the reference's own CUDA kernels
(compiled from its sources by oracle/build_ref.py) replaying its step.
Used by the parity tests, tests/golden/make_ref_fixtures.py and
`bench.py --impl reference`; never by the product.
"""
from __future__ import annotations

import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"


def available(variant: str) -> bool:
    return (REF_DIR / variant / "librefpath.so").exists()


def box_floats(box) -> np.ndarray:
    """wcsph.Box -> 38 floats: min[3], max[3], model[16], model_inv[16]."""
    return np.array(list(box.min) + list(box.max) + list(box.model) + list(box.model_inv), np.float32)


class RefSim:
    """One reference-path simulation (one per process: the harness is a singleton)."""

    def __init__(self, variant: str, pos, vel, bpos, box, device: int = 0):
        """box: a wcsph.Box or its 38 floats (min, max, model, model_inv)."""
        path = REF_DIR / variant / "librefpath.so"
        if not path.exists():
            raise OSError(f"reference harness {path} not built (oracle/build_ref.py)")
        L = C.CDLL(str(path))
        vp = C.c_void_p
        L.ref_create.argtypes = [vp, vp, C.c_uint, vp, C.c_uint, vp, C.c_int]
        L.ref_step.argtypes = [C.c_float]
        L.ref_set_box.argtypes = [vp]
        L.ref_time_steps.argtypes = [C.c_int, C.c_float, vp]
        L.ref_time_steps.restype = C.c_float
        L.ref_get_fields.argtypes = [vp] * 12 + [C.c_ulonglong, vp, vp]
        L.ref_get_hash.argtypes = [vp, vp, vp, vp]
        L.ref_get_boundary.argtypes = [vp, vp]
        L.ref_set_state.argtypes = [vp, vp]
        self.L = L
        self.n = pos.shape[0]
        self.nb = 0 if bpos is None else bpos.shape[0]
        self._pos = np.ascontiguousarray(pos, np.float32)
        self._vel = np.ascontiguousarray(vel, np.float32)
        self._bpos = None if bpos is None else np.ascontiguousarray(bpos, np.float32)
        b = np.ascontiguousarray(box, np.float32) if isinstance(box, np.ndarray) else box_floats(box)
        st = L.ref_create(self._pos.ctypes.data, self._vel.ctypes.data, self.n,
                          None if self._bpos is None else self._bpos.ctypes.data, self.nb, b.ctypes.data, device)
        if st != 0:
            raise RuntimeError(f"ref_create failed ({st}): variant {variant} was built for other particle counts")

    def step(self, delta: float):
        if self.L.ref_step(delta) != 0:
            raise RuntimeError("ref_step failed")

    def set_box(self, box):
        b = box_floats(box)
        self.L.ref_set_box(b.ctypes.data)

    def time_steps(self, k: int, delta: float, boxes=None) -> float:
        """boxes: per-step wcsph.Box objects or a [k, 38] float array."""
        arr = None
        if boxes is not None:
            arr = (np.ascontiguousarray(boxes, np.float32) if isinstance(boxes, np.ndarray)
                   else np.ascontiguousarray(np.stack([box_floats(b) for b in boxes]), np.float32))
        return self.L.ref_time_steps(k, delta, None if arr is None else arr.ctypes.data)

    def set_state(self, pos, vel):
        """Next step starts from this state (float32 [n, 4] each)."""
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        if self.L.ref_set_state(pos.ctypes.data, vel.ctypes.data) != 0:
            raise RuntimeError("ref_set_state failed")

    def _get(self, **want):
        """ref_get_fields with only the requested host arrays (others NULL)."""
        order = ("position", "velocity", "density", "pressure", "pressure_accel", "non_pressure_accel", "normal",
                 "sorted_keys", "permutation", "nbr_counts", "nbr_offsets", "nbr_idx")
        ptr = [None if want.get(k) is None else want[k].ctypes.data for k in order]
        total = C.c_ulonglong()
        cap = want["nbr_idx"].size if want.get("nbr_idx") is not None else 0
        dt = want.get("dt")
        self.L.ref_get_fields(*ptr, cap, C.byref(total), None if dt is None else dt.ctypes.data)
        return total.value

    def state(self):
        """(positions, velocities) of the last step, in its sorted order."""
        pos = np.empty((self.n, 4), np.float32)
        vel = np.empty((self.n, 4), np.float32)
        self._get(position=pos, velocity=vel)
        return pos, vel

    def last_dt(self):
        dt = np.empty(2, np.float32)
        self._get(dt=dt)
        return float(dt[0]), float(dt[1])

    def fields(self) -> dict:
        n = self.n
        out = {k: np.empty((n, 4), np.float32) for k in ("position", "velocity", "pressure_accel",
                                                          "non_pressure_accel", "normal")}
        out["density"] = np.empty(n, np.float32)
        out["pressure"] = np.empty(n, np.float32)
        out["sorted_keys"] = np.empty(n, np.uint64)
        out["permutation"] = np.empty(n, np.uint32)
        cnt = np.empty(n, np.uint32)
        off = np.empty(n, np.uint32)
        cap = n * 96
        nbr = np.empty(cap, np.uint32)
        total = C.c_ulonglong()
        dt = np.empty(2, np.float32)
        p = lambda a: a.ctypes.data  # noqa: E731
        self.L.ref_get_fields(p(out["position"]), p(out["velocity"]), p(out["density"]), p(out["pressure"]),
                              p(out["pressure_accel"]), p(out["non_pressure_accel"]), p(out["normal"]),
                              p(out["sorted_keys"]), p(out["permutation"]), p(cnt), p(off), p(nbr), cap,
                              C.byref(total), p(dt))
        out["neighbors"] = (cnt, off, nbr[: total.value].copy())
        out["dt"] = (float(dt[0]), float(dt[1]))
        T = C.c_uint()
        self.L.ref_get_hash(None, None, None, C.byref(T))
        tab = np.empty(T.value, np.uint64)
        cs = np.empty(T.value, np.uint32)
        ce = np.empty(T.value, np.uint32)
        self.L.ref_get_hash(p(tab), p(cs), p(ce), None)
        out["hash_table"], out["hash_cell_start"], out["hash_cell_end"] = tab, cs, ce
        if self.nb:
            bp = np.empty((self.nb, 4), np.float32)
            bm = np.empty(self.nb, np.float32)
            self.L.ref_get_boundary(p(bp), p(bm))
            out["boundary_position"], out["boundary_mass"] = bp, bm
        return out

    def close(self):
        self.L.ref_destroy()


_TIME_VARIANT = r"""
import json, sys, time
import numpy as np
sys.path.insert(0, sys.argv[1])
import refpath
variant, npz, warmup, steps = sys.argv[2], sys.argv[3], int(sys.argv[4]), int(sys.argv[5])
d = np.load(npz)
bpos = d["bpos"] if d["bpos"].size else None
boxes = d["boxes"] if d["boxes"].size else None
sim = refpath.RefSim(variant, d["pos"], d["vel"], bpos, d["box0"], device=0)
delta = float(d["delta"])
sim.time_steps(warmup, delta, None if boxes is None else boxes[:warmup])
t0 = time.perf_counter()
ms = sim.time_steps(steps, delta, None if boxes is None else boxes[warmup:warmup + steps])
wall = time.perf_counter() - t0
sim.close()
print(json.dumps({"ms": ms, "wall": wall, "own_library_mapped": refpath.own_library_mapped()}))
"""


def own_library_mapped() -> bool:
    """True when this project's library (libwcsph) is mapped into the calling
    process: the reference arm's timing processes must never load it."""
    try:
        with open("/proc/self/maps") as fh:
            return any("libwcsph" in line for line in fh)
    except OSError:
        return False


def bench_line(args, metric: str, config_of) -> dict:
    """`bench.py --impl reference`: the reference CUDA path on the same workload.

    The scene comes from oracle/scenes.py (numpy, bit-identical to the
    library's preset), so no process of this arm loads the library. Every
    built block size of the reference tuner's space (the frozen config of its
    largest shipped scene uses 32; variants `<workload>_b<block>`) runs the
    same warm-up + timed steps from the same initial state, each in a process
    of its own (every harness library carries its own CUDA runtime and
    Thrust); the fastest is the line's value and all are listed.
    `config_of(particles, dt, ms_per_step)` builds the configuration block the
    way bench.py builds its own line's, so that both lines carry the same keys."""
    import subprocess
    import tempfile

    import scenes

    variants = [v for v in [args.workload] + [f"{args.workload}_b{b}" for b in (64, 128, 256, 512)] if available(v)]
    if not variants:
        return {"impl": "reference", "unavailable": f"reference harness for {args.workload} not built "
                                                    f"(oracle/build_ref.py needs the reference sources)"}
    sc = scenes.scene(args.workload, seed=args.seed)
    n = sc.pos.shape[0]
    total = args.warmup + args.steps
    boxes = np.stack([sc.box_at(k + 1) for k in range(total)]) if sc.moving else np.zeros((0, 38), np.float32)
    sweep = {}
    best = None
    mapped = False
    with tempfile.TemporaryDirectory() as tmp:
        npz = Path(tmp) / "scene.npz"
        np.savez(npz, pos=sc.pos, vel=sc.vel, bpos=sc.bpos if sc.bpos is not None else np.zeros((0, 4), np.float32),
                 box0=sc.box0, boxes=boxes, delta=np.float32(sc.delta))
        for variant in variants:
            block = 32 if variant == args.workload else int(variant.rsplit("_b", 1)[1])
            r = subprocess.run([sys.executable, "-c", _TIME_VARIANT, str(HERE), variant, str(npz),
                                str(args.warmup), str(args.steps)],
                               capture_output=True, text=True, timeout=900)
            if r.returncode != 0 or not r.stdout.strip():
                sweep[str(block)] = f"failed (exit {r.returncode})"
                continue
            t = json.loads(r.stdout.strip().splitlines()[-1])
            mapped = mapped or bool(t["own_library_mapped"])
            sweep[str(block)] = t["ms"] / args.steps
            if best is None or t["ms"] < best[0]:
                best = (t["ms"], t["wall"], block)
    if best is None:
        return {"impl": "reference", "unavailable": f"every reference harness variant failed: {sweep}"}
    ms, wall, block = best
    value = n * args.steps / (ms * 1e-3)
    return {
        "impl": "reference", "metric": metric, "value": value, "unit": metric, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: the same seeded scene as --impl ours (oracle/scenes.py, bit-identical to the preset)",
        "config": config_of(n, sc.delta, ms / args.steps),
        "reference": {"path": "reference kernels (src/cuda/tuning/kernels; neighbour lists, table mult 4, cell mult 1 "
                              "as in the largest shipped scene's frozen config) + Thrust sort/gather/scan/reduce, "
                              "host CFL readback",
                      "block": block, "ms_per_step_by_block": sweep, "wall_s": wall,
                      "own_library_mapped": mapped},
        "cpu_baseline": {"value": value, "unit": metric, "cores": 0, "kind": "reference",
                         "sample": f"{args.steps} steps of the reference CUDA path, fastest block size "
                                   f"(the reference has no CPU solver)"},
        "e2e": {"value": value, "unit": metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
