"""ctypes binding of the CPU oracle (liboracle.so built from sph_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker. The product never imports it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
LIB_PATH = ORACLE_DIR / "lib" / "liboracle.so"

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise OSError(f"{LIB_PATH} not built; run `make -C oracle`")
        L = C.CDLL(str(LIB_PATH))
        vp = C.c_void_p
        L.oracle_morton_keys.argtypes = [vp, C.c_uint32, C.c_float, vp]
        L.oracle_sort_perm.argtypes = [vp, C.c_uint32, vp]
        L.oracle_cell_ranges.argtypes = [vp, C.c_uint32, C.c_float, vp, vp, vp]
        L.oracle_cell_ranges.restype = C.c_uint32
        L.oracle_boundary_init.argtypes = [vp, C.c_uint32, vp, vp, vp]
        L.oracle_step_flat.argtypes = [vp, vp, C.c_uint32, vp, vp, C.c_uint32, vp, vp, C.c_float,
                                       vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, C.c_uint64, vp]
        L.oracle_step_flat.restype = C.c_int
        L.oracle_metrics.argtypes = [vp, C.c_uint32, vp, vp, vp]
        L.oracle_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def morton_keys(pos: np.ndarray, cell_size: float) -> np.ndarray:
    pos = np.ascontiguousarray(pos, np.float32)
    out = np.empty(pos.shape[0], np.uint64)
    lib().oracle_morton_keys(_p(pos), pos.shape[0], cell_size, _p(out))
    return out


def sort_perm(keys: np.ndarray) -> np.ndarray:
    keys = np.ascontiguousarray(keys, np.uint64)
    out = np.empty(keys.shape[0], np.uint32)
    lib().oracle_sort_perm(_p(keys), keys.shape[0], _p(out))
    return out


def cell_ranges(sorted_pos: np.ndarray, cell_size: float):
    sorted_pos = np.ascontiguousarray(sorted_pos, np.float32)
    n = sorted_pos.shape[0]
    k = np.empty(max(n, 1), np.uint64)
    s = np.empty(max(n, 1), np.uint32)
    e = np.empty(max(n, 1), np.uint32)
    nc = lib().oracle_cell_ranges(_p(sorted_pos), n, cell_size, _p(k), _p(s), _p(e))
    return k[:nc], s[:nc], e[:nc]


def boundary_init(params, bpos: np.ndarray):
    bpos = np.ascontiguousarray(bpos, np.float32)
    nb = bpos.shape[0]
    out = np.empty_like(bpos)
    mass = np.empty(nb, np.float64)
    lib().oracle_boundary_init(C.byref(params), nb, _p(bpos), _p(out), _p(mass))
    return out, mass


@dataclass
class StepResult:
    keys: np.ndarray
    perm: np.ndarray
    rho: np.ndarray
    prs: np.ndarray
    ap: np.ndarray
    anp: np.ndarray
    normal: np.ndarray
    pos: np.ndarray
    vel: np.ndarray
    dt_p: float
    np_dt: float
    nbr_counts: np.ndarray
    nbr_offsets: np.ndarray
    nbr_idx: np.ndarray


def step(params, box, pos, vel, bpos_sorted=None, bmass=None, delta=0.01, nbr_cap=None) -> StepResult:
    """One FP64 oracle step; outputs in sorted order (like the CUDA path)."""
    pos = np.ascontiguousarray(pos, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    n = pos.shape[0]
    nb = 0 if bpos_sorted is None else bpos_sorted.shape[0]
    bpos_sorted = np.zeros((1, 4), np.float32) if nb == 0 else np.ascontiguousarray(bpos_sorted, np.float32)
    bmass = np.zeros(1, np.float64) if nb == 0 else np.ascontiguousarray(bmass, np.float64)
    cap = nbr_cap if nbr_cap is not None else max(n * 96, 1)
    r = StepResult(keys=np.empty(n, np.uint64), perm=np.empty(n, np.uint32), rho=np.empty(n),
                   prs=np.empty(n), ap=np.empty((n, 4)), anp=np.empty((n, 4)), normal=np.empty((n, 4)),
                   pos=np.empty((n, 4)), vel=np.empty((n, 4)), dt_p=0.0, np_dt=0.0,
                   nbr_counts=np.empty(n, np.uint32), nbr_offsets=np.empty(n, np.uint32),
                   nbr_idx=np.empty(cap, np.uint32))
    dt = np.empty(2, np.float64)
    total = C.c_uint64()
    lib().oracle_step_flat(C.byref(params), C.byref(box), n, _p(pos), _p(vel), nb, _p(bpos_sorted), _p(bmass),
                           delta, _p(r.keys), _p(r.perm), _p(r.rho), _p(r.prs), _p(r.ap), _p(r.anp),
                           _p(r.normal), _p(r.pos), _p(r.vel), _p(dt), _p(r.nbr_counts), _p(r.nbr_offsets),
                           _p(r.nbr_idx), cap, C.byref(total))
    if total.value > cap:
        raise RuntimeError("oracle neighbour capacity exceeded")
    r.nbr_idx = r.nbr_idx[: total.value]
    r.dt_p, r.np_dt = float(dt[0]), float(dt[1])
    return r


def metrics(params, vel: np.ndarray):
    vel = np.ascontiguousarray(vel, np.float32)
    a, b = C.c_double(), C.c_double()
    lib().oracle_metrics(C.byref(params), vel.shape[0], _p(vel), C.byref(a), C.byref(b))
    return a.value, b.value


def num_threads() -> int:
    return lib().oracle_num_threads()
