"""Python binding of the WCSPH C ABI (include/wcsph.h) via ctypes.

Mirrors the reference's solver interface so tests and tools read like the
reference's own code:

    reference (petbab/fluid-simulation)          here
    FluidSimulator / CUDASPHSimulator            CUDASPHSimulator
      update(delta)  sph.cu:31-60                  .update(delta)
      reset()        sph.cu:73-82                  .reset()
      get_fluid_particles()                        .get_fluid_particles()
      compute_state_metrics() sph.cu:180-197       .compute_state_metrics()
    Snapshot::save / Snapshot::load              .snapshot_save / .snapshot_load
      snapshot.cu:10-106                           (raise SnapshotError with the
                                                    reference's message text)

The native library is ``lib/libwcsph.so`` next to this package; importing
this module fails loudly when it has not been built. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from dataclasses import dataclass
from pathlib import Path

import numpy as np

_PKG_ROOT = Path(__file__).resolve().parent.parent
# WCSPH_LIBRARY selects another build of the same ABI for a process, e.g. the
# bounds-checked lib/libwcsph_checked.so (`make -C fluid-simulation_b200 checked`).
CHECKED_LIB_PATH = _PKG_ROOT / "lib" / "libwcsph_checked.so"
LIB_PATH = Path(os.environ["WCSPH_LIBRARY"]) if os.environ.get("WCSPH_LIBRARY") else _PKG_ROOT / "lib" / "libwcsph.so"
HEADER_PATH = _PKG_ROOT.parent / "include" / "wcsph.h"

# ---- status codes (enum wcsph_status) ---------------------------------------
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_CUDA = 2
ERR_OUT_OF_MEMORY = 3
ERR_IO = 4
ERR_SNAPSHOT_MAGIC = 5
ERR_SNAPSHOT_VERSION = 6
ERR_SNAPSHOT_APP_NAME = 7
ERR_SNAPSHOT_COUNT = 8
ERR_SNAPSHOT_TRUNCATED = 9
ERR_HASH_FULL = 10
ERR_NEIGHBOR_OVERFLOW = 11
ERR_DEVICE_TIMEOUT = 12
ERR_NO_DEVICE = 13
ERR_CONFIG = 14
ERR_NOT_SUPPORTED = 15
ERR_STATE = 16
ERR_BOUNDS = 17   # bounds-checked build only: a device index guard fired

FORCE_NONE, FORCE_CONSTANT, FORCE_FOUNTAIN, FORCE_VORTEX = 0, 1, 2, 3
SEARCH_MCMC, SEARCH_RANDOM, SEARCH_FULL = 0, 1, 2

FIELD = {
    "position": 0, "velocity": 1, "density": 2, "pressure": 3, "pressure_accel": 4,
    "non_pressure_accel": 5, "normal": 6, "morton_keys": 7, "permutation": 8,
    "hash_table": 9, "hash_cell_start": 10, "hash_cell_end": 11,
    "boundary_position": 12, "boundary_mass": 13,
}
_FIELD_DTYPE = {
    0: (np.float32, 4), 1: (np.float32, 4), 2: (np.float32, 1), 3: (np.float32, 1),
    4: (np.float32, 4), 5: (np.float32, 4), 6: (np.float32, 4), 7: (np.uint64, 1),
    8: (np.uint32, 1), 9: (np.uint64, 1), 10: (np.uint32, 1), 11: (np.uint32, 1),
    12: (np.float32, 4), 13: (np.float32, 1),
}


class WcsphError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status
        self.message = message


class SnapshotError(WcsphError):
    """Snapshot::load / Snapshot::save failure (reference returns the text)."""


class Params(C.Structure):
    _fields_ = [
        ("particle_radius", C.c_float), ("rest_density", C.c_float), ("stiffness", C.c_float),
        ("exponent", C.c_float), ("max_density_ratio", C.c_float), ("viscosity", C.c_float),
        ("surface_tension", C.c_float), ("gravity", C.c_float * 3), ("cfl_factor", C.c_float),
        ("max_time_step", C.c_float), ("min_time_step", C.c_float),
        ("non_pressure_max_time_step", C.c_float), ("collision_buffer_mult", C.c_float),
        ("elasticity", C.c_float), ("cell_size_mult", C.c_float), ("table_size_mult", C.c_uint32),
        ("external_force", C.c_int32), ("external_force_param", C.c_float * 4),
    ]


class Box(C.Structure):
    _fields_ = [("min", C.c_float * 3), ("max", C.c_float * 3), ("model", C.c_float * 16),
                ("model_inv", C.c_float * 16)]


class Scene(C.Structure):
    _fields_ = [("fluid_n", C.c_uint32), ("fluid_pos", C.POINTER(C.c_float)),
                ("fluid_vel", C.POINTER(C.c_float)), ("boundary_n", C.c_uint32),
                ("boundary_pos", C.POINTER(C.c_float)), ("box", Box)]


class Camera(C.Structure):
    """wcsph_camera: column-major projection and view matrices, eye position."""
    _fields_ = [("projection", C.c_float * 16), ("view", C.c_float * 16), ("eye", C.c_float * 3)]


class RenderOpts(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("radius", C.c_float),
                ("show_boundary", C.c_int), ("field", C.c_int), ("normalize", C.c_int),
                ("min_value", C.c_float), ("max_value", C.c_float), ("background", C.c_float * 3),
                ("max_pixels", C.c_int)]


class PresetInfo(C.Structure):
    _fields_ = [("params", Params), ("box", Box), ("fluid_n", C.c_uint32), ("boundary_n", C.c_uint32),
                ("delta", C.c_float), ("steps", C.c_int32), ("sim_time", C.c_float), ("moving_box", C.c_int32)]


class BatchScene(C.Structure):
    _fields_ = [("fluid_n", C.c_uint32), ("fluid_pos", C.POINTER(C.c_float)),
                ("fluid_vel", C.POINTER(C.c_float)), ("boundary_n", C.c_uint32),
                ("boundary_pos", C.POINTER(C.c_float)), ("box", Box), ("gravity", C.c_float * 3),
                ("viscosity", C.c_float)]


_lib = None


def load_library(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads libwcsph.so (raises OSError when it is missing: no fallback)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise OSError(f"native library {p} is not built; run `make -C fluid-simulation_b200`")
    lib = C.CDLL(str(p))
    f = C.POINTER(C.c_float)
    vp = C.c_void_p
    sig = {
        "wcsph_abi_version": (C.c_int, []),
        "wcsph_default_params": (None, [C.POINTER(Params)]),
        "wcsph_identity_box": (None, [f, f, C.POINTER(Box)]),
        "wcsph_status_string": (C.c_char_p, [C.c_int]),
        "wcsph_create": (C.c_int, [C.POINTER(Params), C.POINTER(Scene), C.c_int, C.POINTER(vp)]),
        "wcsph_destroy": (C.c_int, [vp]),
        "wcsph_last_error": (C.c_char_p, [vp]),
        "wcsph_step": (C.c_int, [vp, C.c_float]),
        "wcsph_step_n": (C.c_int, [vp, C.c_int, C.c_float]),
        "wcsph_synchronize": (C.c_int, [vp]),
        "wcsph_reset": (C.c_int, [vp]),
        "wcsph_set_box": (C.c_int, [vp, C.POINTER(Box)]),
        "wcsph_set_params": (C.c_int, [vp, C.POINTER(Params)]),
        "wcsph_get_params": (C.c_int, [vp, C.POINTER(Params)]),
        "wcsph_get_state": (C.c_int, [vp, f, f]),
        "wcsph_set_state": (C.c_int, [vp, f, f]),
        "wcsph_snapshot_save": (C.c_int, [vp, C.c_char_p, C.c_char_p]),
        "wcsph_snapshot_load": (C.c_int, [vp, C.c_char_p, C.c_char_p]),
        "wcsph_snapshot_read_header": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_uint32)]),
        "wcsph_snapshot_read": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint32, f, f]),
        "wcsph_snapshot_write": (C.c_int, [C.c_char_p, C.c_char_p, C.c_uint32, f, f]),
        "wcsph_metrics": (C.c_int, [vp, f, f]),
        "wcsph_last_dt": (C.c_int, [vp, f, f]),
        "wcsph_field_size": (C.c_int, [vp, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32)]),
        "wcsph_get_field": (C.c_int, [vp, C.c_int, vp, C.c_uint64]),
        "wcsph_get_device_field": (C.c_int, [vp, C.c_int, C.POINTER(vp)]),
        "wcsph_get_neighbors": (C.c_int, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                          C.POINTER(C.c_uint32), C.c_uint64, C.POINTER(C.c_uint64)]),
        "wcsph_get_stream": (C.c_int, [vp, C.POINTER(vp)]),
        "wcsph_time_steps": (C.c_int, [vp, C.c_int, C.c_float, f]),
        "wcsph_kernel_timings": (C.c_int, [vp, C.POINTER(C.c_char_p), f, C.c_int]),
        "wcsph_launches_per_step": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "wcsph_set_tuning": (C.c_int, [vp, C.c_int, C.c_float, C.c_char_p]),
        "wcsph_was_tuning_step": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "wcsph_save_config": (C.c_int, [vp, C.c_char_p]),
        "wcsph_save_tuning_results": (C.c_int, [vp, C.c_char_p]),
        "wcsph_reset_tuning": (C.c_int, [vp]),
        "wcsph_make_lattice": (C.c_int, [f, C.POINTER(C.c_uint32), C.c_float, C.c_float, C.c_uint64, f]),
        "wcsph_make_velocities": (C.c_int, [C.c_uint32, C.c_float, C.c_uint64, f]),
        "wcsph_sample_box_walls": (C.c_int, [f, f, C.c_float, f, C.POINTER(C.c_uint32)]),
        "wcsph_sample_icosphere": (C.c_int, [f, C.c_float, C.c_int, C.c_float, f, C.POINTER(C.c_uint32)]),
        "wcsph_sample_triangles": (C.c_int, [f, C.c_uint32, C.c_float, f, C.POINTER(C.c_uint32)]),
        "wcsph_load_obj": (C.c_int, [C.c_char_p, C.c_int, f, f, C.POINTER(C.c_uint32)]),
        "wcsph_preset": (C.c_int, [C.c_char_p, C.c_uint64, C.POINTER(PresetInfo), f, f, f]),
        "wcsph_preset_box": (C.c_int, [C.c_char_p, C.c_int64, C.c_float, C.POINTER(Box)]),
        "wcsph_preset_ensemble": (C.c_int, [C.c_uint64, C.c_uint32, C.POINTER(PresetInfo), f, f, f]),
        "wcsph_batch_create": (C.c_int, [C.POINTER(Params), C.POINTER(BatchScene), C.c_uint32, C.c_int,
                                         C.POINTER(vp)]),
        "wcsph_batch_destroy": (C.c_int, [vp]),
        "wcsph_batch_set_persistent": (C.c_int, [vp, C.c_int]),
        "wcsph_batch_step_n": (C.c_int, [vp, C.c_int, C.c_float]),
        "wcsph_batch_time_steps": (C.c_int, [vp, C.c_int, C.c_float, f]),
        "wcsph_batch_get_state": (C.c_int, [vp, C.c_uint32, f, f]),
        "wcsph_batch_metrics": (C.c_int, [vp, f, f]),
        "wcsph_batch_last_error": (C.c_char_p, [vp]),
        "wcsph_rollout_forward": (C.c_int, [vp, C.c_int, C.c_float, C.c_int, f, f]),
        "wcsph_rollout_backward": (C.c_int, [vp, f, f, f]),
        "wcsph_sort_keys_static": (C.c_int, [vp, C.c_uint32, vp, vp]),
        "wcsph_test_stall_sort": (C.c_int, [C.c_int]),
        "wcsph_camera_look": (None, [f, C.c_float, C.c_float, C.c_uint32, C.c_uint32, C.POINTER(Camera)]),
        "wcsph_default_render_opts": (None, [C.POINTER(RenderOpts)]),
        "wcsph_render": (C.c_int, [vp, C.POINTER(Camera), C.POINTER(RenderOpts), vp, f]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def header_symbols(header: Path = HEADER_PATH) -> list[str]:
    """Every function the C header declares."""
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wcsph_[a-z0-9_]+)\s*\(", text)))


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def default_params(**overrides) -> Params:
    p = Params()
    load_library().wcsph_default_params(C.byref(p))
    for k, v in overrides.items():
        if k == "gravity":
            p.gravity[:] = [float(x) for x in v]
        elif k == "external_force_param":
            p.external_force_param[:] = [float(x) for x in v] + [0.0] * (4 - len(v))
        else:
            setattr(p, k, v)
    return p


def box(mn, mx, model: np.ndarray | None = None) -> Box:
    """Collision box; `model` is a 4x4 (row-major numpy) model matrix."""
    b = Box()
    lib = load_library()
    lib.wcsph_identity_box((C.c_float * 3)(*mn), (C.c_float * 3)(*mx), C.byref(b))
    if model is not None:
        m = np.asarray(model, dtype=np.float64)
        inv = np.linalg.inv(m)
        b.model[:] = [float(x) for x in m.T.reshape(-1)]       # column-major like glm
        b.model_inv[:] = [float(x) for x in inv.T.reshape(-1)]
    return b


def rotation_z(angle: float) -> np.ndarray:
    c, s = np.cos(angle), np.sin(angle)
    m = np.eye(4)
    m[0, 0], m[0, 1], m[1, 0], m[1, 1] = c, -s, s, c
    return m


def make_lattice(origin, dims, radius, jitter=0.0, seed=0) -> np.ndarray:
    n = int(dims[0]) * int(dims[1]) * int(dims[2])
    out = np.empty((n, 4), np.float32)
    st = load_library().wcsph_make_lattice((C.c_float * 3)(*origin), (C.c_uint32 * 3)(*dims),
                                           radius, jitter, seed, fptr(out))
    _check(st, None)
    return out


def make_velocities(n, sigma, seed=0) -> np.ndarray:
    out = np.empty((n, 4), np.float32)
    _check(load_library().wcsph_make_velocities(n, sigma, seed, fptr(out)), None)
    return out


def sample_box_walls(mn, mx, spacing) -> np.ndarray:
    lib = load_library()
    cnt = C.c_uint32()
    _check(lib.wcsph_sample_box_walls((C.c_float * 3)(*mn), (C.c_float * 3)(*mx), spacing, None,
                                      C.byref(cnt)), None)
    out = np.empty((cnt.value, 4), np.float32)
    _check(lib.wcsph_sample_box_walls((C.c_float * 3)(*mn), (C.c_float * 3)(*mx), spacing, fptr(out),
                                      C.byref(cnt)), None)
    return out


def sample_icosphere(center, radius, level, voxel) -> np.ndarray:
    lib = load_library()
    cnt = C.c_uint32()
    _check(lib.wcsph_sample_icosphere((C.c_float * 3)(*center), radius, level, voxel, None, C.byref(cnt)), None)
    out = np.empty((cnt.value, 4), np.float32)
    _check(lib.wcsph_sample_icosphere((C.c_float * 3)(*center), radius, level, voxel, fptr(out),
                                      C.byref(cnt)), None)
    return out


def load_obj(path, normalize: bool = False, model: np.ndarray | None = None) -> np.ndarray:
    """Triangles [n, 3, 3] of the first shape of a .obj mesh (wcsph_load_obj:
    the reference's Geometry::from_file + load_triangles)."""
    lib = load_library()
    m = None if model is None else np.ascontiguousarray(model, np.float32).reshape(16)
    n = C.c_uint32()
    _check(lib.wcsph_load_obj(str(path).encode(), int(normalize), fptr(m), None, C.byref(n)), None)
    out = np.empty((n.value, 3, 3), np.float32)
    _check(lib.wcsph_load_obj(str(path).encode(), int(normalize), fptr(m), fptr(out), C.byref(n)), None)
    return out


def sample_triangles(tris: np.ndarray, voxel: float) -> np.ndarray:
    """Boundary particles of a triangle soup by surface voxelisation (wcsph_sample_triangles)."""
    lib = load_library()
    t = np.ascontiguousarray(tris, np.float32).reshape(-1, 9)
    n = C.c_uint32()
    _check(lib.wcsph_sample_triangles(fptr(t), t.shape[0], voxel, None, C.byref(n)), None)
    out = np.empty((n.value, 4), np.float32)
    _check(lib.wcsph_sample_triangles(fptr(t), t.shape[0], voxel, fptr(out), C.byref(n)), None)
    return out


@dataclass
class Preset:
    name: str
    info: PresetInfo
    pos: np.ndarray
    vel: np.ndarray
    bpos: np.ndarray | None

    @property
    def params(self) -> Params:
        return self.info.params

    @property
    def box(self) -> Box:
        return self.info.box

    def box_at(self, updates: int) -> Box:
        b = Box()
        _check(load_library().wcsph_preset_box(self.name.encode(), updates, self.info.delta, C.byref(b)), None)
        return b

    def simulator(self, device: int = -1) -> "CUDASPHSimulator":
        return CUDASPHSimulator(self.params, self.pos, self.box, fluid_vel=self.vel, boundary_pos=self.bpos,
                                device=device)


def _fill(info, fn):
    pos = np.empty((info.fluid_n, 4), np.float32)
    vel = np.empty((info.fluid_n, 4), np.float32)
    bpos = np.empty((info.boundary_n, 4), np.float32) if info.boundary_n else None
    _check(fn(fptr(pos), fptr(vel), fptr(bpos)), None)
    return pos, vel, bpos


def preset(name: str, seed: int = 0) -> Preset:
    """Named scene (wcsph_preset): reference apps and benchmark workloads."""
    lib = load_library()
    info = PresetInfo()
    _check(lib.wcsph_preset(name.encode(), seed, C.byref(info), None, None, None), None)
    pos, vel, bpos = _fill(info, lambda a, b, c: lib.wcsph_preset(name.encode(), seed, C.byref(info), a, b, c))
    return Preset(name, info, pos, vel, bpos)


def preset_ensemble(seed: int, k: int) -> Preset:
    lib = load_library()
    info = PresetInfo()
    _check(lib.wcsph_preset_ensemble(seed, k, C.byref(info), None, None, None), None)
    pos, vel, bpos = _fill(info, lambda a, b, c: lib.wcsph_preset_ensemble(seed, k, C.byref(info), a, b, c))
    return Preset(f"ensemble_{k}", info, pos, vel, bpos)


def _check(status: int, ctx, lib=None):
    if status == OK:
        return
    lib = lib or load_library()
    msg = lib.wcsph_last_error(ctx).decode(errors="replace") if lib else ""
    if status in (ERR_SNAPSHOT_MAGIC, ERR_SNAPSHOT_VERSION, ERR_SNAPSHOT_APP_NAME, ERR_SNAPSHOT_COUNT,
                  ERR_SNAPSHOT_TRUNCATED) or (status == ERR_IO and "Snapshot" in msg):
        raise SnapshotError(status, msg)
    raise WcsphError(status, msg or lib.wcsph_status_string(status).decode())


def camera_look(position=(0.0, 0.0, 2.5), yaw=np.radians(270.0), pitch=0.0, width=640, height=480) -> Camera:
    """The reference's Camera(position, yaw, pitch, width, height); the default
    is its start view (src/application.cu:16)."""
    cam = Camera()
    pos = (C.c_float * 3)(*[float(x) for x in position])
    load_library().wcsph_camera_look(pos, float(yaw), float(pitch), width, height, C.byref(cam))
    return cam


def render_opts(**kw) -> RenderOpts:
    o = RenderOpts()
    load_library().wcsph_default_render_opts(C.byref(o))
    for k, v in kw.items():
        if k == "field" and isinstance(v, str):
            v = FIELD[v]
        if k == "background":
            v = (C.c_float * 3)(*v)
        setattr(o, k, v)
    return o


def write_ppm(path, rgba: np.ndarray) -> None:
    """Binary PPM (P6) of an RGBA image [H, W, 4]."""
    h, w = rgba.shape[:2]
    with open(path, "wb") as fh:
        fh.write(b"P6\n%d %d\n255\n" % (w, h))
        fh.write(np.ascontiguousarray(rgba[..., :3]).tobytes())


STATIC_SORT_MAX_KEYS = 65536
STATIC_SORT_FAILED = 0xFFFFFFFF   # every perm entry after a sort whose bounded wait ran out


def sort_keys_static(keys_ptr: int, n: int, perm_ptr: int, stream: int | None = None) -> None:
    """Stable sort permutation of n device-resident uint64 keys into the device
    uint32 array at perm_ptr, without allocating device memory (for callers
    that cannot allocate while they run; see wcsph_sort_keys_static in
    include/wcsph.h). Enqueued on `stream` (a cudaStream_t handle, None = the
    default stream); the call does not wait for the GPU."""
    _check(load_library().wcsph_sort_keys_static(keys_ptr, n, perm_ptr, stream), None)


class stall_sort:
    """Error-path test hook (wcsph_test_stall_sort): inside the block, sorts
    enqueued afterwards make their look-back waits run out (bounded, no hang),
    so a step reports ERR_DEVICE_TIMEOUT and the static sort marks its output
    with STATIC_SORT_FAILED."""

    def __enter__(self):
        load_library().wcsph_test_stall_sort(1)
        return self

    def __exit__(self, *exc):
        load_library().wcsph_test_stall_sort(0)
        return False


def snapshot_read(path, app_name: str, fluid_n: int):
    pos = np.empty((fluid_n, 4), np.float32)
    vel = np.empty((fluid_n, 4), np.float32)
    _check(load_library().wcsph_snapshot_read(str(path).encode(), app_name.encode(), fluid_n, fptr(pos),
                                              fptr(vel)), None)
    return pos, vel


def snapshot_header(path):
    name = C.create_string_buffer(64)
    n = C.c_uint32()
    _check(load_library().wcsph_snapshot_read_header(str(path).encode(), name, C.byref(n)), None)
    return name.value.decode(), n.value


def snapshot_write(path, app_name: str, pos: np.ndarray, vel: np.ndarray):
    pos = np.ascontiguousarray(pos, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    _check(load_library().wcsph_snapshot_write(str(path).encode(), app_name.encode(), pos.shape[0], fptr(pos),
                                               fptr(vel)), None)


class CUDASPHSimulator:
    """One simulation context (CUDASPHSimulator of src/cuda/SPH/sph.cuh:14-86)."""

    def __init__(self, params: Params, fluid_pos: np.ndarray, box_: Box, fluid_vel=None,
                 boundary_pos=None, device: int = -1):
        self._lib = load_library()
        self._ctx = None
        self.fluid_pos0 = np.ascontiguousarray(fluid_pos, np.float32)
        self.fluid_vel0 = None if fluid_vel is None else np.ascontiguousarray(fluid_vel, np.float32)
        self.boundary_pos0 = (np.zeros((0, 4), np.float32) if boundary_pos is None
                              else np.ascontiguousarray(boundary_pos, np.float32))
        sc = Scene()
        sc.fluid_n = self.fluid_pos0.shape[0]
        sc.fluid_pos = fptr(self.fluid_pos0)
        sc.fluid_vel = fptr(self.fluid_vel0)
        sc.boundary_n = self.boundary_pos0.shape[0]
        sc.boundary_pos = fptr(self.boundary_pos0) if sc.boundary_n else None
        sc.box = box_
        self.params = params
        ctx = C.c_void_p()
        _check(self._lib.wcsph_create(C.byref(params), C.byref(sc), device, C.byref(ctx)), None)
        self._ctx = ctx

    def close(self):
        if self._ctx is not None:
            self._lib.wcsph_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, status):
        _check(status, self._ctx, self._lib)

    # FluidSimulator interface
    def update(self, delta: float):
        self._c(self._lib.wcsph_step(self._ctx, delta))

    def step_n(self, n: int, delta: float):
        self._c(self._lib.wcsph_step_n(self._ctx, n, delta))

    def reset(self):
        self._c(self._lib.wcsph_reset(self._ctx))

    def synchronize(self):
        self._c(self._lib.wcsph_synchronize(self._ctx))

    def get_fluid_particles(self) -> int:
        return self.fluid_pos0.shape[0]

    def set_box(self, b: Box):
        self._c(self._lib.wcsph_set_box(self._ctx, C.byref(b)))

    def set_params(self, p: Params):
        self._c(self._lib.wcsph_set_params(self._ctx, C.byref(p)))
        self.params = p

    def get_state(self, out=None):
        """(positions, velocities) float32 [n, 4] in the current order; `out`
        = (pos, vel) arrays to fill (e.g. views of pinned host memory)."""
        n = self.get_fluid_particles()
        if out is None:
            pos = np.empty((n, 4), np.float32)
            vel = np.empty((n, 4), np.float32)
        else:
            pos, vel = out
            for a in (pos, vel):
                if a.shape != (n, 4) or a.dtype != np.float32 or not a.flags.c_contiguous:
                    raise ValueError("out arrays must be contiguous float32 [n, 4]")
        self._c(self._lib.wcsph_get_state(self._ctx, fptr(pos), fptr(vel)))
        return pos, vel

    def set_state(self, pos, vel=None):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = None if vel is None else np.ascontiguousarray(vel, np.float32)
        self._c(self._lib.wcsph_set_state(self._ctx, fptr(pos), fptr(vel)))

    def snapshot_save(self, path, app_name: str):
        self._c(self._lib.wcsph_snapshot_save(self._ctx, str(path).encode(), app_name.encode()))

    def snapshot_load(self, path, app_name: str):
        self._c(self._lib.wcsph_snapshot_load(self._ctx, str(path).encode(), app_name.encode()))

    def compute_state_metrics(self):
        ms, ke = C.c_float(), C.c_float()
        self._c(self._lib.wcsph_metrics(self._ctx, C.byref(ms), C.byref(ke)))
        return ms.value, ke.value

    def last_dt(self):
        a, b = C.c_float(), C.c_float()
        self._c(self._lib.wcsph_last_dt(self._ctx, C.byref(a), C.byref(b)))
        return a.value, b.value

    def field(self, name: str) -> np.ndarray:
        fid = FIELD[name]
        n = C.c_uint64()
        eb = C.c_uint32()
        self._c(self._lib.wcsph_field_size(self._ctx, fid, C.byref(n), C.byref(eb)))
        dt, comps = _FIELD_DTYPE[fid]
        out = np.empty((n.value, comps) if comps > 1 else (n.value,), dt)
        if n.value:
            self._c(self._lib.wcsph_get_field(self._ctx, fid, C.c_void_p(out.ctypes.data), out.nbytes))
        return out

    def neighbors(self):
        """CSR neighbour lists of the last step: (counts, offsets, indices)."""
        n = self.get_fluid_particles()
        counts = np.empty(n, np.uint32)
        offsets = np.empty(n, np.uint32)
        total = C.c_uint64()
        u = C.POINTER(C.c_uint32)
        # first call sizes the list, second fills it
        st = self._lib.wcsph_get_neighbors(self._ctx, counts.ctypes.data_as(u), offsets.ctypes.data_as(u), None,
                                           0, C.byref(total))
        if st not in (OK, ERR_NEIGHBOR_OVERFLOW):
            self._c(st)
        idx = np.empty(max(total.value, 1), np.uint32)
        self._c(self._lib.wcsph_get_neighbors(self._ctx, counts.ctypes.data_as(u), offsets.ctypes.data_as(u),
                                              idx.ctypes.data_as(u), idx.size, C.byref(total)))
        return counts, offsets, idx[: total.value]

    def stream_handle(self) -> int:
        """cudaStream_t of this context (for torch.cuda.ExternalStream)."""
        v = C.c_void_p()
        self._c(self._lib.wcsph_get_stream(self._ctx, C.byref(v)))
        return v.value or 0

    def time_steps(self, n: int, delta: float) -> float:
        ms = C.c_float()
        self._c(self._lib.wcsph_time_steps(self._ctx, n, delta, C.byref(ms)))
        return ms.value

    def render(self, camera: Camera, opts: RenderOpts | None = None, with_depth: bool = False):
        """Headless particle view of the current state -> rgba [H, W, 4] (and depth [H, W])."""
        o = opts or render_opts()
        rgba = np.empty((o.height, o.width, 4), np.uint8)
        depth = np.empty((o.height, o.width), np.float32) if with_depth else None
        self._c(self._lib.wcsph_render(self._ctx, C.byref(camera), C.byref(o), rgba.ctypes.data_as(C.c_void_p),
                                       fptr(depth)))
        return (rgba, depth) if with_depth else rgba

    def kernel_timings(self):
        names = (C.c_char_p * 16)()
        ms = (C.c_float * 16)()
        k = self._lib.wcsph_kernel_timings(self._ctx, names, ms, 16)
        if k < 0:
            self._c(-k)
        return {names[i].decode(): ms[i] for i in range(k)}

    def launches_per_step(self) -> int:
        v = C.c_int()
        self._c(self._lib.wcsph_launches_per_step(self._ctx, C.byref(v)))
        return v.value

    def set_tuning(self, searcher: int = SEARCH_MCMC, budget: float = 0.1, frozen_config=None):
        fz = None if frozen_config is None else str(frozen_config).encode()
        self._c(self._lib.wcsph_set_tuning(self._ctx, searcher, budget, fz))

    def was_scheduled_step(self) -> bool:
        v = C.c_int()
        self._c(self._lib.wcsph_was_tuning_step(self._ctx, C.byref(v)))
        return bool(v.value)

    def save_config(self, path):
        self._c(self._lib.wcsph_save_config(self._ctx, str(path).encode()))

    def save_tuning_results(self, path):
        self._c(self._lib.wcsph_save_tuning_results(self._ctx, str(path).encode()))

    def reset_tuning(self):
        self._c(self._lib.wcsph_reset_tuning(self._ctx))

    def rollout_forward(self, steps: int, dt: float, checkpoint_every: int, target: np.ndarray) -> float:
        t = np.ascontiguousarray(target, np.float32)
        loss = C.c_float()
        self._c(self._lib.wcsph_rollout_forward(self._ctx, steps, dt, checkpoint_every, fptr(t), C.byref(loss)))
        return loss.value

    def rollout_backward(self):
        n = self.get_fluid_particles()
        gv = np.zeros((n, 4), np.float32)
        gnu, gk = C.c_float(), C.c_float()
        self._c(self._lib.wcsph_rollout_backward(self._ctx, fptr(gv), C.byref(gnu), C.byref(gk)))
        return gv, gnu.value, gk.value


def shard_scenes(counts, world: int) -> list[list[int]]:
    """Greedy longest-processing-time bin packing of independent scenes onto
    `world` ranks by particle count (the ensemble shards with no data-path
    collective). Deterministic: ties go to the lowest rank."""
    loads = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for k in sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i)):
        r = min(range(world), key=lambda q: (loads[q], q))
        shards[r].append(k)
        loads[r] += int(counts[k])
    return [sorted(s) for s in shards]


@dataclass
class BatchSceneSpec:
    fluid_pos: np.ndarray
    box: Box
    gravity: tuple = (0.0, -9.81, 0.0)
    viscosity: float = 0.01
    fluid_vel: np.ndarray | None = None
    boundary_pos: np.ndarray | None = None


class BatchSimulator:
    """Many independent scenes advanced together (wcsph_batch_*)."""

    def __init__(self, params: Params, scenes: list[BatchSceneSpec], device: int = -1):
        self._lib = load_library()
        self._b = None
        self._keep = []
        arr = (BatchScene * len(scenes))()
        for k, s in enumerate(scenes):
            pos = np.ascontiguousarray(s.fluid_pos, np.float32)
            vel = None if s.fluid_vel is None else np.ascontiguousarray(s.fluid_vel, np.float32)
            bp = None if s.boundary_pos is None else np.ascontiguousarray(s.boundary_pos, np.float32)
            self._keep += [pos, vel, bp]
            arr[k].fluid_n = pos.shape[0]
            arr[k].fluid_pos = fptr(pos)
            arr[k].fluid_vel = fptr(vel)
            arr[k].boundary_n = 0 if bp is None else bp.shape[0]
            arr[k].boundary_pos = fptr(bp)
            arr[k].box = s.box
            arr[k].gravity[:] = list(s.gravity)
            arr[k].viscosity = s.viscosity
        self.counts = [s.fluid_pos.shape[0] for s in scenes]
        b = C.c_void_p()
        st = self._lib.wcsph_batch_create(C.byref(params), arr, len(scenes), device, C.byref(b))
        if st != OK:
            raise WcsphError(st, self._lib.wcsph_batch_last_error(None).decode())
        self._b = b

    def _c(self, st):
        if st != OK:
            raise WcsphError(st, self._lib.wcsph_batch_last_error(self._b).decode())

    def set_persistent(self, enable: bool):
        """True (default): n steps in one persistent cooperative launch;
        False: one launch per stage and step (wcsph_batch_set_persistent)."""
        self._c(self._lib.wcsph_batch_set_persistent(self._b, 1 if enable else 0))

    def step_n(self, n, delta):
        self._c(self._lib.wcsph_batch_step_n(self._b, n, delta))

    def time_steps(self, n, delta) -> float:
        ms = C.c_float()
        self._c(self._lib.wcsph_batch_time_steps(self._b, n, delta, C.byref(ms)))
        return ms.value

    def get_state(self, scene: int):
        n = self.counts[scene]
        pos = np.empty((n, 4), np.float32)
        vel = np.empty((n, 4), np.float32)
        self._c(self._lib.wcsph_batch_get_state(self._b, scene, fptr(pos), fptr(vel)))
        return pos, vel

    def metrics(self):
        k = len(self.counts)
        ms = np.empty(k, np.float32)
        ke = np.empty(k, np.float32)
        self._c(self._lib.wcsph_batch_metrics(self._b, fptr(ms), fptr(ke)))
        return ms, ke

    def close(self):
        if self._b is not None:
            self._lib.wcsph_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
