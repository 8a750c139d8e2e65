"""ctypes binding of libarcsim.so, the B200 batched world step.

`Sim` has the reference binding's constructor, attributes and methods
(arc/native.py:73-157): the same float64 output buffers, reused by
`observe()`, the same argument checks. It adds what the GPU library offers
beyond the reference: precision and kernel choice, state snapshots,
per-world terrain, custom models and device-pointer calls.

There is no CPU fallback: if the library is missing or no CUDA device is
usable, construction raises.
"""

from __future__ import annotations

import ctypes
import functools
import os
import re
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
# ARC_SIM_LIB selects another build of the library, e.g. the checked build
# libarcsim_checked.so (arc_demo_b200/build.py)
LIB_PATH = Path(os.environ["ARC_SIM_LIB"]) if os.environ.get("ARC_SIM_LIB") else HERE / "libarcsim.so"
HEADER = HERE.parent / "include" / "arc_sim.h"

_f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_int, _uint, _dbl = ctypes.c_int, ctypes.c_uint, ctypes.c_double

ROOT_SIZE = 13  # pos(3) quat wxyz(4) linvel(3) angvel(3)
FP64 = 1
PLAIN = 2
KERNEL_PLAIN = 0
KERNEL_LEGS = 1
KERNEL_WARPS = 2


class ArcSimError(RuntimeError):
    pass


def _declare(lib, name, restype, *argtypes):
    fn = getattr(lib, name)
    fn.restype = restype
    fn.argtypes = list(argtypes)


@functools.cache
def sim_lib() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise OSError(f"{LIB_PATH} not found: build it with `python -m arc_demo_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    d = functools.partial(_declare, lib)
    # the reference's symbols (csrc/arc_sim.h:25-56), declared as arc/native.py:38-55 does
    d("arc_sim_create", _vp, _int, _dbl, _int, _int, _dbl)
    d("arc_sim_destroy", None, _vp)
    d("arc_sim_set_threads", None, _vp, _int)
    d("arc_sim_num_worlds", _int, _vp)
    d("arc_sim_num_joints", _int)
    d("arc_sim_num_legs", _int)
    d("arc_sim_robot_info", None, _vp, _f64, _f64, _f64, _f64)
    d("arc_sim_reset", None, _vp, _i32, _int, _u32, _f64)
    d("arc_sim_step", None, _vp, _vp)
    d("arc_sim_observe", None, _vp, _vp, _vp, _vp, _vp, _vp)
    d("arc_sim_heights", None, _vp, _vp, _int, _vp)
    d("arc_sim_terrain_at", None, _vp, _i32, _f64, _int, _f64)
    d("arc_sim_world", _vp, _vp, _int)
    # additive
    d("arc_sim_create_ex", _vp, _int, _dbl, _int, _int, _dbl, _uint)
    d("arc_sim_last_error", _int, _vp)
    d("arc_sim_error_message", ctypes.c_char_p, _vp)
    d("arc_sim_set_kernel", _int, _vp, _int, _int)
    d("arc_sim_get_kernel", _int, _vp, ctypes.POINTER(_int), ctypes.POINTER(_int))
    d("arc_sim_real_size", _int, _vp)
    d("arc_sim_model_info", _int, _vp, ctypes.POINTER(_int), ctypes.POINTER(_int), ctypes.POINTER(_int),
      ctypes.POINTER(_int))
    d("arc_sim_state_size", _int, _vp)
    d("arc_sim_get_state", _int, _vp, _i32, _int, _f64)
    d("arc_sim_set_state", _int, _vp, _i32, _int, _f64)
    d("arc_sim_set_terrain", _int, _vp, _int, _int, _int, _dbl, _dbl, _f64)
    d("arc_sim_get_terrain", _int, _vp, _int, _i32, _f64, _f64)
    d("arc_sim_set_world_params", _int, _vp, _f64, _dbl, _dbl)
    d("arc_sim_set_joint", _int, _vp, _int, _dbl, _dbl, _dbl, _dbl, _dbl)
    d("arc_model_create", _vp)
    d("arc_model_destroy", None, _vp)
    d("arc_model_add_body", _int, _vp, _dbl, _f64, _f64, _f64)
    d("arc_model_add_sphere", _int, _vp, _int, _f64, _dbl)
    d("arc_model_add_hinge", _int, _vp, _int, _int, _f64, _f64)
    d("arc_model_add_visual", _int, _vp, _int, _int, _f64, _f64, _dbl, _dbl, _dbl, _int,
      np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS"))
    d("arc_sim_create_model", _vp, _vp, _int, _dbl, _int, _int, _dbl, _uint)
    d("arc_sim_set_pose", _int, _vp, _int, _f64, _f64, _vp)
    d("arc_sim_stream", _vp, _vp)
    d("arc_sim_step_device", _int, _vp, _vp, _vp)
    d("arc_sim_step_actions", _int, _vp, _vp, _vp)
    d("arc_sim_observe_device", _int, _vp, _vp, _vp, _vp, _vp, _vp, _vp)
    d("arc_sim_synchronize", _int, _vp)
    d("arc_sim_create_sized", _vp, _int, _i32, _dbl, _int, _dbl, _uint)
    d("arc_sim_step_ids", _int, _vp, _vp, _int, _vp, _vp, _vp)
    d("arc_sim_set_work_queue", _int, _vp, _int)
    d("arc_sim_set_substep_tile", _int, _vp, _int)
    d("arc_device_checks", _int, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(_int),
      ctypes.POINTER(ctypes.c_longlong), _int)
    return lib


def device_checks(clear: bool = False) -> dict:
    """The loaded library's record of failed index checks (arc_device_checks):
    whether it is the checked build, how many checks failed since the last
    clear, and the site and index of the first."""
    failures, site, index = ctypes.c_ulonglong(), _int(), ctypes.c_longlong()
    rc = sim_lib().arc_device_checks(ctypes.byref(failures), ctypes.byref(site), ctypes.byref(index), int(clear))
    if rc < 0:
        raise ArcSimError(f"arc_device_checks failed: {rc}")
    return {"checked": rc == 1, "failures": failures.value, "site": site.value, "index": index.value}


def header_symbols() -> list[str]:
    """Every function declared in the library's headers (include/*.h)."""
    names = set()
    for h in sorted(HEADER.parent.glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"\b(arc_\w+)\s*\(", text))
    return sorted(names)


class Model:
    """A custom model (bodies, hinges, spheres), as with csrc/arc_phys.h's builders."""

    def __init__(self):
        self._lib = sim_lib()
        self.ptr = self._lib.arc_model_create()

    def add_body(self, mass, inertia, pos, q=(1.0, 0.0, 0.0, 0.0)) -> int:
        return self._lib.arc_model_add_body(self.ptr, mass, _vec(inertia), _vec(pos), _vec(q))

    def add_sphere(self, body, pos, radius) -> int:
        return self._lib.arc_model_add_sphere(self.ptr, body, _vec(pos), radius)

    def add_hinge(self, parent, child, anchor, axis) -> int:
        return self._lib.arc_model_add_hinge(self.ptr, parent, child, _vec(anchor), _vec(axis))

    def add_visual(self, type, body, p0, p1, radius, radius2=0.0, aspect=1.0, material=0,
                   color=(0.5, 0.5, 0.5)) -> int:
        """A render-only shape on `body` (types and materials as in include/arc_sim.h)."""
        return self._lib.arc_model_add_visual(self.ptr, type, body, _vec(p0), _vec(p1), radius, radius2,
                                              aspect, material, np.asarray(color, dtype=np.float32))

    def close(self):
        if self.ptr:
            self._lib.arc_model_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()


def _vec(v) -> np.ndarray:
    return np.ascontiguousarray(v, dtype=np.float64)


class Sim:
    """N independent worlds, each with the quadruped on its own terrain."""

    def __init__(self, num_worlds: int, dt: float = 1.0 / 30.0, substeps: int = 20,
                 grid: int = 64, cell: float = 0.4, threads: int = 1, *, fp64: bool = False,
                 plain: bool = False, model: Model | None = None, grids=None):
        """grids: optional per-world terrain sizes (1..64); grid is then
        their maximum and world i holds grids[i] x grids[i] columns."""
        self._lib = sim_lib()
        if grids is not None:
            grids = np.ascontiguousarray(grids, dtype=np.int32)
            assert len(grids) == num_worlds
            grid = int(grids.max()) if num_worlds else grid
        self.grids = grids
        self.num_worlds = num_worlds
        self.grid = min(grid, 64)
        self.cell = cell
        self.dt, self.substeps = dt, substeps
        self.num_joints = self._lib.arc_sim_num_joints()
        self.num_legs = self._lib.arc_sim_num_legs()
        flags = (FP64 if fp64 else 0) | (PLAIN if plain else 0)
        if model is not None:
            self._ptr = self._lib.arc_sim_create_model(model.ptr, num_worlds, dt, substeps, grid, cell, flags)
        elif grids is not None:
            self._ptr = self._lib.arc_sim_create_sized(num_worlds, grids, dt, substeps, cell, flags)
        else:
            self._ptr = self._lib.arc_sim_create_ex(num_worlds, dt, substeps, grid, cell, flags)
        if not self._ptr:
            raise MemoryError("arc_sim_create failed (no CUDA device, or out of memory)")
        self._lib.arc_sim_set_threads(self._ptr, int(threads))
        nb, nj_, ns, nch = _int(), _int(), _int(), _int()
        self._lib.arc_sim_model_info(self._ptr, ctypes.byref(nb), ctypes.byref(nj_), ctypes.byref(ns),
                                     ctypes.byref(nch))
        self.num_bodies, self.num_spheres, self.num_channels = nb.value, ns.value, nch.value
        if model is not None:
            self.num_joints = nj_.value

        nj = self.num_joints
        self.default_angles = np.zeros(max(nj, 12))
        self.lo, self.hi, misc = np.zeros(max(nj, 12)), np.zeros(max(nj, 12)), np.zeros(2)
        self._lib.arc_sim_robot_info(self._ptr, self.default_angles, self.lo, self.hi, misc)
        self.default_angles, self.lo, self.hi = self.default_angles[:nj], self.lo[:nj], self.hi[:nj]
        self.stand_height = float(misc[0])
        self.total_mass = float(misc[1])
        self.state_size = self._lib.arc_sim_state_size(self._ptr)

        # output buffers, reused by observe()
        self.root = np.zeros((num_worlds, ROOT_SIZE))
        self.rot = np.zeros((num_worlds, 3, 3))
        self.joints = np.zeros((num_worlds, 3 * nj))
        self.contacts = np.zeros((num_worlds, self.num_channels if model is not None else self.num_legs + 2))
        self.flags = np.zeros(num_worlds, dtype=np.int32)
        self._observe_args = (self._ptr, self.root.ctypes.data, self.rot.ctypes.data,
                              self.joints.ctypes.data, self.contacts.ctypes.data,
                              self.flags.ctypes.data)

    # -- errors ---------------------------------------------------------------

    def _check(self, rc: int | None = None) -> None:
        err = self._lib.arc_sim_last_error(self._ptr) if rc is None else rc
        if err:
            msg = self._lib.arc_sim_error_message(self._ptr).decode()
            raise ArcSimError(f"libarcsim error {err}: {msg}")

    # -- the reference's interface (arc/native.py:73-157) ---------------------

    @property
    def ptr(self) -> int:
        return self._ptr

    @property
    def half_extent(self) -> float:
        return 0.5 * self.grid * self.cell

    def reset(self, ids: np.ndarray, seeds: np.ndarray, difficulty: np.ndarray) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        difficulty = np.ascontiguousarray(difficulty, dtype=np.float64)
        assert len(ids) == len(seeds) == len(difficulty)
        if len(ids):
            self._lib.arc_sim_reset(self._ptr, ids, len(ids), seeds, difficulty)
            self._check()

    def step(self, targets: np.ndarray) -> None:
        targets = np.ascontiguousarray(targets, dtype=np.float64)
        assert targets.shape == (self.num_worlds, self.num_joints)
        self._lib.arc_sim_step(self._ptr, targets.ctypes.data)
        self._check()

    def observe(self) -> tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """root (N, 13), joints (N, 3*J), contacts (N, legs + 2), flags (N,);
        also refreshes rot (N, 3, 3)."""
        self._lib.arc_sim_observe(*self._observe_args)
        self._check()
        return self.root, self.joints, self.contacts, self.flags

    def heights(self, offsets: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        offsets = np.ascontiguousarray(offsets, dtype=np.float64)
        if out is None:
            out = np.empty((self.num_worlds, len(offsets)))
        assert out.shape == (self.num_worlds, len(offsets)) and out.dtype == np.float64
        assert out.flags.c_contiguous
        self._lib.arc_sim_heights(self._ptr, offsets.ctypes.data, len(offsets), out.ctypes.data)
        self._check()
        return out

    def terrain_at(self, ids: np.ndarray, xy: np.ndarray) -> np.ndarray:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        xy = np.ascontiguousarray(xy, dtype=np.float64)
        out = np.zeros(len(ids))
        if len(ids):
            self._lib.arc_sim_terrain_at(self._ptr, ids, xy, len(ids), out)
            self._check()
        return out

    def close(self) -> None:
        if getattr(self, "_ptr", None):
            self._lib.arc_sim_destroy(self._ptr)
            self._ptr = None

    def __del__(self):
        self.close()

    # -- additive -------------------------------------------------------------

    def set_kernel(self, kernel: int, worlds_per_cta: int = 16) -> None:
        self._check(self._lib.arc_sim_set_kernel(self._ptr, kernel, worlds_per_cta))

    def kernel(self) -> tuple[int, int]:
        k, w = _int(), _int()
        self._lib.arc_sim_get_kernel(self._ptr, ctypes.byref(k), ctypes.byref(w))
        return k.value, w.value

    @property
    def real_size(self) -> int:
        return self._lib.arc_sim_real_size(self._ptr)

    def get_state(self, ids=None) -> np.ndarray:
        ids = np.arange(self.num_worlds) if ids is None else ids
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros((len(ids), self.state_size))
        self._check(self._lib.arc_sim_get_state(self._ptr, ids, len(ids), out))
        return out

    def set_state(self, state, ids=None) -> None:
        ids = np.arange(self.num_worlds) if ids is None else ids
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        st = np.ascontiguousarray(state, dtype=np.float64).reshape(len(ids), self.state_size)
        self._check(self._lib.arc_sim_set_state(self._ptr, ids, len(ids), st))

    def set_terrain(self, i: int, heights: np.ndarray, cell: float, outside: float = -100.0) -> None:
        h = np.ascontiguousarray(heights, dtype=np.float64)
        ny, nx = h.shape
        self._check(self._lib.arc_sim_set_terrain(self._ptr, int(i), nx, ny, cell, outside, h.ravel()))

    def get_terrain(self, i: int):
        nxy = np.zeros(2, dtype=np.int32)
        geom = np.zeros(4)
        h = np.zeros(64 * 64)
        self._check(self._lib.arc_sim_get_terrain(self._ptr, int(i), nxy, geom, h))
        nx, ny = int(nxy[0]), int(nxy[1])
        return h[: nx * ny].reshape(ny, nx), geom

    def set_world_params(self, gravity=(0.0, 0.0, -9.81), mu_static=1.0, mu_dynamic=0.8) -> None:
        self._check(self._lib.arc_sim_set_world_params(self._ptr, _vec(gravity), mu_static, mu_dynamic))

    def set_joint(self, j, lo, hi, kp, kd, max_torque) -> None:
        self._check(self._lib.arc_sim_set_joint(self._ptr, j, lo, hi, kp, kd, max_torque))

    def set_pose(self, i, pos, q=(1.0, 0.0, 0.0, 0.0), angles=None) -> None:
        a = None if angles is None else _vec(angles)
        self._check(self._lib.arc_sim_set_pose(self._ptr, int(i), _vec(pos), _vec(q),
                                               None if a is None else a.ctypes.data))

    def synchronize(self) -> None:
        self._check(self._lib.arc_sim_synchronize(self._ptr))

    def step_ids(self, d_ids: int, n_ids: int, d_targets: int = 0, d_actions: int = 0, stream: int = 0) -> None:
        """Steps the n_ids worlds listed at device address d_ids, with device
        targets (N x 12 FP64) or actions (N x 12 FP32); asynchronous."""
        self._check(self._lib.arc_sim_step_ids(self._ptr, d_ids or None, n_ids, d_targets or None,
                                               d_actions or None, stream or None))

    def set_work_queue(self, on: bool) -> None:
        self._check(self._lib.arc_sim_set_work_queue(self._ptr, int(bool(on))))

    def set_substep_tile(self, tile: int) -> None:
        """Warp-per-leg kernel: `tile` substeps per launch (0: the whole
        control step in one launch)."""
        self._check(self._lib.arc_sim_set_substep_tile(self._ptr, int(tile)))
