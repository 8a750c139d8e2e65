"""ctypes front end of the CPU checkers. TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module; the product (arc_demo_b200) never does.

- `OracleSim`: the C restatement in oracle/arc_oracle.c, FP64 (`bits=64`,
  the reference's arithmetic) or FP32 (`bits=32`, the CUDA kernel's
  arithmetic and operation order).
- `RefSim`: the reference's own csrc/ compiled from its sources by
  oracle/Makefile into oracle/_ref/ (its batched C API, csrc/arc_sim.h:25-56),
  with read/write access to each world through the reference's `arc_world`
  layout (csrc/arc_phys.h:25-112), mirrored here as ctypes structures.

Both expose the same snapshot format (387 doubles per world, see
`STATE_SIZE`) so states can be moved between them for teacher forcing.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
NJ, NLEGS, NB, NS = 12, 4, 13, 21
STATE_SIZE = NB * 13 + NS * 8 + NJ * 4 + 2  # 387
ROOT_SIZE = 13

_f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
_vp = ctypes.c_void_p
_int, _dbl = ctypes.c_int, ctypes.c_double


def build(ref: str | None = None) -> None:
    """Builds the oracle (and, when the reference sources exist, oracle/_ref)."""
    cmd = ["make", "-s", "-C", str(HERE)]
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


def ref_available() -> bool:
    return (HERE / "_ref" / "libarcsim_ref.so").exists()


def host_has_avx512() -> bool:
    try:
        flags = Path("/proc/cpuinfo").read_text().split()
    except OSError:
        return False
    return "avx512f" in flags and "avx512bw" in flags and "avx512vl" in flags and "avx512dq" in flags


def fastest_ref_variant() -> str:
    """The reference build for timing: AVX-512 where the host runs it (the
    reference's own -march=native would use it there), else AVX2."""
    if host_has_avx512() and (HERE / "_ref" / "libarcsim_ref_v4.so").exists():
        return "_v4"
    return ""


# -- the restatement ----------------------------------------------------------

_oracle_libs: dict[int, ctypes.CDLL] = {}


def oracle_lib(bits: int) -> ctypes.CDLL:
    if bits in _oracle_libs:
        return _oracle_libs[bits]
    path = HERE / f"liboracle{bits}.so"
    if not path.exists():
        build()
    lib = ctypes.CDLL(str(path))
    p = f"orc{bits}_"

    def d(name, res, *args):
        fn = getattr(lib, p + name)
        fn.restype = res
        fn.argtypes = list(args)

    d("create", _vp, _int, _dbl, _int, _int, _dbl)
    d("destroy", None, _vp)
    d("num_worlds", _int, _vp)
    d("real_size", _int)
    d("robot_info", None, _vp, _f64, _f64, _f64, _f64)
    d("reset", None, _vp, _i32, _int, _u32, _f64)
    d("step", None, _vp, _f64)
    d("step_some", None, _vp, _i32, _int, _f64)
    d("observe", None, _vp, _f64, _f64, _f64, _f64, _i32)
    d("heights", None, _vp, _f64, _int, _f64)
    d("terrain_at", None, _vp, _i32, _f64, _int, _f64)
    d("state_size", _int, _vp)
    d("get_state", None, _vp, _i32, _int, _f64)
    d("margins", None, _vp, _f64)
    d("set_state", None, _vp, _i32, _int, _f64)
    d("set_terrain", None, _vp, _int, _int, _int, _dbl, _dbl, _f64)
    d("get_terrain", None, _vp, _int, _i32, _f64, _f64)
    d("terrain_generate", None, _int, _dbl, _dbl, ctypes.c_uint, _f64, _f64)
    d("model_dump", _int, _vp, _f64)
    d("n_contacts", _int, _vp, _int)
    _oracle_libs[bits] = lib
    return lib


class _SimBase:
    """Shared numpy-facing helpers (mirrors arc/native.py's Sim)."""

    num_joints = NJ
    num_legs = NLEGS

    def _alloc_outputs(self, n: int) -> None:
        self.root = np.zeros((n, ROOT_SIZE))
        self.rot = np.zeros((n, 3, 3))
        self.joints = np.zeros((n, 3 * NJ))
        self.contacts = np.zeros((n, NLEGS + 2))
        self.flags = np.zeros(n, dtype=np.int32)

    @property
    def half_extent(self) -> float:
        return 0.5 * self.grid * self.cell


class OracleSim(_SimBase):
    def __init__(self, n: int, dt: float = 1.0 / 30.0, substeps: int = 20, grid: int = 64,
                 cell: float = 0.4, bits: int = 64):
        self.lib = oracle_lib(bits)
        self.p = f"orc{bits}_"
        self.bits = bits
        self.num_worlds, self.dt, self.substeps = n, dt, substeps
        self.grid, self.cell = min(grid, 64), cell
        self.ptr = self._f("create")(n, dt, substeps, grid, cell)
        if not self.ptr:
            raise MemoryError("oracle create failed")
        self.default_angles = np.zeros(NJ)
        self.lo, self.hi, misc = np.zeros(NJ), np.zeros(NJ), np.zeros(3)
        self._f("robot_info")(self.ptr, self.default_angles, self.lo, self.hi, misc)
        self.stand_height, self.total_mass, self.footprint = (float(v) for v in misc)
        self._alloc_outputs(n)

    def _f(self, name):
        return getattr(self.lib, self.p + name)

    def reset(self, ids, seeds, difficulty) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        diff = np.ascontiguousarray(difficulty, dtype=np.float64)
        if len(ids):
            self._f("reset")(self.ptr, ids, len(ids), seeds, diff)

    def step(self, targets) -> None:
        t = np.ascontiguousarray(targets, dtype=np.float64)
        assert t.shape == (self.num_worlds, NJ)
        self._f("step")(self.ptr, t)

    def step_some(self, ids, targets) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        t = np.ascontiguousarray(targets, dtype=np.float64)
        self._f("step_some")(self.ptr, ids, len(ids), t)

    def observe(self):
        self._f("observe")(self.ptr, self.root, self.rot, self.joints, self.contacts, self.flags)
        return self.root, self.joints, self.contacts, self.flags

    def heights(self, offsets, out=None):
        off = np.ascontiguousarray(offsets, dtype=np.float64)
        if out is None:
            out = np.empty((self.num_worlds, len(off)))
        self._f("heights")(self.ptr, off, len(off), out)
        return out

    def terrain_at(self, ids, xy):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        xy = np.ascontiguousarray(xy, dtype=np.float64)
        out = np.zeros(len(ids))
        if len(ids):
            self._f("terrain_at")(self.ptr, ids, xy, len(ids), out)
        return out

    def margins(self) -> np.ndarray:
        """Threshold margins of each world's last step (N x (NS + 3)):
        per sphere the closest contact on/off decision in metres, then the
        closest anchor reset, static/dynamic friction and limit decisions
        (1e30 where none was taken)."""
        out = np.zeros((self.num_worlds, NS + 3))
        self._f("margins")(self.ptr, out)
        return out

    def get_state(self, ids=None) -> np.ndarray:
        ids = np.arange(self.num_worlds) if ids is None else ids
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros((len(ids), STATE_SIZE))
        self._f("get_state")(self.ptr, ids, len(ids), out)
        return out

    def set_state(self, state, ids=None) -> None:
        ids = np.arange(self.num_worlds) if ids is None else ids
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        st = np.ascontiguousarray(state, dtype=np.float64).reshape(len(ids), STATE_SIZE)
        self._f("set_state")(self.ptr, ids, len(ids), st)

    def set_terrain(self, i: int, heights: np.ndarray, cell: float, outside: float = -100.0) -> None:
        h = np.ascontiguousarray(heights, dtype=np.float64)
        ny, nx = h.shape
        self._f("set_terrain")(self.ptr, i, nx, ny, cell, outside, h.ravel())

    def get_terrain(self, i: int):
        nxy = np.zeros(2, dtype=np.int32)
        geom = np.zeros(4)
        h = np.zeros(64 * 64)
        self._f("get_terrain")(self.ptr, i, nxy, geom, h)
        nx, ny = int(nxy[0]), int(nxy[1])
        return h[: nx * ny].reshape(ny, nx), geom

    def model_dump(self) -> np.ndarray:
        out = np.zeros(4096)
        n = self._f("model_dump")(self.ptr, out)
        return out[:n].copy()

    def n_contacts(self, i: int) -> int:
        return int(self._f("n_contacts")(self.ptr, i))

    def close(self) -> None:
        if getattr(self, "ptr", None):
            self._f("destroy")(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()


def oracle_terrain(n: int, cell: float, difficulty: float, seed: int, bits: int = 64):
    lib = oracle_lib(bits)
    out = np.zeros(n * n)
    geom = np.zeros(4)
    getattr(lib, f"orc{bits}_terrain_generate")(n, cell, difficulty, seed, out, geom)
    nx = int(geom[0])
    return out[: nx * nx].reshape(nx, nx), geom


# -- the reference, built from its own sources --------------------------------

class Vec3(ctypes.Structure):
    _fields_ = [("x", _dbl), ("y", _dbl), ("z", _dbl)]


class Quat(ctypes.Structure):
    _fields_ = [("w", _dbl), ("x", _dbl), ("y", _dbl), ("z", _dbl)]


class Mat3(ctypes.Structure):
    _fields_ = [("m", _dbl * 9)]


class Body(ctypes.Structure):  # csrc/arc_phys.h:25-36
    _fields_ = [("x", Vec3), ("x_prev", Vec3), ("q", Quat), ("q_prev", Quat), ("v", Vec3),
                ("w", Vec3), ("mass", _dbl), ("inv_mass", _dbl), ("inertia", Vec3),
                ("inv_inertia", Vec3), ("rot", Mat3), ("inv_iw", Mat3)]


class Sphere(ctypes.Structure):  # csrc/arc_phys.h:38-46
    _fields_ = [("body", _int), ("pos", Vec3), ("radius", _dbl), ("touch", _int),
                ("anchored", _int), ("anchor", Vec3), ("anchor_n", Vec3)]


class Joint(ctypes.Structure):  # csrc/arc_phys.h:48-63
    _fields_ = [("parent", _int), ("child", _int), ("r1", Vec3), ("r2", Vec3), ("a1", Vec3),
                ("a2", Vec3), ("b1", Vec3), ("b2", Vec3), ("q_rel0", Quat), ("lo", _dbl),
                ("hi", _dbl), ("kp", _dbl), ("kd", _dbl), ("max_torque", _dbl),
                ("target", _dbl), ("angle", _dbl), ("rate", _dbl), ("torque", _dbl),
                ("torque_acc", _dbl), ("lim", _dbl * 4)]


class Contact(ctypes.Structure):  # csrc/arc_phys.h:65-69
    _fields_ = [("body", _int), ("local", Vec3), ("n", Vec3)]


class Visual(ctypes.Structure):  # csrc/arc_phys.h:92-100
    _fields_ = [("type", _int), ("body", _int), ("p0", Vec3), ("p1", Vec3), ("radius", _dbl),
                ("radius2", _dbl), ("aspect", _dbl), ("material", _int),
                ("color", ctypes.c_float * 3)]


class Terrain(ctypes.Structure):  # csrc/arc_terrain.h:13-19
    _fields_ = [("nx", _int), ("ny", _int), ("cell", _dbl), ("ox", _dbl), ("oy", _dbl),
                ("outside", _dbl), ("h", _dbl * (64 * 64))]


class World(ctypes.Structure):  # csrc/arc_phys.h:102-112
    _fields_ = [("gravity", Vec3), ("mu_static", _dbl), ("mu_dynamic", _dbl),
                ("n_bodies", _int), ("n_joints", _int), ("n_spheres", _int),
                ("n_contacts", _int), ("n_visuals", _int), ("unstable", _int), ("time", _dbl),
                ("bodies", Body * 16), ("joints", Joint * 16), ("spheres", Sphere * 48),
                ("contacts", Contact * 128), ("visuals", Visual * 80), ("terrain", Terrain)]


def world_state(w: World) -> np.ndarray:
    """Snapshot (STATE_SIZE doubles) of one reference world."""
    out = []
    for i in range(w.n_bodies):
        b = w.bodies[i]
        out += [b.x.x, b.x.y, b.x.z, b.q.w, b.q.x, b.q.y, b.q.z, b.v.x, b.v.y, b.v.z,
                b.w.x, b.w.y, b.w.z]
    for i in range(w.n_spheres):
        s = w.spheres[i]
        out += [s.anchored, s.anchor.x, s.anchor.y, s.anchor.z, s.anchor_n.x, s.anchor_n.y,
                s.anchor_n.z, s.touch]
    for i in range(w.n_joints):
        j = w.joints[i]
        out += [j.target, j.angle, j.rate, j.torque]
    out += [w.unstable, w.time]
    return np.array(out, dtype=np.float64)


def set_world_state(w: World, st: np.ndarray) -> None:
    """Writes a snapshot into a reference world (x_prev/q_prev follow x/q)."""
    p = 0
    for i in range(w.n_bodies):
        b = w.bodies[i]
        b.x.x, b.x.y, b.x.z = st[p:p + 3]
        b.q.w, b.q.x, b.q.y, b.q.z = st[p + 3:p + 7]
        b.v.x, b.v.y, b.v.z = st[p + 7:p + 10]
        b.w.x, b.w.y, b.w.z = st[p + 10:p + 13]
        b.x_prev.x, b.x_prev.y, b.x_prev.z = st[p:p + 3]
        b.q_prev.w, b.q_prev.x, b.q_prev.y, b.q_prev.z = st[p + 3:p + 7]
        p += 13
    for i in range(w.n_spheres):
        s = w.spheres[i]
        s.anchored = int(st[p] != 0)
        s.anchor.x, s.anchor.y, s.anchor.z = st[p + 1:p + 4]
        s.anchor_n.x, s.anchor_n.y, s.anchor_n.z = st[p + 4:p + 7]
        s.touch = int(st[p + 7])
        p += 8
    for i in range(w.n_joints):
        j = w.joints[i]
        j.target, j.angle, j.rate, j.torque = st[p:p + 4]
        p += 4
    w.unstable = int(st[p] != 0)
    w.time = st[p + 1]


_ref_libs: dict[str, ctypes.CDLL] = {}


def ref_lib(variant: str = "") -> ctypes.CDLL:
    """variant "" (reference flags, AVX2), "_v4" (the same with AVX-512) or
    "_strict" (no FMA contraction)."""
    if variant in _ref_libs:
        return _ref_libs[variant]
    path = HERE / "_ref" / f"libarcsim_ref{variant}.so"
    if not path.exists():
        raise FileNotFoundError(f"{path} not built (needs the reference sources)")
    lib = ctypes.CDLL(str(path))

    def d(name, res, *args):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)

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
    d("arc_sim_world", ctypes.POINTER(World), _vp, _int)
    d("arc_world_step", None, ctypes.POINTER(World), _dbl, _int)
    _ref_libs[variant] = lib
    return lib


class RefSim(_SimBase):
    """The reference's batched simulation (csrc/arc_sim.c), same methods as OracleSim."""

    def __init__(self, n: int, dt: float = 1.0 / 30.0, substeps: int = 20, grid: int = 64,
                 cell: float = 0.4, threads: int = 1, variant: str = ""):
        self.lib = ref_lib(variant)
        self.num_worlds, self.dt, self.substeps = n, dt, substeps
        self.grid, self.cell = min(grid, 64), cell
        self.ptr = self.lib.arc_sim_create(n, dt, substeps, grid, cell)
        if not self.ptr:
            raise MemoryError("arc_sim_create failed")
        self.lib.arc_sim_set_threads(self.ptr, int(threads))
        self.default_angles = np.zeros(NJ)
        self.lo, self.hi, misc = np.zeros(NJ), np.zeros(NJ), np.zeros(2)
        self.lib.arc_sim_robot_info(self.ptr, self.default_angles, self.lo, self.hi, misc)
        self.stand_height, self.total_mass = float(misc[0]), float(misc[1])
        self._alloc_outputs(n)

    def set_threads(self, threads: int) -> None:
        self.lib.arc_sim_set_threads(self.ptr, int(threads))

    def world(self, i: int) -> World:
        return self.lib.arc_sim_world(self.ptr, i).contents

    def reset(self, ids, seeds, difficulty) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        diff = np.ascontiguousarray(difficulty, dtype=np.float64)
        if len(ids):
            self.lib.arc_sim_reset(self.ptr, ids, len(ids), seeds, diff)

    def step(self, targets) -> None:
        t = np.ascontiguousarray(targets, dtype=np.float64)
        assert t.shape == (self.num_worlds, NJ)
        self.lib.arc_sim_step(self.ptr, t.ctypes.data)

    def observe(self):
        self.lib.arc_sim_observe(self.ptr, self.root.ctypes.data, self.rot.ctypes.data,
                                 self.joints.ctypes.data, self.contacts.ctypes.data,
                                 self.flags.ctypes.data)
        return self.root, self.joints, self.contacts, self.flags

    def heights(self, offsets, out=None):
        off = np.ascontiguousarray(offsets, dtype=np.float64)
        if out is None:
            out = np.empty((self.num_worlds, len(off)))
        self.lib.arc_sim_heights(self.ptr, off.ctypes.data, len(off), out.ctypes.data)
        return out

    def terrain_at(self, ids, xy):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        xy = np.ascontiguousarray(xy, dtype=np.float64)
        out = np.zeros(len(ids))
        if len(ids):
            self.lib.arc_sim_terrain_at(self.ptr, ids, xy, len(ids), out)
        return out

    def get_state(self, ids=None) -> np.ndarray:
        ids = range(self.num_worlds) if ids is None else ids
        return np.stack([world_state(self.world(int(i))) for i in ids])

    def set_state(self, state, ids=None) -> None:
        ids = range(self.num_worlds) if ids is None else ids
        st = np.asarray(state, dtype=np.float64).reshape(-1, STATE_SIZE)
        for k, i in enumerate(ids):
            set_world_state(self.world(int(i)), st[k])

    def set_terrain(self, i: int, heights: np.ndarray, cell: float, outside: float = -100.0) -> None:
        t = self.world(i).terrain
        h = np.asarray(heights, dtype=np.float64)
        ny, nx = h.shape
        t.nx, t.ny, t.cell = nx, ny, cell
        t.ox, t.oy = -0.5 * nx * cell, -0.5 * ny * cell
        t.outside = outside
        flat = h.ravel()
        for k in range(nx * ny):
            t.h[k] = flat[k]

    def get_terrain(self, i: int):
        t = self.world(i).terrain
        h = np.ctypeslib.as_array(t.h)[: t.nx * t.ny].reshape(t.ny, t.nx).copy()
        return h, np.array([t.cell, t.ox, t.oy, t.outside])

    def close(self) -> None:
        if getattr(self, "ptr", None):
            self.lib.arc_sim_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        self.close()


# ---- the renderer's restatement (render_oracle.c)

VIEW_YAW = (0.5, 1.4, 2.6)  # camera presets behind, side, front (csrc/arc_render.c:962-968)


def render_lib() -> ctypes.CDLL:
    path = HERE / "liborender.so"
    if not path.exists():
        subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    lib = ctypes.CDLL(str(path))
    fn = lib.oracle_render
    fn.restype = _int
    fn.argtypes = [ctypes.POINTER(World), _vp, _int, _int, _f64, _dbl, _dbl, _dbl, _int, _int, _int, _vp]
    return lib


class RenderOracle:
    """One camera following a world, as the reference's renderer keeps one:
    frame(world, markers, active) -> (H, W, 3) uint8."""

    def __init__(self, width: int, height: int, samples: int = 4, view: int = 0, dist: float = 4.0):
        self.lib = render_lib()
        self.width, self.height, self.samples = width, height, samples
        self.yaw, self.pitch, self.dist = VIEW_YAW[view % 3], 0.3, dist
        self.cam = np.zeros(5)

    def frame(self, world: World, markers=None, active: int = -1) -> np.ndarray:
        img = np.zeros((self.height, self.width, 3), dtype=np.uint8)
        m_ptr, n = None, 0
        if markers is not None and len(markers):
            markers = np.ascontiguousarray(markers, dtype=np.float64).reshape(-1, 4)
            m_ptr, n = markers.ctypes.data, len(markers)
        self.lib.oracle_render(ctypes.byref(world), m_ptr, n, active, self.cam, self.yaw, self.pitch, self.dist,
                               self.width, self.height, self.samples, img.ctypes.data)
        return img
