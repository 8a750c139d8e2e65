"""The task layer of arc/task.py, computed on the GPU.

`TaskConfig`, `CAUSES` and `HEIGHT_OFFSETS` are the reference's
(arc/task.py:17-76). `ArcTask` has the reference class's constructor,
methods and attributes (arc/task.py:88-267), so arc/env.py's ArcVecEnv and
ArcEnv can sit on it unchanged; its observations, rewards and terminations
come from libarcsim.so's task kernels instead of numpy. It hands host numpy
arrays across, like the reference. `arc_demo_b200.torch_env.DeviceVecEnv`
keeps them on the device instead.

Deviation, by design: reset seeds and checkpoint positions are drawn on the
device from a counter-based stream seeded from `seed`, not from numpy's
PCG64 stream; the distributions are the reference's.
"""

from __future__ import annotations

import ctypes
from dataclasses import asdict, dataclass

import numpy as np

from .native import Sim, sim_lib

_vp, _int, _dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double


@dataclass
class TaskConfig:  # arc/task.py:17-66
    dt: float = 1.0 / 30.0
    substeps: int = 20
    grid: int = 64
    cell: float = 0.4
    max_steps: int = 1000
    action_scale: float = 0.6
    checkpoint_radius: float = 0.5
    checkpoint_min_dist: float = 3.0
    checkpoint_max_dist: float = 6.0
    border: float = 1.5
    w_progress: float = 10.0
    max_speed: float = 1.2
    fov: float = 45.0
    w_turn: float = 1.0
    w_checkpoint: float = 10.0
    w_time: float = 0.05
    w_fall: float = 20.0
    w_energy: float = 0.002
    w_action_rate: float = 0.005
    w_body_contact: float = 0.02
    w_torso_contact: float = 0.5
    w_body_rate: float = 0.01
    w_bounce: float = 0.05
    flip_up_z: float = 0.3
    beached_steps: int = 30
    void_z: float = -2.0
    curriculum: bool = True
    difficulty: float = 0.0
    max_difficulty: float = 1.0
    level_step: float = 0.1
    level_up_checkpoints: int = 3
    level_down_steps: int = 300


CAUSES = ("", "unstable", "void", "flip", "beached")  # arc/task.py:70
_F = np.arange(-1.0, 1.41, 0.2)
_L = np.arange(-1.0, 1.01, 0.2)
HEIGHT_OFFSETS = np.array([(f, l) for f in _F for l in _L])  # arc/task.py:74-76
OBS_SIZE = 195
TASK_STATE_SIZE = 25

# buffer ids of include/arc_sim.h
OBS, TERMINAL_OBS, REWARD, TERMINATED, TRUNCATED, CAUSE, DONE_LIST, DONE_COUNT, ACTIONS, \
    ENDED_CHECKPOINTS, ENDED_STEPS, ENDED_DIFFICULTY = range(12)


class CTaskConfig(ctypes.Structure):
    """arc_task_config of include/arc_sim.h."""
    _fields_ = [("dt", _dbl), ("max_steps", _int), ("action_scale", _dbl), ("checkpoint_radius", _dbl),
                ("checkpoint_min_dist", _dbl), ("checkpoint_max_dist", _dbl), ("border", _dbl),
                ("w_progress", _dbl), ("max_speed", _dbl), ("fov", _dbl), ("w_turn", _dbl),
                ("w_checkpoint", _dbl), ("w_time", _dbl), ("w_fall", _dbl), ("w_energy", _dbl),
                ("w_action_rate", _dbl), ("w_body_contact", _dbl), ("w_torso_contact", _dbl),
                ("w_body_rate", _dbl), ("w_bounce", _dbl), ("flip_up_z", _dbl), ("beached_steps", _int),
                ("void_z", _dbl), ("curriculum", _int), ("difficulty", _dbl), ("max_difficulty", _dbl),
                ("level_step", _dbl), ("level_up_checkpoints", _int), ("level_down_steps", _int)]

    @classmethod
    def of(cls, cfg: TaskConfig) -> "CTaskConfig":
        d = asdict(cfg)
        c = cls()
        for name, typ in cls._fields_:
            setattr(c, name, int(d[name]) if typ is _int else float(d[name]))
        return c


def env_lib() -> ctypes.CDLL:
    lib = sim_lib()
    if getattr(lib, "_env_declared", False):
        return lib
    f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")

    def d(name, res, *args):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)

    d("arc_env_init", _int, _vp, ctypes.POINTER(CTaskConfig), ctypes.c_ulonglong)
    d("arc_env_reset", _int, _vp, _vp, _int, _vp)
    d("arc_env_step", _int, _vp, _vp, _vp)
    d("arc_env_set_fused", _int, _vp, _int)
    d("arc_env_set_step_order", _int, _vp, _int)
    d("arc_env_get_step_order", _int, _vp, _vp)
    d("arc_env_step_host", _int, _vp, _vp, _vp, _vp, _vp, _vp, _int)
    d("arc_env_part_range", _int, _vp, _int, _int, ctypes.POINTER(_int), ctypes.POINTER(_int))
    d("arc_env_step_part", _int, _vp, _int, _int, _vp)
    d("arc_env_merge_parts", _int, _vp, _int, _vp)
    d("arc_env_task_step", _int, _vp, _vp, _vp)
    d("arc_env_observe", _int, _vp, _vp)
    d("arc_env_buffer", _int, _vp, _int, ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_longlong * 2),
      ctypes.POINTER(_int), ctypes.POINTER(_int), ctypes.POINTER(_int))
    d("arc_env_dlpack", _int, _vp, _int, ctypes.POINTER(_vp))
    d("arc_env_download", _int, _vp, _int, _vp)
    d("arc_env_upload", _int, _vp, _int, _vp)
    d("arc_env_get_task_state", _int, _vp, i32, _int, f64)
    d("arc_env_set_task_state", _int, _vp, i32, _int, f64)
    d("arc_env_set_targets", _int, _vp, i32, _int, f64)
    lib._env_declared = True
    return lib


class GpuTask:
    """The device task layer of one Sim: init, buffers, host-side state access."""

    def __init__(self, sim: Sim, cfg: TaskConfig, seed: int):
        self.sim, self.cfg = sim, cfg
        self.lib = env_lib()
        c = CTaskConfig.of(cfg)
        sim._check(self.lib.arc_env_init(sim.ptr, ctypes.byref(c), ctypes.c_ulonglong(seed & (2**64 - 1))))

    def buffer(self, which: int):
        ptr, shape = _vp(), (ctypes.c_longlong * 2)()
        nd, code, bits = _int(), _int(), _int()
        self.sim._check(self.lib.arc_env_buffer(self.sim.ptr, which, ctypes.byref(ptr), ctypes.byref(shape),
                                                ctypes.byref(nd), ctypes.byref(code), ctypes.byref(bits)))
        dt = {(2, 32): np.float32, (2, 64): np.float64, (1, 8): np.uint8, (0, 8): np.int8,
              (0, 32): np.int32}[(code.value, bits.value)]
        return ptr.value, tuple(shape[: nd.value]), dt

    def download(self, which: int) -> np.ndarray:
        _, shape, dt = self.buffer(which)
        out = np.empty(shape, dtype=dt)
        self.sim._check(self.lib.arc_env_download(self.sim.ptr, which, out.ctypes.data))
        return out

    def upload(self, which: int, arr: np.ndarray) -> None:
        _, shape, dt = self.buffer(which)
        a = np.ascontiguousarray(arr, dtype=dt).reshape(shape)
        self.sim._check(self.lib.arc_env_upload(self.sim.ptr, which, a.ctypes.data))

    def get_state(self, ids=None) -> np.ndarray:
        ids = np.arange(self.sim.num_worlds) if ids is None else ids
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        out = np.zeros((len(ids), TASK_STATE_SIZE))
        self.sim._check(self.lib.arc_env_get_task_state(self.sim.ptr, ids, len(ids), out))
        return out

    def set_state(self, state, ids=None) -> None:
        ids = np.arange(self.sim.num_worlds) if ids is None else ids
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        st = np.ascontiguousarray(state, dtype=np.float64).reshape(len(ids), TASK_STATE_SIZE)
        self.sim._check(self.lib.arc_env_set_task_state(self.sim.ptr, ids, len(ids), st))

    def set_targets(self, ids, xy) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        xy = np.ascontiguousarray(xy, dtype=np.float64)
        self.sim._check(self.lib.arc_env_set_targets(self.sim.ptr, ids, len(ids), xy))


class ArcTask:
    """arc/task.py's ArcTask with the task math on the GPU (host numpy in/out)."""

    def __init__(self, num_worlds: int, config: TaskConfig | None = None, threads: int = 1,
                 seed: int | None = None, *, fp64: bool = False):
        self.cfg = cfg = config or TaskConfig()
        self.sim = Sim(num_worlds, cfg.dt, cfg.substeps, cfg.grid, cfg.cell, threads, fp64=fp64)
        self.nj = self.sim.num_joints
        self.rng = np.random.default_rng(seed)
        self.gpu = GpuTask(self.sim, cfg, int(self.rng.integers(0, 2**63)))
        self.obs_size = OBS_SIZE
        self._ids_all = np.arange(num_worlds, dtype=np.int32)

    # task state, read from the device (arc/task.py:98-108)
    def _col(self, k):
        return self.gpu.get_state()[:, k]

    @property
    def target(self):
        return self.gpu.get_state()[:, 0:2]

    @property
    def target_z(self):
        return self._col(2)

    @property
    def prev_dist(self):
        return self._col(3)

    @property
    def prev_gaze(self):
        return self._col(4)

    @property
    def prev_action(self):
        return self.gpu.get_state()[:, 5:17]

    @property
    def torso_steps(self):
        return self._col(17).astype(np.int64)

    @property
    def steps(self):
        return self._col(18).astype(np.int64)

    @property
    def checkpoints(self):
        return self._col(19).astype(np.int64)

    @property
    def level(self):
        return self._col(20)

    @property
    def difficulty(self):
        return self._col(21)

    @property
    def in_view(self):
        return self._col(22).astype(bool)

    def reset(self, ids) -> None:
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        if not len(ids):
            return
        self.sim._check(self.gpu.lib.arc_env_reset(self.sim.ptr, ids.ctypes.data, len(ids), None))
        self.sim.observe()

    def step(self, actions):
        a = np.ascontiguousarray(np.asarray(actions, dtype=np.float32).reshape(self.sim.num_worlds, self.nj))
        self.gpu.upload(ACTIONS, a)
        self.sim._check(self.gpu.lib.arc_env_task_step(self.sim.ptr, None, None))
        self.sim.observe()
        reward = self.gpu.download(REWARD)
        terminated = self.gpu.download(TERMINATED).astype(bool)
        truncated = self.gpu.download(TRUNCATED).astype(bool)
        st = self.gpu.get_state()
        fell = terminated
        stats = {"checkpoints": st[:, 19].astype(np.int64), "difficulty": st[:, 21].copy(),
                 "fell": fell.copy(), "cause": self.gpu.download(CAUSE).astype(np.int64),
                 "steps": st[:, 18].astype(np.int64)}
        ended = np.flatnonzero(terminated | truncated)
        if len(ended):
            stats["difficulty"][ended] = self.gpu.download(ENDED_DIFFICULTY)[ended]
            stats["steps"][ended] = self.gpu.download(ENDED_STEPS)[ended]
        return reward, terminated, truncated, stats

    def observe(self) -> np.ndarray:
        self.sim._check(self.gpu.lib.arc_env_observe(self.sim.ptr, None))
        return self.gpu.download(OBS)

    def markers(self, i: int) -> np.ndarray:
        st = self.gpu.get_state([i])[0]
        return np.array([[st[0], st[1], st[2], self.cfg.checkpoint_radius]])

    def close(self) -> None:
        self.sim.close()
