"""Device-resident vectorised env over libarcsim.so, for PyTorch training loops.

`DeviceVecEnv` runs ArcVecEnv.step_wait's work (arc/env.py:99-117) on the GPU:
actuation, physics, rewards, terminations, checkpoints, curriculum,
observations and the auto-reset of ended worlds, in one CUDA graph per
control step (or, with step_parts, in ranges of worlds on side-by-side
streams, each after its share of the policy). Observations, rewards and done flags are torch tensors that
alias the library's device buffers through DLPack: no copies, no host
round trip. Torch is only the consumer here; the step itself is the
library's CUDA kernels.
"""

from __future__ import annotations

import ctypes

import torch

from .native import Sim
from .task import (ACTIONS, CAUSE, DONE_COUNT, DONE_LIST, ENDED_CHECKPOINTS, ENDED_DIFFICULTY, ENDED_STEPS, OBS,
                   REWARD, TERMINAL_OBS, TERMINATED, TRUNCATED, GpuTask, TaskConfig)

_capsule_new = ctypes.pythonapi.PyCapsule_New
_capsule_new.restype = ctypes.py_object
_capsule_new.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_void_p]

CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: torch's default stream has handle 0


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = (stream or torch.cuda.current_stream()).cuda_stream
    return s if s else CUDA_STREAM_LEGACY


def dlpack_tensor(gpu: GpuTask, which: int) -> torch.Tensor:
    """A torch tensor aliasing one of the library's device buffers."""
    p = ctypes.c_void_p()
    gpu.sim._check(gpu.lib.arc_env_dlpack(gpu.sim.ptr, which, ctypes.byref(p)))
    return torch.utils.dlpack.from_dlpack(_capsule_new(p, b"dltensor", None))


class DeviceVecEnv:
    def __init__(self, num_envs: int, config: TaskConfig | None = None, seed: int = 0, *, fp64: bool = False,
                 kernel: int | None = None, worlds_per_cta: int = 16):
        self.cfg = cfg = config or TaskConfig()
        self.num_envs = num_envs
        self.sim = Sim(num_envs, cfg.dt, cfg.substeps, cfg.grid, cfg.cell, fp64=fp64)
        if kernel is not None:
            self.sim.set_kernel(kernel, worlds_per_cta)
        self.gpu = GpuTask(self.sim, cfg, seed)
        self.obs = dlpack_tensor(self.gpu, OBS)
        self.terminal_obs = dlpack_tensor(self.gpu, TERMINAL_OBS)
        self.reward = dlpack_tensor(self.gpu, REWARD)
        self.terminated = dlpack_tensor(self.gpu, TERMINATED)
        self.truncated = dlpack_tensor(self.gpu, TRUNCATED)
        self.cause = dlpack_tensor(self.gpu, CAUSE)
        self.actions = dlpack_tensor(self.gpu, ACTIONS)
        self.done_list = dlpack_tensor(self.gpu, DONE_LIST)
        self.done_count = dlpack_tensor(self.gpu, DONE_COUNT)
        self.ended_checkpoints = dlpack_tensor(self.gpu, ENDED_CHECKPOINTS)
        self.ended_steps = dlpack_tensor(self.gpu, ENDED_STEPS)
        self.ended_difficulty = dlpack_tensor(self.gpu, ENDED_DIFFICULTY)

    def set_kernel(self, kernel: int, worlds_per_cta: int = 16) -> None:
        self.sim.set_kernel(kernel, worlds_per_cta)

    def set_fused(self, mode: int) -> None:
        """With the warp-per-leg kernel: 0 the step kernel, then the task,
        heights and reset kernels; 1 the step and the task layer fused per
        group of 32 worlds, the resets after; 2 the resets fused too (one
        launch per control step). Forms 1 and 2 agree with form 0 to FP32
        rounding (their physics is compiled into their own kernel)."""
        self.sim._check(self.gpu.lib.arc_env_set_fused(self.sim.ptr, int(mode)))

    def set_step_order(self, mode: int) -> None:
        """1 (the default): the step kernels take each range's worlds by
        difficulty band, hardest first; 0: in index order. The results are
        the same bit for bit."""
        self.sim._check(self.gpu.lib.arc_env_set_step_order(self.sim.ptr, int(mode)))

    def step_order(self):
        """The order (numpy int32 permutation) a whole control step hands the
        step kernels now."""
        import numpy as np
        out = np.empty(self.num_envs, dtype=np.int32)
        self.sim._check(self.gpu.lib.arc_env_get_step_order(self.sim.ptr, out.ctypes.data))
        return out

    def set_levels(self, levels) -> None:
        """Per-world terrain difficulty levels (the curriculum state)."""
        import numpy as np
        st = self.gpu.get_state()
        st[:, 20] = np.asarray(levels, dtype=np.float64)
        st[:, 21] = st[:, 20]
        self.gpu.set_state(st)

    def reset(self) -> torch.Tensor:
        self.sim._check(self.gpu.lib.arc_env_reset(self.sim.ptr, None, -1, ctypes.c_void_p(stream_handle())))
        return self.obs

    def step(self, actions: torch.Tensor | None = None, *, graph: bool = True):
        """One control step of every world on the current torch stream.

        actions: N x 12 float32 on the device, or None when the policy
        already wrote `self.actions`. Returns (obs, reward, terminated,
        truncated) views; ended worlds are already reset, their last
        observation is in `terminal_obs`."""
        st = ctypes.c_void_p(stream_handle())
        if graph:
            if actions is not None:
                self.actions.copy_(actions)
            rc = self.gpu.lib.arc_env_step(self.sim.ptr, None, st)
        else:
            a = self.actions if actions is None else actions.contiguous()
            rc = self.gpu.lib.arc_env_step(self.sim.ptr, ctypes.c_void_p(a.data_ptr()), st)
        self.sim._check(rc)
        return self.obs, self.reward, self.terminated, self.truncated

    def part_range(self, part: int, parts: int) -> tuple[int, int]:
        """(first, count): the worlds of part `part` of `parts` (arc_env_part_range)."""
        first, count = ctypes.c_int(), ctypes.c_int()
        self.sim._check(self.gpu.lib.arc_env_part_range(self.sim.ptr, part, parts, ctypes.byref(first),
                                                        ctypes.byref(count)))
        return first.value, count.value

    def step_parts(self, policy, parts: int = 4):
        """One control step of every world in `parts` ranges, each on a stream
        of its own: policy(part, obs, actions) writes the part's actions (obs
        and actions are that part's rows of self.obs and self.actions), then
        the part steps (arc_env_step_part). A part's policy starts once the
        policy of the part before it has finished, so it runs beside that
        part's step, and its own step fills the last wave of the steps before
        it. The part streams start after the work queued on the current
        stream, which waits for all of them; the ended-world list is merged
        in part order. World for world the results equal step()'s. Returns
        (obs, reward, terminated, truncated)."""
        cached = getattr(self, "_parts", None)
        if cached is None or cached[0] != parts:
            ranges = [self.part_range(p, parts) for p in range(parts)]
            cached = self._parts = (parts, ranges, [torch.cuda.Stream() for _ in range(parts)])
        _, ranges, streams = cached
        cur = torch.cuda.current_stream()
        start = torch.cuda.Event()
        start.record(cur)
        ends, acted = [], None
        for p, ((first, count), st) in enumerate(zip(ranges, streams)):
            st.wait_event(start)
            if acted is not None:
                st.wait_event(acted)
            with torch.cuda.stream(st):
                policy(p, self.obs[first:first + count], self.actions[first:first + count])
                acted = torch.cuda.Event()
                acted.record(st)
                self.sim._check(self.gpu.lib.arc_env_step_part(self.sim.ptr, p, parts,
                                                               ctypes.c_void_p(stream_handle(st))))
                end = torch.cuda.Event()
                end.record(st)
            ends.append(end)
        for end in ends:
            cur.wait_event(end)
        self.sim._check(self.gpu.lib.arc_env_merge_parts(self.sim.ptr, parts, ctypes.c_void_p(stream_handle(cur))))
        return self.obs, self.reward, self.terminated, self.truncated

    def step_host(self, actions: torch.Tensor, chunks: int = 3):
        """One control step with host tensors: actions (N x 12 float32, on
        the host, ideally pinned) in; (obs, reward, terminated, truncated)
        out as pinned host tensors, reused by the next call. The worlds go
        in `chunks` ranges whose copies overlap the next range's step
        (arc_env_step_host); the results equal step() followed by copies."""
        n = self.num_envs
        if getattr(self, "_host_out", None) is None:
            self._host_out = (torch.empty((n, 195), dtype=torch.float32, pin_memory=True),
                              torch.empty(n, dtype=torch.float32, pin_memory=True),
                              torch.empty(n, dtype=torch.uint8, pin_memory=True),
                              torch.empty(n, dtype=torch.uint8, pin_memory=True))
        a = actions.contiguous()
        assert a.device.type == "cpu" and a.dtype == torch.float32 and a.shape == (n, 12)
        obs, rew, term, trunc = self._host_out
        self.sim._check(self.gpu.lib.arc_env_step_host(self.sim.ptr, a.data_ptr(), obs.data_ptr(), rew.data_ptr(),
                                                      term.data_ptr(), trunc.data_ptr(), chunks))
        return self._host_out

    def render(self, ids: torch.Tensor | None = None, width: int = 640, height: int = 360) -> torch.Tensor:
        """Frames of the worlds (all, or the int32 CUDA tensor ids) with their
        checkpoints, as the reference's rgb_array mode draws one world
        (arc/env.py:38-50): a (n, height, width, 3) uint8 CUDA tensor. Each
        world keeps its own following camera across calls."""
        from .render import Renderer
        r = getattr(self, "_renderer", None)
        if r is None or r.size() != (width, height):
            r = self._renderer = Renderer(width, height, visible=False)
        return r.env_frames(self, ids)

    def close(self) -> None:
        r = getattr(self, "_renderer", None)
        if r is not None:
            r.close()
            self._renderer = None
        self.sim.close()
