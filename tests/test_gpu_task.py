"""Parity of the device task layer (arc/task.py on the GPU) with the numpy oracle.

The physics state and the task state are teacher-forced: after each GPU
step, the oracle's simulation is given the GPU's post-step physics state and
the task state the GPU started from, and oracle/task_oracle.py computes the
rewards, terminations and observations from the same inputs. The task math
is FP64 on both sides; observations are float32 on both sides.

Tolerances: rewards 1e-5 absolute (FP64 math, float32 output);
terminations, truncations and causes exact; observations 1e-5 absolute.
Checkpoints drawn after a reached checkpoint come from the device stream,
not numpy's, so those worlds' targets are checked for the reference's
placement rule (3-6 m away, inside the terrain) instead.
"""

import ctypes

import numpy as np
import pytest

from arc_demo_b200.native import Sim
from arc_demo_b200.task import (ACTIONS, CAUSE, OBS, REWARD, TERMINATED, TRUNCATED, GpuTask, TaskConfig)
from oracle.oracle import OracleSim
from oracle.task_oracle import TaskConfig as OracleConfig
from oracle.task_oracle import TaskOracle

pytestmark = pytest.mark.gpu


def load_task_state(t: TaskOracle, st: np.ndarray) -> None:
    t.target[:] = st[:, 0:2]
    t.target_z[:] = st[:, 2]
    t.prev_dist[:] = st[:, 3]
    t.prev_gaze[:] = st[:, 4]
    t.prev_action[:] = st[:, 5:17]
    t.torso_steps[:] = st[:, 17].astype(np.int64)
    t.steps[:] = st[:, 18].astype(np.int64)
    t.checkpoints[:] = st[:, 19].astype(np.int64)
    t.level[:] = st[:, 20]
    t.difficulty[:] = st[:, 21]
    t.in_view[:] = st[:, 22] != 0


def make(n, curriculum=True, fp64=False):
    cfg = TaskConfig(curriculum=curriculum)
    sim = Sim(n, fp64=fp64)
    gpu = GpuTask(sim, cfg, seed=42)
    osim = OracleSim(n, bits=64 if fp64 else 32)
    task = TaskOracle(osim, OracleConfig(curriculum=curriculum), seed=0)
    return cfg, sim, gpu, osim, task


@pytest.mark.parametrize("fp64", [False, True])
def test_task_step_and_observe_match_oracle(fp64):
    n = 64
    cfg, sim, gpu, osim, task = make(n, curriculum=True, fp64=fp64)
    lib = gpu.lib
    rng = np.random.default_rng(0)
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    diffs = np.round(rng.uniform(0, 1, n), 1)
    sim.reset(np.arange(n), seeds, diffs)
    osim.reset(np.arange(n), seeds, diffs)
    osim.set_state(sim.get_state())
    osim.observe()
    # checkpoints from the oracle's numpy stream, injected on both sides
    task.new_targets(np.arange(n))
    gpu.set_targets(np.arange(n), task.target)
    st = gpu.get_state()
    st[:, 20] = diffs
    st[:, 21] = diffs
    # provoke events: beached soon, truncation soon, a checkpoint under some robots
    st[0:4, 17] = 29
    st[4:8, 18] = cfg.max_steps - 1
    gpu.set_state(st)
    root = sim.observe()[0]
    near = np.arange(8, 16)
    gpu.set_targets(near, root[near, :2] + 0.1)
    checked_hits = 0
    for step in range(25):
        st0 = gpu.get_state()
        a = rng.uniform(-1.3, 1.3, (n, 12)).astype(np.float32)
        gpu.upload(ACTIONS, a)
        sim._check(lib.arc_env_task_step(sim.ptr, None, None))
        sim._check(lib.arc_env_observe(sim.ptr, None))
        r_g = gpu.download(REWARD)
        te_g = gpu.download(TERMINATED).astype(bool)
        tr_g = gpu.download(TRUNCATED).astype(bool)
        c_g = gpu.download(CAUSE)
        obs_g = gpu.download(OBS)
        st1 = gpu.get_state()
        # oracle from the same inputs
        osim.set_state(sim.get_state())
        load_task_state(task, st0)
        r_o, te_o, tr_o, stats = task.after_step(np.clip(a.astype(np.float64), -1, 1))
        hit = np.flatnonzero(stats["reached"] & ~te_o)
        # device draws for reached checkpoints: rule check, then align the oracle
        for i in hit:
            d = np.hypot(*(st1[i, 0:2] - osim.root[i, :2]))
            inside = np.all(np.abs(st1[i, 0:2]) < osim.half_extent - cfg.border)
            fallback = np.allclose(st1[i, 0:2], 0.5 * osim.root[i, :2])
            assert (3.0 - 1e-9 <= d <= 6.0 + 1e-9 and inside) or fallback
            checked_hits += 1
        task.set_targets(hit, st1[hit, 0:2]) if len(hit) else None
        obs_o = task.observe()
        assert np.array_equal(te_g, te_o), step
        assert np.array_equal(tr_g, tr_o), step
        assert np.array_equal(c_g.astype(np.int64), stats["cause"]), step
        assert np.allclose(r_g, r_o, rtol=0, atol=1e-5), (step, np.abs(r_g - r_o).max())
        assert np.allclose(st1[:, 3], task.prev_dist, atol=1e-9)
        assert np.allclose(st1[:, 4], task.prev_gaze, atol=1e-9)
        assert np.array_equal(st1[:, 17], task.torso_steps)
        assert np.array_equal(st1[:, 18], task.steps)
        assert np.array_equal(st1[:, 19], task.checkpoints)
        assert np.array_equal(st1[:, 20], task.level)
        assert np.allclose(obs_g, obs_o, rtol=0, atol=1e-5), (step, np.abs(obs_g - obs_o).max())
    assert checked_hits >= 1


def test_reset_places_checkpoints_by_the_reference_rule():
    n = 256
    cfg, sim, gpu, _, _ = make(n)
    sim._check(gpu.lib.arc_env_reset(sim.ptr, None, -1, None))
    st = gpu.get_state()
    root = sim.observe()[0]
    d = np.hypot(st[:, 0] - root[:, 0], st[:, 1] - root[:, 1])
    limit = sim.half_extent - cfg.border
    inside = np.all(np.abs(st[:, 0:2]) < limit, axis=1)
    fallback = np.all(np.isclose(st[:, 0:2], 0.5 * root[:, :2]), axis=1)
    assert np.all(((d >= 3.0) & (d <= 6.0) & inside) | fallback)
    assert np.all(st[:, 23] == 1)  # one episode started per world
    assert np.all(st[:, 18] == 0) and np.all(st[:, 5:17] == 0)
    # device-drawn seeds give distinct terrains
    h0, h1 = sim.get_terrain(0)[0], sim.get_terrain(1)[0]
    assert st[0, 21] == 0.0 or not np.array_equal(h0, h1)


@pytest.mark.parametrize("queue", [False, True])
def test_env_graph_step_equals_eager_step(queue):
    """The control step as one CUDA graph (captured once, replayed) equals
    the same launches made eagerly, also with the step kernel's work queue
    (its counter must come back to zero at the end of every replay)."""
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv
    n = 96
    envs = [DeviceVecEnv(n, TaskConfig(curriculum=True), seed=7) for _ in range(2)]
    envs[0].sim.set_work_queue(queue)
    for e in envs:
        e.set_levels(np.linspace(0, 1, n))
        e.reset()
    rng = np.random.default_rng(1)
    for _ in range(12):
        a = torch.from_numpy(rng.uniform(-1, 1, (n, 12)).astype(np.float32)).cuda()
        envs[0].step(a, graph=True)
        envs[1].step(a, graph=False)
        torch.cuda.synchronize()
        for x, y in ((envs[0].obs, envs[1].obs), (envs[0].reward, envs[1].reward),
                     (envs[0].terminated, envs[1].terminated), (envs[0].truncated, envs[1].truncated)):
            assert torch.equal(x, y)
    assert np.array_equal(envs[0].sim.get_state(), envs[1].sim.get_state(), equal_nan=True)


def test_dlpack_tensors_alias_the_library_buffers():
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv
    n = 40
    env = DeviceVecEnv(n, seed=3)
    for which, t in ((OBS, env.obs), (REWARD, env.reward), (ACTIONS, env.actions)):
        ptr, shape, dt = env.gpu.buffer(which)
        assert t.data_ptr() == ptr and tuple(t.shape) == shape and t.is_cuda
    env.reset()
    env.actions.fill_(0.0)
    obs, rew, term, trunc = env.step()
    torch.cuda.synchronize()
    assert obs.shape == (n, 195) and torch.isfinite(obs).all()
    host = env.gpu.download(OBS)
    assert np.array_equal(host, obs.cpu().numpy())


def test_env_auto_reset_writes_terminal_observation():
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv
    n = 32
    env = DeviceVecEnv(n, TaskConfig(curriculum=False, max_steps=5), seed=9)
    env.reset()
    zeros = torch.zeros((n, 12), device="cuda")
    for t in range(5):
        obs, rew, term, trunc = env.step(zeros)
    torch.cuda.synchronize()
    assert bool((trunc.bool() | term.bool()).all())
    assert int(env.done_count.item()) == n
    st = env.gpu.get_state()
    assert np.all(st[:, 18] == 0)        # new episodes started
    assert np.all(st[:, 23] == 2)        # second episode of every world
    assert torch.isfinite(env.terminal_obs).all()
    assert not torch.equal(env.terminal_obs, env.obs)


@pytest.mark.parametrize("queue,form", [(False, 1), (True, 1), (False, 2), (True, 2)])
def test_fused_control_step_agrees_with_separate_kernels(queue, form):
    """The fused control step (k_control_step's fused forms: each group's
    physics, then its rewards, observations and heights, and with form 2 its
    resets, in the same kernel) against the physics-only kernel followed by
    the task, heights and reset kernels, one control step at a time from the
    same world and task states, through the graph step, the step in parts and
    the host-buffer step, with resets on most steps (max_steps 6, curriculum
    on). The task functions are one compiled copy, but the physics is inlined
    into each form's kernel, whose code around it differs, so the two steps
    agree to FP32 rounding rather than bit for bit: body positions within
    1e-5 relative at p99, and rewards, observations, done flags, causes and
    ended worlds equal but for the few worlds that a threshold decided within
    that rounding."""
    import torch
    from arc_demo_b200.native import KERNEL_WARPS
    from arc_demo_b200.torch_env import DeviceVecEnv
    from parity_checks import body_errors
    n = 200
    envs = [DeviceVecEnv(n, TaskConfig(curriculum=True, max_steps=6), seed=13) for _ in range(2)]
    envs[0].set_fused(form)
    envs[1].set_fused(0)
    for e in envs:
        e.set_kernel(KERNEL_WARPS)
        e.sim.set_work_queue(queue)
        e.set_levels(np.linspace(0, 1, n))
        e.reset()
    rng = np.random.default_rng(8)
    ranges = [envs[0].part_range(p, 3) for p in range(3)]
    x, y = envs
    ended, odd = 0, 0
    for k in range(15):
        # the same states in both
        x.sim.set_state(y.sim.get_state())
        x.gpu.set_state(y.gpu.get_state())
        a = rng.uniform(-1.2, 1.2, (n, 12)).astype(np.float32)
        d_a = torch.from_numpy(a).cuda()
        torch.cuda.synchronize()

        def policy(p, obs, act):
            first, count = ranges[p]
            act.copy_(d_a[first:first + count])
        for e in envs:
            if k % 3 == 0:
                e.step(d_a)
            elif k % 3 == 1:
                e.step_parts(policy, 3)
            else:
                e.step_host(torch.from_numpy(a))
        torch.cuda.synchronize()
        # worlds whose episodes, causes or rewards came out differently: a
        # threshold that FP32 rounding decided; they are few and counted
        flags = [(u != v).reshape(n, -1).any(1).cpu().numpy() for u, v in
                 ((x.terminated, y.terminated), (x.truncated, y.truncated), (x.cause, y.cause))]
        diff = np.logical_or.reduce(flags)
        diff |= (x.reward - y.reward).abs().cpu().numpy() > 1e-3
        odd += int(diff.sum())
        same = ~diff
        dx, dq = body_errors(x.sim.get_state()[same], y.sim.get_state()[same])
        assert np.percentile(dx, 99) <= 1e-5 and np.percentile(dq, 99) <= 1e-5, (k, dx.max(), dq.max())
        obs_d = (x.obs - y.obs).abs().amax(1).cpu().numpy()[same]
        assert np.percentile(obs_d, 99) <= 1e-3, (k, obs_d.max())
        nd, ny = int(x.done_count.item()), int(y.done_count.item())
        ended += ny
        ex, ey = set(x.done_list[:nd].tolist()), set(y.done_list[:ny].tolist())
        assert len(ex ^ ey) <= diff.sum(), k
    assert odd <= 0.01 * 15 * n, odd
    assert ended > n  # most worlds went through at least one reset
