"""The batched-uneven configuration: 4,096 worlds, difficulty U[0, 1] per
world, Ornstein-Uhlenbeck actions (theta 0.15, sigma 0.3, clipped to
[-1, 1], seed 1, one control step per OU step), every world reset when its
episode ends by a fall (the task layer's terminations, arc/task.py:185-212)
or at max_steps (truncation), each control step one CUDA-graph launch.

Per-step parity of the task math is teacher-forced in test_gpu_task.py; this
test runs the loop at scale and checks its bookkeeping on every step: the
observation stays finite, the ended-world list is exactly the worlds that
terminated or truncated, every termination carries a cause, and an ended
world starts a fresh episode (step counter 0, episode count + 1).
"""

import numpy as np
import pytest

from arc_demo_b200.task import TaskConfig

pytestmark = pytest.mark.gpu


def ou_actions(n, steps, seed=1, theta=0.15, sigma=0.3):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 12))
    for _ in range(steps):
        x += theta * (0.0 - x) + sigma * rng.standard_normal((n, 12))
        yield np.clip(x, -1.0, 1.0).astype(np.float32)


@pytest.mark.parametrize("max_steps", [1000, 40])
def test_ou_rollout_4096_worlds_with_resets(max_steps):
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv

    n, steps = 4096, 120 if max_steps == 1000 else 90
    env = DeviceVecEnv(n, TaskConfig(curriculum=False, max_steps=max_steps), seed=1)
    env.set_levels(np.random.default_rng(1).uniform(0.0, 1.0, n))
    env.reset()
    ended_total, terminated_total = 0, 0
    st = env.gpu.get_state()
    for a in ou_actions(n, steps):
        obs, rew, term, trunc = env.step(torch.from_numpy(a).cuda(), graph=True)
        torch.cuda.synchronize()
        ended = (term.bool() | trunc.bool()).cpu().numpy()
        cause = env.cause.cpu().numpy()
        count = int(env.done_count.item())
        assert torch.isfinite(obs).all() and torch.isfinite(rew).all()
        assert count == int(ended.sum())
        assert np.array_equal(np.sort(env.done_list[:count].cpu().numpy()), np.flatnonzero(ended))
        assert np.all(cause[term.bool().cpu().numpy()] > 0)
        st1 = env.gpu.get_state()
        assert np.all(st1[ended, 18] == 0)                      # fresh episodes
        assert np.array_equal(st1[ended, 23], st[ended, 23] + 1)
        assert np.array_equal(st1[~ended, 18], st[~ended, 18] + 1)
        st = st1
        ended_total += count
        terminated_total += int(term.sum().item())
    assert terminated_total > 0  # falls happen under OU actions on rough terrain
    if max_steps < steps:
        # every episode ends by max_steps at the latest
        assert ended_total >= n * (steps // max_steps)


def test_vec_normalize_over_the_device_env():
    """The SB3-style adapter and VecNormalize keep everything on the device:
    normalised observations inside +-10, statistics that move, terminal
    observations of ended worlds normalised with the same statistics."""
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv
    from arc_demo_b200.vec_env import DeviceVecEnvAdapter, DeviceVecNormalize

    n = 512
    venv = DeviceVecEnv(n, TaskConfig(curriculum=False, max_steps=15), seed=4)
    env = DeviceVecNormalize(DeviceVecEnvAdapter(venv))
    obs = env.reset()
    assert obs.is_cuda and obs.shape == (n, 195)
    count0 = env.obs_rms.count
    ended = False
    for a in ou_actions(n, 20, seed=2):
        obs, rew, done, info = env.step(torch.from_numpy(a).cuda())
        ended |= bool(done.any())
        assert obs.is_cuda and rew.is_cuda and done.is_cuda
        assert torch.isfinite(obs).all() and obs.abs().max() <= 10.0
        assert torch.isfinite(rew).all() and rew.abs().max() <= 10.0
        assert info["terminal_observation"].abs().max() <= 10.0
    assert env.obs_rms.count == pytest.approx(count0 + 20 * n)
    assert ended  # max_steps 15: every world has ended once


@pytest.mark.parametrize("chunks", [1, 3, 4])
def test_host_step_in_chunks_equals_the_device_step(chunks):
    """arc_env_step_host (actions in, observations, rewards and done flags
    out through host buffers, the worlds stepped in ranges whose copies
    overlap) gives, world for world and bit for bit, what arc_env_step's
    graph gives on a twin env, through episode ends and auto-resets."""
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv

    n, steps = 1000, 30
    cfg = TaskConfig(curriculum=False, max_steps=12)
    a = DeviceVecEnv(n, cfg, seed=9)
    b = DeviceVecEnv(n, cfg, seed=9)
    for env in (a, b):
        env.set_levels(np.random.default_rng(2).uniform(0.0, 1.0, n))
        env.reset()
    torch.cuda.synchronize()
    ended_total = 0
    for act in ou_actions(n, steps, seed=4):
        ho = torch.from_numpy(act).pin_memory()
        obs, rew, term, trunc = a.step(ho.cuda(), graph=True)
        torch.cuda.synchronize()
        hobs, hrew, hterm, htrunc = b.step_host(ho, chunks=chunks)
        assert torch.equal(obs.cpu(), hobs)
        assert torch.equal(rew.cpu(), hrew)
        assert torch.equal(term.cpu(), hterm) and torch.equal(trunc.cpu(), htrunc)
        ca, cb = int(a.done_count.item()), int(b.done_count.item())
        assert ca == cb
        assert np.array_equal(np.sort(a.done_list[:ca].cpu().numpy()), np.sort(b.done_list[:cb].cpu().numpy()))
        assert torch.equal(a.terminal_obs[term.bool() | trunc.bool()], b.terminal_obs[term.bool() | trunc.bool()])
        ended_total += ca
    assert ended_total >= n  # max_steps 12: every world ended at least twice
    a.close()
    b.close()


@pytest.mark.parametrize("parts,queue", [(2, True), (4, False), (7, True)])
def test_step_in_parts_equals_the_device_step(parts, queue):
    """DeviceVecEnv.step_parts (each range of worlds' policy, then its step,
    on a stream of its own, the ranges running side by side) gives, world
    for world and bit for bit, what the policy followed by arc_env_step's
    graph gives on a twin env, through episode ends and auto-resets. The
    policy reads the observations, so a part whose rows were misplaced
    would act differently from then on."""
    import torch
    from arc_demo_b200.native import ArcSimError
    from arc_demo_b200.torch_env import DeviceVecEnv

    n, steps = 1000, 30
    cfg = TaskConfig(curriculum=False, max_steps=12)
    a = DeviceVecEnv(n, cfg, seed=9)
    b = DeviceVecEnv(n, cfg, seed=9)
    for env in (a, b):
        env.sim.set_work_queue(queue)
        env.set_levels(np.random.default_rng(2).uniform(0.0, 1.0, n))
        env.reset()
    ranges = [b.part_range(p, parts) for p in range(parts)]
    assert ranges[0][0] == 0 and sum(c for _, c in ranges) == n
    assert all(f0 + c0 == f1 for (f0, c0), (f1, _) in zip(ranges, ranges[1:]))
    torch.cuda.synchronize()
    ended_total = 0
    for act in ou_actions(n, steps, seed=4):
        ou = torch.from_numpy(act).cuda()
        torch.cuda.synchronize()

        def policy(p, obs, actions):
            first, count = ranges[p]
            actions.copy_(torch.clamp(ou[first:first + count] + 0.3 * torch.tanh(obs[:, 9:21]), -1.0, 1.0))

        a.actions.copy_(torch.clamp(ou + 0.3 * torch.tanh(a.obs[:, 9:21]), -1.0, 1.0))
        a.step()
        b.step_parts(policy, parts)
        torch.cuda.synchronize()
        assert torch.equal(a.actions, b.actions)
        assert torch.equal(a.obs, b.obs) and torch.equal(a.reward, b.reward)
        assert torch.equal(a.terminated, b.terminated) and torch.equal(a.truncated, b.truncated)
        ca, cb = int(a.done_count.item()), int(b.done_count.item())
        assert ca == cb
        assert np.array_equal(np.sort(a.done_list[:ca].cpu().numpy()), np.sort(b.done_list[:cb].cpu().numpy()))
        ended = a.terminated.bool() | a.truncated.bool()
        assert torch.equal(a.terminal_obs[ended], b.terminal_obs[ended])
        ended_total += ca
    assert ended_total >= n  # max_steps 12: every world ended at least twice
    with pytest.raises(ArcSimError):
        b.part_range(0, 17)  # at most 16 parts
    a.close()
    b.close()


def test_large_configuration_2048_step_rollout():
    """The large configuration at full size: 65,536 worlds, difficulty in
    {0, 0.1, ..., 1.0} per world, 2,048 control steps of uniform random
    actions through the CUDA-graph step with auto-reset. Observations and
    rewards stay finite on every step (checked on the device), and every
    world ends an episode at least twice (max_steps 1,000)."""
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv

    n, steps = 65536, 2048
    env = DeviceVecEnv(n, TaskConfig(curriculum=False), seed=7)
    env.set_levels(np.random.default_rng(7).integers(0, 11, n) / 10.0)
    env.reset()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    bad = torch.zeros((), dtype=torch.bool, device="cuda")
    ended = torch.zeros((), dtype=torch.int64, device="cuda")
    for _ in range(steps):
        a = torch.rand((n, 12), device="cuda", generator=gen) * 2.0 - 1.0
        obs, rew, term, trunc = env.step(a)
        bad |= ~(torch.isfinite(obs).all() & torch.isfinite(rew).all())
        ended += env.done_count[0]
    torch.cuda.synchronize()
    assert not bool(bad.item())
    assert int(ended.item()) >= 2 * n
    st = env.gpu.get_state()
    assert (st[:, 18] < 1000).all()          # no episode outlives max_steps
    assert ((st[:, 20] >= 0.0) & (st[:, 20] <= 1.0)).all()
    env.close()
