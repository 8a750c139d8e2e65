"""The step order of the env's control step (arc_env_set_step_order): the
worlds of each range the step kernels take, by difficulty band, hardest
first, and the results, which must not depend on it.

A world's step reads and writes only its own record, terrain and task state
(csrc/arc_phys.c:707-747, arc/task.py:155-259), so which worlds share a CTA
cannot change it: the order is a schedule, and both orders must give the same
worlds bit for bit, through every form of the control step."""

import numpy as np
import pytest

from arc_demo_b200.native import KERNEL_PLAIN, KERNEL_WARPS
from arc_demo_b200.task import TaskConfig

pytestmark = pytest.mark.gpu

BANDS = 16


def bands_of(difficulty):
    d = np.asarray(difficulty, dtype=np.float64)
    b = np.where(d >= 1.0, BANDS - 1, np.where(d > 0.0, np.floor(d * BANDS), 0)).astype(np.int64)
    return np.clip(b, 0, BANDS - 1)


def test_step_order_is_by_band_hardest_first():
    from arc_demo_b200.torch_env import DeviceVecEnv
    n = 3000  # two whole chunks of the order kernels and a part chunk
    env = DeviceVecEnv(n, TaskConfig(curriculum=False), seed=3)
    rng = np.random.default_rng(5)
    levels = rng.uniform(0.0, 1.0, n)
    levels[:7] = [0.0, 1.0, 1.0 / 16, 0.5, 15.999 / 16, 0.0625 - 1e-12, 0.999999]
    env.set_levels(levels)
    env.reset()
    env.set_kernel(KERNEL_WARPS)
    order = env.step_order()
    assert sorted(order.tolist()) == list(range(n))
    bands = bands_of(env.gpu.get_state()[:, 21])  # column 21: difficulty
    assert order.tolist() == sorted(range(n), key=lambda w: (-bands[w], w))
    env.set_step_order(0)
    assert env.step_order().tolist() == list(range(n))
    env.close()


@pytest.mark.parametrize("kernel,queue,form", [(KERNEL_WARPS, False, 0), (KERNEL_WARPS, True, 0),
                                               (KERNEL_WARPS, True, 1), (KERNEL_PLAIN, False, 0)])
def test_step_order_gives_the_same_worlds(kernel, queue, form):
    """Difficulty order against index order, with resets on most steps
    (max_steps 6, curriculum on, so difficulties move): the graph step, the
    step in two parts and the host-buffer step in three chunks (each range in
    its own order) all give the same outputs, ended worlds and states."""
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv
    n = 6500
    envs = [DeviceVecEnv(n, TaskConfig(curriculum=True, max_steps=6), seed=21) for _ in range(2)]
    envs[1].set_step_order(0)
    for e in envs:
        e.set_kernel(kernel)
        e.sim.set_work_queue(queue)
        e.set_fused(form)
        e.set_levels(np.random.default_rng(2).uniform(0.0, 1.0, n))
        e.reset()
    ranges = [envs[0].part_range(p, 2) for p in range(2)]
    assert not np.array_equal(envs[0].step_order(), envs[1].step_order())
    rng = np.random.default_rng(9)
    ended = 0
    for k in range(12):
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
                e.step_parts(policy, 2)
            else:
                e.step_host(torch.from_numpy(a))
        torch.cuda.synchronize()
        x, y = envs
        for name, u, v in (("obs", x.obs, y.obs), ("reward", x.reward, y.reward),
                           ("terminated", x.terminated, y.terminated), ("truncated", x.truncated, y.truncated),
                           ("cause", x.cause, y.cause)):
            assert torch.equal(u, v), f"step {k}: {name} differs"
        if k % 3 == 2:
            for u, v in zip(x._host_out, y._host_out):
                assert torch.equal(u, v), k
        nd = int(x.done_count.item())
        assert nd == int(y.done_count.item())
        ended += nd
        assert sorted(x.done_list[:nd].tolist()) == sorted(y.done_list[:nd].tolist())
        assert np.array_equal(x.sim.get_state(), y.sim.get_state(), equal_nan=True)
        assert np.array_equal(x.gpu.get_state(), y.gpu.get_state(), equal_nan=True)
    assert ended > n
    for e in envs:
        e.close()
