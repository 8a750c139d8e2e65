"""Edge cases of the drop-in API and the device env: no worlds at all, empty
id, offset and point lists, fewer worlds than one warp's 32 lanes, the grid
cap of the reference (csrc/arc_sim.c:36), and a world range split finer than
the worlds allow."""

import numpy as np
import pytest

from arc_demo_b200.native import ArcSimError, Sim
from arc_demo_b200.task import HEIGHT_OFFSETS, TaskConfig

pytestmark = pytest.mark.gpu


def test_no_worlds():
    sim = Sim(0)
    assert sim.num_worlds == 0
    sim.reset(np.zeros(0, np.int32), np.zeros(0, np.uint32), np.zeros(0))
    sim.step(np.zeros((0, 12)))
    root, joints, contacts, flags = sim.observe()
    assert root.shape == (0, 13) and joints.shape == (0, 36) and flags.shape == (0,)
    assert sim.heights(HEIGHT_OFFSETS).shape == (0, len(HEIGHT_OFFSETS))
    assert sim.get_state().shape == (0, sim.state_size)
    sim.close()


def test_empty_lists_on_a_batch_smaller_than_a_warp():
    n = 5
    sim = Sim(n)
    sim.reset(np.arange(n), np.arange(n, dtype=np.uint32), np.full(n, 0.5))
    before = sim.get_state()
    sim.reset(np.zeros(0, np.int32), np.zeros(0, np.uint32), np.zeros(0))  # resets nothing
    assert np.array_equal(sim.get_state(), before)
    sim.step(np.tile(sim.default_angles, (n, 1)))
    assert sim.heights(np.zeros((0, 2))).shape == (n, 0)
    assert sim.terrain_at(np.zeros(0, np.int32), np.zeros((0, 2))).shape == (0,)
    root, _, _, flags = sim.observe()
    assert np.all(np.isfinite(root)) and not flags.any()
    with pytest.raises(ArcSimError):
        sim.get_state(np.array([n]))  # one past the last world
    sim.close()


def test_grid_is_capped_at_64():
    sim = Sim(2, grid=100)
    assert sim.grid == 64 and sim.half_extent == pytest.approx(0.5 * 64 * 0.4)
    sim.reset(np.arange(2), np.arange(2, dtype=np.uint32), np.ones(2))
    heights, geom = sim.get_terrain(1)
    assert heights.shape == (64, 64) and geom[1] == pytest.approx(-0.5 * 64 * 0.4)
    sim.close()


def test_device_env_of_three_worlds_in_parts():
    """Three worlds stepped whole and in three one-world parts, through
    resets; four parts of three worlds are refused."""
    import torch
    from arc_demo_b200.torch_env import DeviceVecEnv

    env = DeviceVecEnv(3, TaskConfig(curriculum=False, max_steps=4), seed=2)
    env.reset()
    for k in range(9):
        if k % 2 == 0:
            env.step(torch.zeros((3, 12), device="cuda"))
        else:
            env.step_parts(lambda part, obs, actions: actions.zero_(), 3)
    torch.cuda.synchronize()
    assert np.all(np.isfinite(env.obs.cpu().numpy()))
    assert np.all(env.gpu.get_state()[:, 18] < 4)  # every episode restarted by max_steps
    with pytest.raises(ArcSimError):
        env.step_parts(lambda part, obs, actions: actions.zero_(), 4)
    env.close()
