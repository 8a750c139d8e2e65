"""Host-side logic that needs no GPU: the serving load generator's request
shapes, the serving engine's per-slot byte count, and the task weights'
balance."""

import math

import numpy as np

from arc_demo_b200.serve import WORLD_BYTES, request_shape


def test_request_shapes_are_log_uniform_within_bounds():
    rng = np.random.default_rng(0)
    shapes = np.array([request_shape(rng) for _ in range(20000)])
    n, k = shapes[:, 0], shapes[:, 1]
    assert n.min() >= 1 and n.max() <= 8192
    assert k.min() == 1 and k.max() == 32
    # log-uniform: each factor-of-two band of sizes gets about the same share
    bands = np.bincount(np.floor(np.log2(n)).astype(int), minlength=14)[:13]
    assert bands.min() > 0.6 * bands.mean() and bands.max() < 1.4 * bands.mean()
    assert abs(k.mean() - 16.5) < 0.5


def test_state_budget_holds_about_1_7_million_worlds():
    # 40 GB of FP32 worlds with 64 x 64 terrains and the task layer's rows:
    # the serving configuration
    assert 22_000 < WORLD_BYTES < 25_000
    assert math.isclose(40e9 / WORLD_BYTES, 1.71e6, rel_tol=0.02)


def test_no_reward_for_ending_episodes_on_purpose():
    """tests/test_env.py:148-153 of the reference: under PPO's discount,
    standing still forever costs less than falling once (the task weights
    are the reference's, arc/task.py:17-66)."""
    from arc_demo_b200.task import TaskConfig
    cfg = TaskConfig()
    gamma = 0.99
    assert cfg.w_time / (1 - gamma) < cfg.w_fall
