"""DeviceVecNormalize against a numpy restatement of Stable-Baselines3's
VecNormalize (running mean/variance by the parallel-variance merge, clip 10,
gamma 0.99, epsilon 1e-8), on CPU tensors from a synthetic env."""

import numpy as np
import pytest
import torch

from arc_demo_b200.vec_env import DeviceRunningMeanStd, DeviceVecEnvAdapter, DeviceVecNormalize


class NumpyRMS:
    def __init__(self, shape=()):
        self.mean, self.var, self.count = np.zeros(shape), np.ones(shape), 1e-4

    def update(self, x):
        bm, bv, bc = x.mean(0), x.var(0), x.shape[0]
        d = bm - self.mean
        tot = self.count + bc
        self.mean = self.mean + d * bc / tot
        self.var = (self.var * self.count + bv * bc + d**2 * self.count * bc / tot) / tot
        self.count = tot


class FakeEnv:
    """n worlds, 5-float observations, random rewards and ends (CPU tensors)."""

    def __init__(self, n, seed):
        self.num_envs, self.g = n, torch.Generator().manual_seed(seed)
        self.terminal_obs = torch.zeros(n, 5)

    def _obs(self):
        return torch.randn(self.num_envs, 5, generator=self.g) * 3.0 + 1.5

    def reset(self):
        return self._obs()

    def step(self, actions):
        obs = self._obs()
        rew = torch.randn(self.num_envs, generator=self.g)
        term = torch.rand(self.num_envs, generator=self.g) < 0.05
        trunc = torch.rand(self.num_envs, generator=self.g) < 0.02
        self.terminal_obs = torch.randn(self.num_envs, 5, generator=self.g)
        return obs, rew, term, trunc


def test_running_mean_std_matches_numpy():
    rng = np.random.default_rng(0)
    a, b = DeviceRunningMeanStd((3,)), NumpyRMS((3,))
    for _ in range(20):
        x = rng.normal(2.0, 5.0, (int(rng.integers(1, 50)), 3))
        a.update(torch.from_numpy(x))
        b.update(x)
    assert np.allclose(a.mean.numpy(), b.mean, rtol=1e-12, atol=1e-12)
    assert np.allclose(a.var.numpy(), b.var, rtol=1e-12, atol=1e-12)
    assert a.count == pytest.approx(b.count)


def test_vec_normalize_matches_the_published_algorithm():
    n = 64
    env = DeviceVecNormalize(DeviceVecEnvAdapter(FakeEnv(n, 1)))
    ref_env = FakeEnv(n, 1)
    obs_rms, ret_rms, returns = NumpyRMS((5,)), NumpyRMS(), np.zeros(n)

    def norm(o):
        return np.clip((o - obs_rms.mean) / np.sqrt(obs_rms.var + 1e-8), -10, 10)

    o = ref_env.reset().double().numpy()
    obs_rms.update(o)
    got = env.reset()
    assert np.allclose(got.numpy(), norm(o), atol=1e-6)
    for _ in range(30):
        got_obs, got_rew, got_done, got_info = env.step(torch.zeros(n, 12))
        o, r, te, tr = ref_env.step(None)
        o, r, done = o.double().numpy(), r.double().numpy(), (te | tr).numpy()
        obs_rms.update(o)
        returns = returns * 0.99 + r
        ret_rms.update(returns)
        want_rew = np.clip(r / np.sqrt(ret_rms.var + 1e-8), -10, 10)
        assert np.allclose(got_obs.numpy(), norm(o), atol=1e-6)
        assert np.allclose(got_rew.numpy(), want_rew, atol=1e-6)
        assert np.array_equal(got_done.numpy(), done)
        assert np.allclose(got_info["terminal_observation"].numpy(),
                           norm(ref_env.terminal_obs.double().numpy()), atol=1e-6)
        returns[done] = 0.0


def test_frozen_statistics_and_checkpoint_round_trip():
    n = 16
    env = DeviceVecNormalize(DeviceVecEnvAdapter(FakeEnv(n, 2)))
    env.reset()
    for _ in range(5):
        env.step(torch.zeros(n, 12))
    saved = env.state_dict()
    env.training = False
    for _ in range(5):
        env.step(torch.zeros(n, 12))
    assert torch.equal(env.obs_rms.mean, saved["obs_rms"]["mean"])
    other = DeviceVecNormalize(DeviceVecEnvAdapter(FakeEnv(n, 3)), training=False)
    other.load_state_dict(saved)
    x = torch.randn(n, 5)
    assert torch.equal(other.normalize_obs(x), env.normalize_obs(x))
