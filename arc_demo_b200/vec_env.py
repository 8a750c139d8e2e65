"""A vectorised-env adapter and observation/reward normalisation on the device.

The reference trains through Stable-Baselines3: `ArcVecEnv` (an SB3 `VecEnv`
with auto-reset and terminal observations, arc/env.py:74-141) wrapped in SB3's
`VecNormalize` (scripts/train.py:116-142). Both keep their data in host numpy
arrays. This module gives the same interface on device tensors, over
`DeviceVecEnv` (or any env with `reset()` and `step(actions)` returning torch
tensors):

- `DeviceVecEnvAdapter`: `num_envs`, `reset()`, `step_async(actions)` /
  `step_wait()` returning (obs, rewards, dones, infos) as device tensors;
  `infos` is one dict of tensors ("terminal_observation", "truncated") rather
  than one dict per world, which would bring every step back to the host.
- `DeviceVecNormalize`: running mean/variance of the observations and of the
  discounted returns, observations normalised and clipped to +-clip_obs,
  rewards scaled by the returns' standard deviation and clipped to
  +-clip_reward, the statistics frozen when `training` is False - the
  behaviour of SB3's VecNormalize with its defaults (clip 10, gamma 0.99,
  epsilon 1e-8). The statistics are FP64, as SB3's numpy ones are.
"""

from __future__ import annotations

import torch


class DeviceRunningMeanStd:
    """Running mean and (population) variance over batches, merged with the
    parallel-variance formula of Chan, Golub and LeVeque (1979), starting
    from mean 0, variance 1 and a count of `epsilon`."""

    def __init__(self, shape=(), epsilon: float = 1e-4, device=None):
        self.mean = torch.zeros(shape, dtype=torch.float64, device=device)
        self.var = torch.ones(shape, dtype=torch.float64, device=device)
        self.count = epsilon

    def update(self, x: torch.Tensor) -> None:
        x = x.to(torch.float64)
        batch_mean = x.mean(dim=0)
        batch_var = x.var(dim=0, unbiased=False)
        self.update_from_moments(batch_mean, batch_var, x.shape[0])

    def update_from_moments(self, batch_mean, batch_var, batch_count: int) -> None:
        delta = batch_mean - self.mean
        total = self.count + batch_count
        new_mean = self.mean + delta * (batch_count / total)
        m2 = self.var * self.count + batch_var * batch_count + delta.square() * (self.count * batch_count / total)
        self.mean, self.var, self.count = new_mean, m2 / total, total

    def state_dict(self) -> dict:
        return {"mean": self.mean.clone(), "var": self.var.clone(), "count": self.count}

    def load_state_dict(self, d: dict) -> None:
        self.mean = d["mean"].to(self.mean.device, torch.float64).clone()
        self.var = d["var"].to(self.var.device, torch.float64).clone()
        self.count = float(d["count"])


class DeviceVecEnvAdapter:
    """SB3's VecEnv calling convention over a device env: step_async stores
    the actions, step_wait steps and returns device tensors."""

    def __init__(self, env):
        self.env = env
        self.num_envs = env.num_envs
        self._actions = None

    def reset(self) -> torch.Tensor:
        return self.env.reset()

    def step_async(self, actions: torch.Tensor) -> None:
        self._actions = actions

    def step_wait(self):
        obs, reward, terminated, truncated = self.env.step(self._actions)
        dones = terminated.bool() | truncated.bool()
        infos = {"terminal_observation": self.env.terminal_obs, "truncated": truncated.bool() & ~terminated.bool()}
        return obs, reward, dones, infos

    def step(self, actions: torch.Tensor):
        self.step_async(actions)
        return self.step_wait()


class DeviceVecNormalize:
    """SB3's VecNormalize on device tensors over a `DeviceVecEnvAdapter`-like
    env (reset, step_async/step_wait returning (obs, rewards, dones, infos))."""

    def __init__(self, venv, training: bool = True, norm_obs: bool = True, norm_reward: bool = True,
                 clip_obs: float = 10.0, clip_reward: float = 10.0, gamma: float = 0.99, epsilon: float = 1e-8):
        self.venv = venv
        self.num_envs = venv.num_envs
        self.training, self.norm_obs, self.norm_reward = training, norm_obs, norm_reward
        self.clip_obs, self.clip_reward, self.gamma, self.epsilon = clip_obs, clip_reward, gamma, epsilon
        self.obs_rms = None
        self.ret_rms = None
        self.returns = None
        self.old_obs = self.old_reward = None

    def _init_stats(self, obs: torch.Tensor) -> None:
        if self.obs_rms is None:
            self.obs_rms = DeviceRunningMeanStd(shape=obs.shape[1:], device=obs.device)
            self.ret_rms = DeviceRunningMeanStd(shape=(), device=obs.device)
            self.returns = torch.zeros(self.num_envs, dtype=torch.float64, device=obs.device)

    def normalize_obs(self, obs: torch.Tensor) -> torch.Tensor:
        if not self.norm_obs:
            return obs
        z = (obs.to(torch.float64) - self.obs_rms.mean) / torch.sqrt(self.obs_rms.var + self.epsilon)
        return z.clamp(-self.clip_obs, self.clip_obs).to(obs.dtype)

    def normalize_reward(self, reward: torch.Tensor) -> torch.Tensor:
        if not self.norm_reward:
            return reward
        r = reward.to(torch.float64) / torch.sqrt(self.ret_rms.var + self.epsilon)
        return r.clamp(-self.clip_reward, self.clip_reward).to(reward.dtype)

    def reset(self) -> torch.Tensor:
        obs = self.venv.reset()
        self._init_stats(obs)
        self.old_obs = obs
        self.returns.zero_()
        if self.training and self.norm_obs:
            self.obs_rms.update(obs)
        return self.normalize_obs(obs)

    def step_async(self, actions: torch.Tensor) -> None:
        self.venv.step_async(actions)

    def step_wait(self):
        obs, rewards, dones, infos = self.venv.step_wait()
        self._init_stats(obs)
        self.old_obs, self.old_reward = obs, rewards
        if self.training and self.norm_obs:
            self.obs_rms.update(obs)
        norm_obs = self.normalize_obs(obs)
        if self.training:
            self.returns = self.returns * self.gamma + rewards.to(torch.float64)
            self.ret_rms.update(self.returns)
        norm_rewards = self.normalize_reward(rewards)
        infos = dict(infos)
        if "terminal_observation" in infos:
            infos["terminal_observation"] = self.normalize_obs(infos["terminal_observation"])
        self.returns = torch.where(dones.bool(), torch.zeros_like(self.returns), self.returns)
        return norm_obs, norm_rewards, dones, infos

    def step(self, actions: torch.Tensor):
        self.step_async(actions)
        return self.step_wait()

    def state_dict(self) -> dict:
        return {"obs_rms": self.obs_rms.state_dict(), "ret_rms": self.ret_rms.state_dict()}

    def load_state_dict(self, d: dict) -> None:
        if self.obs_rms is None:
            dev = d["obs_rms"]["mean"].device
            self.obs_rms = DeviceRunningMeanStd(shape=d["obs_rms"]["mean"].shape, device=dev)
            self.ret_rms = DeviceRunningMeanStd(shape=(), device=dev)
            self.returns = torch.zeros(self.num_envs, dtype=torch.float64, device=dev)
        self.obs_rms.load_state_dict(d["obs_rms"])
        self.ret_rms.load_state_dict(d["ret_rms"])
