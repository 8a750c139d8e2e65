"""Numpy restatement of arc/task.py's ArcTask. TEST INFRASTRUCTURE ONLY.

Observations, rewards, terminations, checkpoints and the terrain curriculum
of the reference's task layer (arc/task.py:17-259), computed in float64 over
any simulation object with the reference `Sim` interface (arc/native.py:73-157):
the oracle's `OracleSim`, the reference build's `RefSim`, or the CUDA
library's `Sim`. It checks the CUDA task epilogue and is the task half of
bench.py's CPU baseline. Checkpoint placement draws from numpy's PCG64
exactly as the reference does (arc/task.py:127-151).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


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

# heightmap sample grid (arc/task.py:74-76): 13 forward x 11 left offsets
_FWD = np.arange(-1.0, 1.41, 0.2)
_LEFT = np.arange(-1.0, 1.01, 0.2)
HEIGHT_OFFSETS = np.array([(f, l) for f in _FWD for l in _LEFT])


def gaze_error(rot, pos, target):
    """|angle| between body +x projected on the ground and the direction to the target."""
    fx, fy = rot[:, 0, 0], rot[:, 1, 0]
    dx, dy = target[:, 0] - pos[:, 0], target[:, 1] - pos[:, 1]
    return np.abs(np.arctan2(fx * dy - fy * dx, fx * dx + fy * dy))


class TaskOracle:
    """Task state and math of ArcTask for the N worlds of `sim`."""

    def __init__(self, sim, config: TaskConfig | None = None, seed: int | None = None):
        self.cfg = cfg = config or TaskConfig()
        self.sim = sim
        self.nj = sim.num_joints
        self.nl = sim.num_legs
        self.rng = np.random.default_rng(seed)
        n = sim.num_worlds
        self.obs_size = 9 + 3 * self.nj + 3 + len(HEIGHT_OFFSETS) + self.nl
        self.target = np.zeros((n, 2))
        self.target_z = np.zeros(n)
        self.prev_dist = np.zeros(n)
        self.prev_gaze = np.zeros(n)
        self.in_view = np.zeros(n, dtype=bool)
        self.prev_action = np.zeros((n, self.nj))
        self.torso_steps = np.zeros(n, dtype=np.int64)
        self.steps = np.zeros(n, dtype=np.int64)
        self.checkpoints = np.zeros(n, dtype=np.int64)
        self.level = np.full(n, 0.0 if cfg.curriculum else cfg.difficulty)
        self.difficulty = self.level.copy()
        self._heights = np.empty((n, len(HEIGHT_OFFSETS)))

    # arc/task.py:113-125
    def reset(self, ids) -> None:
        ids = np.asarray(ids, dtype=np.int64)
        if not len(ids):
            return
        seeds = self.rng.integers(0, 2**32, size=len(ids), dtype=np.uint32)
        self.difficulty[ids] = self.level[ids]
        self.sim.reset(ids, seeds, self.difficulty[ids])
        self.prev_action[ids] = 0.0
        self.torso_steps[ids] = 0
        self.steps[ids] = 0
        self.checkpoints[ids] = 0
        self.sim.observe()
        self.new_targets(ids)

    # arc/task.py:127-151
    def new_targets(self, ids) -> None:
        cfg = self.cfg
        pos = self.sim.root[ids, :2]
        limit = self.sim.half_extent - cfg.border
        target = np.zeros((len(ids), 2))
        pending = np.ones(len(ids), dtype=bool)
        for _ in range(20):
            k = np.flatnonzero(pending)
            if not len(k):
                break
            ang = self.rng.uniform(-np.pi, np.pi, len(k))
            dist = self.rng.uniform(cfg.checkpoint_min_dist, cfg.checkpoint_max_dist, len(k))
            cand = pos[k] + dist[:, None] * np.stack([np.cos(ang), np.sin(ang)], 1)
            ok = np.all(np.abs(cand) < limit, axis=1)
            target[k[ok]] = cand[ok]
            pending[k[ok]] = False
        k = np.flatnonzero(pending)
        target[k] = 0.5 * pos[k]
        self.set_targets(ids, target)

    def set_targets(self, ids, target) -> None:
        pos = self.sim.root[ids, :2]
        self.target[ids] = target
        self.target_z[ids] = self.sim.terrain_at(ids, target)
        self.prev_dist[ids] = np.linalg.norm(target - pos, axis=1)
        self.prev_gaze[ids] = gaze_error(self.sim.rot[ids], pos, target)
        self.in_view[ids] = self.prev_gaze[ids] < np.radians(self.cfg.fov)

    # arc/task.py:155-220, split into the physics step and the task math
    def step(self, actions):
        cfg, sim = self.cfg, self.sim
        a = np.clip(np.asarray(actions, dtype=np.float64), -1.0, 1.0)
        sim.step(sim.default_angles + cfg.action_scale * a)
        return self.after_step(a)

    def after_step(self, a):
        """Reward, terminations, bookkeeping after the physics step (a: clipped actions)."""
        cfg, sim = self.cfg, self.sim
        nj, nl = self.nj, self.nl
        root, joints, contacts, flags = sim.observe()
        rot = sim.rot
        self.steps += 1
        pos = root[:, :3]
        to_target = self.target - pos[:, :2]
        dist = np.hypot(to_target[:, 0], to_target[:, 1])
        gaze = gaze_error(rot, pos, self.target)
        cos_fov = np.cos(np.radians(cfg.fov))
        view = np.clip((np.cos(gaze) - cos_fov) / (1.0 - cos_fov), 0.0, 1.0)
        self.in_view = gaze < np.radians(cfg.fov)
        progress = np.minimum(self.prev_dist - dist, cfg.max_speed * cfg.dt)
        progress = np.where(progress > 0, progress * view, progress)
        turn = self.prev_gaze - gaze
        reached = (dist < cfg.checkpoint_radius) & self.in_view
        # torso angular velocity in the body frame: R^T w, roll and pitch
        body_rate = np.einsum("ni,nij->nj", root[:, 10:13], rot)[:, :2]
        torso = contacts[:, nl] > 0
        self.torso_steps = np.where(torso, self.torso_steps + 1, 0)
        power = np.abs(joints[:, nj:2 * nj] * joints[:, 2 * nj:]).sum(1)
        rate = np.square(a - self.prev_action).sum(1)
        reward = (cfg.w_progress * progress
                  + cfg.w_turn * turn
                  + cfg.w_checkpoint * reached
                  - cfg.w_time
                  - cfg.w_energy * power * cfg.dt
                  - cfg.w_action_rate * rate
                  - cfg.w_body_contact * (contacts[:, nl + 1] > 0)
                  - cfg.w_torso_contact * torso
                  - cfg.w_body_rate * np.square(body_rate).sum(1)
                  - cfg.w_bounce * np.square(root[:, 9]))
        bad = (flags != 0) | ~np.all(np.isfinite(root), axis=1)
        void = np.any(np.abs(pos[:, :2]) > sim.half_extent, axis=1) | (pos[:, 2] < cfg.void_z)
        flip = rot[:, 2, 2] < cfg.flip_up_z
        beached = self.torso_steps > cfg.beached_steps
        fell = flip | beached | void | bad
        cause = np.where(bad, 1, np.where(void, 2, np.where(flip, 3, np.where(beached, 4, 0))))
        reward = np.where(fell, reward - cfg.w_fall, reward)
        reward = np.where(bad, -cfg.w_fall, reward)
        self.prev_dist = dist
        self.prev_gaze = gaze
        self.prev_action = a
        self.checkpoints += reached
        hit = np.flatnonzero(reached & ~fell)
        if len(hit):
            self.new_targets(hit)
        terminated = fell
        truncated = (self.steps >= cfg.max_steps) & ~terminated
        stats = {"checkpoints": self.checkpoints.copy(), "difficulty": self.difficulty.copy(),
                 "fell": fell.copy(), "cause": cause, "steps": self.steps.copy(), "reached": reached}
        done = np.flatnonzero(terminated | truncated)
        if len(done) and cfg.curriculum:
            self.update_levels(done, fell)
        return reward.astype(np.float32), terminated, truncated, stats

    # arc/task.py:222-227
    def update_levels(self, done, fell) -> None:
        cfg = self.cfg
        up = self.checkpoints[done] >= cfg.level_up_checkpoints
        down = fell[done] & (self.checkpoints[done] == 0) & (self.steps[done] < cfg.level_down_steps)
        lvl = self.level[done] + cfg.level_step * (up.astype(float) - down.astype(float))
        self.level[done] = np.clip(np.round(lvl, 6), 0.0, cfg.max_difficulty)

    # arc/task.py:231-259
    def observe(self) -> np.ndarray:
        sim, nj, nl = self.sim, self.nj, self.nl
        root, joints, contacts, rot = sim.root, sim.joints, sim.contacts, sim.rot
        gravity = -rot[:, 2, :]
        lin = np.einsum("ni,nij->nj", root[:, 7:10], rot)
        ang = np.einsum("ni,nij->nj", root[:, 10:13], rot)
        heading = np.arctan2(rot[:, 1, 0], rot[:, 0, 0])
        d = self.target - root[:, :2]
        c, s = np.cos(heading), np.sin(heading)
        fwd, left = c * d[:, 0] + s * d[:, 1], -s * d[:, 0] + c * d[:, 1]
        dist = np.maximum(np.hypot(fwd, left), 1e-6)
        tgt = np.stack([fwd / dist, left / dist, np.minimum(dist, 6.0) / 6.0], 1)
        heights = sim.heights(HEIGHT_OFFSETS, out=self._heights)
        rel = np.clip(root[:, 2:3] - sim.stand_height - heights, -1.0, 1.0)
        obs = np.concatenate([gravity, lin, 0.25 * ang, joints[:, :nj] - sim.default_angles,
                              0.1 * joints[:, nj:2 * nj], self.prev_action, tgt, rel,
                              contacts[:, :nl]], axis=1, dtype=np.float32)
        obs[~np.isfinite(obs)] = 0.0
        return obs
