"""The reference's own robot and environment checks, restated on the CUDA path.

Robot checks of csrc/tests/test_robot.c (standing still on flat ground,
surviving random actions on rough terrain, determinism) through the
reference's C ABI (`Sim`), and the environment checks of tests/test_env.py
(observation at rest, auto-reset, falls, the void, checkpoints, curriculum,
reward shaping, the field of view) through the device env, with the same
thresholds. The reference's tests set task fields directly (task.target,
prev_dist, ...); here the same values go through the task-state accessors
(arc_env_{get,set}_task_state), and the void test moves the robot past the
terrain edge instead of patching `observe`.
"""

import numpy as np
import pytest

from arc_demo_b200.native import Sim
from arc_demo_b200.task import CAUSES, HEIGHT_OFFSETS, TaskConfig

pytestmark = pytest.mark.gpu

DT, SUBSTEPS = 1.0 / 30.0, 20
# task state columns (include/arc_sim.h, ARC_TASK_STATE_SIZE)
TARGET, PREV_DIST, PREV_GAZE, TORSO_STEPS, STEPS, CHECKPOINTS, LEVEL = slice(0, 2), 3, 4, 17, 18, 19, 20
BODY_VALUES, SPHERE_VALUES = 13, 8  # world-state snapshot: bodies (x3 q4 v3 w3), spheres (anchored, ...)


def reset_all(sim, seed, difficulty):
    n = sim.num_worlds
    sim.reset(np.arange(n), seed + np.arange(n), np.full(n, difficulty))


# -- csrc/tests/test_robot.c --------------------------------------------------

@pytest.mark.parametrize("fp64", [False, True])
def test_robot_stands_still_on_flat_ground(fp64):
    """test_robot.c:30-59: default stance held for 8 s on flat ground."""
    sim = Sim(1, DT, SUBSTEPS, 32, 0.4, fp64=fp64)
    reset_all(sim, 1, 0.0)
    targets = sim.default_angles[None].copy()
    maxv = 0.0
    for i in range(240):
        sim.step(targets)
        root, _, contacts, flags = sim.observe()
        if i >= 180:
            maxv = max(maxv, float(np.linalg.norm(root[0, 7:10])))
    assert flags[0] == 0
    assert root[0, 2] > 0.8 * sim.stand_height
    assert maxv < 2e-3
    assert np.all(contacts[0, :4] > 0.99)       # all feet in contact
    assert contacts[0, sim.num_legs] <= 0.0      # no torso contact
    assert 1.0 - 2.0 * (root[0, 4] ** 2 + root[0, 5] ** 2) > 0.99  # upright
    sim.close()


def run_random(sim, seed, steps):
    """test_robot.c:62-95: new targets anywhere in each joint's range every
    3 steps; returns the largest torso speed and the unstable world-steps."""
    rng = np.random.default_rng(seed)
    n = sim.num_worlds
    targets = np.tile(sim.default_angles, (n, 1))
    maxspeed, unstable = 0.0, 0
    for k in range(steps):
        if k % 3 == 0:
            targets = rng.uniform(sim.lo, sim.hi, (n, sim.num_joints))
        sim.step(targets)
        root, _, _, flags = sim.observe()
        maxspeed = max(maxspeed, float(np.linalg.norm(root[:, 7:10], axis=1).max()))
        unstable += int(flags.sum())
    return maxspeed, unstable


def test_random_actions_on_hard_terrain_and_determinism():
    """test_robot.c:97-126: 16 worlds x 20 s of random targets at difficulty 1
    stay stable and below 6 m/s; a second sim stepped with the same inputs,
    its kernel taking groups from the work queue, ends bitwise identical."""
    a = Sim(16, DT, SUBSTEPS, 48, 0.4)
    b = Sim(16, DT, SUBSTEPS, 48, 0.4)
    b.set_work_queue(True)
    for sim in (a, b):
        reset_all(sim, 100, 1.0)
    maxspeed, unstable = run_random(a, 7, 600)
    assert unstable == 0
    assert maxspeed < 6.0
    run_random(b, 7, 600)
    assert np.array_equal(a.get_state(), b.get_state())
    a.close()
    b.close()


# -- tests/test_env.py ---------------------------------------------------------

def make_env(n, seed, **cfg):
    from arc_demo_b200.torch_env import DeviceVecEnv
    env = DeviceVecEnv(n, TaskConfig(**cfg), seed=seed)
    if not cfg.get("curriculum", True) and "difficulty" in cfg:
        env.set_levels(np.full(n, cfg["difficulty"]))
    env.reset()
    return env


def hold(env):
    """Zero actions: every joint holds the default stance."""
    import torch
    return torch.zeros((env.num_envs, 12), device="cuda")


def step(env, actions=None):
    import torch
    obs, rew, term, trunc = env.step(hold(env) if actions is None else actions)
    torch.cuda.synchronize()
    return (obs.cpu().numpy(), rew.cpu().numpy(), term.cpu().numpy().astype(bool),
            trunc.cpu().numpy().astype(bool), env.cause.cpu().numpy())


def set_task(env, col, values, ids=None):
    st = env.gpu.get_state()
    if ids is None:
        st[:, col] = values
    else:
        st[ids, col] = values
    env.gpu.set_state(st)


def test_obs_at_rest_is_sane():
    """test_env.py:28-41."""
    env = make_env(4, 0, curriculum=False)
    assert np.all(np.isfinite(env.obs.cpu().numpy()))
    for _ in range(180):
        obs, *_ = step(env)
    assert np.allclose(obs[:, :3], [0, 0, -1], atol=0.05)   # gravity down in the body frame
    assert np.abs(obs[:, 3:9]).max() < 0.1                   # small velocities
    nh = len(HEIGHT_OFFSETS)
    assert np.abs(obs[:, -4 - nh:-4]).max() < 0.1            # flat heightmap
    assert np.all(obs[:, -4:] > 0.99)                        # all feet touching
    env.close()


def test_auto_reset_and_terminal_obs():
    """test_env.py:44-56."""
    env = make_env(3, 1, max_steps=20, curriculum=False)
    for _ in range(20):
        obs, rew, term, trunc, _ = step(env)
    assert np.all(term | trunc) and np.all(trunc)
    term_obs = env.terminal_obs.cpu().numpy()
    assert term_obs.shape == obs.shape and np.all(np.isfinite(term_obs))
    assert np.all(env.gpu.get_state()[:, STEPS] == 0)   # new episodes started
    env.close()


def test_falls_terminate():
    """test_env.py:59-69: random flailing on hard terrain tips robots over."""
    import torch
    env = make_env(8, 2, curriculum=False, difficulty=1.0)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0)
    falls = 0
    for _ in range(300):
        _, rew, term, _, _ = step(env, torch.rand((8, 12), device="cuda", generator=gen) * 2 - 1)
        assert np.all(np.isfinite(rew))
        falls += int(term.sum())
    assert falls > 0
    env.close()


def test_void_terminates():
    """test_env.py:72-89: the torso past the terrain's edge ends the episode
    as a fall, cause "void"."""
    env = make_env(2, 0, curriculum=False)
    st = env.sim.get_state()
    dx = env.sim.half_extent + 0.1 - st[1, 0]
    for b in range(env.sim.num_bodies):
        st[1, b * BODY_VALUES] += dx                     # the whole robot of world 1 moves
    base = env.sim.num_bodies * BODY_VALUES
    st[1, base:base + env.sim.num_spheres * SPHERE_VALUES:SPHERE_VALUES] = 0.0  # no anchors
    env.sim.set_state(st)
    _, rew, term, trunc, cause = step(env)
    assert not (term[0] or trunc[0])
    assert term[1] and CAUSES[cause[1]] == "void"
    assert rew[1] < -env.cfg.w_fall + 1.0
    env.close()


def test_determinism():
    """test_env.py:92-106: the same seed and actions give the same episode."""
    import torch

    def rollout():
        env = make_env(4, 123, curriculum=False, difficulty=0.5)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(5)
        total = 0.0
        for _ in range(100):
            obs, rew, *_ = step(env, torch.rand((4, 12), device="cuda", generator=gen) * 2 - 1)
            total += float(rew.sum())
        env.close()
        return obs, total

    (o1, r1), (o2, r2) = rollout(), rollout()
    assert np.array_equal(o1, o2) and r1 == r2


def test_checkpoint_reached_moves_target():
    """test_env.py:109-121, with the checkpoint 0.1 m in front of the robot
    rather than right under it: straight below, whether it is in view
    depends on which way the torso drifts in the next step."""
    env = make_env(1, 3, curriculum=False)
    place_target(env, 0.0, 0.1)
    set_task(env, PREV_DIST, 0.5)
    old = env.gpu.get_state()[0, TARGET].copy()
    _, rew, *_ = step(env)
    st = env.gpu.get_state()
    assert rew[0] > 0.8 * env.cfg.w_checkpoint
    assert st[0, CHECKPOINTS] == 1
    assert np.linalg.norm(st[0, TARGET] - old) >= env.cfg.checkpoint_min_dist - 0.5
    env.close()


def test_curriculum_levels():
    """test_env.py:124-132: an episode with enough checkpoints moves its world
    one level up; a fall at level 0 stays at 0. Here both episodes end in a
    real step: world 0 by the time limit, world 1 in the void."""
    cfg = TaskConfig()
    env = make_env(2, 4)
    set_task(env, CHECKPOINTS, [cfg.level_up_checkpoints, 0])
    set_task(env, LEVEL, [0.0, 0.0])
    set_task(env, STEPS, cfg.max_steps - 1, ids=[0])
    st = env.sim.get_state()
    dx = env.sim.half_extent + 0.1 - st[1, 0]
    for b in range(env.sim.num_bodies):
        st[1, b * BODY_VALUES] += dx
    env.sim.set_state(st)
    _, _, term, trunc, _ = step(env)
    assert trunc[0] and term[1]
    level = env.gpu.get_state()[:, LEVEL]
    assert level[0] == pytest.approx(cfg.level_step) and level[1] == 0.0
    env.close()


def gaze_error(env, target):
    """|angle| between the torso's heading and the target (arc/task.py:79-85)."""
    root, _, _, _ = env.sim.observe()
    f = env.sim.rot[:, :2, 0]
    d = target - root[:, :2]
    return np.abs(np.arctan2(f[:, 0] * d[:, 1] - f[:, 1] * d[:, 0], f[:, 0] * d[:, 0] + f[:, 1] * d[:, 1]))


def test_hovering_near_a_checkpoint_costs():
    """test_env.py:156-167. The reference moves the checkpoint but leaves
    prev_gaze at the old checkpoint's gaze error, so its first step pays a
    turn reward of either sign, depending on where the old checkpoint was;
    here prev_gaze is the new checkpoint's, as the reference's
    _place_target sets it."""
    env = make_env(4, 5, curriculum=False)
    for _ in range(150):
        step(env)
    root = env.sim.observe()[0]
    r = env.cfg.checkpoint_radius
    target = root[:, :2] + [r + 0.3, 0.0]   # just outside the radius
    set_task(env, TARGET, target)
    set_task(env, PREV_DIST, r + 0.3)
    set_task(env, PREV_GAZE, gaze_error(env, target))
    rewards = [step(env)[1] for _ in range(30)]
    assert np.all(np.sum(rewards, axis=0) < 0)
    env.close()


def test_progress_reward_is_capped():
    """test_env.py:170-179: 1 m of progress in one step is worth only
    max_speed * dt."""
    cfg = TaskConfig(curriculum=False)
    env = make_env(1, 6, curriculum=False)
    set_task(env, PREV_DIST, env.gpu.get_state()[0, PREV_DIST] + 1.0)
    _, rew, *_ = step(env)
    assert rew[0] <= cfg.w_progress * cfg.max_speed * cfg.dt + 1e-6
    env.close()


def test_torso_contact_is_penalized_then_terminal():
    """test_env.py:182-201: femurs up, shins out: the torso drops onto the
    ground; touching alone does not end the episode, staying down does."""
    import torch
    cfg = TaskConfig(curriculum=False)
    env = make_env(1, 7, curriculum=False)
    fold = torch.tensor(np.tile([0.0, 1.0, 1.0], 4)[None], dtype=torch.float32, device="cuda")
    first_contact, end, end_cause = None, None, None
    for t in range(120):
        _, _, term, trunc, cause = step(env, fold)
        if first_contact is None and env.gpu.get_state()[0, TORSO_STEPS] > 0:
            first_contact = t
            assert not (term[0] or trunc[0])
        if term[0] or trunc[0]:
            end, end_cause = t, CAUSES[cause[0]]
            break
    assert first_contact is not None and end is not None
    assert end_cause == "beached" and end - first_contact >= cfg.beached_steps
    env.close()


def standing_env(seed):
    env = make_env(1, seed, curriculum=False)
    for _ in range(150):
        step(env)
    return env


def place_target(env, angle, dist):
    """The checkpoint at `angle` (rad) from the gaze, `dist` m away."""
    root, _, _, _ = env.sim.observe()
    rot = env.sim.rot[0]
    heading = np.arctan2(rot[1, 0], rot[0, 0]) + angle
    set_task(env, TARGET, root[0, :2] + dist * np.array([np.cos(heading), np.sin(heading)]))
    set_task(env, PREV_DIST, dist)
    set_task(env, PREV_GAZE, abs(angle))


def test_progress_pays_only_when_target_in_view():
    """test_env.py:222-230."""
    env = standing_env(8)
    rewards = {}
    for angle in (0.0, np.pi):
        place_target(env, angle, 3.0)
        set_task(env, PREV_DIST, 3.0 + 0.03)   # as if the robot just walked 3 cm towards it
        rewards[angle] = step(env)[1][0]
    assert rewards[0.0] > rewards[np.pi] + 0.8 * env.cfg.w_progress * 0.03
    env.close()


def test_turning_towards_target_pays():
    """test_env.py:233-239."""
    env = standing_env(9)
    place_target(env, np.pi / 2, 3.0)
    set_task(env, PREV_GAZE, np.pi / 2 + 0.2)  # as if the gaze just turned 0.2 rad towards it
    rew = step(env)[1][0]
    assert rew > 0.8 * env.cfg.w_turn * 0.2 - env.cfg.w_time
    env.close()


def test_checkpoint_counts_only_when_seen():
    """test_env.py:242-250."""
    env = standing_env(10)
    place_target(env, np.pi, 0.3)   # right behind: not seen
    step(env)
    assert env.gpu.get_state()[0, CHECKPOINTS] == 0
    place_target(env, 0.0, 0.3)     # right in front
    step(env)
    assert env.gpu.get_state()[0, CHECKPOINTS] == 1
    env.close()
