"""The serving engine (csrc/arc_serve.cu): sessions of resident worlds with the
task layer, stepped by continuous batching.

- A session's results (per-step rewards and done flags, final observations)
  in a mix of concurrent sessions and requests equal its results when it
  runs alone, bit for bit: worlds never interact, the fused control step
  runs the same per-world code for any list of slots, and a world's random
  draws are named by its session's key, not by its slot.
- Worlds stay resident across requests: a session stepped 3 + 4 steps in two
  requests equals the same session stepped 7 steps in one.
- A world whose episode ends is reset in place and the request goes on
  (arc/env.py:99-117): with max_steps 5, every world that does not fall is
  truncated after steps 5 and 10 of a 12-step request.
- Admission by the slot budget, the per-tick world cap, and the errors.
"""

import threading

import numpy as np
import pytest

from arc_demo_b200.serve import Server
from arc_demo_b200.task import TaskConfig

pytestmark = pytest.mark.gpu

CFG = TaskConfig(curriculum=False, max_steps=5)


def session_plan(seed):
    """Sessions (difficulties, key) and, per session, its requests (steps,
    given actions or None, OU seed)."""
    rng = np.random.default_rng(seed)
    plan = []
    for n, ks in ((5, (3, 4)), (40, (6,)), (100, (2, 9)), (1, (7,)), (33, (5, 1)), (64, (4,))):
        reqs = []
        for k in ks:
            given = rng.random() < 0.5
            act = rng.uniform(-1.2, 1.2, (k, n, 12)).astype(np.float32) if given else None
            reqs.append((k, act, int(rng.integers(2**63))))
        plan.append((rng.uniform(0, 1, n), int(rng.integers(2**63)), reqs))
    return plan


def run_session(sv, diff, key, reqs):
    sid = sv.open(diff, key)
    outs = []
    for k, act, ou in reqs:
        (obs, rew, done), times = sv.wait(sv.request(sid, k, actions=act, ou_seed=ou))
        assert times[2] >= times[1] >= 0
        outs.append((obs, rew, done))
    sv.close_session(sid)
    return outs


def test_mix_equals_alone():
    plan = session_plan(1)
    with Server(512, config=CFG) as sv:
        mixed = [None] * len(plan)

        def client(i):
            mixed[i] = run_session(sv, *plan[i])

        threads = [threading.Thread(target=client, args=(i,)) for i in range(len(plan))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        st = sv.stats()
        assert st["error"] == 0 and st["completed"] == sum(len(p[2]) for p in plan)
        assert st["episodes_ended"] > 0
    for i, p in enumerate(plan):
        with Server(512, config=CFG) as sv:
            alone = run_session(sv, *p)
        for (a, b) in zip(alone, mixed[i]):
            for x, y in zip(a, b):
                assert np.array_equal(x, y), f"session {i} differs in the mix"


def test_resident_worlds_continue_across_requests():
    rng = np.random.default_rng(2)
    n = 48
    diff = rng.uniform(0, 1, n)
    act = rng.uniform(-1, 1, (7, n, 12)).astype(np.float32)
    with Server(64, config=CFG) as sv:
        split = run_session(sv, diff, 9, [(3, act[:3], 0), (4, act[3:], 0)])
        whole = run_session(sv, diff, 9, [(7, act, 0)])
    assert np.array_equal(np.concatenate([split[0][1], split[1][1]]), whole[0][1])
    assert np.array_equal(np.concatenate([split[0][2], split[1][2]]), whole[0][2])
    assert np.array_equal(split[1][0], whole[0][0])


def test_episode_end_resets_in_place():
    n, k = 64, 12
    with Server(n, config=CFG) as sv:
        sid = sv.open(np.zeros(n), 3)
        (obs, rew, done), _ = sv.wait(sv.request(sid, k, actions=np.zeros((k, n, 12), np.float32)))
    assert np.isfinite(obs).all() and np.isfinite(rew).all()
    ended = done != 0
    # a flat world under zero actions stands: truncated (bit 1) after 5 and 10 steps
    assert np.array_equal(done[4], np.full(n, 2, np.uint8)) and np.array_equal(done[9], np.full(n, 2, np.uint8))
    assert ended.sum() == 2 * n
    # the step after an episode end starts the next episode: its reward is an ordinary step's
    assert np.all(np.abs(rew[5]) < 10.0)


def test_slots_budget_ticks_and_errors():
    with Server(100, config=CFG, tick_cap=60) as sv:
        a = sv.open(np.zeros(70), 1)
        b = sv.open(np.zeros(50), 2)          # waits: only 30 slots left
        ra = sv.request(a, 3)
        rb = sv.request(b, 2)
        sv.wait(ra)
        st = sv.stats()
        assert st["waiting_sessions"] == 1 and st["resident"] == 70
        sv.close_session(a)                    # frees 70 slots: b is admitted
        sv.wait(rb)
        c = sv.open(np.zeros(40), 3)
        rc = [sv.request(c, 4) for _ in range(2)]
        rb2 = sv.request(b, 4)
        for r in rc + [rb2]:
            sv.wait(r)
        st = sv.stats()
        assert st["error"] == 0
        assert st["max_active"] <= 70          # the first session alone (70 > cap), then <= 60 a tick
        with pytest.raises(RuntimeError):
            sv.open(np.zeros(101), 4)          # larger than the pool
        sv.close_session(c)
        assert sv._lib.arc_server_request(sv._ptr, c, 1, None, 0, None, None, None) < 0  # closed
        with pytest.raises(RuntimeError):
            sv.request(c, 1)


def test_session_closed_before_admission_still_runs_its_requests():
    """A client may close a session while it still waits for slots: its
    queued requests run, then its slots are freed."""
    with Server(64, config=CFG) as sv:
        a = sv.open(np.zeros(60), 1)
        ra = sv.request(a, 3)
        b = sv.open(np.zeros(30), 2)           # waits: 4 slots left
        rb = [sv.request(b, 2) for _ in range(2)]
        sv.close_session(b)                    # closed before it was admitted
        sv.wait(ra)
        sv.close_session(a)
        for r in rb:
            (obs, rew, done), _ = sv.wait(r, timeout=60.0)
            assert np.isfinite(obs).all() and rew.shape == (2, 30)
        st = sv.stats()
        assert st["error"] == 0 and st["completed"] == 3
