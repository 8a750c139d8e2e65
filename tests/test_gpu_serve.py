"""The serving engine (csrc/arc_serve.cu): continuous batching over a pool of
world slots must not change any request's results.

- A request's final states in a mix of concurrent requests equal its final
  states when it runs alone, bit for bit (worlds never interact; the step
  runs the same per-world code for any list of slots).
- A request with explicit actions equals the same worlds reset and stepped
  directly through arc_sim_step_ids with those actions.
"""

import threading

import numpy as np
import pytest

from arc_demo_b200.native import KERNEL_WARPS, Sim
from arc_demo_b200.serve import Server

pytestmark = pytest.mark.gpu


def make_requests(seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for n, k in ((5, 3), (40, 6), (100, 2), (1, 7), (33, 5), (64, 4), (17, 1)):
        seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        reqs.append((seeds, rng.uniform(0, 1, n), k, int(rng.integers(2**63))))
    return reqs


def test_mix_equals_alone():
    reqs = make_requests(1)
    with Server(256) as sv:
        ids = [None] * len(reqs)

        def submit(i):
            s, d, k, ou = reqs[i]
            ids[i] = sv.submit(s, d, k, ou_seed=ou)

        threads = [threading.Thread(target=submit, args=(i,)) for i in range(len(reqs))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        mixed = [sv.wait(ids[i])[0] for i in range(len(reqs))]
        st = sv.stats()
        assert st["error"] == 0 and st["completed"] == len(reqs)
    with Server(256) as sv:
        for i, (s, d, k, ou) in enumerate(reqs):
            alone, times = sv.wait(sv.submit(s, d, k, ou_seed=ou))
            assert np.array_equal(alone, mixed[i]), f"request {i} differs in the mix"
            assert times[2] >= times[1] >= 0


def test_given_actions_equal_direct_stepping():
    import torch

    rng = np.random.default_rng(2)
    n, k = 45, 4
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    diff = rng.uniform(0, 1, n)
    actions = rng.uniform(-1.2, 1.2, (k, n, 12)).astype(np.float32)
    with Server(64) as sv:
        served, _ = sv.wait(sv.submit(seeds, diff, k, actions=actions))
    sim = Sim(n)
    sim.set_kernel(KERNEL_WARPS)
    sim.reset(np.arange(n), seeds, diff)
    d_ids = torch.arange(n, dtype=torch.int32, device="cuda")
    for t in range(k):
        d_a = torch.as_tensor(actions[t], device="cuda")
        torch.cuda.synchronize()
        sim.step_ids(d_ids.data_ptr(), n, d_actions=d_a.data_ptr())
        sim.synchronize()
    assert np.array_equal(served, sim.get_state())


def test_observation_results_match_observe():
    """A server returning observations gives, per world, the blocks
    arc_sim_observe gives for the same worlds stepped the same way."""
    rng = np.random.default_rng(3)
    n, k = 37, 3
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    diff = rng.uniform(0, 1, n)
    actions = rng.uniform(-1, 1, (k, n, 12)).astype(np.float32)
    with Server(128, result="state") as a, Server(128, result="observe") as b:
        state, _ = a.wait(a.submit(seeds, diff, k, actions=actions))
        obs, _ = b.wait(b.submit(seeds, diff, k, actions=actions))
    sim = Sim(n)
    sim.set_state(state)
    root, joints, contacts, flags = sim.observe()
    assert obs.shape == (n, 65)
    assert np.array_equal(obs[:, :13], root)
    assert np.array_equal(obs[:, 13:22], sim.rot.reshape(n, 9))
    assert np.array_equal(obs[:, 22:58], joints)
    assert np.array_equal(obs[:, 58:64], contacts)
    assert np.array_equal(obs[:, 64], flags.astype(np.float64))


def test_request_larger_than_the_pool_is_refused():
    with Server(16) as sv:
        with pytest.raises(RuntimeError):
            sv.submit(np.arange(17, dtype=np.uint32), np.zeros(17), 1)
        # the engine keeps serving
        out, _ = sv.wait(sv.submit(np.arange(16, dtype=np.uint32), np.zeros(16), 2))
        assert np.isfinite(out).all()


def test_malformed_requests_are_refused_and_the_engine_keeps_serving():
    """Faults made on the host: bad sizes are refused at submit, an unknown
    request id at wait, and none of it disturbs the engine."""
    import ctypes

    from arc_demo_b200.serve import serve_lib

    lib = serve_lib()
    with Server(32) as sv:
        seeds = np.arange(4, dtype=np.uint32)
        diff = np.zeros(4)
        for n, k in ((0, 1), (4, 0), (4, -3), (33, 1)):
            rid = lib.arc_server_submit(sv._ptr, n, k, seeds, diff, None, 0, None)
            assert rid < 0, (n, k)
        assert lib.arc_server_wait(sv._ptr, 123456, 0.1, None, None) < 0
        out, _ = sv.wait(sv.submit(seeds, diff, 3))
        assert np.isfinite(out).all() and sv.stats()["error"] == 0


def test_client_that_never_waits_leaves_the_server_clean():
    """A client that submits and goes away: its request still runs, its
    result is dropped with the server, and other clients are served."""
    with Server(64) as sv:
        sv.submit(np.arange(20, dtype=np.uint32), np.zeros(20), 5)     # never waited for
        out, _ = sv.wait(sv.submit(np.arange(8, dtype=np.uint32), np.zeros(8), 2))
        assert np.isfinite(out).all()
    # the engine thread and every buffer were released by the close above
