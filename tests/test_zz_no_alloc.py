"""arc_step_noalloc, the entry point for callers that cannot allocate device
memory, gives the same worlds as the regular path (arc_sim_step) over two
control steps in a row.

Callers that own all device memory through their own arena, or that must
not let a library call cudaMalloc inside a latency-critical loop, pass their
own buffers; the entry point works in a fixed static device array instead of
allocating. It runs the same leg-parallel kernel as arc_sim_step, so the
states must agree bit for bit.
"""

import ctypes

import numpy as np
import pytest

from arc_demo_b200.native import KERNEL_LEGS, Sim, sim_lib

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    fn = sim_lib().arc_step_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                   ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
    return fn


def _compare_two_steps(n, seed, stream=None):
    """n worlds stepped twice by arc_sim_step (leg-parallel kernel, library
    buffers) and twice by arc_step_noalloc (caller buffers) from the same
    reset: the states must agree bit for bit after each step."""
    import torch

    fn = _noalloc_fn()
    grid, cell = 64, 0.4
    rng = np.random.default_rng(seed)
    sim = Sim(n, grid=grid, cell=cell)
    sim.set_kernel(KERNEL_LEGS, 8)
    sim.reset(np.arange(n), rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32),
              np.round(rng.uniform(0, 1, n), 1))
    s0 = sim.get_state()
    heights = np.stack([sim.get_terrain(i)[0] for i in range(n)]).astype(np.float32)
    t1 = sim.default_angles + 0.6 * rng.uniform(-1, 1, (n, 12))
    t2 = sim.default_angles + 0.6 * rng.uniform(-1, 1, (n, 12))

    # the regular path: library-owned buffers
    sim.step(t1)
    a1 = sim.get_state()
    sim.step(t2)
    a2 = sim.get_state()
    sim.close()

    # the allocation-free path: every buffer is the caller's
    d_state = torch.from_numpy(s0).cuda()
    d_heights = torch.from_numpy(heights).cuda()
    d_t1, d_t2 = torch.from_numpy(t1).cuda(), torch.from_numpy(t2).cuda()
    torch.cuda.synchronize()
    handle = None if stream is None else stream.cuda_stream
    results = []
    for d_t in (d_t1, d_t2):
        rc = fn(d_state.data_ptr(), d_heights.data_ptr(), grid, cell, -100.0, d_t.data_ptr(), n, 1.0 / 30.0, 20,
                handle)
        assert rc == 0
        if stream is None:
            torch.cuda.synchronize()
        else:
            stream.synchronize()
        results.append(d_state.cpu().numpy().copy())
    assert np.array_equal(results[0], a1)
    assert np.array_equal(results[1], a2)


def test_noalloc_step_matches_regular_step_twice():
    _compare_two_steps(300, 2024)


def test_noalloc_at_its_capacity_on_a_caller_stream():
    """The full 1,024 worlds the static array holds, on a stream of the
    caller's: the array's last byte offsets and the stream argument."""
    import torch

    _compare_two_steps(1024, 7, torch.cuda.Stream())


def test_noalloc_rejects_requests_beyond_its_static_capacity():
    fn = _noalloc_fn()
    dummy = ctypes.c_void_p(16)
    assert fn(dummy, dummy, 64, 0.4, -100.0, dummy, 1025, 1 / 30, 20, None) != 0   # too many worlds
    assert fn(dummy, dummy, 65, 0.4, -100.0, dummy, 8, 1 / 30, 20, None) != 0      # grid too large
    assert fn(dummy, dummy, 64, 0.2, -100.0, dummy, 8, 1 / 30, 20, None) != 0      # cells too small
