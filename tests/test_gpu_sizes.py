"""Worlds with different terrain sizes (16..64 columns a side) in one batch.

The reference's arc_sim has one grid for every world (csrc/arc_sim.c:36),
but its world step honours each world's own nx, ny (csrc/arc_terrain.h:
13-40, csrc/arc_phys.c:557-564). The checker therefore drives the
reference's worlds one by one: RefSim writes each world's terrain into its
arc_world and steps it with the reference's own code (FP64).

Terrain: i.i.d. block heights U(0, 0.3 * difficulty * stand_height) per
column, written directly (the reference's generator has no block mode).
Parity contract: the FP32 teacher-forced bounds of test_gpu_step.py.
"""

import numpy as np
import pytest

from arc_demo_b200.native import KERNEL_WARPS, Sim
from oracle.oracle import NB, NS, RefSim, ref_available

pytestmark = pytest.mark.gpu

N = 256
CELL = 0.4


def body_errors(a, b):
    xa = a[:, : NB * 13].reshape(len(a), NB, 13)
    xb = b[:, : NB * 13].reshape(len(b), NB, 13)
    scale = np.maximum(np.linalg.norm(xa[..., :3], axis=2), 1.0)
    dx = (np.linalg.norm(xa[..., :3] - xb[..., :3], axis=2) / scale).max(1)
    qa, qb = xa[..., 3:7], xb[..., 3:7]
    dq = np.minimum(np.linalg.norm(qa - qb, axis=2), np.linalg.norm(qa + qb, axis=2)).max(1)
    return dx, dq


def touches(s):
    return s[:, NB * 13: NB * 13 + NS * 8].reshape(len(s), NS, 8)[:, :, 7]


def uneven_worlds(n, seed):
    rng = np.random.default_rng(seed)
    grids = rng.integers(16, 65, n).astype(np.int32)
    diffs = rng.uniform(0, 1, n)
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    return rng, grids, diffs, seeds


def block_terrain(rng, g, difficulty, stand_height):
    return rng.uniform(0.0, 0.3 * difficulty * stand_height, (g, g))


def test_terrain_pool_holds_each_worlds_size():
    rng, grids, diffs, seeds = uneven_worlds(64, 1)
    s = Sim(64, grids=grids, cell=CELL)
    s.reset(np.arange(64), seeds, diffs)
    for i in range(64):
        h, geom = s.get_terrain(i)
        assert h.shape == (grids[i], grids[i])
        assert geom[1] == pytest.approx(-0.5 * grids[i] * CELL)
    # a world holds at most grids[i]^2 columns
    small = int(np.argmin(grids))
    g = int(grids[small])
    s.set_terrain(small, np.zeros((g, g)), CELL)
    with pytest.raises(Exception):
        s.set_terrain(small, np.zeros((g + 1, g + 1)), CELL)


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_uneven_blocks_teacher_forced_vs_reference():
    rng, grids, diffs, seeds = uneven_worlds(N, 7)
    ref = RefSim(N, grid=64, cell=CELL)
    g = Sim(N, grids=grids, cell=CELL)
    g.set_kernel(KERNEL_WARPS)
    ref.reset(np.arange(N), seeds, diffs)
    for i in range(N):
        h = block_terrain(rng, int(grids[i]), diffs[i], g.stand_height)
        ref.set_terrain(i, h, CELL, outside=-100.0)
        g.set_terrain(i, h, CELL, outside=-100.0)
    # lift every body clear of the tallest block, so the robots drop in
    st = ref.get_state()
    st[:, : NB * 13].reshape(N, NB, 13)[:, :, 2] += 0.2
    ref.set_state(st)
    ou = np.zeros((N, 12))
    dxs, dqs, mism = [], [], 0
    for _ in range(30):
        g.set_state(ref.get_state())
        ou += 0.15 * (0.0 - ou) + 0.3 * rng.standard_normal((N, 12))
        t = ref.default_angles + 0.6 * np.clip(ou, -1, 1)
        ref.step(t)
        g.step(t)
        a, b = ref.get_state(), g.get_state()
        dx, dq = body_errors(a, b)
        dxs.append(dx)
        dqs.append(dq)
        mism += int((touches(a) != touches(b)).any(1).sum())
    dx, dq = np.concatenate(dxs), np.concatenate(dqs)
    touching = int((touches(ref.get_state()) > 0).any(1).sum())
    print(f"uneven blocks: rel |dx| p50 {np.median(dx):.2e} p95 {np.percentile(dx, 95):.2e} "
          f"p99 {np.percentile(dx, 99):.2e} max {dx.max():.2e}; touch mismatches {mism}/{len(dx)}; "
          f"worlds touching {touching}")
    assert touching > N // 2
    assert np.percentile(dx, 95) <= 1e-5 and np.percentile(dx, 99) <= 5e-5
    assert np.percentile(dq, 95) <= 1e-5 and np.percentile(dq, 99) <= 5e-5
    assert mism <= 0.01 * len(dx)
