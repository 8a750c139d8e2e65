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
from oracle.oracle import NB, NS, OracleSim, RefSim, ref_available
from parity_checks import fp32_bound

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
    o32 = OracleSim(N, grid=64, cell=CELL, bits=32)
    g = Sim(N, grids=grids, cell=CELL)
    g.set_kernel(KERNEL_WARPS)
    ref.reset(np.arange(N), seeds, diffs)
    for i in range(N):
        h = block_terrain(rng, int(grids[i]), diffs[i], g.stand_height)
        ref.set_terrain(i, h, CELL, outside=-100.0)
        o32.set_terrain(i, h, CELL, outside=-100.0)
        g.set_terrain(i, h, CELL, outside=-100.0)
    # lift every body clear of the tallest block, so the robots drop in
    st = ref.get_state()
    st[:, : NB * 13].reshape(N, NB, 13)[:, :, 2] += 0.2
    ref.set_state(st)
    ou = np.zeros((N, 12))
    dxs, dqs, rxs, rqs, mism, rmism = [], [], [], [], 0, 0
    for _ in range(30):
        s0 = ref.get_state()
        g.set_state(s0)
        o32.set_state(s0)
        ou += 0.15 * (0.0 - ou) + 0.3 * rng.standard_normal((N, 12))
        t = ref.default_angles + 0.6 * np.clip(ou, -1, 1)
        ref.step(t)
        g.step(t)
        o32.step(t)
        a, b, c = ref.get_state(), g.get_state(), o32.get_state()
        dx, dq = body_errors(a, b)
        rx, rq = body_errors(a, c)
        dxs.append(dx)
        dqs.append(dq)
        rxs.append(rx)
        rqs.append(rq)
        mism += int((touches(a) != touches(b)).any(1).sum())
        rmism += int((touches(a) != touches(c)).any(1).sum())
    dx, dq = np.concatenate(dxs), np.concatenate(dqs)
    rx, rq = np.concatenate(rxs), np.concatenate(rqs)
    touching = int((touches(ref.get_state()) > 0).any(1).sum())
    print(f"uneven blocks: rel |dx| p50 {np.median(dx):.2e} p95 {np.percentile(dx, 95):.2e} "
          f"p99 {np.percentile(dx, 99):.2e} max {dx.max():.2e}; touch mismatches {mism}/{len(dx)}; "
          f"worlds touching {touching}")
    print(f"  strict FP32 restatement: rel |dx| p50 {np.median(rx):.2e} p95 {np.percentile(rx, 95):.2e} "
          f"p99 {np.percentile(rx, 99):.2e} max {rx.max():.2e}; touch mismatches {rmism}/{len(rx)}")
    assert touching > N // 2
    assert np.percentile(dx, 95) <= 1e-5 and np.percentile(dq, 95) <= 1e-5
    fp32_bound("position", dx, rx)
    fp32_bound("orientation", dq, rq)
    assert mism <= max(1.5 * rmism, 0.01 * len(dx))


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_full_uneven_batch_subset_vs_reference():
    """The configuration at its stated size: 16,384 worlds of 16..64 columns
    a side in one batch, every control step one launch over all of them; a
    256-world subset spread over the batch is teacher-forced against the
    reference stepping those worlds on their own grids."""
    n_all = 16384
    rng, grids, diffs, seeds = uneven_worlds(n_all, 11)
    g = Sim(n_all, grids=grids, cell=CELL)
    g.set_kernel(KERNEL_WARPS)
    g.reset(np.arange(n_all), seeds, diffs)
    subset = np.sort(rng.choice(n_all, N, replace=False)).astype(np.int32)
    ref = RefSim(N, grid=64, cell=CELL)
    o32 = OracleSim(N, grid=64, cell=CELL, bits=32)
    ref.reset(np.arange(N), seeds[subset], diffs[subset])
    for i in range(n_all):
        h = block_terrain(rng, int(grids[i]), diffs[i], g.stand_height)
        g.set_terrain(i, h, CELL, outside=-100.0)
        k = np.searchsorted(subset, i)
        if k < N and subset[k] == i:
            ref.set_terrain(int(k), h, CELL, outside=-100.0)
            o32.set_terrain(int(k), h, CELL, outside=-100.0)
    st = g.get_state()
    st[:, : NB * 13].reshape(n_all, NB, 13)[:, :, 2] += 0.2
    g.set_state(st)
    ref.set_state(st[subset])
    ou = np.zeros((n_all, 12))
    dxs, dqs, rxs, rqs = [], [], [], []
    for _ in range(20):
        s0 = ref.get_state()
        g.set_state(s0, ids=subset)
        o32.set_state(s0)
        ou += 0.15 * (0.0 - ou) + 0.3 * rng.standard_normal((n_all, 12))
        t = g.default_angles + 0.6 * np.clip(ou, -1, 1)
        ref.step(t[subset])
        o32.step(t[subset])
        g.step(t)
        a, b, c = ref.get_state(), g.get_state(ids=subset), o32.get_state()
        dx, dq = body_errors(a, b)
        rx, rq = body_errors(a, c)
        dxs.append(dx)
        dqs.append(dq)
        rxs.append(rx)
        rqs.append(rq)
    dx, dq = np.concatenate(dxs), np.concatenate(dqs)
    rx, rq = np.concatenate(rxs), np.concatenate(rqs)
    whole = g.get_state()
    print(f"16,384-world uneven batch, 256-world subset: rel |dx| p50 {np.median(dx):.2e} "
          f"p95 {np.percentile(dx, 95):.2e} p99 {np.percentile(dx, 99):.2e} max {dx.max():.2e}; "
          f"restatement p95 {np.percentile(rx, 95):.2e} p99 {np.percentile(rx, 99):.2e}")
    assert np.all(np.isfinite(whole)) and int(whole[:, -2].sum()) == 0  # no world of the batch blew up
    assert np.percentile(dx, 95) <= 1e-5 and np.percentile(dq, 95) <= 1e-5
    fp32_bound("position", dx, rx)
    fp32_bound("orientation", dq, rq)
