"""Pins the CPU oracle to the reference (no GPU needed).

The fixtures in tests/golden/ come from the reference itself
(tests/golden/make_golden.py): golden_strict.npz from its csrc/ built
without FMA contraction, the way the FP64 oracle is built, so those must
match bit for bit; golden_shipped.npz from its csrc/ built with its own
flags (FMA contraction on), matched to rounding.
"""

from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import NB, NJ, NS, OracleSim, RefSim, oracle_terrain, ref_available
from oracle.task_oracle import HEIGHT_OFFSETS, TaskConfig, TaskOracle

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def strict():
    return dict(np.load(GOLDEN / "golden_strict.npz"))


@pytest.fixture(scope="module")
def shipped():
    return dict(np.load(GOLDEN / "golden_shipped.npz"))


def test_robot_template_matches_reference(strict):
    o = OracleSim(1, bits=64)
    assert np.array_equal(o.default_angles, strict["robot_default"])
    assert np.array_equal(o.lo, strict["robot_lo"]) and np.array_equal(o.hi, strict["robot_hi"])
    assert np.array_equal([o.stand_height, o.total_mass], strict["robot_misc"])
    dump = o.model_dump()
    bodies = dump[: NB * 11].reshape(NB, 11)
    assert np.array_equal(bodies[:, :4], strict["robot_bodies"])
    joints = dump[NB * 11: NB * 11 + NJ * 29].reshape(NJ, 29)
    assert np.array_equal(joints, strict["robot_joints"])
    spheres = dump[NB * 11 + NJ * 29:].reshape(NS, 5)
    assert np.array_equal(spheres, strict["robot_spheres"])
    assert np.array_equal(o.get_state()[0], strict["robot_state"])


def test_terrain_generator_matches_reference(shipped):
    import hashlib
    for (seed, diff, grid), want in zip(shipped["terrain_combos"], shipped["terrain_sha"]):
        h, _ = oracle_terrain(int(grid), 0.4, float(diff), int(seed))
        got = hashlib.sha256(np.ascontiguousarray(h).tobytes()).hexdigest()
        assert got == want, (seed, diff, grid)
    for key in shipped:
        if key.startswith("terrain_") and key.count("_") == 3 and "geom" not in key and "sha" not in key \
                and "combos" not in key:
            _, seed, diff, grid = key.split("_")
            h, geom = oracle_terrain(int(grid), 0.4, float(diff), int(seed))
            assert np.array_equal(h, shipped[key])


@pytest.mark.parametrize("which", ["strict", "shipped"])
def test_reset_matches_reference(which, strict, shipped):
    g = strict if which == "strict" else shipped
    n = len(g["reset_seeds"])
    o = OracleSim(n, bits=64)
    o.reset(np.arange(n), g["reset_seeds"], g["reset_diffs"])
    if which == "strict":
        assert np.array_equal(o.get_state(), g["reset_state"])
    else:
        assert np.allclose(o.get_state(), g["reset_state"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("which", ["strict", "shipped"])
def test_teacher_forced_steps_match_reference(which, strict, shipped):
    g = strict if which == "strict" else shipped
    n = len(g["step_seeds"])
    o = OracleSim(n, bits=64)
    o.reset(np.arange(n), g["step_seeds"], g["step_diffs"])
    for before, t, after in zip(g["step_before"], g["step_targets"], g["step_after"]):
        o.set_state(before)
        o.step(t)
        got = o.get_state()
        if which == "strict":
            assert np.array_equal(got, after)
        else:
            assert np.allclose(got, after, rtol=1e-9, atol=1e-9)


def test_rollout_matches_reference_bitwise(strict):
    g = strict
    n = len(g["step_seeds"])
    o = OracleSim(n, bits=64)
    o.reset(np.arange(n), g["step_seeds"], g["step_diffs"])
    rng = np.random.default_rng(7)
    for k in range(len(g["rollout"])):
        o.step(o.lo + (o.hi - o.lo) * rng.uniform(0, 1, (n, NJ)))
        root, joints, contacts, flags = o.observe()
        assert np.array_equal(np.concatenate([root, contacts, flags[:, None]], 1), g["rollout"][k]), k


def test_task_oracle_matches_reference_task(strict):
    """oracle/task_oracle.py over the FP64 oracle replays the reference's
    ArcTask (arc/task.py) run over the reference build."""
    g = strict
    n = int(g["task_n"])
    assert np.array_equal(HEIGHT_OFFSETS, g["height_offsets"])
    sim = OracleSim(n, bits=64)
    t = TaskOracle(sim, TaskConfig(curriculum=True), seed=int(g["task_seed"]))
    t.reset(np.arange(n))
    assert np.array_equal(t.observe(), g["task_obs0"])
    for k in range(len(g["task_actions"])):
        r, te, tr, st = t.step(g["task_actions"][k])
        o = t.observe()
        done = np.flatnonzero(te | tr)
        if len(done):
            t.reset(done)
        # einsum and matmul may sum the 3-term products in a different order
        assert np.allclose(o, g["task_obs"][k], rtol=2e-7, atol=1e-7), k
        assert np.allclose(r, g["task_reward"][k], rtol=1e-6, atol=1e-6), k
        assert np.array_equal(te, g["task_terminated"][k]) and np.array_equal(tr, g["task_truncated"][k])
        assert np.array_equal(st["cause"], g["task_cause"][k])
        assert np.array_equal(t.target, g["task_target"][k])
        assert np.array_equal(t.level, g["task_level"][k])


def test_fp32_oracle_error_budget(shipped):
    """The FP32 restatement, teacher-forced from FP64 reference states, stays
    inside the FP32 parity contract (p99 position error <= 1e-5 m)."""
    g = shipped
    n = len(g["step_seeds"])
    o = OracleSim(n, bits=32)
    o.reset(np.arange(n), g["step_seeds"], g["step_diffs"])
    errs = []
    for before, t, after in zip(g["step_before"], g["step_targets"], g["step_after"]):
        o.set_state(before)
        o.step(t)
        a = after[:, : NB * 13].reshape(n, NB, 13)
        b = o.get_state()[:, : NB * 13].reshape(n, NB, 13)
        errs.append(np.linalg.norm(a[..., :3] - b[..., :3], axis=2).max(1))
    e = np.concatenate(errs)
    assert np.percentile(e, 99) <= 1e-5


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_oracle_bitwise_equals_reference_build_live():
    n = 16
    o, r = OracleSim(n, bits=64), RefSim(n, variant="_strict")
    ids, seeds, diffs = np.arange(n), np.arange(n, dtype=np.uint32) * 7 + 3, np.linspace(0, 1, n)
    o.reset(ids, seeds, diffs)
    r.reset(ids, seeds, diffs)
    rng = np.random.default_rng(0)
    for _ in range(60):
        t = o.default_angles + 0.6 * rng.uniform(-1, 1, (n, NJ))
        o.step(t)
        r.step(t)
    assert np.array_equal(o.get_state(), r.get_state())
    for x, y in zip(o.observe(), r.observe()):
        assert np.array_equal(x, y)
    assert np.array_equal(o.heights(HEIGHT_OFFSETS), r.heights(HEIGHT_OFFSETS))


def test_oracle_unstable_world_is_flagged_and_frozen():
    """csrc/tests/test_phys.c:304-324: NaN / huge / too fast states are
    flagged unstable and then skipped (csrc/arc_sim.c:135)."""
    n = 4
    o = OracleSim(n, bits=64)
    o.reset(np.arange(n), np.arange(n, dtype=np.uint32), np.zeros(n))
    st = o.get_state()
    st[1, 0], st[2, 0], st[3, 7] = np.nan, 1e12, 1000.0
    o.set_state(st)
    o.step(np.broadcast_to(o.default_angles, (n, NJ)))
    assert list(o.observe()[3]) == [0, 1, 1, 1]
