"""Generates tests/golden/*.npz from the reference itself.

Runs only where the reference sources are, given as ARC_REFERENCE (or
--ref): oracle/Makefile builds the reference's csrc/ into
oracle/_ref, and the reference's Python task layer (arc/task.py) is imported
from the reference tree with its `Sim` bound to that build. The fixtures
are what the tests compare the oracle and the CUDA library with on machines
without the reference.

    ARC_REFERENCE=<reference checkout> python tests/golden/make_golden.py
"""

from __future__ import annotations

import hashlib
import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
REF = Path(os.environ.get("ARC_REFERENCE", ""))
OUT = Path(__file__).resolve().parent

from oracle.oracle import NB, NJ, NS, RefSim, build  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def import_reference_task(variant: str):
    """arc/task.py from the reference tree, with arc.native.Sim -> RefSim."""
    pkg = types.ModuleType("arcref")
    pkg.__path__ = []
    native = types.ModuleType("arcref.native")

    class Sim(RefSim):
        def __init__(self, n, dt, substeps, grid, cell, threads=1):
            super().__init__(n, dt, substeps, grid, cell, threads, variant=variant)

    native.Sim = Sim
    sys.modules["arcref"] = pkg
    sys.modules["arcref.native"] = native
    spec = importlib.util.spec_from_file_location("arcref.task", REF / "arc" / "task.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["arcref.task"] = mod
    spec.loader.exec_module(mod)
    return mod


def robot(variant: str) -> dict:
    s = RefSim(1, variant=variant)
    w = s.world(0)
    bodies = np.array([[w.bodies[i].mass, w.bodies[i].inertia.x, w.bodies[i].inertia.y,
                        w.bodies[i].inertia.z] for i in range(w.n_bodies)])
    joints = []
    for i in range(w.n_joints):
        j = w.joints[i]
        row = [j.parent, j.child]
        for v in (j.r1, j.r2, j.a1, j.a2, j.b1, j.b2):
            row += [v.x, v.y, v.z]
        row += [j.q_rel0.w, j.q_rel0.x, j.q_rel0.y, j.q_rel0.z, j.lo, j.hi, j.kp, j.kd, j.max_torque]
        joints.append(row)
    spheres = np.array([[w.spheres[i].body, w.spheres[i].pos.x, w.spheres[i].pos.y,
                         w.spheres[i].pos.z, w.spheres[i].radius] for i in range(w.n_spheres)])
    return {"robot_default": s.default_angles, "robot_lo": s.lo, "robot_hi": s.hi,
            "robot_misc": np.array([s.stand_height, s.total_mass]),
            "robot_bodies": bodies, "robot_joints": np.array(joints), "robot_spheres": spheres,
            "robot_state": s.get_state()[0]}


def terrains(variant: str) -> dict:
    combos = [(seed, diff, grid) for seed in (0, 1, 7, 123456789, 4294967295)
              for diff in (0.0, 0.1, 0.5, 0.7, 1.0) for grid in (16, 33, 48, 64)]
    hashes, full = [], {}
    s = RefSim(1, grid=64)
    for k, (seed, diff, grid) in enumerate(combos):
        sg = RefSim(1, grid=grid)
        sg.reset([0], [seed], [diff])
        h, geom = sg.get_terrain(0)
        hashes.append(sha(h))
        if (seed, diff, grid) in ((7, 1.0, 64), (1, 0.5, 33), (123456789, 0.7, 16)):
            full[f"terrain_{seed}_{diff}_{grid}"] = h
            full[f"terrain_geom_{seed}_{diff}_{grid}"] = geom
    del s
    return {"terrain_combos": np.array(combos, dtype=np.float64),
            "terrain_sha": np.array(hashes), **full}


def resets(variant: str) -> dict:
    n = 32
    rng = np.random.default_rng(123)
    seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    diffs = np.round(rng.uniform(0, 1, n), 2)
    s = RefSim(n, variant=variant)
    s.reset(np.arange(n), seeds, diffs)
    return {"reset_seeds": seeds, "reset_diffs": diffs, "reset_state": s.get_state()}


def steps(variant: str) -> dict:
    """Teacher-forcing pairs and a short rollout, mixed terrain, random targets."""
    n = 8
    rng = np.random.default_rng(7)
    seeds = np.arange(n, dtype=np.uint32) * 1000 + 5
    diffs = np.linspace(0.0, 1.0, n)
    s = RefSim(n, variant=variant)
    s.reset(np.arange(n), seeds, diffs)
    before, targets, after, roll = [], [], [], []
    for k in range(30):
        t = s.lo + (s.hi - s.lo) * rng.uniform(0, 1, (n, NJ))
        if k % 6 == 5:
            before.append(s.get_state())
        s.step(t)
        if k % 6 == 5:
            targets.append(t)
            after.append(s.get_state())
        root, joints, contacts, flags = s.observe()
        roll.append(np.concatenate([root, contacts, flags[:, None]], 1))
    return {"step_seeds": seeds, "step_diffs": diffs, "step_before": np.stack(before),
            "step_targets": np.stack(targets), "step_after": np.stack(after),
            "rollout": np.stack(roll)}


def task(variant: str) -> dict:
    """The reference's ArcTask over the reference build: actions in, outputs out."""
    mod = import_reference_task(variant)
    n, T = 4, 30
    cfg = mod.TaskConfig(curriculum=True)
    t = mod.ArcTask(n, cfg, threads=1, seed=11)
    t.reset(np.arange(n))
    rng = np.random.default_rng(3)
    acts, obs, rew, term, trunc, cause, tgt, level = [], [], [], [], [], [], [], []
    obs0 = t.observe()
    for _ in range(T):
        a = rng.uniform(-1.2, 1.2, (n, 12)).astype(np.float32)
        r, te, tr, st = t.step(a)
        o = t.observe()
        done = np.flatnonzero(te | tr)
        if len(done):
            t.reset(done)
        acts.append(a)
        obs.append(o)
        rew.append(r)
        term.append(te)
        trunc.append(tr)
        cause.append(st["cause"])
        tgt.append(t.target.copy())
        level.append(t.level.copy())
    return {"task_n": np.array(n), "task_seed": np.array(11), "task_obs0": obs0,
            "task_actions": np.stack(acts), "task_obs": np.stack(obs), "task_reward": np.stack(rew),
            "task_terminated": np.stack(term), "task_truncated": np.stack(trunc),
            "task_cause": np.stack(cause), "task_target": np.stack(tgt), "task_level": np.stack(level),
            "height_offsets": mod.HEIGHT_OFFSETS}


def main() -> None:
    global REF
    if len(sys.argv) > 2 and sys.argv[1] == "--ref":
        REF = Path(sys.argv[2])
    if not str(REF) or not (REF / "csrc").is_dir():
        sys.exit("give the reference checkout with ARC_REFERENCE=<dir> or --ref <dir>")
    build(str(REF))
    # bitwise pins: the reference built without FMA contraction, like the oracle
    strict = {**robot("_strict"), **resets("_strict"), **steps("_strict"), **task("_strict")}
    # the reference as shipped (its own flags): terrain, resets, a few steps
    shipped = {**terrains(""), **resets("")}
    st = steps("")
    shipped.update({k: st[k] for k in ("step_seeds", "step_diffs", "step_before", "step_targets",
                                       "step_after")})
    for name, data in (("golden_strict.npz", strict), ("golden_shipped.npz", shipped)):
        np.savez_compressed(OUT / name, **data)
        print(f"wrote {OUT / name} ({(OUT / name).stat().st_size // 1024} KB)")


if __name__ == "__main__":
    main()
