"""Shared parity measures of the FP32 step against the FP64 reference.

Two things the FP32 tests hold the CUDA step to, besides plain tolerances:

1. Its error against the FP64 reference is no worse than FP32 arithmetic
   itself: the strict FP32 C restatement of the reference (oracle/, no FMA,
   IEEE division) is stepped from the same states, and the kernel's error
   percentiles are bounded by a factor of the restatement's (`fp32_bound`).
   A regression of the kernel therefore shows even while it stays inside a
   flat tolerance.

2. Every sphere whose touch count differs from the reference's sits at a
   threshold the FP64 step decided within FP32 resolution
   (`classify_touch_mismatches`): the discrete outputs may only differ where
   the reference itself was a rounding away from the other outcome. The
   margins come from the FP64 restatement (bitwise the reference built
   without FMA contraction) stepped from the same state, which records for
   each decision of csrc/arc_phys.c how far it was from flipping: contact
   on/off (:570, :572-581, :587), friction anchor reset (:519),
   static/dynamic friction (:534) and limit activation (:437-443).
"""

from __future__ import annotations

import numpy as np

from oracle.oracle import NB, NS

# How close to a threshold an FP64 decision must be for FP32 to flip it.
# Positions: the FP32 step differs from the FP64 one by up to ~2e-5 of
# max(|x|, 1 m) after a control step (p99); 1e-4 of it is 5x that. Dot
# products of unit normals and the joint-limit sines carry FP32 errors of
# ~1e-6; 1e-4 leaves two orders of magnitude. The static/dynamic friction
# test compares two impulses whose FP32 relative error reaches 1e-4 when the
# tangential slip is small; 1e-3 relative.
CONTACT_RES = 1e-4   # of max(|x|, 1 m), metres
ANCHOR_RES = 1e-4    # dot product
FRICTION_RES = 1e-3  # relative
LIMIT_RES = 1e-4     # sine / radians


def body_errors(a: np.ndarray, b: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Per world, the largest body position error relative to max(|x|, 1 m)
    and the largest (sign-aligned) quaternion error."""
    xa = a[:, : NB * 13].reshape(len(a), NB, 13)
    xb = b[:, : NB * 13].reshape(len(b), NB, 13)
    scale = np.maximum(np.linalg.norm(xa[..., :3], axis=2), 1.0)
    dx = (np.linalg.norm(xa[..., :3] - xb[..., :3], axis=2) / scale).max(1)
    qa, qb = xa[..., 3:7], xb[..., 3:7]
    dq = np.minimum(np.linalg.norm(qa - qb, axis=2), np.linalg.norm(qa + qb, axis=2)).max(1)
    return dx, dq


def touches(s: np.ndarray) -> np.ndarray:
    return s[:, NB * 13: NB * 13 + NS * 8].reshape(len(s), NS, 8)[:, :, 7]


def position_scale(s: np.ndarray) -> np.ndarray:
    """max(|x|, 1 m) over each world's bodies."""
    x = s[:, : NB * 13].reshape(len(s), NB, 13)[..., :3]
    return np.maximum(np.linalg.norm(x, axis=2).max(1), 1.0)


def fp32_bound(name: str, kernel: np.ndarray, restatement: np.ndarray, factor: float = 1.25,
               floor: float = 1e-7, percentiles=(50, 95, 99)) -> None:
    """The kernel's error percentiles are at most `factor` times the strict
    FP32 restatement's (or `floor`, below which both are FP32 rounding of the
    start state)."""
    for p in percentiles:
        k, r = float(np.percentile(kernel, p)), float(np.percentile(restatement, p))
        assert k <= max(factor * r, floor), f"{name}: p{p} {k:.3e} > {factor} x restatement {r:.3e}"


def classify_touch_mismatches(kernel_state: np.ndarray, ref_state: np.ndarray, margins: np.ndarray,
                              start_state: np.ndarray) -> tuple[list[dict], int]:
    """Every sphere whose touch count differs between the kernel and the FP64
    reference after one teacher-forced step, with the FP64 margins of that
    step (OracleSim.margins(), one row per world: NS contact margins, then
    anchor, friction, limit). A mismatch is explained when its own contact
    decision was within CONTACT_RES of flipping, or when an earlier decision
    of the same world's step was within the resolution of its kind (a flip
    there moves the whole world's trajectory). Returns the rows and how many
    sphere-steps of the whole batch had their own contact margin within
    resolution (how selective the explanation is)."""
    tk, tr = touches(kernel_state), touches(ref_state)
    scale = position_scale(start_state)
    rows = []
    for w, s in np.argwhere(tk != tr):
        own = margins[w, s] / scale[w]
        others = np.delete(margins[w, :NS], s) / scale[w]
        norm = {"contact": own / CONTACT_RES, "other contact": others.min() / CONTACT_RES,
                "anchor": margins[w, NS] / ANCHOR_RES, "friction": margins[w, NS + 1] / FRICTION_RES,
                "limit": margins[w, NS + 2] / LIMIT_RES}
        closest = min(norm, key=norm.get)
        rows.append({"world": int(w), "sphere": int(s), "touch": (int(tk[w, s]), int(tr[w, s])),
                     "contact_margin_m": float(margins[w, s]), "closest": closest,
                     "normalised": float(norm[closest]), "explained": bool(norm[closest] < 1.0)})
    near = int((margins[:, :NS] / scale[:, None] < CONTACT_RES).sum())
    return rows, near


def report_mismatches(name: str, rows: list[dict], near: int, sphere_steps: int) -> None:
    kinds = {}
    for r in rows:
        kinds[r["closest"]] = kinds.get(r["closest"], 0) + 1
    worst = max((r["normalised"] for r in rows), default=0.0)
    print(f"{name}: {len(rows)} touch mismatches in {sphere_steps} sphere-steps; closest threshold {kinds}; "
          f"largest margin / resolution {worst:.2e}; sphere-steps within contact resolution {near} "
          f"({near / max(sphere_steps, 1):.1%})")
