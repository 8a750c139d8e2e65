"""The renderer's host side without a GPU: the ABI the reference binds, and
its CPU restatement (oracle/render_oracle.c) on worlds of the reference
build, whose pictures must show the scene of csrc/arc_render.c."""

import ctypes
import subprocess

import numpy as np
import pytest

from arc_demo_b200 import native
from arc_demo_b200.build import LIB, RENDER_LIB, build

# csrc/arc_render.h:11-39, bound by arc/native.py:59-70
REFERENCE_RENDER_SYMBOLS = [
    "arc_render_create", "arc_render_destroy", "arc_render_frame", "arc_render_size",
    "arc_render_keys", "arc_render_set_title", "arc_render_set_view",
]


@pytest.fixture(scope="module")
def rlib():
    if not RENDER_LIB.exists() or not LIB.exists():
        build()
    return ctypes.CDLL(str(RENDER_LIB))


def test_render_library_resolves_the_reference_symbols(rlib):
    for s in REFERENCE_RENDER_SYMBOLS + ["arc_render_frames", "arc_render_set_samples", "arc_render_reset_cameras"]:
        assert s in native.header_symbols()
        getattr(rlib, s)
    needed = subprocess.run(["readelf", "-d", str(RENDER_LIB)], capture_output=True, text=True, check=True).stdout
    assert "libarcsim.so" in needed


def test_visible_renderer_is_refused_without_touching_cuda(rlib):
    rlib.arc_render_create.restype = ctypes.c_void_p
    rlib.arc_render_create.argtypes = [ctypes.c_int] * 3
    assert not rlib.arc_render_create(640, 360, 1)
    assert not rlib.arc_render_create(0, 360, 0)
    assert not rlib.arc_render_create(640, -1, 0)


def _ref_world(seed=3, difficulty=0.6):
    from oracle.oracle import RefSim
    try:
        sim = RefSim(1, grid=24)
    except FileNotFoundError as e:
        pytest.skip(str(e))
    sim.reset(np.arange(1), np.array([seed], dtype=np.uint32), np.array([difficulty]))
    return sim


def test_oracle_draws_the_scene():
    from oracle.oracle import RenderOracle
    sim = _ref_world()
    img = RenderOracle(96, 54, samples=1).frame(sim.world(0))
    assert img.shape == (54, 96, 3) and img.dtype == np.uint8
    # the void above the arena is black; the terrain below is lit
    assert img[:4].max() == 0
    assert img[36:].mean() > 40
    # the robot stands at the camera's target, in the middle of the frame
    mid = img[18:40, 36:60].astype(int)
    assert np.abs(mid - img[40:, :].mean(axis=(0, 1))).mean() > 5


def test_oracle_markers_views_and_determinism():
    from oracle.oracle import RenderOracle
    sim = _ref_world()
    w = sim.world(0)
    markers = np.array([[0.8, -0.6, 0.0, 0.4]])
    a = RenderOracle(64, 36, samples=1).frame(w, markers, 0)
    b = RenderOracle(64, 36, samples=1).frame(w, markers, 0)
    assert np.array_equal(a, b)
    seen = a.astype(int)
    unseen = RenderOracle(64, 36, samples=1).frame(w, markers, -1).astype(int)
    # the seen beacon is orange, the unseen one blue
    assert (seen[..., 0] - seen[..., 2]).sum() > (unseen[..., 0] - unseen[..., 2]).sum()
    side = RenderOracle(64, 36, samples=1, view=1).frame(w, markers, 0)
    assert not np.array_equal(a, side)


def test_oracle_camera_smoothing():
    """The camera starts at the torso + 0.1 m and then moves 15% of the way
    toward it per frame (csrc/arc_render.c:700-716)."""
    from oracle.oracle import RenderOracle
    sim = _ref_world()
    w = sim.world(0)
    r = RenderOracle(16, 9, samples=1)
    r.frame(w)
    target = np.array([w.bodies[0].x.x, w.bodies[0].x.y, w.bodies[0].x.z + 0.1])
    assert r.cam[0] == 1.0 and np.allclose(r.cam[1:4], target)
    r.cam[1:4] = target + np.array([1.0, 0.0, 0.0])
    r.frame(w)
    assert np.allclose(r.cam[1:4], target + np.array([0.85, 0.0, 0.0]))
    r.cam[1:4] = target + np.array([4.0, 0.0, 0.0])  # beyond 3 m: jumps
    r.frame(w)
    assert np.allclose(r.cam[1:4], target)
