"""The GPU renderer (csrc/arc_render.cu) against its CPU restatement
(oracle/render_oracle.c), through the reference's renderer ABI.

Tolerance. The two differ only in arithmetic: FP32 rays and shading on the
GPU, FP64 in the oracle (both evaluate the shader's sin-based hash in
float with the same rounding order). A sample whose ray passes within
rounding of a silhouette or a column edge can land on different surfaces,
and a channel within rounding of a half level can round either way. So a
frame matches when its mean absolute difference is at most 0.1 levels and
at most 0.3% of its channels differ by more than 2 levels (of 255).
"""

import ctypes

import numpy as np
import pytest

from arc_demo_b200.native import Sim
from arc_demo_b200.render import Renderer
from oracle.oracle import RefSim, RenderOracle, World

pytestmark = pytest.mark.gpu

W, H = 128, 72


def world_of(sim: Sim, i: int) -> World:
    lib = sim._lib
    lib.arc_sim_world.restype = ctypes.POINTER(World)
    lib.arc_sim_world.argtypes = [ctypes.c_void_p, ctypes.c_int]
    return lib.arc_sim_world(sim.ptr, i).contents


def assert_frames_match(gpu: np.ndarray, ref: np.ndarray, what: str = ""):
    assert gpu.shape == ref.shape and gpu.dtype == np.uint8
    d = np.abs(gpu.astype(np.int32) - ref.astype(np.int32))
    assert d.mean() <= 0.1, f"{what}: mean abs difference {d.mean():.3f}"
    assert (d > 2).mean() <= 0.003, f"{what}: {(d > 2).mean():.4%} of channels differ by more than 2"
    # the picture is not trivially empty: terrain and robot are lit
    assert ref.mean() > 20.0


def make_sim(n=4, grid=32, fp64=False):
    sim = Sim(n, grid=grid, fp64=fp64)
    seeds = np.arange(11, 11 + n, dtype=np.uint32)
    sim.reset(np.arange(n), seeds, np.linspace(0.0, 1.0, n))
    return sim


def test_visuals_match_the_reference_robot():
    sim = make_sim(1)
    ref = RefSim(1)
    a, b = world_of(sim, 0), ref.world(0)
    assert a.n_visuals == b.n_visuals == 74
    for i in range(a.n_visuals):
        va, vb = a.visuals[i], b.visuals[i]
        assert (va.type, va.body, va.material) == (vb.type, vb.body, vb.material), i
        for f in ("p0", "p1"):
            pa, pb = getattr(va, f), getattr(vb, f)
            assert np.allclose([pa.x, pa.y, pa.z], [pb.x, pb.y, pb.z], rtol=0, atol=1e-12), (i, f)
        assert np.allclose([va.radius, va.radius2, va.aspect], [vb.radius, vb.radius2, vb.aspect], rtol=0, atol=1e-12)
        assert list(va.color) == list(vb.color), i


@pytest.mark.parametrize("samples", [1, 4])
@pytest.mark.parametrize("world", [0, 1, 2, 3])
def test_frame_matches_oracle(samples, world):
    sim = make_sim()
    markers = np.array([[1.5, -1.0, 0.0, 0.5]])
    active = 0 if world % 2 else -1
    r = Renderer(W, H, visible=False)
    r.set_samples(samples)
    gpu = r.frame(sim, world, markers, active, rgb=True)
    ref = RenderOracle(W, H, samples=samples).frame(world_of(sim, world), markers, active)
    assert_frames_match(gpu, ref, f"world {world}, {samples} samples")


@pytest.mark.parametrize("view", [1, 2, 5])
def test_view_presets_match_oracle(view):
    sim = make_sim()
    r = Renderer(W, H, visible=False)
    r.set_view(view)
    r.set_samples(1)
    gpu = r.frame(sim, 2, None, -1, rgb=True)
    ref = RenderOracle(W, H, samples=1, view=view).frame(world_of(sim, 2))
    assert_frames_match(gpu, ref, f"view {view}")


def test_camera_follows_a_moving_robot():
    """The camera's smoothing state carries from frame to frame as the
    reference's does: five steps of random drive targets, one frame each."""
    sim = make_sim(2)
    rng = np.random.default_rng(5)
    r = Renderer(W, H, visible=False)
    r.set_samples(1)
    ora = RenderOracle(W, H, samples=1)
    markers = np.array([[3.0, 2.0, 0.2, 0.5], [-2.0, 1.0, 0.0, 0.4]])
    for k in range(5):
        targets = np.tile(sim.default_angles, (2, 1)) + rng.uniform(-0.6, 0.6, (2, 12))
        for _ in range(3):
            sim.step(targets)
        gpu = r.frame(sim, 1, markers, k % 2, rgb=True)
        ref = ora.frame(world_of(sim, 1), markers, k % 2)
        assert_frames_match(gpu, ref, f"frame {k}")


def test_fallen_robot_and_fp64_worlds():
    """An upside-down robot on rough terrain, in an FP64 simulation."""
    sim = make_sim(2, fp64=True)
    s = np.sqrt(0.5)
    sim.set_pose(1, (0.3, -0.2, 0.6), (0.0, s, s, 0.0), sim.default_angles)
    r = Renderer(W, H, visible=False)
    gpu = r.frame(sim, 1, None, -1, rgb=True)
    ref = RenderOracle(W, H, samples=4).frame(world_of(sim, 1))
    assert_frames_match(gpu, ref, "fallen")


def test_batched_frames_equal_single_frames():
    """arc_render_frames with fresh cameras gives, for each world, the bytes
    arc_render_frame gives on a fresh renderer."""
    import torch

    sim = make_sim(5)
    ids = torch.tensor([4, 0, 2], dtype=torch.int32, device="cuda")
    markers = torch.tensor([[[1.0, 1.0, 0.0, 0.5]], [[-1.0, 2.0, 0.1, 0.3]], [[0.0, -2.0, 0.0, 0.6]]],
                           dtype=torch.float32, device="cuda")
    active = torch.tensor([0, -1, 0], dtype=torch.int32, device="cuda")
    r = Renderer(W, H, visible=False)
    batch = r.frames(sim, ids, markers, active).cpu().numpy()
    for k, w in enumerate(ids.tolist()):
        one = Renderer(W, H, visible=False)
        img = one.frame(sim, w, markers[k].cpu().numpy().astype(np.float64), int(active[k]), rgb=True)
        assert np.array_equal(batch[k], img), k


def test_errors_are_reported_not_faults():
    import torch

    sim = make_sim(2)
    with pytest.raises(RuntimeError):
        Renderer(W, H, visible=True)
    r = Renderer(W, H, visible=False)
    with pytest.raises(ValueError):
        r.set_samples(3)
    from arc_demo_b200.native import ArcSimError
    with pytest.raises(ArcSimError):
        r.frame(sim, 7, None, -1, rgb=True)
    lib = r._lib
    out = torch.empty((2, H, W, 3), dtype=torch.uint8, device="cuda")
    m = torch.zeros((2, 5, 4), dtype=torch.float32, device="cuda")
    assert lib.arc_render_frames(r._ptr, sim.ptr, None, 2, m.data_ptr(), 5, None, out.data_ptr(), None) < 0
    assert lib.arc_render_frames(r._ptr, sim.ptr, None, 3, None, 0, None, out.data_ptr(), None) < 0
    assert r.keys() == []
    # and it still renders
    assert r.frame(sim, 1, None, -1, rgb=True).mean() > 20.0


def test_device_env_frames_show_each_world_checkpoint():
    """arc_env_render takes each world's checkpoint and in-view flag from the
    device task layer: the bytes equal arc_render_frames given the same
    markers from the task state (target x, y, z, radius; active 0 while in
    view, arc/env.py:45-47)."""
    import torch
    from arc_demo_b200.task import TaskConfig
    from arc_demo_b200.torch_env import DeviceVecEnv

    n = 6
    env = DeviceVecEnv(n, TaskConfig(curriculum=False), seed=3)
    env.reset()
    for _ in range(3):
        env.step(torch.zeros((n, 12), dtype=torch.float32, device="cuda"))
    torch.cuda.synchronize()
    ids = torch.tensor([5, 1, 3], dtype=torch.int32, device="cuda")
    a = Renderer(W, H, visible=False)
    got = a.env_frames(env, ids).cpu().numpy()
    st = env.gpu.get_state()[ids.cpu().numpy()]
    markers = np.stack([st[:, 0], st[:, 1], st[:, 2], np.full(3, env.cfg.checkpoint_radius)], axis=1)
    markers = torch.tensor(markers[:, None, :].astype(np.float32), device="cuda")
    active = torch.tensor(np.where(st[:, 22] != 0, 0, -1).astype(np.int32), device="cuda")
    b = Renderer(W, H, visible=False)
    want = b.frames(env.sim, ids, markers, active).cpu().numpy()
    assert np.array_equal(got, want)
    frames = env.render(width=W, height=H)
    assert frames.shape == (n, H, W, 3) and frames.is_cuda
    env.close()


def test_per_world_terrain_sizes_match_oracle():
    """Worlds of different grid sizes in one sim (the uneven-size
    configuration's packed terrain pool), each frame against the oracle."""
    grids = np.array([16, 37, 64], dtype=np.int32)
    sim = Sim(3, grids=grids)
    sim.reset(np.arange(3), np.array([7, 8, 9], dtype=np.uint32), np.array([0.9, 0.5, 1.0]))
    r = Renderer(W, H, visible=False)
    r.set_samples(1)
    for w in range(3):
        gpu = r.frame(sim, w, None, -1, rgb=True)
        r.reset_cameras()
        ref = RenderOracle(W, H, samples=1).frame(world_of(sim, w))
        assert_frames_match(gpu, ref, f"grid {grids[w]}")


def test_custom_model_visuals_match_oracle():
    """A custom model's own visuals, one of each shape and several
    materials, on a plain-kernel sim."""
    from arc_demo_b200.native import Model

    m = Model()
    b0 = m.add_body(2.0, (0.1, 0.1, 0.1), (0.0, 0.0, 0.6))
    b1 = m.add_body(1.0, (0.05, 0.05, 0.05), (0.4, 0.0, 0.6))
    m.add_sphere(b0, (0, 0, 0), 0.2)
    m.add_sphere(b1, (0, 0, 0), 0.1)
    m.add_hinge(b0, b1, (0.2, 0.0, 0.6), (0.0, 1.0, 0.0))
    m.add_visual(0, b0, (0, 0, 0), (0, 0, 0), 0.2, material=1, color=(0.5, 0.45, 0.4))        # panelled sphere
    m.add_visual(1, b1, (0, 0, 0), (0.1, 0.08, 0.06), 0.0, material=0, color=(0.3, 0.3, 0.35))  # rounded box
    m.add_visual(2, b0, (0, 0, -0.2), (0, 0, -0.5), 0.08, 0.04, aspect=0.7, material=2, color=(0.6, 0.6, 0.6))
    m.add_visual(3, b1, (0, -0.15, 0), (0, 0.15, 0), 0.03, material=5, color=(0.3, 0.3, 0.3))  # ribbed cylinder
    m.add_visual(4, b0, (0.2, 0, 0), (1, 0, 0), 0.09, 0.015, material=6, color=(1.0, 0.2, 0.1))  # glowing ring
    sim = Sim(2, grid=24, model=m)
    rng = np.random.default_rng(4)
    sim.set_terrain(1, np.round(rng.uniform(-0.1, 0.2, (24, 24)) / 0.05) * 0.05, 0.4, -100.0)
    sim.set_pose(1, (0.0, 0.0, 0.9), (0.96, 0.1, 0.2, 0.15), np.zeros(1))
    r = Renderer(W, H, visible=False)
    gpu = r.frame(sim, 1, None, -1, rgb=True)
    w = world_of(sim, 1)
    assert w.n_visuals == 5
    ref = RenderOracle(W, H, samples=4).frame(w)
    assert_frames_match(gpu, ref, "custom model")


def test_larger_frame_on_the_full_grid_and_determinism():
    """A 320 x 180 frame on a 64 x 64 terrain against the oracle; the same
    batch rendered twice from the same camera state is byte-identical."""
    import torch

    sim = make_sim(2, grid=64)
    r = Renderer(320, 180, visible=False)
    r.set_samples(1)
    gpu = r.frame(sim, 1, np.array([[2.0, -1.0, 0.0, 0.5]]), 0, rgb=True)
    ref = RenderOracle(320, 180, samples=1).frame(world_of(sim, 1), np.array([[2.0, -1.0, 0.0, 0.5]]), 0)
    assert_frames_match(gpu, ref, "320x180")
    a = Renderer(320, 180, visible=False)
    b = Renderer(320, 180, visible=False)
    fa = a.frames(sim).cpu().numpy()
    fb = b.frames(sim).cpu().numpy()
    assert np.array_equal(fa, fb)


def test_calls_on_different_streams_are_ordered():
    """Consecutive calls of one renderer on different streams share its
    frame records and cameras; each waits for the previous one, so the
    frames equal those of the same calls on one stream."""
    import torch

    sim = make_sim(4)
    a = Renderer(W, H, visible=False)
    b = Renderer(W, H, visible=False)
    side = torch.cuda.Stream()
    ids1 = torch.tensor([0, 2], dtype=torch.int32, device="cuda")
    ids2 = torch.tensor([1, 3, 0], dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        f1 = a.frames(sim, ids1)
    f2 = a.frames(sim, ids2)
    side.synchronize()
    torch.cuda.synchronize()
    g1 = b.frames(sim, ids1)
    g2 = b.frames(sim, ids2)
    torch.cuda.synchronize()
    assert torch.equal(f1, g1) and torch.equal(f2, g2)
