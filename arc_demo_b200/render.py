"""ctypes binding of the GPU renderer (include/arc_render.h).

`Renderer` has the constructor and methods of the reference's binding
(arc/native.py:160-200): `size()`, `frame(sim, world, markers, active,
rgb)` returning an (H, W, 3) uint8 image, `keys()`, `set_title()`,
`set_view()`, `close()`. There is no window system, so `visible=True`
raises like the reference does without a display, `keys()` is always empty
and titles are ignored. `frames()` renders many worlds in one launch into a
device tensor, one camera per world.
"""

from __future__ import annotations

import ctypes
import functools

import numpy as np

from .native import ArcSimError, HERE, Sim, _declare, _vp

RENDER_LIB_PATH = HERE / "libarcrender.so"
_int = ctypes.c_int
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
MAX_MARKERS = 4
CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy


@functools.cache
def render_lib() -> ctypes.CDLL:
    """libarcrender.so, as the reference loads it (arc/native.py:59-70); its
    symbols come from libarcsim.so, on which it depends."""
    if not RENDER_LIB_PATH.exists():
        raise OSError(f"{RENDER_LIB_PATH} not found: build it with `python -m arc_demo_b200.build`")
    lib = ctypes.CDLL(str(RENDER_LIB_PATH))
    d = functools.partial(_declare, lib)
    d("arc_render_create", _vp, _int, _int, _int)
    d("arc_render_destroy", None, _vp)
    d("arc_render_frame", _int, _vp, _vp, _int, _vp, _int, _int, _vp)
    d("arc_render_size", None, _vp, ctypes.POINTER(_int), ctypes.POINTER(_int))
    d("arc_render_keys", _int, _vp, _i32, _int)
    d("arc_render_set_title", None, _vp, ctypes.c_char_p)
    d("arc_render_set_view", None, _vp, _int)
    d("arc_render_set_samples", _int, _vp, _int)
    d("arc_render_reset_cameras", _int, _vp)
    d("arc_render_frames", _int, _vp, _vp, _vp, _int, _vp, _int, _vp, _vp, _vp)
    d("arc_env_render", _int, _vp, _vp, _vp, _int, _vp, _vp)
    return lib


class Renderer:
    """Offscreen renderer of the worlds of a `Sim`."""

    def __init__(self, width: int = 1280, height: int = 720, visible: bool = True):
        self._lib = render_lib()
        self._ptr = self._lib.arc_render_create(width, height, int(visible))
        if not self._ptr:
            raise RuntimeError("cannot create renderer (no window system here; use visible=False)")
        self.closed = False

    def size(self) -> tuple[int, int]:
        w, h = ctypes.c_int(), ctypes.c_int()
        self._lib.arc_render_size(self._ptr, ctypes.byref(w), ctypes.byref(h))
        return w.value, h.value

    def frame(self, sim: Sim, world: int = 0, markers: np.ndarray | None = None,
              active: int = -1, rgb: bool = False) -> np.ndarray | None:
        """Draws the world with checkpoint markers given as rows of (x, y, z,
        radius); returns an (H, W, 3) uint8 image if rgb is set."""
        img = None
        img_ptr = None
        if rgb:
            w, h = self.size()
            img = np.empty((h, w, 3), dtype=np.uint8)
            img_ptr = img.ctypes.data
        m_ptr, n = None, 0
        if markers is not None and len(markers):
            markers = np.ascontiguousarray(markers, dtype=np.float64).reshape(-1, 4)
            m_ptr, n = markers.ctypes.data, len(markers)
        if not self._lib.arc_render_frame(self._ptr, sim.ptr, world, m_ptr, n, active, img_ptr):
            raise ArcSimError(f"arc_render_frame failed for world {world}")
        return img

    def frames(self, sim: Sim, ids=None, markers=None, active=None, out=None, stream: int | None = None):
        """Renders many worlds at once on the GPU: a (n, H, W, 3) uint8 CUDA
        tensor. ids: a CUDA int32 tensor of distinct world indices (None:
        every world); markers: a CUDA float32 tensor (n, m, 4) of (x, y, z,
        radius), m <= 4; active: a CUDA int32 tensor (n,) of highlighted
        marker indices (-1: none). Runs on torch's current stream unless a
        stream handle is given."""
        import torch

        if not stream:
            # torch's default stream has handle 0, which the C call reads as
            # "the sim's stream": name it as the legacy default stream (0x1)
            stream = torch.cuda.current_stream().cuda_stream or CUDA_STREAM_LEGACY
        n = sim.num_worlds if ids is None else int(ids.numel())
        w, h = self.size()
        if out is None:
            out = torch.empty((n, h, w, 3), dtype=torch.uint8, device="cuda")
        assert out.is_cuda and out.dtype == torch.uint8 and out.is_contiguous() and out.numel() == n * h * w * 3
        ids_ptr = None
        if ids is not None:
            assert ids.is_cuda and ids.dtype == torch.int32 and ids.is_contiguous()
            ids_ptr = ids.data_ptr()
        m_ptr, mpw = None, 0
        if markers is not None:
            assert markers.is_cuda and markers.dtype == torch.float32 and markers.is_contiguous()
            assert markers.dim() == 3 and markers.shape[0] == n and markers.shape[2] == 4
            m_ptr, mpw = markers.data_ptr(), int(markers.shape[1])
        a_ptr = None
        if active is not None:
            assert active.is_cuda and active.dtype == torch.int32 and active.numel() == n
            a_ptr = active.data_ptr()
        rc = self._lib.arc_render_frames(self._ptr, sim.ptr, ids_ptr, n, m_ptr, mpw, a_ptr, out.data_ptr(),
                                         stream)
        if rc != 0:
            raise ArcSimError(f"arc_render_frames failed ({rc})")
        return out

    def env_frames(self, env, ids=None, out=None, stream: int | None = None):
        """Frames of a `DeviceVecEnv`'s worlds with their checkpoints, as the
        reference's Viewer draws them: a (n, H, W, 3) uint8 CUDA tensor."""
        import torch

        if not stream:
            stream = torch.cuda.current_stream().cuda_stream or CUDA_STREAM_LEGACY
        sim = env.sim
        n = sim.num_worlds if ids is None else int(ids.numel())
        w, h = self.size()
        if out is None:
            out = torch.empty((n, h, w, 3), dtype=torch.uint8, device="cuda")
        assert out.is_cuda and out.dtype == torch.uint8 and out.is_contiguous() and out.numel() == n * h * w * 3
        ids_ptr = None
        if ids is not None:
            assert ids.is_cuda and ids.dtype == torch.int32 and ids.is_contiguous()
            ids_ptr = ids.data_ptr()
        rc = self._lib.arc_env_render(self._ptr, sim.ptr, ids_ptr, n, out.data_ptr(), stream)
        if rc != 0:
            raise ArcSimError(f"arc_env_render failed ({rc})")
        return out

    def set_samples(self, samples: int) -> None:
        """Rays per pixel: 4 (default, the reference's multisampling) or 1."""
        if self._lib.arc_render_set_samples(self._ptr, samples) != 0:
            raise ValueError("samples must be 1 or 4")

    def reset_cameras(self) -> None:
        self._lib.arc_render_reset_cameras(self._ptr)

    def keys(self) -> list[int]:
        buf = np.zeros(32, dtype=np.int32)
        n = self._lib.arc_render_keys(self._ptr, buf, 32)
        return [int(k) for k in buf[:n]]

    def set_title(self, title: str) -> None:
        self._lib.arc_render_set_title(self._ptr, title.encode())

    def set_view(self, preset: int) -> None:
        self._lib.arc_render_set_view(self._ptr, preset)

    def close(self) -> None:
        if self._ptr:
            self._lib.arc_render_destroy(self._ptr)
            self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
