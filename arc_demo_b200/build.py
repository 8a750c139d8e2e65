"""Builds arc_demo_b200/libarcsim.so, the drop-in batched step library.

nvcc compiles every .cu under csrc/ for sm_100a only (no other targets, no
PTX fallback) and links them with the static CUDA runtime into one shared
library with a plain C ABI (include/arc_sim.h). Objects go to _build/.
build(checked=True) makes the checked build, libarcsim_checked.so (objects
in _build_checked/): the same sources with ARC_DEVICE_CHECKS, whose kernels
test their data-dependent indexes (csrc/arc_checks.cuh).

    python -m arc_demo_b200.build          # or: python arc_demo_b200/build.py [-f] [--checked]
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
BUILD = HERE / "_build"
LIB = HERE / "libarcsim.so"
BUILD_CHECKED = HERE / "_build_checked"
LIB_CHECKED = HERE / "libarcsim_checked.so"
# the reference loads its renderer from a second library (arc/native.py:59-70);
# this one only depends on libarcsim.so, which exports the arc_render_* calls
RENDER_LIB = HERE / "libarcrender.so"
INCLUDE = HERE.parent / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-Xptxas", "-warn-spills", f"-I{INCLUDE}", f"-I{CSRC}"]
# per-file flags: the warp-per-leg FP32 step (arc_step_warps.cuh, compiled
# into arc_task.cu's control-step kernel) divides and takes square roots with
# the full-range approximate instructions (at most 2 ulp), whose errors are
# far below the FP32 parity bounds its tests hold it to, and flushes denormals
# to zero (no fix-up code for them: 3% less code and time); the task layer's
# own arithmetic there is FP64, which these flags do not touch
FILE_FLAGS = {"arc_task.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
              # the renderer: the same, for code size (its output is 8-bit colour)
              "arc_render.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src, *CSRC.glob("*.cuh"), *CSRC.glob("*.h"), *INCLUDE.glob("*.h"), Path(__file__)]
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra: list[str] | None = None, checked: bool = False) -> Path:
    build_dir, lib = (BUILD_CHECKED, LIB_CHECKED) if checked else (BUILD, LIB)
    build_dir.mkdir(exist_ok=True)
    cc = nvcc()
    extra = (extra or []) + (["-DARC_DEVICE_CHECKS"] if checked else [])
    jobs = []
    for src in sources():
        obj = build_dir / (src.stem + ".o")
        if force or _stale(obj, src):
            jobs.append([cc, *ARCH, *FLAGS, *FILE_FLAGS.get(src.name, []), *extra, "-c", str(src), "-o", str(obj)])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, file=sys.stderr)
        return r

    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        list(ex.map(run, jobs))
    objs = [str(build_dir / (s.stem + ".o")) for s in sources()]
    if jobs or not lib.exists():
        run([cc, *ARCH, "-shared", "-o", str(lib), *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    if checked:
        return lib
    if jobs or not RENDER_LIB.exists():
        cxx = shutil.which("gcc") or "gcc"
        run([cxx, "-shared", "-fPIC", "-o", str(RENDER_LIB), "-x", "c", os.devnull, f"-L{HERE}",
             "-Wl,--no-as-needed", "-larcsim", "-Wl,-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, checked="--checked" in sys.argv))
