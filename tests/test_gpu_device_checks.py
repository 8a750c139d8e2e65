"""The checked build of the library (libarcsim_checked.so: the same kernels
testing their data-dependent indexes, arc_demo_b200/csrc/arc_checks.cuh)
runs every kernel form and entry point of the step (the allocation-free one
included) over the configurations' terrain kinds, with resets, without a
single failed check. This stands in for
a memory checker over the test workloads: a terrain column outside its
world's slice of the pool, or a contact record outside its lane's slice of
the spill buffer, would be counted (and skipped) instead of read or written.
The workload runs in a child process that loads the checked build in place
of the regular one (ARC_SIM_LIB).
"""

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

from arc_demo_b200.build import LIB_CHECKED

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

WORKLOAD = r"""
import json
import numpy as np
import torch
from arc_demo_b200.native import KERNEL_LEGS, KERNEL_PLAIN, KERNEL_WARPS, Sim, device_checks
from arc_demo_b200.task import HEIGHT_OFFSETS, TaskConfig
from arc_demo_b200.torch_env import DeviceVecEnv

assert device_checks(clear=True)["checked"]
rng = np.random.default_rng(0)

# the reference ABI: every kernel form, flat and rough terrain, 64 x 64 grids
for fp64, kernels in ((False, ((KERNEL_WARPS, 16), (KERNEL_LEGS, 8), (KERNEL_LEGS, 16), (KERNEL_PLAIN, 16))),
                      (True, ((KERNEL_LEGS, 16), (KERNEL_PLAIN, 16)))):
    for kernel, wpc in kernels:
        n = 96
        sim = Sim(n, fp64=fp64)
        sim.set_kernel(kernel, wpc)
        sim.reset(np.arange(n), np.arange(n, dtype=np.uint32) * 3 + 1, np.linspace(0.0, 1.0, n))
        for _ in range(25):
            sim.step(rng.uniform(sim.lo, sim.hi, (n, 12)))
        sim.observe()
        sim.heights(HEIGHT_OFFSETS)
        sim.terrain_at(np.arange(n), rng.uniform(-15.0, 15.0, (n, 2)))
        sim.close()

# per-world terrain sizes (16 x 16 to 64 x 64) through one launch
n = 512
grids = rng.integers(16, 65, n).astype(np.int32)
sim = Sim(n, grids=grids)
sim.reset(np.arange(n), np.arange(n, dtype=np.uint32), rng.uniform(0.0, 1.0, n))
for _ in range(25):
    sim.step(rng.uniform(sim.lo, sim.hi, (n, 12)))
sim.observe()
sim.heights(HEIGHT_OFFSETS)
sim.close()

# the allocation-free entry point: state, terrain and targets in caller
# memory, the kernel's records and contact spill in the library's static array
import ctypes
from arc_demo_b200.native import sim_lib
noalloc = sim_lib().arc_step_noalloc
noalloc.restype = ctypes.c_int
noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                    ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
n = 256
sim = Sim(n)
sim.reset(np.arange(n), np.arange(n, dtype=np.uint32) * 5 + 3, np.linspace(0.0, 1.0, n))
d_state = torch.from_numpy(sim.get_state()).cuda()
d_heights = torch.from_numpy(np.stack([sim.get_terrain(i)[0] for i in range(n)]).astype(np.float32)).cuda()
for _ in range(25):
    d_t = torch.from_numpy(rng.uniform(sim.lo, sim.hi, (n, 12))).cuda()
    assert noalloc(d_state.data_ptr(), d_heights.data_ptr(), 64, 0.4, -100.0, d_t.data_ptr(), n, 1.0 / 30.0, 20,
                   None) == 0
torch.cuda.synchronize()
sim.close()

# the device env: graph step, host-buffer step and step in parts, with resets
n = 4096
env = DeviceVecEnv(n, TaskConfig(curriculum=False, max_steps=15), seed=1)
env.set_levels(rng.uniform(0.0, 1.0, n))
env.reset()
gen = torch.Generator(device="cuda")
gen.manual_seed(1)
def policy(part, obs, actions):
    actions.copy_(torch.rand(actions.shape, device="cuda", generator=gen) * 2 - 1)
for k in range(40):
    if k % 3 == 0:
        env.step(torch.rand((n, 12), device="cuda", generator=gen) * 2 - 1)
    elif k % 3 == 1:
        env.step_parts(policy, 3)
    else:
        env.step_host(torch.rand((n, 12), generator=torch.Generator().manual_seed(k)) * 2 - 1)
torch.cuda.synchronize()
env.close()

print(json.dumps(device_checks()))
"""


def test_checked_build_reports_no_failed_check():
    assert LIB_CHECKED.exists(), "build it with arc_demo_b200.build.build(checked=True)"
    env = dict(os.environ, ARC_SIM_LIB=str(LIB_CHECKED))
    r = subprocess.run([sys.executable, "-c", WORKLOAD], env=env, cwd=ROOT, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    record = json.loads(r.stdout.strip().splitlines()[-1])
    assert record["checked"]
    assert record["failures"] == 0, record
