"""The drop-in library loads without a GPU and exports its whole C ABI."""

import ctypes
import subprocess

import pytest

from arc_demo_b200 import native
from arc_demo_b200.build import LIB, LIB_CHECKED, build

# the reference's batched API (csrc/arc_sim.h:25-56), bound by arc/native.py:38-55
REFERENCE_SYMBOLS = [
    "arc_sim_create", "arc_sim_destroy", "arc_sim_set_threads", "arc_sim_num_worlds",
    "arc_sim_num_joints", "arc_sim_num_legs", "arc_sim_robot_info", "arc_sim_reset",
    "arc_sim_step", "arc_sim_observe", "arc_sim_heights", "arc_sim_terrain_at", "arc_sim_world",
]


@pytest.fixture(scope="module")
def lib():
    if not LIB.exists():
        build()
    return ctypes.CDLL(str(LIB))


def test_header_declares_reference_api():
    syms = native.header_symbols()
    for s in REFERENCE_SYMBOLS:
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in native.header_symbols() if s not in exported]
    assert not missing, missing
    for s in native.header_symbols():
        getattr(lib, s)


def test_checked_build_exports_the_same_abi():
    """libarcsim_checked.so (the kernels testing their indexes) is a drop-in
    for libarcsim.so: every declared symbol, and it says it is the checked
    build only through arc_device_checks, which needs a device."""
    if not LIB_CHECKED.exists():
        build(checked=True)
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_CHECKED)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [s for s in native.header_symbols() if s not in exported]
    assert not missing, missing


def test_regular_build_checks_nothing():
    """The regular build compiles the index checks away: arc_device_checks
    reports 0 (not the checked build) and no failures, without a device."""
    record = native.device_checks()
    assert not record["checked"] and record["failures"] == 0


def test_constants_without_a_device(lib):
    assert lib.arc_sim_num_joints() == 12
    assert lib.arc_sim_num_legs() == 4


def test_arc_world_layout_matches_reference_size():
    """include/arc_world.h mirrors csrc/arc_phys.h's arc_world: 62,960 bytes."""
    from oracle.oracle import World
    assert ctypes.sizeof(World) == 62960
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "arc_world.h"
int main(void) { printf("%zu %zu %zu\n", sizeof(arc_world), offsetof(arc_world, terrain),
                 offsetof(arc_world, bodies)); return 0; }
'''
    import tempfile
    from pathlib import Path
    inc = Path(native.HEADER).parent
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "t.c"
        c.write_text(src)
        exe = Path(d) / "t"
        subprocess.run(["gcc", "-I", str(inc), str(c), "-o", str(exe)], check=True)
        size, terrain, bodies = map(int, subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.split())
    assert size == 62960
    assert terrain == World.terrain.offset
    assert bodies == World.bodies.offset
