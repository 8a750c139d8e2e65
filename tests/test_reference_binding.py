"""The reference's own ctypes binding (arc/native.py:38-70), as recorded from
the reference by tests/golden/make_binding.py, binds to this library.

CPU: every function the reference declares is exported by libarcsim.so (or
libarcrender.so), and each ctypes type the reference passes agrees with the C
prototype in include/*.h (int with int, double with double, a float64 /
int32 / uint32 array with a pointer to double / int / unsigned, an opaque
handle with a pointer).

GPU: a fresh handle of the library, declared exactly as the reference
declares it, runs the reference's Sim call sequence (arc/native.py:73-157:
create, robot info, reset, step, observe, heights, terrain_at, destroy) and
gives the same numbers as this repository's binding.
"""

import ctypes
import json
import re
from pathlib import Path

import numpy as np
import pytest

from arc_demo_b200.build import LIB, RENDER_LIB

ROOT = Path(__file__).resolve().parents[1]
BINDING = json.loads((ROOT / "tests" / "golden" / "reference_binding.json").read_text())
LIBS = {"libarcsim.so": LIB, "libarcrender.so": RENDER_LIB}


def prototypes() -> dict:
    """name -> (return type, [parameter types]) of every function in include/*.h."""
    out = {}
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for ret, name, params in re.findall(r"([\w\s\*]+?)\s*\b(arc_\w+)\s*\(([^)]*)\)\s*;", text):
            ps = [p.strip() for p in params.split(",") if p.strip() and p.strip() != "void"]
            # drop the parameter names: the type is everything but the last word
            types = [re.sub(r"\s*\b\w+$", "", p) if re.search(r"[\w\*]\s+\**\w+$", p) else p for p in ps]
            out[name] = (" ".join(ret.split()), [" ".join(t.replace("*", " * ").split()) for t in types])
    return out


def compatible(ctype: str, ctext: str) -> bool:
    """Whether a ctypes type name recorded from the reference fits a C type."""
    c = ctext.replace("const ", "").strip()
    if ctype == "void":
        return c == "void"
    if ctype == "c_int":
        return c == "int"
    if ctype == "c_double":
        return c == "double"
    if ctype == "c_char_p":
        return c == "char *"
    if ctype == "c_void_p":
        return c.endswith("*")
    if ctype.startswith("ndpointer:"):
        dt = ctype.split(":")[1]
        return c.replace("unsigned int", "unsigned") == {"float64": "double *", "int32": "int *", "uint32": "unsigned *"}[dt]
    if ctype.startswith("POINTER:"):
        return c == {"c_int": "int *", "c_double": "double *"}[ctype.split(":")[1]]
    return False


def test_fixture_holds_the_reference_declarations():
    sim = BINDING["libraries"]["libarcsim.so"]
    assert {"arc_sim_create", "arc_sim_step", "arc_sim_observe", "arc_sim_heights", "arc_sim_terrain_at"} <= set(sim)
    assert "arc_render_frame" in BINDING["libraries"]["libarcrender.so"]


def test_reference_declarations_match_the_headers_and_exports():
    protos = prototypes()
    for libname, decls in BINDING["libraries"].items():
        lib = ctypes.CDLL(str(LIBS[libname]))
        for name, d in decls.items():
            getattr(lib, name)  # exported (libarcrender.so forwards to libarcsim.so)
            assert name in protos, f"{name} is not declared in include/*.h"
            ret, params = protos[name]
            assert compatible(d["restype"], ret), (name, d["restype"], ret)
            assert len(d["argtypes"]) == len(params), (name, d["argtypes"], params)
            for t, c in zip(d["argtypes"], params):
                assert compatible(t, c), (name, t, c)


def declared(libname: str) -> ctypes.CDLL:
    """A handle of the library with the reference's declarations applied."""
    lib = ctypes.CDLL(str(LIBS[libname]))
    types = {"void": None, "c_int": ctypes.c_int, "c_double": ctypes.c_double, "c_void_p": ctypes.c_void_p,
             "c_char_p": ctypes.c_char_p}
    nd = {"float64": np.float64, "int32": np.int32, "uint32": np.uint32}

    def conv(t):
        if t in types:
            return types[t]
        if t.startswith("ndpointer:"):
            return np.ctypeslib.ndpointer(dtype=nd[t.split(":")[1]], flags="C_CONTIGUOUS")
        if t.startswith("POINTER:"):
            return ctypes.POINTER(types[t.split(":")[1]])
        raise ValueError(t)
    for name, d in BINDING["libraries"][libname].items():
        fn = getattr(lib, name)
        fn.restype = conv(d["restype"])
        fn.argtypes = [conv(t) for t in d["argtypes"]]
    return lib


@pytest.mark.gpu
def test_reference_call_sequence_drives_the_gpu_library():
    from arc_demo_b200.native import Sim
    from arc_demo_b200.task import HEIGHT_OFFSETS

    lib = declared("libarcsim.so")
    n, nj = 64, lib.arc_sim_num_joints()
    legs = lib.arc_sim_num_legs()
    assert (nj, legs) == (12, 4)
    ptr = lib.arc_sim_create(n, 1.0 / 30.0, 20, 64, 0.4)
    assert ptr
    lib.arc_sim_set_threads(ptr, 4)
    default, lo, hi, misc = np.zeros(nj), np.zeros(nj), np.zeros(nj), np.zeros(2)
    lib.arc_sim_robot_info(ptr, default, lo, hi, misc)
    ids = np.arange(n, dtype=np.int32)
    seeds = np.arange(n, dtype=np.uint32) * 11 + 2
    diffs = np.linspace(0.0, 1.0, n)
    lib.arc_sim_reset(ptr, ids, n, seeds, diffs)
    ours = Sim(n)
    ours.reset(ids, seeds, diffs)
    rng = np.random.default_rng(4)
    root, rot = np.zeros((n, 13)), np.zeros((n, 3, 3))
    joints, contacts, flags = np.zeros((n, 3 * nj)), np.zeros((n, legs + 2)), np.zeros(n, dtype=np.int32)
    offsets = np.ascontiguousarray(HEIGHT_OFFSETS, dtype=np.float64)
    heights = np.empty((n, len(offsets)))
    for _ in range(5):
        t = np.ascontiguousarray(default + 0.6 * rng.uniform(-1, 1, (n, nj)))
        lib.arc_sim_step(ptr, t.ctypes.data)
        ours.step(t)
    lib.arc_sim_observe(ptr, root.ctypes.data, rot.ctypes.data, joints.ctypes.data, contacts.ctypes.data,
                        flags.ctypes.data)
    lib.arc_sim_heights(ptr, offsets.ctypes.data, len(offsets), heights.ctypes.data)
    xy = np.ascontiguousarray(rng.uniform(-10, 10, (n, 2)))
    at = np.zeros(n)
    lib.arc_sim_terrain_at(ptr, ids, xy, n, at)
    o_root, o_joints, o_contacts, o_flags = ours.observe()
    assert np.array_equal(root, o_root) and np.array_equal(joints, o_joints)
    assert np.array_equal(contacts, o_contacts) and np.array_equal(flags, o_flags)
    assert np.array_equal(default, ours.default_angles) and misc[0] == ours.stand_height
    assert np.array_equal(heights, ours.heights(offsets))
    assert np.array_equal(at, ours.terrain_at(ids, xy))
    assert np.all(np.isfinite(root)) and not flags.any()
    lib.arc_sim_destroy(ptr)
    ours.close()
