"""Records the reference's own ctypes declarations (arc/native.py sim_lib()
and render_lib(), arc/native.py:38-70) into tests/golden/reference_binding.json.

The reference's native.py is executed as it is, with ctypes.CDLL replaced by a
recorder for the duration, so every `_declare(lib, name, restype, *argtypes)`
it makes is captured with the ctypes types it passes. The tests bind exactly
these declarations to libarcsim.so / libarcrender.so (tests/test_reference_binding.py),
which checks the drop-in claim against the reference's binding itself rather
than against this repository's copy of it.

Needs the reference checkout, given explicitly:

    python tests/golden/make_binding.py --ref <reference checkout>     (or ARC_REFERENCE=<dir>)
"""

from __future__ import annotations

import argparse
import ctypes
import importlib.util
import json
import os
import sys
import tempfile
from pathlib import Path

OUT = Path(__file__).resolve().parent / "reference_binding.json"


def type_name(t) -> str:
    """A stable name for a ctypes type as the reference passes it."""
    if t is None:
        return "void"
    flags = getattr(t, "_flags_", None)
    dtype = getattr(t, "_dtype_", None)
    if dtype is not None:  # numpy.ctypeslib.ndpointer
        return f"ndpointer:{dtype.name}" + (":C_CONTIGUOUS" if flags else "")
    if isinstance(t, type) and issubclass(t, ctypes._Pointer):
        return f"POINTER:{t._type_.__name__}"
    return t.__name__


class _Fn:
    def __init__(self, log, lib, name):
        self._log, self._lib, self._name = log, lib, name
        self.restype, self.argtypes = None, []

    def __setattr__(self, key, value):
        object.__setattr__(self, key, value)
        if key == "argtypes" and not key.startswith("_") and value:
            self._log.setdefault(self._lib, {})[self._name] = {
                "restype": type_name(self.restype), "argtypes": [type_name(a) for a in value]}
        elif key == "argtypes" and value == []:
            self._log.setdefault(self._lib, {})[self._name] = {"restype": type_name(self.restype), "argtypes": []}


class _Recorder:
    def __init__(self, log, path):
        object.__setattr__(self, "_log", log)
        object.__setattr__(self, "_libname", Path(path).name)
        object.__setattr__(self, "_fns", {})

    def __getattr__(self, name):
        fns = object.__getattribute__(self, "_fns")
        if name not in fns:
            fns[name] = _Fn(object.__getattribute__(self, "_log"), object.__getattribute__(self, "_libname"), name)
        return fns[name]


def record(ref: Path) -> dict:
    src = ref / "arc" / "native.py"
    log: dict = {}
    with tempfile.TemporaryDirectory() as tmp:
        # the reference loads its libraries from its own directory; give it
        # placeholder files there so its existence check passes
        for name in ("libarcsim.so", "libarcrender.so"):
            (Path(tmp) / name).write_bytes(b"")
        spec = importlib.util.spec_from_file_location("arc_reference_native", src)
        mod = importlib.util.module_from_spec(spec)
        real = ctypes.CDLL
        ctypes.CDLL = lambda path, *a, **k: _Recorder(log, path)  # noqa: E731
        try:
            spec.loader.exec_module(mod)
            mod._HERE = Path(tmp)
            mod.sim_lib()
            mod.render_lib()
        finally:
            ctypes.CDLL = real
    return {"source": "arc/native.py sim_lib() and render_lib() of the reference, executed with a recording CDLL",
            "libraries": log}


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--ref", default=os.environ.get("ARC_REFERENCE"))
    a = p.parse_args()
    if not a.ref:
        sys.exit("give the reference checkout with --ref or ARC_REFERENCE")
    data = record(Path(a.ref))
    OUT.write_text(json.dumps(data, indent=1) + "\n")
    n = sum(len(v) for v in data["libraries"].values())
    print(f"wrote {OUT} ({n} declarations)")


if __name__ == "__main__":
    main()
