"""Serving engine client and load generator (libarcsim.so arc_server_*).

The engine (csrc/arc_serve.cu) holds a fixed pool of world slots and one
engine thread doing continuous batching; this module wraps it and drives it
with Poisson clients:

    python -m arc_demo_b200.serve --clients 8 --rate 200 --seconds 5

Each client submits requests at exponential inter-arrival times; a request
is 1..8192 worlds (log-uniform) for 1..32 control steps (uniform), mixed
difficulty, OU actions. Reported: per-request latency p50/p99 (submit to
results), the engine's aggregate env-steps/s, and how full the ticks were.
"""

from __future__ import annotations

import argparse
import ctypes
import functools
import json
import math
import threading
import time

import numpy as np

from .native import sim_lib

_vp, _int, _dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
_ll, _ull = ctypes.c_longlong, ctypes.c_ulonglong
_f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")

STATE_SIZE = 387  # arc_sim_state_size of the quadruped
OBS_ROW = 65      # root 13, rot 9, joints 36, contacts 6, flag 1 (arc_sim_observe blocks)
RESULTS = {"state": (0, STATE_SIZE), "observe": (1, OBS_ROW)}
# device bytes of one resident FP32 world slot at 64 x 64 columns of 0.4 m:
# record (344 floats), sphere flags (21), flags and time, a 64 x 64 terrain,
# its offset and geometry, the contact spill (4 lanes x 28 records x 8
# floats) and the engine's per-slot action, OU and seed arrays
WORLD_BYTES = (344 * 4 + 21 * 4 + 4 + 8 + 64 * 64 * 4 + 8 + 24 + 48 + 4 + 4 * 28 * 8 * 4
               + 3 * 12 * 4 + 4 + 8 + 4 + 1)


@functools.cache
def serve_lib() -> ctypes.CDLL:
    lib = sim_lib()
    for name, res, args in (
        ("arc_server_create", _vp, (_int, _dbl, _int, _int, _dbl, _int)),
        ("arc_server_destroy", None, (_vp,)),
        ("arc_server_submit", _ll, (_vp, _int, _int, _u32, _f64, _vp, _ull, _vp)),
        ("arc_server_wait", _int, (_vp, _ll, _dbl, _vp, _vp)),
        ("arc_server_stats", _int, (_vp, _f64)),
    ):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)
    return lib


class Server:
    """capacity world slots; dt, substeps, grid, cell as arc_sim_create;
    result "state" (each world's final state, 387 doubles) or "observe" (its
    final observation row, 65 doubles)."""

    def __init__(self, capacity: int, dt: float = 1.0 / 30.0, substeps: int = 20, grid: int = 64,
                 cell: float = 0.4, result: str = "state"):
        self._lib = serve_lib()
        kind, self.row = RESULTS[result]
        self._ptr = self._lib.arc_server_create(capacity, dt, substeps, grid, cell, kind)
        if not self._ptr:
            raise MemoryError("arc_server_create failed")
        self.capacity = capacity
        self._outs = {}  # request id -> the array the engine writes the final states into

    def submit(self, seeds, difficulty, steps: int, actions=None, ou_seed: int = 0) -> int:
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        diff = np.ascontiguousarray(difficulty, dtype=np.float64)
        act = None
        if actions is not None:
            act = np.ascontiguousarray(actions, dtype=np.float32)
            assert act.shape == (steps, len(seeds), 12)
        out = np.empty((len(seeds), self.row))
        rid = self._lib.arc_server_submit(self._ptr, len(seeds), steps, seeds, diff,
                                          None if act is None else act.ctypes.data, ou_seed, out.ctypes.data)
        if rid < 0:
            raise RuntimeError(f"arc_server_submit failed ({rid})")
        self._outs[rid] = out
        return rid

    def wait(self, rid: int, timeout: float = 60.0):
        """Results (n_worlds x row) and (queued, running, total) seconds."""
        times = np.zeros(3)
        rc = self._lib.arc_server_wait(self._ptr, rid, timeout, None, times.ctypes.data)
        if rc == 0:
            raise TimeoutError(f"request {rid} not done after {timeout} s")
        out = self._outs.pop(rid)
        if rc < 0:
            raise RuntimeError(f"request {rid} failed ({rc})")
        return out, times

    def stats(self) -> dict:
        s = np.zeros(9)
        err = self._lib.arc_server_stats(self._ptr, s)
        return {"ticks": int(s[0]), "world_steps": int(s[1]), "busy_s": float(s[2]),
                "max_active": int(s[3]), "completed": int(s[4]), "queued": int(s[5]),
                "admit_s": float(s[6]), "step_s": float(s[7]), "evict_s": float(s[8]), "error": err}

    def close(self) -> None:
        if getattr(self, "_ptr", None):
            self._lib.arc_server_destroy(self._ptr)
            self._ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        self.close()


def request_shape(rng: np.random.Generator, max_worlds: int = 8192, max_steps: int = 32):
    n = int(math.exp(rng.uniform(0.0, math.log(max_worlds + 1))))
    return max(1, min(n, max_worlds)), int(rng.integers(1, max_steps + 1))


def run_load(server: Server, clients: int, rate: float, seconds: float, seed: int = 0,
             max_worlds: int = 8192, max_steps: int = 32) -> dict:
    """Poisson clients for `seconds`; waits for every request they sent."""
    lat, done_steps, lock = [], [0], threading.Lock()
    t_start = time.perf_counter()

    def client(c: int):
        rng = np.random.default_rng(seed * 1000 + c)
        pending = []
        t_next = t_start
        while True:
            t_next += rng.exponential(1.0 / rate)
            if t_next - t_start > seconds:
                break
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            n, k = request_shape(rng, max_worlds, max_steps)
            seeds = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
            diff = rng.uniform(0.0, 1.0, n)
            pending.append((server.submit(seeds, diff, k, ou_seed=int(rng.integers(2**63))), n, k))
        for rid, n, k in pending:
            _, times = server.wait(rid, timeout=600.0)
            with lock:
                lat.append(times[2])
                done_steps[0] += n * k

    stats0 = server.stats()
    threads = [threading.Thread(target=client, args=(c,)) for c in range(clients)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t_start
    stats = server.stats()
    ticks = stats["ticks"] - stats0["ticks"]
    steps = stats["world_steps"] - stats0["world_steps"]
    busy = stats["busy_s"] - stats0["busy_s"]
    lat_ms = np.array(lat) * 1e3
    return {
        "requests": len(lat),
        "env_steps": int(done_steps[0]),
        "wall_s": wall,
        "env_steps_per_s": done_steps[0] / wall,
        "engine_env_steps_per_s_busy": steps / busy if busy > 0 else 0.0,
        "latency_ms": {"p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                       "max": float(lat_ms.max())} if len(lat) else None,
        "ticks": ticks,
        "busy_split_s": {k: round(stats[k] - stats0[k], 3) for k in ("admit_s", "step_s", "evict_s")},
        "mean_worlds_per_tick": steps / ticks if ticks else 0.0,
        "max_worlds_per_tick": stats["max_active"],
    }


def main() -> None:
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--clients", type=int, default=8)
    p.add_argument("--rate", type=float, default=200.0, help="requests/s per client")
    p.add_argument("--seconds", type=float, default=5.0)
    p.add_argument("--capacity", type=int, default=0, help="world slots (0: from --budget-gb)")
    p.add_argument("--budget-gb", type=float, default=40.0, help="device bytes for resident worlds")
    p.add_argument("--max-worlds", type=int, default=8192)
    p.add_argument("--max-steps", type=int, default=32)
    p.add_argument("--result", choices=sorted(RESULTS), default="observe")
    a = p.parse_args()
    capacity = a.capacity or int(a.budget_gb * 1e9 // WORLD_BYTES)
    with Server(capacity, result=a.result) as sv:
        # warm the kernels and the engine once
        rid = sv.submit(np.arange(64, dtype=np.uint32), np.zeros(64), 2)
        sv.wait(rid)
        out = run_load(sv, a.clients, a.rate, a.seconds, max_worlds=a.max_worlds, max_steps=a.max_steps)
    out.update({"clients": a.clients, "rate_per_client": a.rate, "capacity": capacity, "result": a.result,
                "bytes_per_world": WORLD_BYTES})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
