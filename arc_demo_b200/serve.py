"""Serving engine client and load generator (libarcsim.so arc_server_*).

The engine (csrc/arc_serve.cu) holds a fixed pool of world slots with the
task layer and one engine thread doing continuous batching. Clients open
sessions (resident batches of worlds) and submit requests that step a
session k control steps and return rewards, done flags and observations;
worlds whose episode ends are reset in place. This module wraps it and
drives it with Poisson clients:

    python -m arc_demo_b200.serve --clients 8 --rate 200 --seconds 5

Each client keeps up to four sessions open; a request steps one of them
(a new session, 1..8192 worlds log-uniform at mixed difficulty, replaces the
oldest a quarter of the time) for 1..32 control steps (uniform) with OU
actions, at exponential inter-arrival times. Reported: per-request latency
p50/p99 (submit to results), served env-steps/s, the engine's tick sizes.
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
from .task import CTaskConfig, TaskConfig

_vp, _int, _dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
_ll, _ull = ctypes.c_longlong, ctypes.c_ulonglong
_f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")

OBS = 195
# device bytes of one resident FP32 world slot at 64 x 64 columns of 0.4 m:
# record (344 floats), sphere flags (21), flags and time, a 64 x 64 terrain,
# its offset and geometry, the contact spill (4 lanes x 28 records x 8
# floats), the task layer's rows (observation and terminal observation,
# reward and flags, episode statistics, actions, task state, RNG key) and
# the engine's per-slot OU, action and result staging
WORLD_BYTES = (344 * 4 + 21 * 4 + 4 + 8 + 64 * 64 * 4 + 8 + 24 + 48 + 4 * 28 * 8 * 4
               + 2 * OBS * 4 + 4 + 3 + 16 + 4 + 12 * 4 + 143 + 4
               + 2 * 12 * 4 + 4 + 2 * 8 + 1 + 4 + 4 + 1 + 4)


@functools.cache
def serve_lib() -> ctypes.CDLL:
    lib = sim_lib()
    for name, res, args in (
        ("arc_server_create", _vp, (_int, _dbl, _int, _int, _dbl, ctypes.POINTER(CTaskConfig), _int)),
        ("arc_server_destroy", None, (_vp,)),
        ("arc_server_open", _ll, (_vp, _int, _f64, _ull)),
        ("arc_server_request", _ll, (_vp, _ll, _int, _vp, _ull, _vp, _vp, _vp)),
        ("arc_server_wait", _int, (_vp, _ll, _dbl, _vp)),
        ("arc_server_close", _int, (_vp, _ll)),
        ("arc_server_stats", _int, (_vp, _f64)),
    ):
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = list(args)
    return lib


class Server:
    """capacity world slots; dt, substeps, grid, cell as arc_sim_create;
    config the task (None: defaults, curriculum off); tick_cap the most
    worlds one tick steps (0: capacity)."""

    def __init__(self, capacity: int, dt: float = 1.0 / 30.0, substeps: int = 20, grid: int = 64,
                 cell: float = 0.4, config: TaskConfig | None = None, tick_cap: int = 0):
        self._lib = serve_lib()
        cfg = None
        if config is not None:
            self._cfg = CTaskConfig.of(config)
            cfg = ctypes.byref(self._cfg)
        self._ptr = self._lib.arc_server_create(capacity, dt, substeps, grid, cell, cfg, tick_cap)
        if not self._ptr:
            raise MemoryError("arc_server_create failed")
        self.capacity = capacity
        self._sizes = {}  # session id -> worlds
        self._outs = {}   # request id -> the arrays the engine writes into

    def open(self, difficulty, key: int = 0) -> int:
        """A session of len(difficulty) worlds; returns its id."""
        diff = np.ascontiguousarray(difficulty, dtype=np.float64)
        sid = self._lib.arc_server_open(self._ptr, len(diff), diff, key & (2**64 - 1))
        if sid < 0:
            raise RuntimeError(f"arc_server_open failed ({sid})")
        self._sizes[sid] = len(diff)
        return sid

    def request(self, session: int, steps: int, actions=None, ou_seed: int = 0, obs: bool = True) -> int:
        """Steps a session; actions (steps x n x 12) or an OU process."""
        n = self._sizes.get(session)
        if n is None:
            raise RuntimeError(f"session {session} is not open")
        act = None
        if actions is not None:
            act = np.ascontiguousarray(actions, dtype=np.float32)
            assert act.shape == (steps, n, 12)
        out = (np.empty((n, OBS), dtype=np.float32) if obs else None, np.empty((steps, n), dtype=np.float32),
               np.empty((steps, n), dtype=np.uint8))
        rid = self._lib.arc_server_request(self._ptr, session, steps, None if act is None else act.ctypes.data,
                                           ou_seed & (2**64 - 1), None if out[0] is None else out[0].ctypes.data,
                                           out[1].ctypes.data, out[2].ctypes.data)
        if rid < 0:
            raise RuntimeError(f"arc_server_request failed ({rid})")
        self._outs[rid] = out
        return rid

    def wait(self, rid: int, timeout: float = 60.0):
        """(obs, reward, done) of a request and (queued, running, total) seconds."""
        times = np.zeros(3)
        rc = self._lib.arc_server_wait(self._ptr, rid, timeout, times.ctypes.data)
        if rc == 0:
            raise TimeoutError(f"request {rid} not done after {timeout} s")
        out = self._outs.pop(rid)
        if rc < 0:
            raise RuntimeError(f"request {rid} failed ({rc})")
        return out, times

    def close_session(self, session: int) -> None:
        rc = self._lib.arc_server_close(self._ptr, session)
        if rc < 0:
            raise RuntimeError(f"arc_server_close failed ({rc})")
        self._sizes.pop(session, None)

    def stats(self) -> dict:
        s = np.zeros(12)
        err = self._lib.arc_server_stats(self._ptr, s)
        return {"ticks": int(s[0]), "world_steps": int(s[1]), "busy_s": float(s[2]),
                "max_active": int(s[3]), "completed": int(s[4]), "queued": int(s[5]),
                "admit_s": float(s[6]), "step_s": float(s[7]), "read_s": float(s[8]),
                "episodes_ended": int(s[9]), "resident": int(s[10]), "waiting_sessions": int(s[11]), "error": err}

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


def run_load(server: Server, clients: int, rate: float, seconds: float, seed: int = 0, max_worlds: int = 8192,
             max_steps: int = 32, sessions_per_client: int = 4) -> dict:
    """Poisson clients for `seconds`; waits for every request they sent and
    closes their sessions."""
    lat, lock = [], threading.Lock()
    t_start = time.perf_counter()

    def client(c: int):
        rng = np.random.default_rng(seed * 1000 + c)
        sessions, pending = [], []
        t_next = t_start
        while True:
            t_next += rng.exponential(1.0 / rate)
            if t_next - t_start > seconds:
                break
            delay = t_next - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            n, k = request_shape(rng, max_worlds, max_steps)
            if len(sessions) < sessions_per_client or rng.random() < 0.25:
                if len(sessions) >= sessions_per_client:
                    server.close_session(sessions.pop(0))
                sessions.append(server.open(rng.uniform(0.0, 1.0, n), key=int(rng.integers(2**63))))
                sid = sessions[-1]
            else:
                sid = sessions[int(rng.integers(len(sessions)))]
            pending.append((server.request(sid, k, ou_seed=int(rng.integers(2**63)), obs=True), sid, k))
        for rid, sid, k in pending:
            _, times = server.wait(rid, timeout=600.0)
            with lock:
                lat.append(times[2])
        for sid in sessions:
            server.close_session(sid)

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
        "env_steps": int(steps),
        "wall_s": wall,
        "env_steps_per_s": steps / wall,
        "engine_env_steps_per_s_busy": steps / busy if busy > 0 else 0.0,
        "latency_ms": {"p50": float(np.percentile(lat_ms, 50)), "p99": float(np.percentile(lat_ms, 99)),
                       "max": float(lat_ms.max())} if len(lat) else None,
        "ticks": ticks,
        "busy_split_s": {k: round(stats[k] - stats0[k], 3) for k in ("admit_s", "step_s", "read_s")},
        "mean_worlds_per_tick": steps / ticks if ticks else 0.0,
        "max_worlds_per_tick": stats["max_active"],
        "episodes_ended": stats["episodes_ended"] - stats0["episodes_ended"],
    }


def main() -> None:
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--clients", type=int, default=8)
    p.add_argument("--rate", type=float, default=200.0, help="requests/s per client")
    p.add_argument("--seconds", type=float, default=5.0)
    p.add_argument("--capacity", type=int, default=0, help="world slots (0: from --budget-gb)")
    p.add_argument("--budget-gb", type=float, default=40.0, help="device bytes for resident worlds")
    p.add_argument("--tick-cap", type=int, default=131072, help="most worlds one tick steps")
    p.add_argument("--max-worlds", type=int, default=8192)
    p.add_argument("--max-steps", type=int, default=32)
    a = p.parse_args()
    capacity = a.capacity or int(a.budget_gb * 1e9 // WORLD_BYTES)
    with Server(capacity, tick_cap=a.tick_cap) as sv:
        # warm the kernels and the engine once
        sid = sv.open(np.zeros(64))
        sv.wait(sv.request(sid, 2))
        sv.close_session(sid)
        out = run_load(sv, a.clients, a.rate, a.seconds, max_worlds=a.max_worlds, max_steps=a.max_steps)
    out.update({"clients": a.clients, "rate_per_client": a.rate, "capacity": capacity, "tick_cap": a.tick_cap,
                "bytes_per_world": WORLD_BYTES})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
