"""Serving: a request loop over device-resident complex64 states.

Requests (a Circuit plus "all <Z_i>" or "k shots") are admitted while others
run, as lanes (CUDA streams) and the HBM budget (2^n x 8 B per state) free up;
see nqpu_b200/csrc/server.cpp for the admission and scheduling rules.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import NqpuServerConfig, check
from .state import Circuit

KINDS = {"zall": 0, "shots": 1}


class Server:
    def __init__(self, hbm_budget_bytes: int = 0, max_qubits: int = 28, lanes: int = 16, large_lanes: int = 2,
                 large_qubits: int = 22, max_shots: int = 1024):
        self.lib = _lib.load()
        cfg = NqpuServerConfig(int(hbm_budget_bytes), int(max_qubits), int(lanes), int(large_lanes),
                               int(large_qubits), int(max_shots))
        self.h_ = self.lib.nqpu_server_create(C.byref(cfg))
        if not self.h_:
            raise RuntimeError("nqpu_server_create failed (no CUDA device, bad config or budget too small)")
        self.meta: dict[int, tuple[str, int, int]] = {}

    def close(self):
        if getattr(self, "h_", None):
            self.lib.nqpu_server_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, circuit: Circuit, kind: str = "zall", shots: int = 0, seed: int = 0) -> int:
        rid = C.c_uint64()
        check(self.lib.nqpu_server_submit(self.h_, circuit.h_, KINDS[kind], int(shots), int(seed), C.byref(rid)),
              "server_submit")
        self.meta[rid.value] = (kind, circuit.num_qubits, int(shots))
        return int(rid.value)

    def poll(self, rid: int) -> bool:
        done = C.c_int32()
        check(self.lib.nqpu_server_poll(self.h_, rid, C.byref(done)), "server_poll")
        return bool(done.value)

    def wait(self, rid: int = 0, timeout_s: float = 0.0):
        check(self.lib.nqpu_server_wait(self.h_, rid, float(timeout_s)), "server_wait")

    def cancel(self, rid: int) -> bool:
        """Withdraw a queued request: True when it was still queued (it never
        runs and its id is forgotten), False when it was already admitted."""
        err = self.lib.nqpu_server_cancel(self.h_, rid)
        if err == 2:  # NQPU_INVALID_PARAMETER: already running or finished
            return False
        check(err, "server_cancel")
        self.meta.pop(rid, None)
        return True

    def result(self, rid: int):
        """(values, timing) for a finished request: values = <Z_i> array (zall) or
        outcome array (shots); timing = {queued_ms, running_ms, total_ms}."""
        kind, n, shots = self.meta.pop(rid)
        t = (C.c_double * 3)()
        if kind == "zall":
            z = np.empty(n, dtype=np.float64)
            check(self.lib.nqpu_server_result(self.h_, rid, z.ctypes.data_as(C.POINTER(C.c_double)), n, None, 0, t),
                  "server_result")
            vals = z
        else:
            o = np.empty(shots, dtype=np.uint64)
            check(self.lib.nqpu_server_result(self.h_, rid, None, 0, o.ctypes.data_as(C.POINTER(C.c_uint64)), shots,
                                              t), "server_result")
            vals = o
        return vals, {"queued_ms": t[0], "running_ms": t[1], "total_ms": t[2]}

    def stats(self) -> dict:
        out = (C.c_uint64 * 9)()
        check(self.lib.nqpu_server_stats(self.h_, out, 9), "server_stats")
        keys = ("submitted", "completed", "failed", "running", "queued", "peak_resident_bytes", "arena_bytes",
                "peak_concurrent", "cancelled")
        return {k: int(v) for k, v in zip(keys, out)}
