"""Batched execution: many circuits of different sizes in one persistent,
graph-captured launch, each returning <H> of its own 1D Ising Hamiltonian
H = sum_i J_i Z_i Z_{i+1} + sum_i h_i X_i (complex64 states, FP64 reductions)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check
from .state import Circuit

PARAMS = {"small_max_qubits": 0, "tile_qubits": 1, "queue_order": 2, "ctas_per_sm": 3, "spin_limit": 4,
          "drop_tile": 5}


class Batch:
    def __init__(self):
        self.lib = _lib.load()
        self.h_ = self.lib.nqpu_batch_create()
        if not self.h_:
            raise RuntimeError("nqpu_batch_create failed (no CUDA device)")
        self.count = 0

    def close(self):
        if getattr(self, "h_", None):
            self.lib.nqpu_batch_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_ising(self, circuit: Circuit, J, h) -> int:
        J = np.ascontiguousarray(np.asarray(J, dtype=np.float64))
        h = np.ascontiguousarray(np.asarray(h, dtype=np.float64))
        idx = C.c_uint32()
        check(self.lib.nqpu_batch_add_ising(self.h_, circuit.h_, J.ctypes.data_as(C.POINTER(C.c_double)),
                                            h.ctypes.data_as(C.POINTER(C.c_double)), C.byref(idx)), "batch_add")
        self.count += 1
        return int(idx.value)

    def config(self, **kw):
        for k, v in kw.items():
            check(self.lib.nqpu_batch_config(self.h_, PARAMS[k], int(v)), f"batch_config {k}")

    def prepare(self):
        check(self.lib.nqpu_batch_prepare(self.h_), "batch_prepare")

    def run(self) -> np.ndarray:
        out = np.empty(self.count, dtype=np.float64)
        check(self.lib.nqpu_batch_run(self.h_, out.ctypes.data_as(C.POINTER(C.c_double)), self.count), "batch_run")
        return out

    def last_run_ms(self) -> float:
        """Device time of the last run() (CUDA events around the graph replay)."""
        ms = C.c_float()
        check(self.lib.nqpu_batch_last_run_ms(self.h_, C.byref(ms)), "batch_last_run_ms")
        return float(ms.value)

    def stats(self) -> dict:
        out = (C.c_uint64 * 6)()
        check(self.lib.nqpu_batch_stats(self.h_, out, 6), "batch_stats")
        return {"circuits": out[0], "small": out[1], "tasks": out[2], "arena_bytes": out[3], "passes": out[4],
                "upload_bytes": out[5]}


def ising_terms(n, J, h):
    """Pauli-sum form of H (character q acts on qubit q) for the per-circuit path."""
    terms = []
    for i in range(n - 1):
        s = ["I"] * n
        s[i] = s[i + 1] = "Z"
        terms.append((float(J[i]), "".join(s)))
    for i in range(n):
        s = ["I"] * n
        s[i] = "X"
        terms.append((float(h[i]), "".join(s)))
    return terms
