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

    def add_ising_arrays(self, items) -> int:
        """Add many circuits in one nqpu_batch_add_ising_arrays call.  items:
        (n, (codes [G], qubits [G, 3], params [G, 4]), J [n-1], h [n]) per
        circuit, the gate arrays in the encoding of Circuit.from_arrays (no
        custom-matrix gates).  Returns the index of the first circuit."""
        items = list(items)
        if not items:
            return self.count
        nq = np.array([it[0] for it in items], dtype=np.uint32)
        counts = np.array([len(it[1][0]) for it in items], dtype=np.uint64)
        offs = np.zeros(len(items) + 1, dtype=np.uint64)
        np.cumsum(counts, out=offs[1:])
        codes = np.ascontiguousarray(np.concatenate([np.asarray(it[1][0], dtype=np.uint32) for it in items]))
        qubits = np.ascontiguousarray(np.concatenate([np.asarray(it[1][1], dtype=np.int32).reshape(-1, 3)
                                                      for it in items]))
        params = np.ascontiguousarray(np.concatenate([np.asarray(it[1][2], dtype=np.float64).reshape(-1, 4)
                                                      for it in items]))
        J = np.ascontiguousarray(np.concatenate([np.asarray(it[2], dtype=np.float64) for it in items]))
        h = np.ascontiguousarray(np.concatenate([np.asarray(it[3], dtype=np.float64) for it in items]))
        first = C.c_uint32()
        check(self.lib.nqpu_batch_add_ising_arrays(
            self.h_, len(items), nq.ctypes.data_as(C.POINTER(C.c_uint32)), offs.ctypes.data_as(C.POINTER(C.c_uint64)),
            codes.ctypes.data_as(C.POINTER(C.c_uint32)), qubits.ctypes.data_as(C.POINTER(C.c_int32)),
            params.ctypes.data_as(C.POINTER(C.c_double)), None, J.ctypes.data_as(C.POINTER(C.c_double)),
            h.ctypes.data_as(C.POINTER(C.c_double)), C.byref(first)), "batch_add_arrays")
        self.count += len(items)
        return int(first.value)

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
        out = (C.c_uint64 * 10)()
        check(self.lib.nqpu_batch_stats(self.h_, out, 10), "batch_stats")
        return {"circuits": out[0], "small": out[1], "tasks": out[2], "arena_bytes": out[3], "passes": out[4],
                "upload_bytes": out[5],
                "prepare_s": {"plans": out[6] / 1e6, "pack": out[7] / 1e6, "alloc_upload": out[8] / 1e6,
                              "capture": out[9] / 1e6}}


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
