"""ORACLE — test infrastructure only.

ctypes loader of the CPU restatement (oracle.cpp) of the reference's statevector
path.  Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg
as the checker / reported baseline; never by the engine.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_lib = None


def lib():
    global _lib
    if _lib is None:
        so = HERE / "_build" / "liboracle.so"
        if not so.exists():
            import importlib.util
            spec = importlib.util.spec_from_file_location("oracle_build", HERE / "build.py")
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        L = C.CDLL(str(so))
        vp, d, u64, i = C.c_void_p, C.c_double, C.c_uint64, C.c_int
        pd = C.POINTER(C.c_double)
        sig = {
            "oracle_set_threads": (None, [i]), "oracle_max_threads": (i, []),
            "oracle_state_new": (vp, [i, i]), "oracle_state_free": (None, [vp]),
            "oracle_state_set_basis": (None, [vp, u64]), "oracle_state_get": (None, [vp, pd]),
            "oracle_state_set": (None, [vp, pd]), "oracle_apply_flat": (None, [vp, pd, i]),
            "oracle_reset_qubit": (None, [vp, i]),
            "oracle_expectation_z_all": (None, [vp, pd]), "oracle_expectation_x": (d, [vp, i]),
            "oracle_expectation_y": (d, [vp, i]), "oracle_pauli_string": (d, [vp, C.c_char_p, i]),
            "oracle_norm": (d, [vp]), "oracle_fidelity": (d, [vp, vp]),
            "oracle_probabilities": (None, [vp, pd]),
            "oracle_sample_uniforms": (None, [vp, pd, i, C.POINTER(C.c_uint64)]),
            "oracle_set_seed": (None, [u64]), "oracle_next_random": (d, []),
            "oracle_take_outcomes": (C.c_int, [C.POINTER(C.c_uint32), C.c_int]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class OracleState:
    def __init__(self, n: int, f32: bool = False):
        self.L = lib()
        self.n = n
        self.h = self.L.oracle_state_new(n, 1 if f32 else 0)

    def __del__(self):
        if getattr(self, "h", None):
            self.L.oracle_state_free(self.h)
            self.h = None

    def set_basis(self, idx: int):
        self.L.oracle_state_set_basis(self.h, idx)

    def apply(self, gates):
        from nqpu_b200.circuits import flatten
        flat = np.ascontiguousarray(flatten(gates))
        if len(flat):
            self.L.oracle_apply_flat(self.h, flat.ctypes.data_as(C.POINTER(C.c_double)), len(flat))

    def amplitudes(self) -> np.ndarray:
        out = np.empty(2 << self.n, dtype=np.float64)
        self.L.oracle_state_get(self.h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.view(np.complex128)

    def set_amplitudes(self, arr):
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.complex128)).view(np.float64)
        self.L.oracle_state_set(self.h, a.ctypes.data_as(C.POINTER(C.c_double)))

    def take_outcomes(self, max_count: int = 4096) -> np.ndarray:
        """Outcomes of the 'measure' gates applied since the last call (xorshift64*
        draws from the seed set by set_seed)."""
        out = (C.c_uint32 * max_count)()
        k = self.L.oracle_take_outcomes(out, max_count)
        return np.array(out[:k], dtype=np.uint32)

    def reset_qubit(self, q):
        self.L.oracle_reset_qubit(self.h, q)

    def expectation_z_all(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        self.L.oracle_expectation_z_all(self.h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def expectation_x(self, q):
        return self.L.oracle_expectation_x(self.h, q)

    def expectation_y(self, q):
        return self.L.oracle_expectation_y(self.h, q)

    def pauli_string(self, s: str):
        return self.L.oracle_pauli_string(self.h, s.encode(), len(s))

    def norm(self):
        return self.L.oracle_norm(self.h)

    def fidelity(self, other: "OracleState"):
        return self.L.oracle_fidelity(self.h, other.h)

    def probabilities(self):
        out = np.empty(1 << self.n, dtype=np.float64)
        self.L.oracle_probabilities(self.h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def sample_uniforms(self, u):
        u = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        self.L.oracle_sample_uniforms(self.h, u.ctypes.data_as(C.POINTER(C.c_double)), u.size,
                                      out.ctypes.data_as(C.POINTER(C.c_uint64)))
        return out


def xorshift_uniforms(seed: int, count: int) -> np.ndarray:
    """The reference C FFI's thread-local xorshift64* stream after nqpu_set_seed(seed)."""
    L = lib()
    L.oracle_set_seed(seed)
    return np.array([L.oracle_next_random() for _ in range(count)])


def set_seed(seed: int):
    """Seed the oracle's xorshift64* stream (the draws its 'measure' gates use)."""
    lib().oracle_set_seed(int(seed))


def set_threads(t: int):
    lib().oracle_set_threads(t)


def max_threads() -> int:
    return lib().oracle_max_threads()
