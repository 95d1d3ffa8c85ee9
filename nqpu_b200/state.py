"""Python mirror of the reference's statevector interface over the C ABI.

`StateVector` follows QuantumState + GateOperations (sdk/rust/src/lib.rs:326-1735)
and the C FFI state/gate/measure calls (c_ffi.rs:789-1250); `Circuit` follows the
C FFI circuit API (c_ffi.rs:1259-1400) extended to every GateType.  All work runs
in the CUDA library; the Python layer only marshals arguments.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import NqpuComplex, NqpuMeasurement, check
from .circuits import ARITY, MID_GATES, NPARAMS

C128, C64 = 0, 1
MODES = {"tiled": 0, "pergate": 1, "fused": 2, "tensor": 3, "auto": 4}
DTYPES = {"c128": C128, "complex128": C128, "c64": C64, "complex64": C64}


def _cmat(m, size):
    arr = np.asarray(m, dtype=np.complex128).reshape(-1)
    if arr.size != size:
        raise ValueError(f"matrix needs {size} entries")
    buf = (NqpuComplex * size)()
    for i, v in enumerate(arr):
        buf[i].re = float(v.real)
        buf[i].im = float(v.imag)
    return buf


_GATE_FN = {
    "h": "nqpu_gate_h", "x": "nqpu_gate_x", "y": "nqpu_gate_y", "z": "nqpu_gate_z",
    "s": "nqpu_gate_s", "t": "nqpu_gate_t", "sx": "nqpu_gate_sx", "rx": "nqpu_gate_rx",
    "ry": "nqpu_gate_ry", "rz": "nqpu_gate_rz", "p": "nqpu_gate_phase", "u3": "nqpu_gate_u3",
    "cx": "nqpu_gate_cx", "cz": "nqpu_gate_cz", "swap": "nqpu_gate_swap", "iswap": "nqpu_gate_iswap",
    "cp": "nqpu_gate_cphase", "crx": "nqpu_gate_crx", "cry": "nqpu_gate_cry", "crz": "nqpu_gate_crz",
    "rzz": "nqpu_gate_rzz", "rxx": "nqpu_gate_rxx", "ryy": "nqpu_gate_ryy", "ccx": "nqpu_gate_toffoli",
    "ccz": "nqpu_gate_ccz", "cswap": "nqpu_gate_cswap", "cu": "nqpu_gate_cu",
}
_CIRC_FN = {
    "h": "nqpu_circuit_add_h", "x": "nqpu_circuit_add_x", "y": "nqpu_circuit_add_y",
    "z": "nqpu_circuit_add_z", "s": "nqpu_circuit_add_s", "t": "nqpu_circuit_add_t",
    "sx": "nqpu_circuit_add_sx", "rx": "nqpu_circuit_add_rx", "ry": "nqpu_circuit_add_ry",
    "rz": "nqpu_circuit_add_rz", "p": "nqpu_circuit_add_phase", "u3": "nqpu_circuit_add_u3",
    "cx": "nqpu_circuit_add_cx", "cz": "nqpu_circuit_add_cz", "swap": "nqpu_circuit_add_swap",
    "iswap": "nqpu_circuit_add_iswap", "cp": "nqpu_circuit_add_cphase", "crx": "nqpu_circuit_add_crx",
    "cry": "nqpu_circuit_add_cry", "crz": "nqpu_circuit_add_crz", "rzz": "nqpu_circuit_add_rzz",
    "rxx": "nqpu_circuit_add_rxx", "ryy": "nqpu_circuit_add_ryy", "ccx": "nqpu_circuit_add_toffoli",
    "ccz": "nqpu_circuit_add_ccz", "cswap": "nqpu_circuit_add_cswap", "cu": "nqpu_circuit_add_cu",
    "measure": "nqpu_circuit_add_measure", "reset": "nqpu_circuit_add_reset",
}


class StateVector:
    """Device-resident statevector (complex128 by default, like QuantumState)."""

    def __init__(self, num_qubits: int, dtype: str = "c128"):
        self.lib = _lib.load()
        self.num_qubits = int(num_qubits)
        self.dtype = DTYPES[dtype]
        self.h_ = self.lib.nqpu_state_create_ex(self.num_qubits, self.dtype)
        if not self.h_:
            raise MemoryError(f"nqpu_state_create_ex({num_qubits}) failed (no CUDA device or out of memory)")

    @classmethod
    def _wrap(cls, lib, handle, n, dtype):
        obj = cls.__new__(cls)
        obj.lib, obj.h_, obj.num_qubits, obj.dtype = lib, handle, n, dtype
        return obj

    def close(self):
        if getattr(self, "h_", None):
            self.lib.nqpu_state_destroy(self.h_)
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

    @property
    def dim(self) -> int:
        return 1 << self.num_qubits

    # ---- state management ----
    def clone(self) -> "StateVector":
        h = self.lib.nqpu_state_clone(self.h_)
        if not h:
            raise MemoryError("nqpu_state_clone failed")
        return StateVector._wrap(self.lib, h, self.num_qubits, self.dtype)

    def reset(self):
        check(self.lib.nqpu_state_reset(self.h_), "reset")

    def set_basis(self, index: int):
        check(self.lib.nqpu_state_set_basis(self.h_, int(index)), "set_basis")

    def synchronize(self):
        check(self.lib.nqpu_state_synchronize(self.h_), "synchronize")

    def amplitude(self, index: int) -> complex:
        out = NqpuComplex()
        check(self.lib.nqpu_state_get_amplitude(self.h_, int(index), C.byref(out)), "get_amplitude")
        return complex(out.re, out.im)

    def set_amplitude(self, index: int, value: complex):
        check(self.lib.nqpu_state_set_amplitude(self.h_, int(index), NqpuComplex(value.real, value.imag)),
              "set_amplitude")

    def amplitudes(self) -> np.ndarray:
        out = np.empty(self.dim, dtype=np.complex128)
        check(self.lib.nqpu_state_get_amplitudes(self.h_, out.ctypes.data_as(C.POINTER(NqpuComplex)), self.dim),
              "get_amplitudes")
        return out

    def set_amplitudes(self, arr):
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.complex128).reshape(-1))
        check(self.lib.nqpu_state_set_amplitudes(self.h_, a.ctypes.data_as(C.POINTER(NqpuComplex)), a.size),
              "set_amplitudes")

    def probabilities(self) -> np.ndarray:
        out = np.empty(self.dim, dtype=np.float64)
        check(self.lib.nqpu_state_probabilities(self.h_, out.ctypes.data_as(C.POINTER(C.c_double)), self.dim),
              "probabilities")
        return out

    def norm(self) -> float:
        return float(self.lib.nqpu_state_norm(self.h_))

    def renormalize(self):
        check(self.lib.nqpu_state_renormalize(self.h_), "renormalize")

    # ---- gates (one kernel per gate) ----
    def apply(self, name: str, qubits, params=(), matrix=None):
        qs = [int(q) for q in qubits]
        if name == "custom1":
            return check(self.lib.nqpu_gate_custom_1q(self.h_, qs[0], _cmat(matrix, 4)), name)
        if name == "custom2":
            return check(self.lib.nqpu_gate_custom_2q(self.h_, qs[0], qs[1], _cmat(matrix, 16)), name)
        if name == "u2lo":
            return check(self.lib.nqpu_gate_u2(self.h_, qs[0], qs[1], _cmat(matrix, 16)), name)
        fn = getattr(self.lib, _GATE_FN[name])
        ps = [float(p) for p in tuple(params)[:NPARAMS[name]]]
        if len(ps) != NPARAMS[name]:
            raise ValueError(f"{name} takes {NPARAMS[name]} parameters")
        check(fn(self.h_, *qs, *ps), name)

    def apply_gates(self, gates):
        for g in gates:
            self.apply(g[0], g[1], g[2] if len(g) > 2 else (), g[3] if len(g) > 3 else None)

    def reset_qubit(self, q: int):
        check(self.lib.nqpu_gate_reset_qubit(self.h_, int(q)), "reset_qubit")

    # ---- reductions ----
    def expectation_z(self, q: int) -> float:
        out = C.c_double()
        check(self.lib.nqpu_expectation_z(self.h_, int(q), C.byref(out)), "expectation_z")
        return out.value

    def expectation_z_all(self) -> np.ndarray:
        out = np.empty(self.num_qubits, dtype=np.float64)
        check(self.lib.nqpu_expectation_z_all(self.h_, out.ctypes.data_as(C.POINTER(C.c_double)),
                                              self.num_qubits), "expectation_z_all")
        return out

    def expectation_x(self, q: int) -> float:
        out = C.c_double()
        check(self.lib.nqpu_expectation_x(self.h_, int(q), C.byref(out)), "expectation_x")
        return out.value

    def expectation_y(self, q: int) -> float:
        out = C.c_double()
        check(self.lib.nqpu_expectation_y(self.h_, int(q), C.byref(out)), "expectation_y")
        return out.value

    def expectation_pauli_sum(self, terms) -> float:
        """terms: list of (coeff, pauli_string of length n; char q acts on qubit q)."""
        n = self.num_qubits
        strs = b"".join(s.encode() for _, s in terms)
        if any(len(s) != n for _, s in terms):
            raise ValueError("each Pauli string needs one character per qubit")
        coeffs = (C.c_double * max(1, len(terms)))(*[float(c) for c, _ in terms])
        out = C.c_double()
        check(self.lib.nqpu_expectation_pauli_sum(self.h_, strs, coeffs, len(terms), C.byref(out)),
              "expectation_pauli_sum")
        return out.value

    def expectation_pauli_string(self, s: str) -> float:
        return self.expectation_pauli_sum([(1.0, s)])

    def fidelity(self, other: "StateVector") -> float:
        out = C.c_double()
        check(self.lib.nqpu_fidelity(self.h_, other.h_, C.byref(out)), "fidelity")
        return out.value

    def sample(self, shots: int) -> np.ndarray:
        out = np.empty(shots, dtype=np.uint64)
        check(self.lib.nqpu_sample(self.h_, int(shots), out.ctypes.data_as(C.POINTER(C.c_uint64))), "sample")
        return out

    def sample_with_uniforms(self, u) -> np.ndarray:
        u = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
        out = np.empty(u.size, dtype=np.uint64)
        check(self.lib.nqpu_sample_with_uniforms(self.h_, u.ctypes.data_as(C.POINTER(C.c_double)), u.size,
                                                 out.ctypes.data_as(C.POINTER(C.c_uint64))), "sample")
        return out

    def measure(self, q: int):
        m = NqpuMeasurement()
        check(self.lib.nqpu_measure(self.h_, int(q), C.byref(m)), "measure")
        return int(m.outcome), float(m.probability)

    def measure_all(self):
        out = (C.c_uint32 * self.num_qubits)()
        check(self.lib.nqpu_measure_all(self.h_, out, self.num_qubits), "measure_all")
        return [int(v) for v in out]


class Circuit:
    """Circuit handle (nqpu_circuit_*); `execute` runs it on a StateVector."""

    def __init__(self, num_qubits: int, gates=None, extended: bool = True):
        self.lib = _lib.load()
        self.num_qubits = int(num_qubits)
        create = self.lib.nqpu_circuit_create_ex if extended else self.lib.nqpu_circuit_create
        self.h_ = create(self.num_qubits)
        if not self.h_:
            raise ValueError(f"nqpu_circuit_create({num_qubits}) failed")
        if gates:
            self.extend(gates)

    @classmethod
    def from_arrays(cls, num_qubits: int, codes, qubits, params, matrices=None) -> "Circuit":
        """Circuit from flat arrays in one nqpu_circuit_add_gates call: codes [G]
        (circuits.GATE_CODES), qubits [G, 3], params [G, 4], matrices [G, 16]
        complex (custom gates only) or None."""
        c = cls(num_qubits)
        ca = np.ascontiguousarray(codes, dtype=np.uint32)
        qa = np.ascontiguousarray(qubits, dtype=np.int32).reshape(-1, 3)
        pa = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, 4)
        if not (len(ca) == len(qa) == len(pa)):
            raise ValueError("codes, qubits and params differ in length")
        ma = None
        if matrices is not None:
            ma = np.ascontiguousarray(matrices, dtype=np.complex128).reshape(-1, 16)
            if len(ma) != len(ca):
                raise ValueError("matrices differ in length")
        mp = ma.ctypes.data_as(C.POINTER(NqpuComplex)) if ma is not None else None
        check(c.lib.nqpu_circuit_add_gates(c.h_, ca.ctypes.data_as(C.POINTER(C.c_uint32)),
                                           qa.ctypes.data_as(C.POINTER(C.c_int32)),
                                           pa.ctypes.data_as(C.POINTER(C.c_double)), mp, len(ca)),
              "circuit_add_gates")
        return c

    def close(self):
        if getattr(self, "h_", None):
            self.lib.nqpu_circuit_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, name: str, qubits, params=(), matrix=None):
        qs = [int(q) for q in qubits]
        if name in MID_GATES:
            if len(qs) != 1:
                raise ValueError(f"{name} takes 1 qubit")
            return check(getattr(self.lib, _CIRC_FN[name])(self.h_, qs[0]), name)
        if len(qs) != ARITY[name]:
            raise ValueError(f"{name} takes {ARITY[name]} qubits")
        if name == "custom1":
            return check(self.lib.nqpu_circuit_add_custom_1q(self.h_, qs[0], _cmat(matrix, 4)), name)
        if name == "custom2":
            return check(self.lib.nqpu_circuit_add_custom_2q(self.h_, qs[0], qs[1], _cmat(matrix, 16)), name)
        fn = getattr(self.lib, _CIRC_FN[name])
        ps = [float(p) for p in tuple(params)[:NPARAMS[name]]]
        if len(ps) != NPARAMS[name]:
            raise ValueError(f"{name} takes {NPARAMS[name]} parameters")
        check(fn(self.h_, *qs, *ps), name)

    def extend(self, gates):
        """Append a gate list with one nqpu_circuit_add_gates call."""
        from .circuits import GATE_CODES
        gates = gates if isinstance(gates, list) else list(gates)
        m = len(gates)
        if m == 0:
            return
        names = [g[0] for g in gates]
        codes = np.fromiter(map(GATE_CODES.__getitem__, names), dtype=np.uint32, count=m)
        qls = [g[1] for g in gates]
        qlen = np.fromiter(map(len, qls), dtype=np.int64, count=m)
        ar = np.fromiter((1 if n in MID_GATES else ARITY[n] for n in names), dtype=np.int64, count=m)
        bad = np.nonzero(qlen != ar)[0]
        if bad.size:
            i = int(bad[0])
            raise ValueError(f"{names[i]} takes {ar[i]} qubits")
        qa = np.zeros((m, 3), dtype=np.int32)
        for k in (1, 2, 3):
            idx = np.nonzero(ar == k)[0]
            if idx.size:
                qa[idx, :k] = np.array([qls[i] for i in idx], dtype=np.int64).reshape(-1, k)
        npar = np.fromiter(map(NPARAMS.__getitem__, names), dtype=np.int64, count=m)
        pa = np.zeros((m, 4), dtype=np.float64)
        for k in (1, 2, 3, 4):
            idx = np.nonzero(npar == k)[0]
            if idx.size:
                rows = [tuple(gates[i][2])[:k] if len(gates[i]) > 2 else () for i in idx]
                if any(len(r) != k for r in rows):
                    j = int(idx[[len(r) != k for r in rows].index(True)])
                    raise ValueError(f"{names[j]} takes {k} parameters")
                pa[idx, :k] = np.array(rows, dtype=np.float64)
        mats = None
        cidx = np.nonzero(np.isin(codes, [GATE_CODES["custom1"], GATE_CODES["custom2"], GATE_CODES["u2lo"]]))[0]
        if cidx.size:
            mats = np.zeros((m, 16), dtype=np.complex128)
            for i in cidx:
                mm = np.asarray(gates[i][3], dtype=np.complex128).reshape(-1)
                want = 4 if names[i] == "custom1" else 16
                if mm.size != want:
                    raise ValueError(f"{names[i]} takes a {'2x2' if want == 4 else '4x4'} matrix")
                mats[i, :want] = mm
        mp = mats.ctypes.data_as(C.POINTER(NqpuComplex)) if mats is not None else None
        check(self.lib.nqpu_circuit_add_gates(self.h_, codes.ctypes.data_as(C.POINTER(C.c_uint32)),
                                              qa.ctypes.data_as(C.POINTER(C.c_int32)),
                                              pa.ctypes.data_as(C.POINTER(C.c_double)), mp, m),
              "circuit_add_gates")

    def execute(self, state: StateVector, mode: str = "tiled"):
        check(self.lib.nqpu_circuit_execute_ex(self.h_, state.h_, MODES[mode]), "circuit_execute")

    def optimize(self, level: str = "moderate") -> dict:
        """Rewrite the gate list with the optimizer pre-pass (nqpu_circuit_optimize)."""
        lv = {"none": 0, "basic": 1, "moderate": 2, "aggressive": 3}[level]
        st = (C.c_uint64 * 6)()
        check(self.lib.nqpu_circuit_optimize(self.h_, lv, st, 6), "circuit_optimize")
        keys = ("original_gates", "optimized_gates", "gates_removed", "fusions", "commutations", "cancellations")
        return {k: int(v) for k, v in zip(keys, st)}

    def gates(self) -> list:
        """The gate list as (name, qubits, params[, matrix]) tuples (nqpu_circuit_get_gate)."""
        from .circuits import GATE_CODES, MID_GATES
        names = {v: k for k, v in GATE_CODES.items()}
        out = []
        code = C.c_uint32()
        qs = (C.c_int32 * 3)()
        ps = (C.c_double * 4)()
        mx = (NqpuComplex * 16)()
        for i in range(self.gate_count):
            check(self.lib.nqpu_circuit_get_gate(self.h_, i, C.byref(code), qs, ps, mx), "circuit_get_gate")
            name = names[code.value]
            ar = 1 if name in MID_GATES else ARITY[name]
            g = (name, tuple(int(q) for q in qs[:ar]), tuple(float(p) for p in ps[:NPARAMS[name]]))
            if name in ("custom1", "custom2", "u2lo"):
                k = 4 if name == "custom1" else 16
                m = np.array([complex(mx[j].re, mx[j].im) for j in range(k)])
                g = g + (m.reshape(2, 2) if k == 4 else m.reshape(4, 4),)
            out.append(g)
        return out

    def execute_measured(self, state: StateVector, mode: str = "tiled") -> np.ndarray:
        """Execute and return the outcomes of the mid-circuit measurements in order."""
        nmeas = 64 + self.gate_count
        out = (C.c_uint32 * nmeas)()
        cnt = C.c_uint32()
        check(self.lib.nqpu_circuit_execute_measured(self.h_, state.h_, MODES[mode], out, nmeas, C.byref(cnt)),
              "circuit_execute_measured")
        return np.array(out[:cnt.value], dtype=np.uint32)

    @property
    def gate_count(self) -> int:
        return int(self.lib.nqpu_circuit_gate_count(self.h_))

    @property
    def depth(self) -> int:
        return int(self.lib.nqpu_circuit_depth(self.h_))

    @classmethod
    def from_qasm(cls, text: str) -> "Circuit":
        """Circuit from OpenQASM 2.0 text (nqpu_circuit_from_qasm)."""
        lib = _lib.load()
        line = C.c_uint32()
        h = lib.nqpu_circuit_from_qasm(text.encode(), C.byref(line))
        if not h:
            raise ValueError(f"OpenQASM parse error at line {line.value}")
        obj = cls.__new__(cls)
        obj.lib = lib
        obj.h_ = h
        obj.num_qubits = int(lib.nqpu_circuit_num_qubits(h))
        return obj

    def to_qasm(self) -> str:
        """OpenQASM 2.0 text of the circuit (nqpu_circuit_to_qasm)."""
        need = C.c_uint64()
        self.lib.nqpu_circuit_to_qasm(self.h_, None, 0, C.byref(need))
        buf = C.create_string_buffer(int(need.value) + 1)
        code = self.lib.nqpu_circuit_to_qasm(self.h_, buf, len(buf), C.byref(need))
        if code not in (0, 2):
            check(code, "circuit_to_qasm")
        return buf.value.decode()

    def plan_stats(self, num_qubits: int, dtype: str = "c128", mode: str = "tiled"):
        out = (C.c_uint64 * 4)()
        check(self.lib.nqpu_circuit_plan_stats(self.h_, int(num_qubits), DTYPES[dtype], MODES[mode], out, 4),
              "plan_stats")
        return {"passes": int(out[0]), "ops": int(out[1]), "stages": int(out[2]), "upload_bytes": int(out[3])}
