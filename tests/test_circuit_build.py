"""Bulk circuit construction on CPU (no GPU needed): nqpu_circuit_add_gates
through Circuit.extend and Circuit.from_arrays gives the same gate list as the
one-call-per-gate nqpu_circuit_add_* path, checks every gate the same way, and
appends nothing when any gate is invalid."""
import ctypes as C

import numpy as np
import pytest

from nqpu_b200 import _lib, circuits
from nqpu_b200.state import Circuit


def one_by_one(n, gates):
    c = Circuit(n)
    for g in gates:
        c.add(g[0], g[1], g[2] if len(g) > 2 else (), g[3] if len(g) > 3 else None)
    return c


def test_extend_matches_single_adds():
    rng = np.random.default_rng(7)
    n = 6
    names = [k for k in circuits.ARITY if k not in ("u2lo",)]
    gates = []
    for _ in range(300):
        name = names[int(rng.integers(len(names)))]
        qs = tuple(int(x) for x in rng.choice(n, size=circuits.ARITY[name], replace=False))
        ps = tuple(float(x) for x in rng.uniform(-3, 3, circuits.NPARAMS[name]))
        if name == "custom1":
            gates.append((name, qs, (), rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))))
        elif name == "custom2":
            gates.append((name, qs, (), rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4))))
        else:
            gates.append((name, qs, ps))
    gates.append(("measure", (2,), ()))
    gates.append(("reset", (3,), ()))
    a = Circuit(n, gates).gates()
    b = one_by_one(n, gates).gates()
    assert len(a) == len(b) == len(gates)
    for x, y in zip(a, b):
        assert x[:3] == y[:3]
        if len(x) > 3:
            np.testing.assert_array_equal(x[3], y[3])


def test_from_arrays_matches_gate_lists():
    a = circuits.hea_batch(40, 11)
    b = circuits.hea_batch(40, 11, arrays=True)
    for (n1, g1, J1, h1), (n2, arr, J2, h2) in zip(a, b):
        assert n1 == n2
        np.testing.assert_array_equal(J1, J2)
        np.testing.assert_array_equal(h1, h2)
        assert Circuit(n1, g1).gates() == Circuit.from_arrays(n2, *arr).gates()


def test_bulk_add_rejects_and_appends_nothing():
    lib = _lib.load()
    c = Circuit(4, [("h", (0,), ())])
    def call(codes, qubits, params, mats=None):
        ca = np.asarray(codes, dtype=np.uint32)
        qa = np.asarray(qubits, dtype=np.int32).reshape(-1, 3)
        pa = np.asarray(params, dtype=np.float64).reshape(-1, 4)
        mp = None if mats is None else mats.ctypes.data_as(C.POINTER(_lib.NqpuComplex))
        return lib.nqpu_circuit_add_gates(c.h_, ca.ctypes.data_as(C.POINTER(C.c_uint32)),
                                          qa.ctypes.data_as(C.POINTER(C.c_int32)),
                                          pa.ctypes.data_as(C.POINTER(C.c_double)), mp, len(ca))
    GC = circuits.GATE_CODES
    # unknown gate code
    assert call([GC["x"], 99], [[1, 0, 0], [0, 0, 0]], [0.0] * 8) == 2
    # qubit out of range, repeated qubits, non-finite angle
    assert call([GC["x"], GC["x"]], [[1, 0, 0], [4, 0, 0]], [0.0] * 8) == 1
    assert call([GC["cx"]], [[2, 2, 0]], [0.0] * 4) == 2
    assert call([GC["rx"]], [[1, 0, 0]], [float("nan"), 0, 0, 0]) == 2
    # custom gate without matrices
    assert call([GC["custom1"]], [[1, 0, 0]], [0.0] * 4) == 5
    assert c.gate_count == 1
    # unused qubit slots and parameters are ignored
    assert call([GC["h"], GC["rz"]], [[1, 7, -3], [2, 9, 9]], [5.0, 6, 7, 8, 0.25, 9, 9, 9]) == 0
    assert c.gates() == [("h", (0,), ()), ("h", (1,), ()), ("rz", (2,), (0.25,))]
    # empty call
    assert lib.nqpu_circuit_add_gates(c.h_, None, None, None, None, 0) == 0
    assert lib.nqpu_circuit_add_gates(None, None, None, None, None, 0) == 5


def test_extend_argument_errors():
    with pytest.raises(ValueError):
        Circuit(3, [("cx", (0,), ())])
    with pytest.raises(ValueError):
        Circuit(3, [("rx", (0,), ())])
    with pytest.raises(ValueError):
        Circuit(3, [("custom1", (0,), (), np.eye(4))])
