"""NQPU_MODE_AUTO's engine choice (host-side planning only, no GPU needed):
the tensor-core passes for the random brickwork (dense 1-qubit gates and
CNOTs, where the tensor plan needs few more passes than the tiled one), the
tiled passes for the QFT (controlled phases are diagonal: the tiled passes
apply them without tile bits, 8 passes against 48), the tiled passes for
complex128 and for states below 12 qubits (the tensor mode runs neither)."""
import ctypes as C

import pytest

from nqpu_b200 import _lib, circuits
from nqpu_b200.state import Circuit

TILED, TENSOR, AUTO = 0, 3, 4
C128, C64 = 0, 1


def auto(c, n, dtype):
    m = C.c_int(-1)
    assert _lib.load().nqpu_circuit_auto_mode(c.h_, n, dtype, C.byref(m)) == 0
    return m.value


@pytest.mark.parametrize("n,kind,dtype,want", [
    (30, "brickwork", C64, TENSOR), (26, "brickwork", C64, TENSOR), (30, "qft", C64, TILED),
    (30, "brickwork", C128, TILED), (11, "brickwork", C64, TILED), (24, "qft", C128, TILED)])
def test_choice(n, kind, dtype, want):
    gates = circuits.brickwork(n, 10, 1) if kind == "brickwork" else circuits.qft(n)
    c = Circuit(n, gates)
    assert auto(c, n, dtype) == want
    # the plan statistics of AUTO are those of the mode it picks
    name = {TILED: "tiled", TENSOR: "tensor"}[want]
    dt = "c64" if dtype == C64 else "c128"
    assert c.plan_stats(n, dt, "auto") == c.plan_stats(n, dt, name)


def test_rejects_unknown_mode_and_null():
    lib = _lib.load()
    c = Circuit(12, circuits.brickwork(12, 2, 1))
    out = (C.c_uint64 * 4)()
    assert lib.nqpu_circuit_plan_stats(c.h_, 12, C64, 5, out, 4) == 2  # NQPU_INVALID_PARAMETER
    assert lib.nqpu_circuit_auto_mode(c.h_, 12, C64, None) == 5        # NQPU_NULL_POINTER
    assert lib.nqpu_circuit_auto_mode(c.h_, 11, C64, C.byref(C.c_int())) == 2  # fewer qubits than the circuit
