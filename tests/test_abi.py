"""C ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and the host-side argument checks return the reference's error
codes (c_ffi.rs tests :2068-2120, :2586).  No compute call is made here."""
import ctypes as C
import subprocess

import pytest

from nqpu_b200 import _lib
from nqpu_b200.state import Circuit

OK, INVALID_QUBIT, INVALID_PARAMETER, NULL_POINTER = 0, 1, 2, 5


def test_every_declared_symbol_is_exported():
    decl = set(_lib.parse_header())
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.split()[-2:-1] == ["T"]}
    missing = decl - exported
    assert not missing, f"declared but not exported: {sorted(missing)}"
    assert len(decl) >= 90


def test_library_loads_and_binds(lib):
    for name in _lib.parse_header():
        assert hasattr(lib, name)


def test_version_and_messages(lib):
    v = lib.nqpu_version()
    assert (v.major, v.minor, v.patch) == (0, 1, 0)  # c_ffi.rs:1404
    for code in range(7):
        msg = lib.nqpu_error_message(code)
        assert msg and len(msg) > 0


def test_null_pointer_errors(lib):
    # c_ffi.rs:2068 test_null_pointer_errors
    assert lib.nqpu_gate_h(None, 0) == NULL_POINTER
    assert lib.nqpu_gate_x(None, 0) == NULL_POINTER
    assert lib.nqpu_gate_cx(None, 0, 1) == NULL_POINTER
    assert lib.nqpu_gate_rx(None, 0, 0.5) == NULL_POINTER
    assert lib.nqpu_state_reset(None) == NULL_POINTER
    out = _lib.NqpuComplex()
    assert lib.nqpu_state_get_amplitude(None, 0, C.byref(out)) == NULL_POINTER
    d = C.c_double()
    assert lib.nqpu_expectation_z(None, 0, C.byref(d)) == NULL_POINTER
    assert lib.nqpu_circuit_add_h(None, 0) == NULL_POINTER
    assert lib.nqpu_circuit_add_cx(None, 0, 1) == NULL_POINTER
    assert lib.nqpu_circuit_execute(None, None) == NULL_POINTER
    assert lib.nqpu_state_num_qubits(None) == 0
    assert lib.nqpu_state_norm(None) == -1.0
    assert lib.nqpu_circuit_gate_count(None) == 0
    assert lib.nqpu_circuit_depth(None) == 0
    lib.nqpu_state_destroy(None)
    lib.nqpu_circuit_destroy(None)


def test_create_limits(lib):
    # c_ffi.rs:2426 test_state_create_invalid: 0 and > 30 qubits give NULL
    assert not lib.nqpu_state_create(0)
    assert not lib.nqpu_state_create(31)
    assert not lib.nqpu_state_create(100)
    assert not lib.nqpu_circuit_create(0)
    assert not lib.nqpu_circuit_create(31)
    assert not lib.nqpu_state_create_ex(35, 0)


def test_circuit_api_host_side(lib):
    c = lib.nqpu_circuit_create(3)
    assert c
    assert lib.nqpu_circuit_add_h(c, 0) == OK
    assert lib.nqpu_circuit_add_cx(c, 0, 1) == OK
    assert lib.nqpu_circuit_add_rx(c, 2, 0.785) == OK
    assert lib.nqpu_circuit_gate_count(c) == 3  # c_ffi.rs:1991
    # errors (c_ffi.rs:2107 test_invalid_qubit_errors, :2586 NaN angle)
    assert lib.nqpu_circuit_add_h(c, 3) == INVALID_QUBIT
    assert lib.nqpu_circuit_add_cx(c, 0, 5) == INVALID_QUBIT
    assert lib.nqpu_circuit_add_cx(c, 1, 1) == INVALID_PARAMETER
    assert lib.nqpu_circuit_add_rx(c, 0, float("nan")) == INVALID_PARAMETER
    assert lib.nqpu_circuit_add_rx(c, 0, float("inf")) == INVALID_PARAMETER
    assert lib.nqpu_circuit_gate_count(c) == 3
    lib.nqpu_circuit_destroy(c)


def test_circuit_depth(lib):
    # c_ffi.rs:2054 test_circuit_depth: H(0) H(1) CX(0,1) -> depth 2
    c = lib.nqpu_circuit_create(2)
    lib.nqpu_circuit_add_h(c, 0)
    lib.nqpu_circuit_add_h(c, 1)
    lib.nqpu_circuit_add_cx(c, 0, 1)
    assert lib.nqpu_circuit_depth(c) == 2
    lib.nqpu_circuit_destroy(c)


def test_plan_stats_brickwork():
    from nqpu_b200.circuits import brickwork
    g = brickwork(30, 40, seed=1)
    c = Circuit(30, g)
    assert c.gate_count == 1780
    st = c.plan_stats(30, "c64", "tiled")
    assert st["ops"] == 1780
    assert 1 <= st["passes"] < 200
    pg = c.plan_stats(30, "c64", "pergate")
    assert pg["passes"] == 1780
    # 64 KB complex64 tiles (13 qubits) need no more passes than 64 KB complex128 tiles (12)
    lib = _lib.load()
    old = lib.nqpu_tile_config_get(1)
    assert lib.nqpu_tile_config_set(1, 2) == OK
    try:
        st13 = c.plan_stats(30, "c64", "tiled")
    finally:
        lib.nqpu_tile_config_set(1, old)
    st12 = c.plan_stats(30, "c128", "tiled")
    assert st12["passes"] >= st13["passes"]
    assert lib.nqpu_tile_config_set(1, 3) == INVALID_PARAMETER


def test_batch_bulk_add_rejects_without_a_device_call():
    """Argument checks of nqpu_batch_add_ising_arrays that need no batch
    handle: a NULL batch is NQPU_NULL_POINTER."""
    import ctypes as C
    from nqpu_b200 import _lib
    lib = _lib.load()
    nq = (C.c_uint32 * 1)(6)
    offs = (C.c_uint64 * 2)(0, 0)
    assert lib.nqpu_batch_add_ising_arrays(None, 1, nq, offs, None, None, None, None, None, None, None) == 5
