"""Mid-circuit measurement and reset in circuits (QuantumSimulator::measure_qubit,
lib.rs:1835; GateOperations::reset_qubit, lib.rs:1705) against the oracle: with
the same seed the engine and the oracle draw the same xorshift64* uniforms,
so the outcomes must agree exactly and the final states within the dtype's
tolerance (complex128 1e-12, complex64 1e-5).  In NQPU_MODE_AUTO every gate run
between measurements makes its own mode choice (22 qubits: tensor passes)."""
import ctypes as C

import numpy as np
import pytest

from nqpu_b200 import _lib, circuits
from nqpu_b200.batch import Batch
from nqpu_b200.server import Server
from nqpu_b200.state import Circuit, StateVector
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def mid_circuit(n, seed):
    rng = np.random.default_rng(seed)
    g = circuits.brickwork(n, 3, seed)
    for q in rng.choice(n, size=3, replace=False):
        g.append(("measure", (int(q),), ()))
    g += circuits.brickwork(n, 2, seed + 1)
    g.append(("reset", (int(rng.integers(n)),), ()))
    g += circuits.brickwork(n, 2, seed + 2)
    g.append(("measure", (int(rng.integers(n)),), ()))
    return g


@pytest.mark.parametrize("n,dtype,mode", [(6, "c128", "tiled"), (6, "c128", "pergate"), (11, "c128", "tiled"),
                                          (14, "c64", "tiled"), (14, "c64", "fused"), (14, "c64", "tensor"),
                                          (22, "c64", "auto")])
def test_measured_circuit_matches_oracle(n, dtype, mode):
    lib = _lib.load()
    for seed in (3, 4, 5):
        g = mid_circuit(n, seed)
        c = Circuit(n, g)
        assert c.gate_count == len(g)
        with StateVector(n, dtype) as sv:
            lib.nqpu_set_seed(1000 + seed)
            got = c.execute_measured(sv, mode)
            amps = sv.amplitudes()
        o = O.OracleState(n)
        O.set_seed(1000 + seed)
        o.apply(g)
        want = o.take_outcomes()
        assert np.array_equal(got, want), (seed, got, want)
        tol = 1e-12 if dtype == "c128" else (1e-4 if mode == "fused" else 1e-5)
        assert np.abs(amps - o.amplitudes()).max() < tol


def test_qasm_mid_circuit_measure_and_reset():
    lib = _lib.load()
    text = """OPENQASM 2.0;
include "qelib1.inc";
qreg q[3];
creg c[3];
h q[0];
cx q[0],q[1];
measure q[0] -> c[0];
reset q[1];
h q[2];
cx q[2],q[0];
measure q -> c;
"""
    c = Circuit.from_qasm(text)
    assert c.gate_count == 9
    g = [("h", (0,), ()), ("cx", (0, 1), ()), ("measure", (0,), ()), ("reset", (1,), ()), ("h", (2,), ()),
         ("cx", (2, 0), ()), ("measure", (0,), ()), ("measure", (1,), ()), ("measure", (2,), ())]
    for seed in range(6):
        with StateVector(3, "c128") as sv:
            lib.nqpu_set_seed(seed)
            got = c.execute_measured(sv)
        o = O.OracleState(3)
        O.set_seed(seed)
        o.apply(g)
        assert np.array_equal(got, o.take_outcomes())
        assert got[2] == 0  # q[1] was reset to |0> and nothing touched it since


def test_batch_and_server_refuse_measured_circuits():
    n = 8
    c = Circuit(n, circuits.brickwork(n, 2, 1) + [("measure", (0,), ())])
    b = Batch()
    with pytest.raises(RuntimeError):
        b.add_ising(c, np.zeros(n - 1), np.zeros(n))
    b.close()
    with Server(hbm_budget_bytes=1 << 22, max_qubits=10) as srv:
        with pytest.raises(RuntimeError):
            srv.submit(c, "zall")
