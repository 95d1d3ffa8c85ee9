"""Circuit optimizer pre-pass (nqpu_circuit_optimize) on CPU: the reference's
optimizer tests (circuits/synthesis/circuit_optimizer.rs:840-1200) restated,
plus equivalence of optimized and original random circuits on the oracle at
every level (equal up to a global phase, which the fusion pass may drop)."""
import math

import numpy as np
import pytest

from nqpu_b200 import circuits
from nqpu_b200.state import Circuit
from oracle.oracle import OracleState


def opt(gates, n, level):
    c = Circuit(n, gates)
    st = c.optimize(level)
    return c.gates(), st


def test_clifford_simplification():
    g, _ = opt([("h", (0,), ()), ("h", (0,), ()), ("x", (1,), ()), ("x", (1,), ())], 2, "basic")
    assert g == []


def test_cnot_cancellation_and_different_qubits():
    g, _ = opt([("cx", (0, 1), ()), ("cx", (0, 1), ())], 2, "basic")
    assert g == []
    g, _ = opt([("h", (0,), ()), ("h", (1,), ())], 2, "basic")
    assert len(g) == 2


def test_stats_and_none_level():
    g, st = opt([("h", (0,), ()), ("h", (0,), ()), ("x", (1,), ())], 2, "basic")
    assert len(g) == 1
    assert st["original_gates"] == 3 and st["optimized_gates"] == 1
    assert st["gates_removed"] == 2 and st["cancellations"] == 2
    g, _ = opt([("h", (0,), ()), ("h", (0,), ())], 1, "none")
    assert len(g) == 2


def test_fusion():
    g, _ = opt([("h", (0,), ()), ("x", (0,), ())], 1, "basic")
    assert len(g) == 1 and g[0][0] == "custom1"
    # H then X: the fused matrix is X H (later gates multiply from the left)
    s2 = 1 / math.sqrt(2)
    H = np.array([[s2, s2], [s2, -s2]])
    X = np.array([[0, 1], [1, 0]])
    np.testing.assert_allclose(g[0][3], X @ H, atol=1e-12)
    g, _ = opt([("rz", (0,), (0.3,)), ("ry", (0,), (0.5,)), ("h", (0,), ())], 1, "basic")
    assert len(g) == 1 and g[0][0] == "custom1"
    g, _ = opt([("x", (0,), ()), ("x", (0,), ())], 1, "basic")
    assert g == []


def test_peephole_patterns():
    g, _ = opt([("h", (1,), ()), ("cx", (0, 1), ()), ("h", (1,), ())], 2, "aggressive")
    assert g == [("cz", (0, 1), ())]
    g, _ = opt([("h", (1,), ()), ("cz", (0, 1), ()), ("h", (1,), ())], 2, "aggressive")
    assert g == [("cx", (0, 1), ())]
    g, _ = opt([("cx", (0, 1), ()), ("x", (1,), ()), ("cx", (0, 1), ())], 2, "aggressive")
    assert g == [("x", (1,), ())]
    g, _ = opt([("s", (0,), ()), ("s", (0,), ())], 1, "aggressive")
    assert g == [("z", (0,), ())]
    g, _ = opt([("t", (0,), ()), ("t", (0,), ())], 1, "aggressive")
    assert g == [("s", (0,), ())]


def test_rotation_merging_and_commutation():
    g, _ = opt([("rz", (0,), (0.3,)), ("rz", (0,), (0.5,))], 1, "moderate")
    assert len(g) == 1 and g[0][0] == "rz" and abs(g[0][2][0] - 0.8) < 1e-12
    # Z on the control commutes through the CNOT and cancels the other Z
    g, st = opt([("z", (0,), ()), ("cx", (0, 1), ()), ("z", (0,), ())], 2, "moderate")
    assert g == [("cx", (0, 1), ())] and st["commutations"] >= 1


def test_measurements_are_barriers():
    g, _ = opt([("h", (0,), ()), ("measure", (0,), ()), ("h", (0,), ())], 1, "aggressive")
    assert [x[0] for x in g] == ["h", "measure", "h"]


@pytest.mark.parametrize("level", ["basic", "moderate", "aggressive"])
def test_random_circuits_equivalent(level):
    rng = np.random.default_rng(17)
    n = 5
    names = ["h", "x", "y", "z", "s", "t", "rx", "ry", "rz", "cx", "cz", "swap", "p", "u3"]
    for trial in range(6):
        gates = []
        for _ in range(120):
            name = names[int(rng.integers(len(names)))]
            ar = circuits.ARITY[name]
            qs = tuple(int(x) for x in rng.choice(n, size=ar, replace=False))
            # draw from a small angle set so that merges and cancellations occur
            ps = tuple(float(rng.choice([0.5, -0.5, math.pi / 2])) for _ in range(circuits.NPARAMS[name]))
            gates.append((name, qs, ps))
            if rng.random() < 0.3:
                gates.append(gates[-1])  # adjacent duplicates: cancellations and merges
        g, st = opt(gates, n, level)
        assert st["optimized_gates"] < st["original_gates"]
        a, b = OracleState(n), OracleState(n)
        a.apply(gates)
        b.apply(g)
        fid = abs(np.vdot(a.amplitudes(), b.amplitudes())) ** 2
        assert 1 - fid < 1e-10, (level, trial)
