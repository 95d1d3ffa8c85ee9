"""GPU tests of the fused (precision) mode: <=5-qubit fused unitaries applied as
split-TF32 tcgen05 tensor-core contractions on complex64 states.

Tolerance (complex64, split TF32 with FP32 accumulation): 1-F <= 1e-5 and
max |d<Z_i>| <= 1e-5 against the FP64 oracle."""
import numpy as np
import pytest

from nqpu_b200 import circuits
from nqpu_b200.state import Circuit, StateVector
from oracle.oracle import OracleState

pytestmark = pytest.mark.gpu
TOL = 1e-5


def fid(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def random_circuit(rng, n, g):
    names = [k for k in circuits.ARITY if k not in ("u2lo", "custom1", "custom2")]
    gates = [("u3", (q,), tuple(rng.uniform(0, 6, 3))) for q in range(n)]
    for _ in range(g):
        name = names[int(rng.integers(len(names)))]
        qs = tuple(int(x) for x in rng.choice(n, size=circuits.ARITY[name], replace=False))
        gates.append((name, qs, tuple(rng.uniform(-6, 6, 4))))
    return gates


@pytest.mark.parametrize("n", [12, 13, 14, 16])
def test_fused_random_circuits(n):
    rng = np.random.default_rng(300 + n)
    gates = random_circuit(rng, n, 8 * n)
    sv = StateVector(n, "c64")
    c = Circuit(n, gates)
    c.execute(sv, "fused")
    o = OracleState(n)
    o.apply(gates)
    assert 1 - fid(sv.amplitudes(), o.amplitudes()) <= TOL
    assert np.abs(sv.expectation_z_all() - o.expectation_z_all()).max() <= TOL


# Fused qubit sets that take each operand-layout case of the kernel: qubit 0
# fused (16-byte operand stores), lane qubits 1..5 fused without qubit 0,
# lowest fused qubit at 6 or above (rotated load steps), and mixtures.
@pytest.mark.parametrize("fset", [(0, 1, 2, 3, 4), (0, 2, 9, 10, 11), (1, 2, 10, 11, 12), (3, 6, 7, 12, 13),
                                  (5, 6, 7, 8, 9), (6, 7, 8, 9, 10), (9, 10, 11, 12, 13)])
def test_fused_operand_layouts(fset):
    n = 14
    rng = np.random.default_rng(sum(fset))
    gates = [("u3", (q,), tuple(rng.uniform(0, 6, 3))) for q in range(n)]
    # dense gates confined to the five qubits: one fused unitary on exactly fset
    for _ in range(12):
        a, b = (int(x) for x in rng.choice(fset, size=2, replace=False))
        gates.append(("cx", (a, b), ()))
        gates.append(("u3", (b,), tuple(rng.uniform(0, 6, 3))))
        gates.append(("rzz", (a, b), (float(rng.uniform(-3, 3)),)))
    sv = StateVector(n, "c64")
    Circuit(n, gates).execute(sv, "fused")
    o = OracleState(n)
    o.apply(gates)
    assert 1 - fid(sv.amplitudes(), o.amplitudes()) <= TOL
    assert np.abs(sv.expectation_z_all() - o.expectation_z_all()).max() <= TOL


@pytest.mark.parametrize("n", [12, 17])
def test_fused_brickwork_and_modes_agree(n):
    gates = circuits.brickwork(n, 12, seed=n)
    c = Circuit(n, gates)
    a = StateVector(n, "c64")
    b = StateVector(n, "c64")
    c.execute(a, "fused")
    c.execute(b, "tiled")
    assert 1 - a.fidelity(b) <= TOL
    st = c.plan_stats(n, "c64", "fused")
    assert st["passes"] < len(gates)


def test_fused_tfim_neel_observables():
    # first-order Trotterised TFIM from the Neel state, <Z_i> and <Z0 Z1>
    n = 16
    gates, _ = circuits.tfim_trotter(n, 20, seed=5)
    sv = StateVector(n, "c64")
    sv.set_basis(circuits.neel_index(n))
    Circuit(n, gates).execute(sv, "fused")
    o = OracleState(n)
    o.set_basis(circuits.neel_index(n))
    o.apply(gates)
    assert np.abs(sv.expectation_z_all() - o.expectation_z_all()).max() <= TOL
    zz = "ZZ" + "I" * (n - 2)
    assert abs(sv.expectation_pauli_string(zz) - o.pauli_string(zz)) <= TOL
    assert abs(sv.norm() - 1) <= 1e-5


def test_fused_renormalisation_long_circuit():
    # > 64 fused unitaries exercises the periodic FP64 renormalisation
    n = 13
    gates = circuits.brickwork(n, 80, seed=9)
    c = Circuit(n, gates)
    assert c.plan_stats(n, "c64", "fused")["passes"] > 64
    sv = StateVector(n, "c64")
    c.execute(sv, "fused")
    o = OracleState(n)
    o.apply(gates)
    assert 1 - fid(sv.amplitudes(), o.amplitudes()) <= TOL
    assert abs(sv.norm() - 1) <= 1e-6


def test_fused_mode_rejects_unsupported():
    from nqpu_b200._lib import NqpuErrorException
    c = Circuit(8, circuits.brickwork(8, 2, 1))
    with pytest.raises(NqpuErrorException):
        c.execute(StateVector(8, "c64"), "fused")  # fewer than 12 qubits
    c12 = Circuit(12, circuits.brickwork(12, 2, 1))
    with pytest.raises(NqpuErrorException):
        c12.execute(StateVector(12, "c128"), "fused")  # complex128
