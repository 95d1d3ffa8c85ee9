"""GPU parity of the tensor-core pass mode (NQPU_MODE_TENSOR, tcpass.cu):
up to three fused 5-qubit unitaries per HBM pass, split-FP16 tcgen05 GEMMs on a
shared-memory tile, complex64 states of 12 or more qubits.

Tolerance (complex64 against the FP64 oracle, as every complex64 test):
1-F <= 1e-5 and max |d<Z_i>| <= 1e-5; the norm of the input is kept to 1e-6.
"""
import numpy as np
import pytest

import make_golden
from nqpu_b200 import circuits
from nqpu_b200.state import Circuit, StateVector
from oracle.oracle import OracleState

pytestmark = pytest.mark.gpu

TOL = 1e-5


def fid(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def run_tensor(n, gates, init=None):
    sv = StateVector(n, "c64")
    if init is not None:
        sv.set_amplitudes(init)
    Circuit(n, gates).execute(sv, "tensor")
    out = sv.amplitudes(), sv.expectation_z_all(), sv.norm()
    sv.close()
    return out


def oracle(n, gates, init=None):
    o = OracleState(n)
    if init is not None:
        o.set_amplitudes(init)
    o.apply(gates)
    return o.amplitudes(), o.expectation_z_all()


def random_circuit(rng, n, g):
    names = [k for k in circuits.ARITY if k != "u2lo" and circuits.ARITY[k] <= n]
    gates = [("u3", (q,), tuple(float(x) for x in rng.uniform(0, 6, 3))) for q in range(n)]
    for _ in range(g):
        name = names[int(rng.integers(len(names)))]
        qs = tuple(int(x) for x in rng.choice(n, size=circuits.ARITY[name], replace=False))
        if name == "custom1":
            m = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))[0]
            gates.append((name, qs, (), m))
        elif name == "custom2":
            m = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))[0]
            gates.append((name, qs, (), m))
        else:
            gates.append((name, qs, tuple(float(x) for x in rng.uniform(-6, 6, 4))))
    return gates


@pytest.mark.parametrize("n", [12, 13, 14, 17, 20])
def test_random_circuits(n):
    rng = np.random.default_rng(300 + n)
    gates = random_circuit(rng, n, 12 * n)
    got, z, nrm = run_tensor(n, gates)
    ref, zref = oracle(n, gates)
    assert 1 - fid(got, ref) <= TOL
    assert np.abs(z - zref).max() <= TOL
    assert abs(nrm - 1.0) <= 1e-6


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_brickwork_20q_config(seed):
    n = 20
    gates = circuits.brickwork(n, 20, seed)
    got, z, _ = run_tensor(n, gates)
    ref, zref = oracle(n, gates)
    assert 1 - fid(got, ref) <= TOL
    assert np.abs(z - zref).max() <= TOL


@pytest.mark.parametrize("n,depth", [(24, 16), (26, 10)])
def test_brickwork_large(n, depth):
    gates = circuits.brickwork(n, depth, seed=n)
    got, z, _ = run_tensor(n, gates)
    ref, zref = oracle(n, gates)
    assert 1 - fid(got, ref) <= TOL
    assert np.abs(z - zref).max() <= TOL


def test_qft_and_tfim():
    n = 20
    rng = np.random.default_rng(8)
    prep = [("u3", (q,), tuple(float(x) for x in rng.uniform(0, 6, 3))) for q in range(n)]
    for gates in (prep + circuits.qft(n), circuits.tfim_trotter(n, 10, seed=4)[0]):
        got, z, _ = run_tensor(n, gates)
        ref, zref = oracle(n, gates)
        assert 1 - fid(got, ref) <= TOL
        assert np.abs(z - zref).max() <= TOL


def test_golden_fixtures_tensor_mode():
    for n, gates, ref in make_golden.load_u3_rzz():
        if n < 12:
            continue
        got, _, _ = run_tensor(n, gates)
        assert 1 - fid(got, ref) <= TOL


def test_input_norm_is_kept():
    # renormalisation restores the norm the state had when the run started
    n = 16
    rng = np.random.default_rng(2)
    init = 0.5 * (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)) / np.sqrt(2 << n)
    gates = circuits.brickwork(n, 30, seed=7)
    got, _, nrm = run_tensor(n, gates, init=init)
    ref, _ = oracle(n, gates, init=init)
    assert abs(nrm / np.vdot(init, init).real - 1.0) <= 1e-6
    assert 1 - fid(got, ref) <= TOL


def test_agrees_with_tiled_engine():
    n = 18
    gates = circuits.brickwork(n, 24, seed=11)
    c = Circuit(n, gates)
    a, b = StateVector(n, "c64"), StateVector(n, "c64")
    c.execute(a, "tensor")
    c.execute(b, "tiled")
    assert 1 - a.fidelity(b) <= TOL
    st = c.plan_stats(n, "c64", "tensor")
    assert st["passes"] >= 1 and st["stages"] <= 3 * st["passes"]  # at most three unitaries per pass
    a.close()
    b.close()


def test_rejects_complex128_and_small_states():
    from nqpu_b200._lib import NqpuErrorException
    c = Circuit(11, circuits.brickwork(11, 2, 1))
    with StateVector(11, "c64") as sv, pytest.raises(NqpuErrorException):
        c.execute(sv, "tensor")
    c = Circuit(12, circuits.brickwork(12, 2, 1))
    with StateVector(12, "c128") as sv, pytest.raises(NqpuErrorException):
        c.execute(sv, "tensor")


@pytest.mark.parametrize("n,kind,dtype", [(22, "brickwork", "c64"), (20, "qft", "c64"), (16, "tfim", "c64"),
                                          (18, "brickwork", "c128"), (10, "brickwork", "c64")])
def test_auto_mode_matches_oracle(n, kind, dtype):
    """NQPU_MODE_AUTO runs each gate run in the mode its model picks; the
    result must meet that dtype's tolerance against the FP64 oracle."""
    gates = {"brickwork": lambda: circuits.brickwork(n, 12, 5), "qft": lambda: circuits.qft(n),
             "tfim": lambda: circuits.tfim_trotter(n, 6, 3)[0]}[kind]()
    rng = np.random.default_rng(n)
    init = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    init /= np.linalg.norm(init)
    ref, zref = oracle(n, gates, init)
    sv = StateVector(n, dtype)
    sv.set_amplitudes(init)
    Circuit(n, gates).execute(sv, "auto")
    got, z = sv.amplitudes(), sv.expectation_z_all()
    sv.close()
    tol = TOL if dtype == "c64" else 1e-12
    assert 1 - fid(ref, got) <= tol
    assert np.abs(z - zref).max() <= max(tol, 1e-12)


def test_one_circuit_on_two_states_at_once():
    """The same circuit handle runs on two states from two host threads, so
    the two runs overlap on the GPU; each run's norm partials and error flag
    live in its own state, so both results equal a run on its own, bitwise."""
    import threading
    n = 22
    c = Circuit(n, circuits.brickwork(n, 16, 9))
    with StateVector(n, "c64") as sv:
        c.execute(sv, "tensor")
        alone = sv.amplitudes()
    for _ in range(3):
        svs = [StateVector(n, "c64"), StateVector(n, "c64")]
        errs = []

        def run(sv):
            try:
                c.execute(sv, "tensor")
            except Exception as e:  # reported below
                errs.append(e)

        th = [threading.Thread(target=run, args=(s,)) for s in svs]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert not errs, errs
        for s in svs:
            assert np.array_equal(s.amplitudes(), alone)
            s.close()
