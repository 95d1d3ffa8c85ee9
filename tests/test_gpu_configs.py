"""GPU parity on the configurations the random-circuit tests do not reach.

* the reference-generated golden statevectors (tests/golden: the reference's
  Python statevector, its gate set, and U3 / RZZ through identities of its own
  gates) run through the engine's C ABI, every engine mode;
* the QFT (controlled-phase chains: the diagonal-run fusion of
  gate_fusion.rs:757,905 in the reference) from a random product state;
* long runs of diagonal gates (CZ, CPhase, RZ, RZZ, CRZ) on qubits far outside
  the tiled pass's shared-memory tile, where the engine applies a diagonal from
  the amplitude index instead of a register bit;
* brickwork at 25-26 qubits, where most qubits of every pass lie outside the
  tile, against the FP64 oracle.

Tolerances (as every GPU parity test): complex128 max |amp diff| <= 1e-12 and
1-F <= 1e-12; complex64 1-F <= 1e-5 and max |d<Z_i>| <= 1e-5.  Circuits with
U3 gates are compared with the golden states up to one global phase (the
reference's Python statevector runs U3 as Rz Ry Rz).
"""
import numpy as np
import pytest

import make_golden
from nqpu_b200 import circuits
from nqpu_b200.state import Circuit, StateVector
from oracle.oracle import OracleState

pytestmark = pytest.mark.gpu

TOL = {"c128": 1e-12, "c64": 1e-5}


def fid(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


def align_global_phase(got, ref):
    ov = np.vdot(got, ref)
    return got * (ov / abs(ov))


def product_state_prep(rng, n):
    return [("u3", (q,), tuple(float(x) for x in rng.uniform(0, 6, 3))) for q in range(n)]


def check(got, ref, dtype, z=None, zref=None, phase_free=False):
    if phase_free:
        got = align_global_phase(got, ref)
    if dtype == "c128":
        assert np.abs(got - ref).max() <= 1e-12
    assert 1 - fid(got, ref) <= TOL[dtype]
    if z is not None:
        assert np.abs(z - zref).max() <= TOL[dtype]


@pytest.mark.parametrize("mode", ["tiled", "pergate"])
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_reference_golden_statevectors_on_gpu(dtype, mode):
    cases = make_golden.load()
    assert len(cases) == 16
    for n, gates, ref in cases:
        sv = StateVector(n, dtype)
        Circuit(n, gates).execute(sv, mode)
        check(sv.amplitudes(), ref, dtype)
        sv.close()


@pytest.mark.parametrize("mode", ["tiled", "pergate"])
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_reference_golden_u3_rzz_on_gpu(dtype, mode):
    cases = make_golden.load_u3_rzz()
    assert len(cases) == 22
    for n, gates, ref in cases:
        sv = StateVector(n, dtype)
        Circuit(n, gates).execute(sv, mode)
        check(sv.amplitudes(), ref, dtype, phase_free=any(g[0] == "u3" for g in gates))
        sv.close()


def test_reference_golden_u3_rzz_fused_mode():
    # the fused tensor-core mode needs >= 12 qubits (complex64)
    for n, gates, ref in make_golden.load_u3_rzz():
        if n < 12:
            continue
        sv = StateVector(n, "c64")
        Circuit(n, gates).execute(sv, "fused")
        check(sv.amplitudes(), ref, "c64", phase_free=True)
        sv.close()


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("n", [12, 20, 24])
def test_qft_random_product_state(dtype, n):
    rng = np.random.default_rng(500 + n)
    gates = product_state_prep(rng, n) + circuits.qft(n)
    o = OracleState(n)
    o.apply(gates)
    c = Circuit(n, gates)
    modes = ["tiled", "pergate"] + (["fused"] if dtype == "c64" else [])
    for mode in modes:
        sv = StateVector(n, dtype)
        c.execute(sv, mode)
        check(sv.amplitudes(), o.amplitudes(), dtype, sv.expectation_z_all(), o.expectation_z_all())
        sv.close()


def diagonal_run_circuit(rng, n, layers, runs):
    """U3 layers separated by long runs of diagonal gates on random qubits (most
    of them outside any one shared-memory tile)."""
    gates = []
    for _ in range(layers):
        gates += product_state_prep(rng, n)
        for _ in range(runs):
            kind = ["cz", "cp", "rz", "rzz", "crz", "p", "s", "t", "z"][int(rng.integers(9))]
            if kind in ("rz", "p", "s", "t", "z"):
                q = int(rng.integers(n))
                gates.append((kind, (q,), (float(rng.uniform(-6, 6)),) if kind in ("rz", "p") else ()))
            else:
                a, b = (int(x) for x in rng.choice(n, size=2, replace=False))
                gates.append((kind, (a, b), () if kind == "cz" else (float(rng.uniform(-6, 6)),)))
    return gates


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("n", [16, 22])
def test_long_diagonal_runs_outside_the_tile(dtype, n):
    rng = np.random.default_rng(900 + n)
    gates = diagonal_run_circuit(rng, n, layers=3, runs=6 * n)
    o = OracleState(n)
    o.apply(gates)
    c = Circuit(n, gates)
    st = c.plan_stats(n, dtype, "tiled")
    assert st["passes"] >= 1
    for mode in ("tiled", "pergate"):
        sv = StateVector(n, dtype)
        c.execute(sv, mode)
        check(sv.amplitudes(), o.amplitudes(), dtype, sv.expectation_z_all(), o.expectation_z_all())
        sv.close()


@pytest.mark.parametrize("n,depth,dtype", [(25, 10, "c128"), (26, 8, "c128"), (26, 8, "c64")])
def test_brickwork_large_against_oracle(n, depth, dtype):
    # 25-26 qubits: 13-14 of 26 qubits lie outside every pass's tile
    gates = circuits.brickwork(n, depth, seed=n + depth)
    o = OracleState(n)
    o.apply(gates)
    sv = StateVector(n, dtype)
    Circuit(n, gates).execute(sv, "tiled")
    check(sv.amplitudes(), o.amplitudes(), dtype, sv.expectation_z_all(), o.expectation_z_all())
    sv.close()
