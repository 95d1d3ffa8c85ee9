"""Oracle pinning (CPU): the oracle against the reference's own outputs.

* golden statevectors generated by the reference's Python statevector
  (sdk/python/nqpu/core/simulator.py:193-295) — tests/golden/make_golden.py;
* known-answer tests restated from R/lib.rs:2533-2813 and c_ffi.rs:1646-2660;
* the xorshift64* stream of c_ffi.rs:56-66 and the sampling rule of c_ffi.rs:602.
"""
import math

import numpy as np
import pytest

import make_golden
from oracle.oracle import OracleState, xorshift_uniforms
from nqpu_b200 import circuits

EPS = 1e-10  # c_ffi.rs:1651


@pytest.mark.parametrize("case", range(16))
def test_oracle_matches_reference_python_golden(case):
    n, gates, ref = make_golden.load()[case]
    o = OracleState(n)
    o.apply(gates)
    np.testing.assert_allclose(o.amplitudes(), ref, atol=1e-13, rtol=0)


def align_global_phase(got, ref):
    """got times the one global phase that best matches ref."""
    ov = np.vdot(got, ref)
    return got * (ov / abs(ov))


@pytest.mark.parametrize("case", range(22))
def test_oracle_u3_rzz_match_reference_python_golden(case):
    # U3 (ascii_viz.rs:134-150) and RZZ (gates.rs:486) against the reference's
    # Python statevector running Rz Ry Rz and CX Rz CX: RZZ circuits agree
    # exactly, U3 ones up to one global phase (e^{i(phi+lambda)/2} per U3)
    n, gates, ref = make_golden.load_u3_rzz()[case]
    o = OracleState(n)
    o.apply(gates)
    got = o.amplitudes()
    if any(g[0] == "u3" for g in gates):
        got = align_global_phase(got, ref)
    np.testing.assert_allclose(got, ref, atol=1e-12, rtol=0)


def test_oracle_rzz_alone_matches_exactly():
    # no global-phase freedom: RZZ = CX Rz CX exactly
    cases = [c for c in make_golden.load_u3_rzz() if not any(g[0] == "u3" for g in c[1])]
    assert len(cases) == 4 and all(any(g[0] == "rzz" for g in c[1]) for c in cases)
    for n, gates, ref in cases:
        o = OracleState(n)
        o.apply(gates)
        np.testing.assert_allclose(o.amplitudes(), ref, atol=1e-12, rtol=0)


@pytest.mark.parametrize("case", [3, 9, 15])
def test_oracle_f32_matches_golden_within_f32(case):
    n, gates, ref = make_golden.load()[case]
    o = OracleState(n, f32=True)
    o.apply(gates)
    a = o.amplitudes()
    fid = abs(np.vdot(ref, a)) ** 2
    assert 1 - fid < 1e-6
    assert np.abs(a - ref).max() < 1e-5


def amp(o, i):
    return o.amplitudes()[i]


def test_known_answers_c_ffi():
    s2 = 1 / math.sqrt(2)
    o = OracleState(1)
    o.apply([("h", (0,), ())])  # c_ffi.rs:1706 H|0> = |+>
    assert abs(amp(o, 0) - s2) < EPS and abs(amp(o, 1) - s2) < EPS
    o = OracleState(2)
    o.apply([("h", (0,), ()), ("cx", (0, 1), ())])  # c_ffi.rs:1752 Bell
    a = o.amplitudes()
    assert abs(a[0] - s2) < EPS and abs(a[3] - s2) < EPS and abs(a[1]) < EPS and abs(a[2]) < EPS
    o = OracleState(1)
    o.apply([("rx", (0,), (math.pi,))])  # c_ffi.rs:1775 Rx(pi)|0> = -i|1>
    assert abs(amp(o, 0)) < EPS and abs(amp(o, 1) - (-1j)) < EPS
    o = OracleState(1)
    o.apply([("ry", (0,), (math.pi,))])  # c_ffi.rs:1798 Ry(pi)|0> = |1>
    assert abs(amp(o, 1) - 1) < EPS
    o = OracleState(1)
    o.apply([("x", (0,), ()), ("y", (0,), ())])  # c_ffi Y|0> = i|1>: start |0>
    o = OracleState(1)
    o.apply([("y", (0,), ())])  # c_ffi.rs:2296
    assert abs(amp(o, 1) - 1j) < EPS
    o = OracleState(1)
    o.apply([("x", (0,), ()), ("s", (0,), ())])  # c_ffi.rs:2329 S|1> = i|1>
    assert abs(amp(o, 1) - 1j) < EPS
    o = OracleState(1)
    o.apply([("x", (0,), ()), ("t", (0,), ())])  # c_ffi.rs:2344
    assert abs(amp(o, 1) - complex(math.cos(math.pi / 4), math.sin(math.pi / 4))) < EPS
    o = OracleState(2)
    o.apply([("x", (0,), ()), ("swap", (0, 1), ())])  # c_ffi.rs:2371 |01> -> |10>
    assert abs(amp(o, 2) - 1) < EPS
    # custom 2q SWAP matrix with q1 high (c_ffi.rs:2168)
    sw = np.zeros((4, 4), complex)
    sw[0, 0] = sw[1, 2] = sw[2, 1] = sw[3, 3] = 1
    o = OracleState(2)
    o.apply([("x", (1,), ()), ("custom2", (1, 0), (), sw)])
    assert abs(amp(o, 1) - 1) < EPS and abs(amp(o, 2)) < EPS
    # GHZ (c_ffi.rs:2634)
    o = OracleState(3)
    o.apply([("h", (0,), ()), ("cx", (0, 1), ()), ("cx", (1, 2), ())])
    a = o.amplitudes()
    assert abs(a[0] - s2) < EPS and abs(a[7] - s2) < EPS


def test_known_answers_lib_rs():
    # Bell <ZZ> = <XX> = 1 (R/lib.rs:2560-2580)
    o = OracleState(2)
    o.apply([("h", (0,), ()), ("cx", (0, 1), ())])
    assert abs(o.pauli_string("ZZ") - 1) < EPS
    assert abs(o.pauli_string("XX") - 1) < EPS
    assert abs(o.pauli_string("YY") + 1) < EPS
    # <X> on |+> = 1
    o = OracleState(1)
    o.apply([("h", (0,), ())])
    assert abs(o.expectation_x(0) - 1) < EPS
    assert abs(o.pauli_string("X") - 1) < EPS
    # SX^2 = X
    o = OracleState(1)
    o.apply([("sx", (0,), ()), ("sx", (0,), ())])
    assert abs(abs(amp(o, 1)) - 1) < EPS
    # P(pi)|1> = -|1>
    o = OracleState(1)
    o.apply([("x", (0,), ()), ("p", (0,), (math.pi,))])
    assert abs(amp(o, 1) + 1) < EPS
    # iSWAP|01> = i|10>
    o = OracleState(2)
    o.apply([("x", (0,), ()), ("iswap", (0, 1), ())])
    assert abs(amp(o, 2) - 1j) < EPS
    # CCZ|111> = -|111>
    o = OracleState(3)
    o.apply([("x", (0,), ()), ("x", (1,), ()), ("x", (2,), ()), ("ccz", (0, 1, 2), ())])
    assert abs(amp(o, 7) + 1) < EPS


def test_expectations_consistent():
    rng = np.random.default_rng(5)
    n = 6
    o = OracleState(n)
    o.apply(circuits.brickwork(n, 4, seed=3))
    a = o.amplitudes()
    p = np.abs(a) ** 2
    z = o.expectation_z_all()
    for q in range(n):
        bits = (np.arange(1 << n) >> q) & 1
        assert abs(z[q] - np.sum(p * (1 - 2 * bits))) < 1e-12
        s = ["I"] * n
        s[q] = "Z"
        assert abs(o.pauli_string("".join(s)) - z[q]) < 1e-12
        s[q] = "X"
        assert abs(o.pauli_string("".join(s)) - o.expectation_x(q)) < 1e-12
        s[q] = "Y"
        assert abs(o.pauli_string("".join(s)) - o.expectation_y(q)) < 1e-12
    assert abs(o.norm() - 1) < 1e-12
    del rng


def test_xorshift_stream_and_sampling_rule():
    u1 = xorshift_uniforms(42, 100)
    u2 = xorshift_uniforms(42, 100)
    assert np.array_equal(u1, u2)  # seed determinism (c_ffi.rs:2478)
    assert np.all((u1 >= 0) & (u1 < 1))
    # seed 0 maps to the default state 0x853c49e6748fea9b (c_ffi.rs:1449)
    assert np.array_equal(xorshift_uniforms(0, 5), xorshift_uniforms(0x853c49e6748fea9b, 5))
    o = OracleState(2)
    o.apply([("h", (0,), ()), ("cx", (0, 1), ())])
    u = xorshift_uniforms(7, 2000)
    out = o.sample_uniforms(u)
    assert set(np.unique(out)) <= {0, 3}
    assert abs(np.mean(out == 0) - 0.5) < 0.05  # lib.rs 10000-shot 50/50 style check
    # first i with r < cumsum_i
    assert o.sample_uniforms([0.0])[0] == 0 and o.sample_uniforms([0.4999])[0] == 0
    assert o.sample_uniforms([0.5000001])[0] == 3 and o.sample_uniforms([1.5])[0] == 3


def test_flat_encoding_roundtrip_all_gates():
    # every gate of the set runs through the oracle and preserves the norm
    rng = np.random.default_rng(9)
    n = 5
    gates = []
    for name, ar in circuits.ARITY.items():
        qs = tuple(int(x) for x in rng.choice(n, size=ar, replace=False))
        if name == "custom1":
            q, _ = np.linalg.qr(rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2)))
            gates.append((name, qs, (), q))
        elif name in ("custom2", "u2lo"):
            q, _ = np.linalg.qr(rng.normal(size=(4, 4)) + 1j * rng.normal(size=(4, 4)))
            gates.append((name, qs, (), q))
        else:
            ps = tuple(float(x) for x in rng.uniform(0, 6, size=4))
            gates.append((name, qs, ps))
    o = OracleState(n)
    o.apply([("h", (q,), ()) for q in range(n)] + gates)
    assert abs(o.norm() - 1) < 1e-12
