"""OpenQASM 2.0 import/export (nqpu_circuit_from_qasm / nqpu_circuit_to_qasm).

The reference's parser (circuits/formats/qasm.rs:65, tests :529-576) reads qreg /
creg declarations, gate statements and measurements; these tests restate its
import test (a Bell circuit with a register-level measure) and add the gates
of qelib1.inc, parameter expressions, broadcasting, error reporting and the
export round trip.  The CPU tests need no GPU (parsing and export are host
code); the GPU test runs a parsed circuit against the oracle."""
import math

import numpy as np
import pytest

from nqpu_b200 import circuits
from nqpu_b200.state import Circuit, StateVector

BELL = """
OPENQASM 2.0;
include "qelib1.inc";
qreg q[2];
creg c[2];
h q[0];
cx q[0],q[1];
measure q -> c;
"""


def test_reference_import_example():
    c = Circuit.from_qasm(BELL)
    assert c.num_qubits == 2
    assert c.gate_count == 4  # h, cx, measure q[0], measure q[1] (qasm.rs:556)
    out = c.to_qasm()
    assert "h q[0];" in out and "cx q[0],q[1];" in out
    assert "creg c[2];" in out and "measure q[1] -> c[1];" in out


def test_gate_set_expressions_and_broadcast():
    text = """OPENQASM 2.0;
include "qelib1.inc";
qreg a[2]; qreg b[2];
creg m[4];
u3(pi/2, -pi/4, 2*pi/3) a[0];
u2(0, pi) a[1];
u1(pi^2/10) b[0];
sdg b[1]; tdg a[0]; sx a[1]; sxdg b[0];
rx(-(pi - 0.5)) a[0]; ry(1e-1) a[1]; rz(.25) b[1];
cy a[0], b[0]; ch a[1], b[1]; cu3(0.1, 0.2, 0.3) b[0], a[0]; cu(0.1, 0.2, 0.3, 0.4) a[1], b[1];
crx(0.7) a[0],a[1]; cry(0.7) a[0],a[1]; crz(0.7) a[0],a[1]; cp(0.3) b[0],b[1];
rzz(0.2) a[0],b[1]; rxx(0.2) a[1],b[0]; ryy(0.2) a[0],b[0]; swap a[0],b[1]; iswap a[1],b[0];
ccx a[0],a[1],b[0]; ccz a[0],b[0],b[1]; cswap b[1],a[0],a[1];
h a;
cx a, b;
id b[0];
barrier a, b;
measure a[0] -> m[0];
"""
    c = Circuit.from_qasm(text)
    assert c.num_qubits == 4
    # 3 + 4 + 3 + 4 + 4 + 5 + 3 + 2 (h a) + 2 (cx a, b pairwise) + 1 measure
    assert c.gate_count == 31
    out = c.to_qasm()
    assert "u3(1.5707963267948966,-0.78539816339744828,2.0943951023931953) q[0];" in out
    assert "u3(1.5707963267948966,0,3.1415926535897931) q[1];" in out  # u2(phi, lambda)
    assert "p(-1.5707963267948966) q[3];" in out  # sdg on b[1] = q[3]
    assert "cx q[0],q[2];" in out and "cx q[1],q[3];" in out
    assert "h q[0];" in out and "h q[1];" in out
    # custom (sxdg) has no OpenQASM 2.0 form on export: a comment line
    assert "// gate code" in out


@pytest.mark.parametrize("bad,line", [
    ("qreg q[2];\nfoo q[0];\n", 2),
    ("qreg q[2];\nh q[2];\n", 2),
    ("qreg q[2];\nh r[0];\n", 2),
    ("qreg q[2];\ncx q[0],q[0];\n", 2),
    ("qreg q[2];\n\nrx(pi/0) q[0];\n", 3),
    ("qreg q[2];\nrx(theta) q[0];\n", 2),
    ("qreg q[2];\ngate foo a { h a; }\n", 2),
    ("qreg q[2];\nh q[0]\n", 3),
])
def test_errors_report_line(bad, line):
    from nqpu_b200 import _lib
    import ctypes as C
    lib = _lib.load()
    ln = C.c_uint32()
    assert not lib.nqpu_circuit_from_qasm(bad.encode(), C.byref(ln))
    assert ln.value == line


def test_export_round_trip():
    g = circuits.brickwork(6, 5, seed=4) + [("cp", (0, 3), (0.3,)), ("crz", (2, 5), (1.1,)), ("rzz", (1, 4), (0.7,)),
                                           ("ccx", (0, 1, 2), ()), ("cswap", (3, 4, 5), ()), ("sx", (2,), ())]
    c = Circuit(6, g)
    text = c.to_qasm()
    c2 = Circuit.from_qasm(text)
    assert c2.num_qubits == 6 and c2.gate_count == c.gate_count
    assert c2.to_qasm() == text


@pytest.mark.gpu
def test_parsed_circuit_matches_oracle():
    from oracle.oracle import OracleState
    n = 7
    lines = ["OPENQASM 2.0;", 'include "qelib1.inc";', f"qreg q[{n}];"]
    gates = []
    rng = np.random.default_rng(3)
    for _ in range(60):
        a, b = (int(x) for x in rng.choice(n, 2, replace=False))
        t = float(rng.uniform(-3, 3))
        kind = int(rng.integers(6))
        if kind == 0:
            lines.append(f"u3({t},{t / 2},{-t / 3}) q[{a}];")
            gates.append(("u3", (a,), (t, t / 2, -t / 3)))
        elif kind == 1:
            lines.append(f"cx q[{a}],q[{b}];")
            gates.append(("cx", (a, b), ()))
        elif kind == 2:
            lines.append(f"cu1({t}) q[{a}],q[{b}];")
            gates.append(("cp", (a, b), (t,)))
        elif kind == 3:
            lines.append(f"sdg q[{a}];")
            gates.append(("p", (a,), (-math.pi / 2,)))
        elif kind == 4:
            lines.append(f"rzz({t}) q[{a}],q[{b}];")
            gates.append(("rzz", (a, b), (t,)))
        else:
            lines.append(f"h q[{a}];")
            gates.append(("h", (a,), ()))
    c = Circuit.from_qasm("\n".join(lines))
    for dtype, tol in (("c128", 1e-12), ("c64", 1e-5)):
        sv = StateVector(n, dtype)
        c.execute(sv, "tiled")
        o = OracleState(n)
        o.apply(gates)
        assert np.abs(sv.amplitudes() - o.amplitudes()).max() < tol
        sv.close()
