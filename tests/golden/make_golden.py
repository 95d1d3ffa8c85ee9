"""Generate golden statevectors with the reference's own Python statevector.

The reference's numpy path (sdk/python/nqpu/core/simulator.py:193-295:
`_apply_single_qubit_gate`, `_apply_two_qubit_gate`, `_single_qubit_matrix`) is
imported from a reference checkout and run on seeded random circuits.  Two
fixtures are written next to this script, each with its gate lists, so the
oracle and the engine can be checked against them without the reference:

* golden_statevectors.npz — the reference's gate set (h x y z s t rx ry rz cx
  cz swap);
* golden_u3_rzz.npz — the same gate set plus U3(theta, phi, lambda) and
  RZZ(theta), the gates of the brickwork and Trotter workloads.  The reference
  Python statevector has neither, so it runs them through identities of its
  own gates: U3 = Rz(phi) Ry(theta) Rz(lambda) up to the global phase
  e^{i(phi+lambda)/2} (the nQPU U3 matrix, ascii_viz.rs:134-150), and
  RZZ(theta) = CX(a,b) Rz_b(theta) CX(a,b) exactly (GateType::RZZ,
  gates.rs:486, diag(e^{-i t/2}, e^{i t/2}, e^{i t/2}, e^{-i t/2})).  The
  stored gate lists name u3 and rzz, so a consumer applies them directly and
  compares up to one global phase (U3 cases) or exactly.

    python tests/golden/make_golden.py <reference checkout>
    NQPU_REFERENCE=<reference checkout> python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GATESET_1Q = ["h", "x", "y", "z", "s", "t", "rx", "ry", "rz"]
GATESET_2Q = ["cx", "cz", "swap"]


def random_circuit(n: int, ngates: int, rng: np.random.Generator, extra: bool = False, u3: bool = True):
    one = GATESET_1Q + (["u3", "u3", "u3"] if extra and u3 else [])
    two = GATESET_2Q + (["rzz", "rzz"] if extra else [])
    gates = []
    for _ in range(ngates):
        if n >= 2 and rng.random() < 0.35:
            name = two[int(rng.integers(len(two)))]
            a, b = rng.choice(n, size=2, replace=False)
            params = (float(rng.uniform(-2 * math.pi, 2 * math.pi)),) if name == "rzz" else ()
            gates.append((name, (int(a), int(b)), params))
        else:
            name = one[int(rng.integers(len(one)))]
            q = int(rng.integers(n))
            if name in ("rx", "ry", "rz"):
                params = (float(rng.uniform(-2 * math.pi, 2 * math.pi)),)
            elif name == "u3":
                params = (float(rng.uniform(0, math.pi)), float(rng.uniform(0, 2 * math.pi)),
                          float(rng.uniform(0, 2 * math.pi)))
            else:
                params = ()
            gates.append((name, (q,), params))
    return gates


def reference_ops(name, qs, ps):
    """The gate as a sequence of the reference Python statevector's own gates."""
    if name == "u3":
        th, ph, la = ps
        q = qs[0]
        return [("rz", (q,), (la,)), ("ry", (q,), (th,)), ("rz", (q,), (ph,))]
    if name == "rzz":
        a, b = qs
        return [("cx", (a, b), ()), ("rz", (b,), (ps[0],)), ("cx", (a, b), ())]
    return [(name, qs, ps)]


def run_reference(S, n, gates):
    state = np.zeros(1 << n, dtype=np.complex128)
    state[0] = 1.0
    for g in gates:
        for name, qs, ps in reference_ops(*g):
            op = S.GateOperation(name=name, qubits=tuple(qs), params=tuple(ps))
            if len(qs) == 1:
                state = S._apply_single_qubit_gate(state, n, op)
            else:
                state = S._apply_two_qubit_gate(state, op)
    return state


def save(path: Path, cases) -> None:
    arrays = {}
    meta = []
    for i, c in enumerate(cases):
        arrays[f"state_{i}"] = c["state"]
        meta.append({"n": c["n"], "gates": [[g[0], list(g[1]), list(g[2])] for g in c["gates"]]})
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path, **arrays)
    print(f"wrote {len(cases)} cases to {path.name}")


def main(ref_root: str) -> None:
    sys.path.insert(0, str(Path(ref_root) / "sdk" / "python"))
    from nqpu.core import simulator as S  # the reference implementation

    sizes = [(1, 12), (2, 20), (3, 30), (4, 40), (5, 60), (6, 60), (8, 80), (10, 100)]
    cases = []
    rng = np.random.default_rng(20261203)
    for n, ngates in sizes:
        for rep in range(2):
            gates = random_circuit(n, ngates, rng)
            cases.append({"n": n, "gates": gates, "state": run_reference(S, n, gates)})
    save(HERE / "golden_statevectors.npz", cases)

    cases = []
    rng = np.random.default_rng(20261204)
    for n, ngates in sizes + [(12, 120)]:
        for rep in range(2):
            gates = random_circuit(n, ngates, rng, extra=True)
            cases.append({"n": n, "gates": gates, "state": run_reference(S, n, gates)})
    # RZZ without U3: no global-phase freedom, compared exactly
    for n, ngates in [(3, 30), (5, 60), (8, 80), (10, 100)]:
        gates = random_circuit(n, ngates, rng, extra=True, u3=False)
        cases.append({"n": n, "gates": gates, "state": run_reference(S, n, gates)})
    save(HERE / "golden_u3_rzz.npz", cases)


def _load(path: Path):
    z = np.load(path)
    meta = json.loads(bytes(z["meta"]).decode())
    out = []
    for i, m in enumerate(meta):
        gates = [(g[0], tuple(g[1]), tuple(g[2])) for g in m["gates"]]
        out.append((m["n"], gates, z[f"state_{i}"]))
    return out


def load():
    """Return [(n, gates, state)] from the reference-gate-set fixture."""
    return _load(HERE / "golden_statevectors.npz")


def load_u3_rzz():
    """Return [(n, gates, state)] from the U3/RZZ fixture (U3 cases agree with
    the nQPU U3 matrix up to one global phase per circuit)."""
    return _load(HERE / "golden_u3_rzz.npz")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NQPU_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout> (or set NQPU_REFERENCE)")
    main(root)
