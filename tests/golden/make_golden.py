"""Generate golden statevectors with the reference's own Python statevector.

The reference's numpy path (sdk/python/nqpu/core/simulator.py:193-295:
`_apply_single_qubit_gate`, `_apply_two_qubit_gate`, `_single_qubit_matrix`) is
imported from the reference checkout and run on seeded random circuits over its
gate set (h x y z s t rx ry rz cx cz swap).  The final statevectors are stored in
golden_statevectors.npz next to this script together with the gate lists, so the
oracle and the engine can be checked against them without the reference present.

    python tests/golden/make_golden.py /path/to/reference
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
GATESET_1Q = ["h", "x", "y", "z", "s", "t", "rx", "ry", "rz"]
GATESET_2Q = ["cx", "cz", "swap"]


def random_circuit(n: int, ngates: int, rng: np.random.Generator):
    gates = []
    for _ in range(ngates):
        if n >= 2 and rng.random() < 0.35:
            name = GATESET_2Q[int(rng.integers(len(GATESET_2Q)))]
            a, b = rng.choice(n, size=2, replace=False)
            gates.append((name, (int(a), int(b)), ()))
        else:
            name = GATESET_1Q[int(rng.integers(len(GATESET_1Q)))]
            q = int(rng.integers(n))
            params = (float(rng.uniform(-2 * math.pi, 2 * math.pi)),) if name in ("rx", "ry", "rz") else ()
            gates.append((name, (q,), params))
    return gates


def main(ref_root: str) -> None:
    sys.path.insert(0, str(Path(ref_root) / "sdk" / "python"))
    from nqpu.core import simulator as S  # the reference implementation

    cases = []
    rng = np.random.default_rng(20261203)
    for n, ngates in [(1, 12), (2, 20), (3, 30), (4, 40), (5, 60), (6, 60), (8, 80), (10, 100)]:
        for rep in range(2):
            gates = random_circuit(n, ngates, rng)
            state = np.zeros(1 << n, dtype=np.complex128)
            state[0] = 1.0
            for name, qs, ps in gates:
                op = S.GateOperation(name=name, qubits=tuple(qs), params=tuple(ps))
                if len(qs) == 1:
                    state = S._apply_single_qubit_gate(state, n, op)
                else:
                    state = S._apply_two_qubit_gate(state, op)
            cases.append({"n": n, "gates": gates, "state": state})

    arrays = {}
    meta = []
    for i, c in enumerate(cases):
        arrays[f"state_{i}"] = c["state"]
        meta.append({"n": c["n"], "gates": [[g[0], list(g[1]), list(g[2])] for g in c["gates"]]})
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(HERE / "golden_statevectors.npz", **arrays)
    print(f"wrote {len(cases)} cases")


def load():
    """Return [(n, gates, state)] from the committed fixture."""
    z = np.load(HERE / "golden_statevectors.npz")
    meta = json.loads(bytes(z["meta"]).decode())
    out = []
    for i, m in enumerate(meta):
        gates = [(g[0], tuple(g[1]), tuple(g[2])) for g in m["gates"]]
        out.append((m["n"], gates, z[f"state_{i}"]))
    return out


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
