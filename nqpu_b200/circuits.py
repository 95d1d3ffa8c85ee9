"""Gate lists and the seeded synthetic workloads.

A gate is `(name, qubits, params)` like the reference Python SDK's
`GateOperation(name, qubits, params)` (sdk/python/nqpu/core/simulator.py:22), with
an optional fourth element holding a custom matrix.  Names cover the reference's
GateType set (sdk/rust/src/core/gates/gates.rs:8-62).

Workloads (synthetic, seeded with numpy's PCG64 `default_rng`; draw order documented
per generator) stand in for the configurations the engine is measured on:
  * `brickwork`: U3(theta, phi, lambda) on every qubit then CNOTs on alternating
    even/odd neighbour pairs, per layer; theta~U[0,pi], phi,lambda~U[0,2pi).
  * `tfim_trotter`: first-order Trotterised 1D transverse-field Ising evolution,
    open chain: RZZ(2 J dt) on every bond then RX(2 h_i dt) on every site.
  * `hea`: hardware-efficient ansatz, RY(theta) RZ(phi) on all qubits + CZ ladder.
  * `serving_mix`: Poisson arrivals of brickwork requests of log-uniform size.
  * `qft`: the quantum Fourier transform (H + controlled-phase chains + SWAPs).
"""
from __future__ import annotations

import math

import numpy as np

# Circuit-level gate codes shared with the oracle's flat encoding.
GATE_CODES = {
    "h": 0, "x": 1, "y": 2, "z": 3, "s": 4, "t": 5, "sx": 6, "rx": 7, "ry": 8, "rz": 9, "p": 10,
    "u3": 11, "cx": 12, "cz": 13, "swap": 14, "iswap": 15, "cp": 16, "crx": 17, "cry": 18,
    "crz": 19, "rzz": 20, "rxx": 21, "ryy": 22, "ccx": 23, "ccz": 24, "cswap": 25,
    "custom1": 26, "custom2": 27, "u2lo": 28, "cu": 29, "measure": 30, "reset": 31,
}
# Mid-circuit measurement and reset (circuit-level, one qubit, no parameters);
# ARITY covers the unitary gates only.
MID_GATES = ("measure", "reset")
ARITY = {name: (3 if name in ("ccx", "ccz", "cswap") else
                2 if name in ("cx", "cz", "swap", "iswap", "cp", "crx", "cry", "crz", "rzz", "rxx",
                              "ryy", "custom2", "u2lo", "cu") else 1)
         for name in GATE_CODES if name not in MID_GATES}

NPARAMS = {name: 0 for name in GATE_CODES}
NPARAMS.update({"rx": 1, "ry": 1, "rz": 1, "p": 1, "u3": 3, "cp": 1, "crx": 1, "cry": 1, "crz": 1,
                "rzz": 1, "rxx": 1, "ryy": 1, "cu": 4})

FLAT_WIDTH = 40  # code, q0, q1, q2, p0..p3, 16 complex matrix entries (re, im)


def flatten(gates) -> np.ndarray:
    """Flat float64 encoding [G, 40] consumed by the oracle."""
    out = np.zeros((len(gates), FLAT_WIDTH), dtype=np.float64)
    for i, g in enumerate(gates):
        name, qs, ps = g[0], g[1], g[2]
        out[i, 0] = GATE_CODES[name]
        out[i, 1:1 + len(qs)] = qs
        ps = tuple(ps)[:NPARAMS[name]]
        out[i, 4:4 + len(ps)] = ps
        if len(g) > 3 and g[3] is not None:
            m = np.asarray(g[3], dtype=np.complex128).reshape(-1)
            out[i, 8:8 + 2 * len(m):2] = m.real
            out[i, 9:9 + 2 * len(m):2] = m.imag
    return out


def count_gates(gates) -> int:
    return len(gates)


def algorithmic_bytes(gates, n: int, amp_bytes: int) -> int:
    """Bytes a per-gate pass moves: dense 1q/2q and full diagonals 2S, phase on
    the |1> half S, CNOT/SWAP-like S, CZ/CPhase S/2 (S = 2^n * amp_bytes)."""
    S = (1 << n) * amp_bytes
    tot = 0
    for g in gates:
        name = g[0]
        if name in ("z", "s", "t", "p", "x"):
            tot += S if name != "x" else 2 * S
        elif name in ("cx", "swap"):
            tot += S
        elif name in ("cz", "cp"):
            tot += S // 2
        elif name in ("ccx", "cswap"):
            tot += S // 2
        elif name == "ccz":
            tot += S // 4
        else:
            tot += 2 * S
    return tot


def algorithmic_flops(gates, n: int) -> int:
    """FP32 flops (an FMA counts two) of the plainest formulation of each gate:
    a dense 2x2 complex matrix on an amplitude pair takes 8 FMAs per output
    amplitude (16 flops), a full diagonal one complex product per amplitude (8),
    a phase on the |1> half 4 per amplitude, a controlled dense 1q gate 8, a
    dense 4x4 32; permutations and sign flips (X, CNOT, SWAP, Z, CZ, Toffoli,
    CCZ, CSWAP) none."""
    per_amp = {"z": 0, "x": 0, "cx": 0, "swap": 0, "cz": 0, "ccx": 0, "ccz": 0, "cswap": 0,
               "s": 4, "t": 4, "p": 4, "cp": 2, "rz": 8, "rzz": 8,
               "crx": 8, "cry": 8, "crz": 4, "cu": 8,
               "iswap": 32, "rxx": 32, "ryy": 32, "custom2": 32}
    return sum(per_amp.get(g[0], 16) for g in gates) << n


# ---------------------------------------------------------------------------
# Workload generators
# ---------------------------------------------------------------------------

def brickwork(n: int, layers: int, seed: int):
    """Random brickwork circuit.  Draw order: for each layer, for each qubit
    q = 0..n-1: theta, phi, lambda (three uniform draws).  Layer l applies U3 on
    every qubit, then CNOT(2k, 2k+1) for even l and CNOT(2k+1, 2k+2) for odd l."""
    rng = np.random.default_rng(seed)
    gates = []
    for layer in range(layers):
        draws = rng.random((n, 3))
        for q in range(n):
            th = math.pi * draws[q, 0]
            ph = 2 * math.pi * draws[q, 1]
            la = 2 * math.pi * draws[q, 2]
            gates.append(("u3", (q,), (th, ph, la)))
        start = 0 if layer % 2 == 0 else 1
        for a in range(start, n - 1, 2):
            gates.append(("cx", (a, a + 1), ()))
    return gates


def tfim_trotter(n: int, steps: int, seed: int, J: float = 1.0, dt: float = 0.05,
                 hmin: float = 0.6, hmax: float = 1.0):
    """Trotter steps of H = J sum Z_i Z_{i+1} + sum h_i X_i (open chain); h_i ~ U[hmin, hmax]
    drawn once (i = 0..n-1).  Each step: RZZ(2 J dt) on bonds (i, i+1), then RX(2 h_i dt)."""
    rng = np.random.default_rng(seed)
    h = hmin + (hmax - hmin) * rng.random(n)
    step = []
    for i in range(n - 1):
        step.append(("rzz", (i, i + 1), (2.0 * J * dt,)))
    for i in range(n):
        step.append(("rx", (i,), (2.0 * float(h[i]) * dt,)))
    return step * steps, h


def qft(n: int):
    """Quantum Fourier transform (no input state preparation): for i = n-1..0,
    H(i) then controlled phases CP(pi / 2^(i-j)) from qubit j < i onto i, then
    the qubit-order reversal by n/2 SWAPs.  n(n+1)/2 + n/2 gates."""
    gates = []
    for i in range(n - 1, -1, -1):
        gates.append(("h", (i,), ()))
        for j in range(i - 1, -1, -1):
            gates.append(("cp", (j, i), (math.pi / 2 ** (i - j),)))
    for i in range(n // 2):
        gates.append(("swap", (i, n - 1 - i), ()))
    return gates


def neel_index(n: int) -> int:
    """Basis index of the Neel state |0101...>: qubit i is i mod 2 (qubit 0 = 0)."""
    return sum(1 << i for i in range(n) if i % 2 == 1)


def hea(n: int, layers: int, rng: np.random.Generator):
    """Hardware-efficient ansatz: per layer RY(theta_q) RZ(phi_q) on every qubit
    (draw order q-major: theta, phi), then CZ(q, q+1) for q = 0..n-2."""
    gates = []
    for _ in range(layers):
        ang = 2 * math.pi * rng.random((n, 2))
        for q in range(n):
            gates.append(("ry", (q,), (float(ang[q, 0]),)))
            gates.append(("rz", (q,), (float(ang[q, 1]),)))
        for q in range(n - 1):
            gates.append(("cz", (q, q + 1), ()))
    return gates


def hea_arrays(n: int, layers: int, rng: np.random.Generator):
    """hea() as flat arrays (codes [G], qubits [G, 3], params [G, 4]) for
    Circuit.from_arrays, with the same draws and gate order."""
    per = 3 * n - 1
    codes = np.empty(layers * per, dtype=np.uint32)
    qs = np.zeros((layers * per, 3), dtype=np.int32)
    ps = np.zeros((layers * per, 4), dtype=np.float64)
    q = np.arange(n)
    for layer in range(layers):
        ang = 2 * math.pi * rng.random((n, 2))
        b = layer * per
        codes[b:b + 2 * n:2] = GATE_CODES["ry"]
        codes[b + 1:b + 2 * n:2] = GATE_CODES["rz"]
        qs[b:b + 2 * n:2, 0] = q
        qs[b + 1:b + 2 * n:2, 0] = q
        ps[b:b + 2 * n:2, 0] = ang[:, 0]
        ps[b + 1:b + 2 * n:2, 0] = ang[:, 1]
        codes[b + 2 * n:b + per] = GATE_CODES["cz"]
        qs[b + 2 * n:b + per, 0] = q[:-1]
        qs[b + 2 * n:b + per, 1] = q[1:]
    return codes, qs, ps


def ising_hamiltonian(n: int, rng: np.random.Generator):
    """H = sum_i J_i Z_i Z_{i+1} + sum_i h_i X_i with J_i, h_i ~ U[-1, 1]."""
    J = rng.uniform(-1.0, 1.0, n - 1)
    h = rng.uniform(-1.0, 1.0, n)
    return J, h


def hea_batch(count: int, seed: int, nmin: int = 10, nmax: int = 22, lmin: int = 2, lmax: int = 12,
              arrays: bool = False):
    """Batch of HEA circuits with their Ising Hamiltonians.  Per circuit, draw
    order: n ~ U{nmin..nmax}, L ~ U{lmin..lmax}, the ansatz angles, then J, h.
    arrays=True gives each circuit as hea_arrays' (codes, qubits, params)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        L = int(rng.integers(lmin, lmax + 1))
        g = hea_arrays(n, L, rng) if arrays else hea(n, L, rng)
        J, h = ising_hamiltonian(n, rng)
        out.append((n, g, J, h))
    return out


def serving_mix(count: int, seed: int, rate: float, nmin: int = 8, nmax: int = 28,
                dmin: int = 10, dmax: int = 50):
    """Request stream: arrival times (Poisson, exponential gaps at `rate`/s),
    n = round(exp(U[ln nmin, ln nmax])), brickwork depth ~ U{dmin..dmax}, and half
    the requests ask for 1024 shots, half for all <Z_i>."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        depth = int(rng.integers(dmin, dmax + 1))
        kind = "shots" if rng.random() < 0.5 else "zall"
        cseed = int(rng.integers(0, 2**31 - 1))
        reqs.append({"id": i, "arrival": t, "n": n, "depth": depth, "kind": kind, "seed": cseed})
    return reqs
