"""CPU check of the tiled-pass planner: tests/plan_emulator.cpp executes the
planner's pass/stage/op tables with the kernel's index arithmetic (swizzled
slots, register blocks, affine write-back of deferred permutations) and the
result is compared with the oracle.  No GPU needed."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from nqpu_b200 import circuits
from oracle.oracle import OracleState

ROOT = Path(__file__).resolve().parent.parent
SO = ROOT / "tests" / "_build" / "libplanemu.so"


@pytest.fixture(scope="module")
def emu():
    SO.parent.mkdir(exist_ok=True)
    srcs = [ROOT / "tests" / "plan_emulator.cpp", ROOT / "nqpu_b200" / "csrc" / "planner.cpp",
            ROOT / "nqpu_b200" / "csrc" / "fusion.cpp"]
    deps = srcs + [ROOT / "nqpu_b200" / "csrc" / h for h in ("sv_types.h", "planner.h", "fusion.h")]
    if not SO.exists() or SO.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(ROOT / "nqpu_b200" / "csrc"),
                        *map(str, srcs), "-o", str(SO)], check=True)
    lib = C.CDLL(str(SO))
    lib.emu_run.restype = C.c_int
    lib.emu_run.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]
    lib.emu_fused.restype = C.c_int
    lib.emu_fused.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double)]
    return lib


def run_emu(lib, n, c64, gates):
    flat = np.ascontiguousarray(circuits.flatten(gates))
    st = np.zeros(2 << n)
    st[0] = 1.0
    rc = lib.emu_run(n, 1 if c64 else 0, flat.ctypes.data_as(C.POINTER(C.c_double)), len(flat),
                     st.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc >= 0
    return st.view(np.complex128), rc


def random_unitary(rng, d):
    q, r = np.linalg.qr(rng.normal(size=(d, d)) + 1j * rng.normal(size=(d, d)))
    return q * (np.diag(r) / np.abs(np.diag(r)))


def random_circuit(rng, n, g):
    names = [k for k in circuits.ARITY if circuits.ARITY[k] <= n and k != "u2lo"]
    gates = [("u3", (q,), tuple(rng.uniform(0, 6, 3))) for q in range(n)]
    for _ in range(g):
        name = names[int(rng.integers(len(names)))]
        qs = tuple(int(x) for x in rng.choice(n, size=circuits.ARITY[name], replace=False))
        if name == "custom1":
            gates.append((name, qs, (), random_unitary(rng, 2)))
        elif name == "custom2":
            gates.append((name, qs, (), random_unitary(rng, 4)))
        else:
            gates.append((name, qs, tuple(rng.uniform(-6, 6, 4))))
    return gates


def fid(a, b):
    return abs(np.vdot(a, b)) ** 2 / (np.vdot(a, a).real * np.vdot(b, b).real)


@pytest.mark.parametrize("c64", [False, True])
@pytest.mark.parametrize("n", [5, 6, 8, 12, 13, 14, 16])
def test_emulated_plan_random(emu, c64, n):
    rng = np.random.default_rng(500 + n + 100 * c64)
    gates = random_circuit(rng, n, 10 * n)
    got, _ = run_emu(emu, n, c64, gates)
    o = OracleState(n)
    o.apply(gates)
    assert 1 - fid(got, o.amplitudes()) <= (1e-6 if c64 else 1e-12)


@pytest.mark.parametrize("c64", [False, True])
def test_emulated_plan_brickwork_and_permutation_heavy(emu, c64):
    n = 15
    gates = circuits.brickwork(n, 12, 4)
    rng = np.random.default_rng(9)
    for _ in range(120):  # CNOT/X/SWAP-heavy tail exercises the deferred write-back
        kind = ["cx", "x", "swap", "cx", "u3"][int(rng.integers(5))]
        ar = circuits.ARITY[kind]
        qs = tuple(int(x) for x in rng.choice(n, size=ar, replace=False))
        gates.append((kind, qs, tuple(rng.uniform(0, 6, 3)) if kind == "u3" else ()))
    got, passes = run_emu(emu, n, c64, gates)
    o = OracleState(n)
    o.apply(gates)
    assert 1 - fid(got, o.amplitudes()) <= (1e-6 if c64 else 1e-12)
    assert passes >= 2


@pytest.mark.parametrize("c64", [False, True])
@pytest.mark.parametrize("n", [4, 5, 6, 7, 9])
def test_emulated_plan_many_seeds_small(emu, c64, n):
    if c64 and n < 5:
        pytest.skip("complex64 tiles need >= 5 qubits")
    for seed in range(25):
        rng = np.random.default_rng(10_000 + 97 * seed + n)
        gates = random_circuit(rng, n, 6 * n)
        got, _ = run_emu(emu, n, c64, gates)
        o = OracleState(n)
        o.apply(gates)
        assert 1 - fid(got, o.amplitudes()) <= (1e-6 if c64 else 1e-12), (seed, n, c64)


def run_fused(lib, n, gates):
    flat = np.ascontiguousarray(circuits.flatten(gates))
    st = np.zeros(2 << n)
    st[0] = 1.0
    nf = lib.emu_fused(n, flat.ctypes.data_as(C.POINTER(C.c_double)), len(flat), st.ctypes.data_as(C.POINTER(C.c_double)))
    return st.view(np.complex128), nf


@pytest.mark.parametrize("n", [5, 6, 9, 12])
def test_fusion_pass_matches_oracle(emu, n):
    rng = np.random.default_rng(77 + n)
    gates = random_circuit(rng, n, 12 * n)
    got, nf = run_fused(emu, n, gates)
    o = OracleState(n)
    o.apply(gates)
    assert 1 - fid(got, o.amplitudes()) <= 1e-12
    assert nf < len(gates)


def test_fusion_pass_tfim_cluster_sizes(emu):
    n = 12
    gates, _ = circuits.tfim_trotter(n, 10, seed=3)
    o = OracleState(n)
    o.set_basis(circuits.neel_index(n))
    o.apply(gates)
    flat = np.ascontiguousarray(circuits.flatten(gates))
    st = np.zeros(2 << n)
    st[2 * circuits.neel_index(n)] = 1.0
    nf = emu.emu_fused(n, flat.ctypes.data_as(C.POINTER(C.c_double)), len(flat), st.ctypes.data_as(C.POINTER(C.c_double)))
    assert 1 - fid(st.view(np.complex128), o.amplitudes()) <= 1e-12
    assert len(gates) / nf >= 4  # several gates per fused unitary


def test_split_tf32_product_accuracy():
    """The split-TF32 product used on the tensor cores (hi*hi + hi*lo + lo*hi,
    FP32 accumulation) keeps the relative error of a 64-term dot product near
    FP32 level, far below plain TF32."""
    rng = np.random.default_rng(1)

    def tf32(x):  # round to nearest, as the kernel splits
        b = np.asarray(x, np.float32).view(np.uint32)
        return ((b + np.uint32(0x1000)) & np.uint32(0xFFFFE000)).view(np.float32)

    a = rng.normal(size=(256, 64)).astype(np.float32)
    b = rng.normal(size=(64, 64)).astype(np.float32)
    ah, bh = tf32(a), tf32(b)
    al, bl = tf32(a - ah), tf32(b - bh)
    exact = a.astype(np.float64) @ b.astype(np.float64).T
    split = (ah.astype(np.float64) @ bh.T.astype(np.float64) + ah.astype(np.float64) @ bl.T.astype(np.float64)
             + al.astype(np.float64) @ bh.T.astype(np.float64))
    plain = ah.astype(np.float64) @ bh.T.astype(np.float64)
    rel = lambda x: np.abs(x - exact).max() / np.abs(exact).max()
    assert rel(split) < 5e-7
    assert rel(plain) > 20 * rel(split)
