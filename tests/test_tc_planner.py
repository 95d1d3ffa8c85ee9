"""CPU check of the tensor-core pass mode's planner and addressing.

tests/tc_emulator.cpp executes the planner's pass records (tcplan.cpp) with
the kernel's index arithmetic (tcpass.cu): operand images in the 128-byte
swizzled layout, B-operand copies, the split contraction and the epilogue's
offset tables.  In FP64 the result must equal the oracle to rounding; with the
kernel's FP16 hi/lo split it must stay within the complex64 tolerance.  Every
operand slot and amplitude is written exactly once per tile (the layouts are
bijections), and the 16-byte store pairings the kernel uses must hold."""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

from nqpu_b200 import circuits
from oracle.oracle import OracleState

ROOT = Path(__file__).resolve().parent.parent
SO = ROOT / "tests" / "_build" / "libtcemu.so"
CSRC = ROOT / "nqpu_b200" / "csrc"


@pytest.fixture(scope="module")
def emu():
    SO.parent.mkdir(exist_ok=True)
    srcs = [ROOT / "tests" / "tc_emulator.cpp", CSRC / "tcplan.cpp", CSRC / "planner.cpp", CSRC / "fusion.cpp"]
    deps = srcs + [CSRC / h for h in ("sv_types.h", "planner.h", "fusion.h", "tcpass.h")]
    if not SO.exists() or SO.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", str(CSRC), *map(str, srcs), "-o",
                        str(SO)], check=True)
    lib = C.CDLL(str(SO))
    lib.emu_tc_run.restype = C.c_int
    lib.emu_tc_run.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_int,
                               C.POINTER(C.c_int64)]
    lib.emu_half_bits.restype = C.c_uint16
    lib.emu_half_bits.argtypes = [C.c_float]
    return lib


def run_emu(lib, n, gates, split=False, init=None):
    flat = np.ascontiguousarray(circuits.flatten(gates))
    if init is None:
        st = np.zeros(2 << n)
        st[0] = 1.0
    else:
        st = np.ascontiguousarray(np.asarray(init, dtype=np.complex128).view(np.float64)).copy()
    stats = (C.c_int64 * 3)()
    rc = lib.emu_tc_run(n, flat.ctypes.data_as(C.POINTER(C.c_double)), len(flat),
                        st.ctypes.data_as(C.POINTER(C.c_double)), 1 if split else 0, stats)
    assert rc >= 0, rc
    return st.view(np.complex128), {"passes": stats[0], "unitaries": stats[1]}


def random_circuit(rng, n, g):
    names = [k for k in circuits.ARITY if k not in ("u2lo", "custom1", "custom2") and circuits.ARITY[k] <= n]
    gates = [("u3", (q,), tuple(rng.uniform(0, 6, 3))) for q in range(n)]
    for _ in range(g):
        name = names[int(rng.integers(len(names)))]
        qs = tuple(int(x) for x in rng.choice(n, size=circuits.ARITY[name], replace=False))
        gates.append((name, qs, tuple(float(x) for x in rng.uniform(-6, 6, 4))))
    return gates


@pytest.mark.parametrize("n,depth", [(12, 6), (13, 8), (14, 10), (16, 6)])
def test_brickwork_fp64_matches_oracle(emu, n, depth):
    gates = circuits.brickwork(n, depth, seed=n)
    got, st = run_emu(emu, n, gates)
    o = OracleState(n)
    o.apply(gates)
    assert np.abs(got - o.amplitudes()).max() < 1e-12
    assert st["unitaries"] <= 3 * st["passes"]  # at most three unitaries per pass


@pytest.mark.parametrize("n", [12, 13, 15])
def test_random_gates_fp64_matches_oracle(emu, n):
    rng = np.random.default_rng(40 + n)
    gates = random_circuit(rng, n, 10 * n)
    got, _ = run_emu(emu, n, gates)
    o = OracleState(n)
    o.apply(gates)
    assert np.abs(got - o.amplitudes()).max() < 1e-12


def test_qft_and_tfim_fp64(emu):
    n = 14
    rng = np.random.default_rng(5)
    prep = [("u3", (q,), tuple(rng.uniform(0, 6, 3))) for q in range(n)]
    for gates in (prep + circuits.qft(n), circuits.tfim_trotter(n, 4, seed=2)[0]):
        got, _ = run_emu(emu, n, gates)
        o = OracleState(n)
        o.apply(gates)
        assert np.abs(got - o.amplitudes()).max() < 1e-12


def test_half_rounding_matches_ieee(emu):
    # the planner's host FP16 conversion (unitary hi/lo parts) against numpy's
    rng = np.random.default_rng(3)
    vals = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.uniform(-9, 5, 4000),
                           [0.0, -0.0, 1.0, 65504.0, 65519.0, 65520.0, 1e6, 2.0 ** -24, 2.0 ** -25,
                            3 * 2.0 ** -26, 2.0 ** -14, 6.0e-8, -7.7e-5]]).astype(np.float32)
    got = np.array([emu.emu_half_bits(float(v)) for v in vals], dtype=np.uint16)
    with np.errstate(over="ignore"):
        want = vals.astype(np.float16).view(np.uint16)
    assert np.array_equal(got, want)


def test_fp16_split_within_complex64_tolerance(emu):
    n = 14
    gates = circuits.brickwork(n, 12, seed=3)
    got, _ = run_emu(emu, n, gates, split=True)
    o = OracleState(n)
    o.apply(gates)
    ref = o.amplitudes()
    fid = abs(np.vdot(ref, got)) ** 2 / np.vdot(got, got).real
    assert 1 - fid < 1e-6


def test_nonnormalised_input_state(emu):
    # the planner and addressing do not assume a normalised or basis input
    n = 13
    rng = np.random.default_rng(9)
    init = 0.3 * (rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n))
    gates = circuits.brickwork(n, 4, seed=1)
    got, _ = run_emu(emu, n, gates, init=init)
    o = OracleState(n)
    o.set_amplitudes(init)
    o.apply(gates)
    assert np.abs(got - o.amplitudes()).max() < 1e-12


def store_lines(lib, n, gates):
    lib.emu_tc_store_lines.restype = C.c_int
    lib.emu_tc_store_lines.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int64)]
    flat = np.ascontiguousarray(circuits.flatten(gates))
    out = (C.c_int64 * 3)()
    npass = lib.emu_tc_store_lines(n, flat.ctypes.data_as(C.POINTER(C.c_double)), len(flat), out)
    assert npass > 0
    return out[0] / npass, out[1] / npass, out[2]


@pytest.mark.parametrize("n,depth", [(26, 10), (30, 40)])
def test_lane_exchanges_coalesce_the_last_epilogue_stores(emu, n, depth):
    # a warp store of the last epilogue touches 2^k 128-byte lines (k lane bits
    # on index bits >= 4); the lane exchanges bring the plan near the minimum
    # of 4 (16-byte stores) / 2 (8-byte stores)
    with_x, without_x, exchanges = store_lines(emu, n, circuits.brickwork(n, depth, seed=1))
    assert exchanges > 0
    assert with_x <= 4.0 and with_x < 0.5 * without_x, (with_x, without_x)


@pytest.mark.parametrize("n,seed", [(14, 5), (15, 6)])
def test_lane_exchanges_keep_fp64_parity(emu, n, seed):
    # the emulator replays the kernel's register exchange: parity with the
    # oracle on circuits whose plans make exchanges
    gates = circuits.brickwork(n, 10, seed=seed)
    assert store_lines(emu, n, gates)[2] > 0
    got, _ = run_emu(emu, n, gates)
    o = OracleState(n)
    o.apply(gates)
    assert np.abs(got - o.amplitudes()).max() < 1e-12


def test_raw_landing_is_a_half_preserving_bijection(emu):
    # the two-phase split's landing offsets, on random layouts: distinct
    # 16-byte slots, and each half's raw chunks only where its own outputs go
    emu.emu_tc_raw_landing.restype = C.c_int
    emu.emu_tc_raw_landing.argtypes = [C.c_int, C.c_uint64]
    valid = emu.emu_tc_raw_landing(4000, 12345)
    assert valid > 500, valid
