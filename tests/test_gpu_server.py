"""GPU tests of the serving request loop (continuous batching of mixed-size
circuits on device-resident complex64 states).

Tolerance: each request's result is bitwise the same whether it runs alone or
in a mix, and bitwise the same as the state API run in NQPU_MODE_AUTO (the
server makes the same engine choice: same plan, same kernels, same launch
shapes, same seeded uniforms); against the FP64 oracle, max |d<Z_i>| <= 1e-5
(the complex64 bar)."""
import numpy as np
import pytest

from nqpu_b200 import _lib, circuits
from nqpu_b200.server import Server
from nqpu_b200.state import Circuit, StateVector
from oracle.oracle import OracleState

pytestmark = pytest.mark.gpu


def mix(count, seed, nmin=5, nmax=18, dmin=3, dmax=12):
    reqs = circuits.serving_mix(count, seed, rate=1000.0, nmin=nmin, nmax=nmax, dmin=dmin, dmax=dmax)
    for r in reqs:
        r["gates"] = circuits.brickwork(r["n"], r["depth"], r["seed"])
        r["shots"] = 256 if r["kind"] == "shots" else 0
    return reqs


def run_all(server, reqs):
    ids = []
    for r in reqs:
        c = Circuit(r["n"], r["gates"])
        ids.append(server.submit(c, r["kind"], r["shots"], r["seed"]))
        c.close()  # the server copied the circuit
    server.wait(0, 120.0)
    return [server.result(i)[0] for i in ids]


def test_results_same_alone_in_mix_and_as_state_api():
    reqs = mix(48, seed=2)
    # tight budget: 8 blocks of the largest state, so admission has to wait for memory
    with Server(hbm_budget_bytes=8 << 21, max_qubits=18, lanes=12, large_lanes=2, large_qubits=15,
                max_shots=1024) as srv:
        in_mix = run_all(srv, reqs)
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["failed"] == 0
        assert st["peak_concurrent"] > 1  # requests overlapped on the device
        assert st["peak_resident_bytes"] <= st["arena_bytes"]
    lib = _lib.load()
    for r, got in zip(reqs, in_mix):
        with Server(hbm_budget_bytes=1 << 21, max_qubits=18, lanes=1, large_lanes=1, max_shots=1024) as solo:
            alone = run_all(solo, [r])[0]
        assert np.array_equal(alone, got), r
        with StateVector(r["n"], "c64") as sv:
            Circuit(r["n"], r["gates"]).execute(sv, "auto")
            if r["kind"] == "zall":
                ref = sv.expectation_z_all()
            else:
                lib.nqpu_set_seed(r["seed"])
                ref = sv.sample(r["shots"])
        assert np.array_equal(np.asarray(ref, dtype=got.dtype), got), r


def test_zall_matches_fp64_oracle():
    reqs = [r for r in mix(30, seed=5, nmin=5, nmax=12) if r["kind"] == "zall"]
    with Server(hbm_budget_bytes=1 << 24, max_qubits=12) as srv:
        out = run_all(srv, reqs)
    for r, z in zip(reqs, out):
        o = OracleState(r["n"])
        o.apply(r["gates"])
        assert np.abs(z - o.expectation_z_all()).max() <= 1e-5


def test_budget_bounds_resident_states():
    n = 16
    reqs = [{"n": n, "gates": circuits.brickwork(n, 6, s), "kind": "zall", "shots": 0, "seed": s} for s in range(10)]
    block = (1 << n) * 8
    with Server(hbm_budget_bytes=2 * block, max_qubits=n, lanes=8, large_lanes=8, large_qubits=n) as srv:
        out = run_all(srv, reqs)
        st = srv.stats()
    assert st["arena_bytes"] == 2 * block
    assert st["peak_resident_bytes"] <= 2 * block and st["peak_concurrent"] <= 2
    assert all(np.isfinite(z).all() for z in out)


def test_rejects_invalid_requests():
    with Server(hbm_budget_bytes=1 << 22, max_qubits=16, max_shots=64) as srv:
        big = Circuit(17, [("h", (0,), ())])
        with pytest.raises(RuntimeError):
            srv.submit(big, "zall")
        ok = Circuit(8, [("h", (0,), ())])
        with pytest.raises(RuntimeError):
            srv.submit(ok, "shots", shots=65)
        rid = srv.submit(ok, "shots", shots=64, seed=3)
        srv.wait(rid, 30.0)
        vals, t = srv.result(rid)
        assert vals.shape == (64,) and set(np.unique(vals)) <= {0, 1}
        assert t["total_ms"] >= t["running_ms"] >= 0
