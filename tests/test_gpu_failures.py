"""The engine's bounded waits and timeouts fire, report an error status, and
leave the process usable.

The reference falls back silently to its CPU path on any GPU error
(sdk/rust/src/backends/runtime/auto_simulator.rs:1058-1063); this engine has no
fallback, so its failure statuses must be shown to fire.  Every failure here is
made on the host, never by faulting the GPU:

* batch: the host leaves one pass tile out of the task queue
  (NQPU_BATCH_DROP_TILE), so the next pass's tiles wait on a completion counter
  that never fills; with a short poll limit (NQPU_BATCH_SPIN_LIMIT) their
  bounded waits expire, every CTA stops, and nqpu_batch_run returns
  NQPU_SIMULATION_FAILED.  The same handle, reconfigured, then runs normally.
* server: nqpu_server_wait with a timeout shorter than the request returns
  NQPU_SIMULATION_FAILED and the request still completes; nqpu_server_cancel
  withdraws a queued request.
* tensor passes: nqpu_tensor_wait_limit_set(64, 1) points every engine's first
  wait for its MMAs at a barrier nothing arrives on; the waits expire after 64
  polls, each engine waits out its MMAs in flight and stops, and the run
  returns NQPU_SIMULATION_FAILED.  With the default restored, the same circuit
  and plan run again and match the oracle.
"""
import numpy as np
import pytest

from nqpu_b200 import _lib, circuits
from nqpu_b200._lib import NqpuErrorException
from nqpu_b200.batch import Batch
from nqpu_b200.server import Server
from nqpu_b200.state import Circuit, StateVector
from oracle.oracle import OracleState

pytestmark = pytest.mark.gpu

SIMULATION_FAILED, INVALID_HANDLE = 4, 6


def batch_items():
    # 14-16 qubit circuits run as pass tiles over HBM (small_max_qubits = 13)
    return circuits.hea_batch(12, seed=11, nmin=14, nmax=16, lmin=3, lmax=5)


def make_batch(items, **cfg):
    b = Batch()
    b.config(**cfg)
    for n, g, J, h in items:
        b.add_ising(Circuit(n, g), J, h)
    return b


def test_batch_bounded_wait_expires_and_handle_recovers():
    items = batch_items()
    ref = make_batch(items, small_max_qubits=13).run()
    b = make_batch(items, small_max_qubits=13, spin_limit=1 << 12, drop_tile=1)
    with pytest.raises(NqpuErrorException) as e:
        b.run()
    assert e.value.code == SIMULATION_FAILED
    # a replay of the same faulty queue fails the same way (counters and the
    # error flag are reset by every replay)
    with pytest.raises(NqpuErrorException) as e:
        b.run()
    assert e.value.code == SIMULATION_FAILED
    # the same handle with a complete queue: results equal a fresh batch's
    b.config(drop_tile=0, spin_limit=1 << 26)
    got = b.run()
    assert np.array_equal(got, ref)
    b.close()


def test_batch_short_spin_limit_alone_still_completes():
    # a short poll limit is only a bound: with a complete queue the waits end
    # well before it in practice, or the run reports the expiry; either way no
    # wrong result is returned
    items = batch_items()
    ref = make_batch(items, small_max_qubits=13).run()
    b = make_batch(items, small_max_qubits=13, spin_limit=1 << 20)
    try:
        got = b.run()
        assert np.array_equal(got, ref)
    except NqpuErrorException as e:
        assert e.code == SIMULATION_FAILED
    b.close()


def big_request():
    # 28 qubits, depth 60: a few hundred milliseconds of device time
    return Circuit(28, circuits.brickwork(28, 60, seed=5))


def test_server_wait_timeout_reports_and_request_completes():
    with Server(hbm_budget_bytes=1 << 31, max_qubits=28, lanes=2, large_lanes=1, large_qubits=22) as srv:
        rid = srv.submit(big_request(), "zall")
        with pytest.raises(NqpuErrorException) as e:
            srv.wait(rid, 1e-4)
        assert e.value.code == SIMULATION_FAILED
        srv.wait(rid, 120.0)
        z, t = srv.result(rid)
        assert z.shape == (28,) and np.isfinite(z).all()
        assert srv.stats()["failed"] == 0


def test_server_cancel_queued_request():
    with Server(hbm_budget_bytes=1 << 31, max_qubits=28, lanes=1, large_lanes=1, large_qubits=22) as srv:
        a = srv.submit(big_request(), "zall")
        small = Circuit(10, circuits.brickwork(10, 5, seed=3))
        b = srv.submit(small, "zall")
        c = srv.submit(small, "shots", shots=64, seed=9)
        # one lane, held by the large request: b and c are still queued
        assert srv.cancel(b) is True
        with pytest.raises(NqpuErrorException) as e:
            srv.poll(b)
        assert e.value.code == INVALID_HANDLE
        srv.wait(0, 120.0)  # every request that was not cancelled finishes
        assert srv.cancel(a) is False  # already ran: nothing to withdraw
        za, _ = srv.result(a)
        oc, _ = srv.result(c)
        assert za.shape == (28,) and oc.shape == (64,)
        st = srv.stats()
        assert st["cancelled"] == 1 and st["completed"] == 2 and st["failed"] == 0
        assert srv.lib.nqpu_server_cancel(srv.h_, 12345) == INVALID_HANDLE  # unknown id


def test_tensor_pass_wait_expiry_is_reported_and_the_plan_recovers():
    lib = _lib.load()
    n = 14
    gates = circuits.brickwork(n, 6, 3)
    c = Circuit(n, gates)
    tensor = 3  # NQPU_MODE_TENSOR
    try:
        assert lib.nqpu_tensor_wait_limit_set(64, 1) == 0
        with StateVector(n, "c64") as sv:
            assert lib.nqpu_circuit_execute_ex(c.h_, sv.h_, tensor) == SIMULATION_FAILED
    finally:
        assert lib.nqpu_tensor_wait_limit_set(0, 0) == 0
    o = OracleState(n)
    o.apply(gates)
    ref = o.amplitudes()
    with StateVector(n, "c64") as sv:
        assert lib.nqpu_circuit_execute_ex(c.h_, sv.h_, tensor) == 0  # the cached plan, error flag cleared
        got = sv.amplitudes()
    fid = abs(np.vdot(ref, got)) ** 2
    assert 1 - fid <= 1e-5
    assert lib.nqpu_tensor_wait_limit_set(1 << 31, 0) == 2  # beyond the limit's range
