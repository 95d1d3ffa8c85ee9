"""GPU tests of the batched executor (persistent launch over mixed-size
circuits, each returning <H> of its Ising Hamiltonian).

Tolerance: complex64 states with FP64 reductions, |<H> - <H>_FP64| <= 1e-5 *
(sum |J| + sum |h|) against the oracle; results are bitwise identical whether a
circuit runs alone or in a mix, and across repeated runs."""
import numpy as np
import pytest

from nqpu_b200 import circuits
from nqpu_b200.batch import Batch, ising_terms
from nqpu_b200.state import Circuit, StateVector
from oracle.oracle import OracleState

pytestmark = pytest.mark.gpu


def workload(count, seed, nmin, nmax, lmin=2, lmax=6):
    return circuits.hea_batch(count, seed, nmin=nmin, nmax=nmax, lmin=lmin, lmax=lmax)


def oracle_energy(n, gates, J, h):
    o = OracleState(n)
    o.apply(gates)
    return sum(c * o.pauli_string(s) for c, s in ising_terms(n, J, h))


def make_batch(items, **cfg):
    b = Batch()
    if cfg:
        b.config(**cfg)
    for n, g, J, h in items:
        b.add_ising(Circuit(n, g), J, h)
    return b


def test_batch_matches_oracle_mixed_sizes():
    items = workload(40, seed=3, nmin=5, nmax=17)
    b = make_batch(items)
    res = b.run()
    st = b.stats()
    assert st["small"] > 0 and st["small"] < len(items)  # both execution classes present
    for (n, g, J, h), e in zip(items, res):
        ref = oracle_energy(n, g, J, h)
        scale = np.abs(J).sum() + np.abs(h).sum()
        assert abs(e - ref) <= 1e-5 * scale, (n, e, ref)


def test_batch_matches_plain_per_circuit_path():
    items = workload(12, seed=5, nmin=10, nmax=16)
    res = make_batch(items).run()
    for (n, g, J, h), e in zip(items, res):
        sv = StateVector(n, "c64")
        Circuit(n, g).execute(sv, "pergate")
        ref = sv.expectation_pauli_sum(ising_terms(n, J, h))
        assert abs(e - ref) <= 1e-5 * (np.abs(J).sum() + np.abs(h).sum())


def test_batch_result_same_alone_and_in_mix_and_repeatable():
    items = workload(30, seed=7, nmin=8, nmax=16)
    mix = make_batch(items)
    r1 = mix.run()
    r2 = mix.run()
    assert np.array_equal(r1, r2)  # graph replay is deterministic
    for i in (0, 7, 19, 29):
        alone = make_batch([items[i]]).run()
        assert alone[0] == r1[i]


@pytest.mark.parametrize("cfg", [dict(small_max_qubits=9), dict(queue_order=1), dict(queue_order=2),
                                 dict(tile_qubits=12), dict(ctas_per_sm=1)])
def test_batch_configs_agree(cfg):
    items = workload(24, seed=11, nmin=6, nmax=15)
    base = make_batch(items).run()
    other = make_batch(items, **cfg).run()
    np.testing.assert_allclose(other, base, atol=1e-5, rtol=0)


def test_bulk_add_from_arrays_is_bitwise_the_same():
    """nqpu_batch_add_ising_arrays (every circuit's gate arrays in one call)
    builds the same batch as one nqpu_batch_add_ising per circuit handle."""
    items = workload(48, 21, 5, 16)
    arrs = circuits.hea_batch(48, 21, nmin=5, nmax=16, lmin=2, lmax=6, arrays=True)
    one = make_batch(items)
    r1 = one.run()
    one.close()
    bulk = Batch()
    assert bulk.add_ising_arrays(arrs[:20]) == 0
    assert bulk.add_ising_arrays(arrs[20:]) == 20
    r2 = bulk.run()
    bulk.close()
    assert np.array_equal(r1, r2)
