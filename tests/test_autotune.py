"""Tests of the batch autotuner (nqpu_b200/autotune.py).

CPU: the coordinate descent, the correctness filter and the cache, with the
device timing replaced by a deterministic fake (no GPU needed).
GPU: the real tuner on a small stratified sample: its choice lies in the
search space, its results equal the default configuration's within the
batch tolerance, a second call hits the cache, a changed workload misses it.
"""
import numpy as np
import pytest

from nqpu_b200 import autotune, circuits


def small_items(count=48, seed=21):
    return circuits.hea_batch(count, seed, nmin=8, nmax=16, lmin=2, lmax=4)


def test_stratified_sample_covers_every_size():
    items = small_items(200)
    idx = autotune.stratified_sample(items, 40)
    assert len(idx) == 40 and len(set(idx)) == 40
    sizes = {items[i][0] for i in idx}
    assert sizes == {n for n, *_ in items}
    assert autotune.stratified_sample(items, 0) == []
    assert sorted(autotune.stratified_sample(items, 10**6)) == list(range(200))


def test_signature_depends_on_workload_only():
    a, b = small_items(30, 1), small_items(30, 1)
    assert autotune.signature(a) == autotune.signature(b)
    assert autotune.signature(a) != autotune.signature(small_items(31, 1))


def test_coordinate_descent_and_cache_with_fake_timer(monkeypatch, tmp_path):
    monkeypatch.setenv("NQPU_B200_CACHE", str(tmp_path / "tune.json"))
    items = small_items(20)
    # fake device: tile_qubits 12 and queue_order 2 are fastest; small_max 9
    # is faster still but returns wrong results, so it must be rejected
    calls = []

    def fake_time(entries, cfg, reps=3):
        calls.append(dict(cfg))
        ms = 10.0
        ms -= 2.0 if cfg["tile_qubits"] == 12 else 0.0
        ms -= 1.0 if cfg["queue_order"] == 2 else 0.0
        ms -= 5.0 if cfg["small_max_qubits"] == 9 else 0.0
        res = np.ones(len(entries)) + (1.0 if cfg["small_max_qubits"] == 9 else 0.0)
        return ms, res

    monkeypatch.setattr(autotune, "time_config", fake_time)
    monkeypatch.setattr(autotune, "Circuit", lambda n, g: object())
    cfg, rep = autotune.tune(items, sample_size=8, reps=1)
    assert cfg["tile_qubits"] == 12 and cfg["queue_order"] == 2 and cfg["small_max_qubits"] == 13
    for k, v in cfg.items():
        assert v in autotune.SPACE[k]
    assert rep["cached"] is False and rep["trials"] == len(calls)
    n_calls = len(calls)
    cfg2, rep2 = autotune.tune(items, sample_size=8, reps=1)
    assert rep2["cached"] is True and cfg2 == cfg and len(calls) == n_calls  # no timing on a hit
    cfg3, rep3 = autotune.tune(small_items(21), sample_size=8, reps=1)
    assert rep3["cached"] is False and len(calls) > n_calls


@pytest.mark.gpu
def test_tuner_on_gpu(monkeypatch, tmp_path):
    from nqpu_b200.batch import Batch
    from nqpu_b200.state import Circuit
    monkeypatch.setenv("NQPU_B200_CACHE", str(tmp_path / "tune.json"))
    items = small_items(48)
    cfg, rep = autotune.tune(items, sample_size=24, reps=1, max_sweeps=1)
    assert rep["cached"] is False and rep["trials"] >= 1
    for k, v in cfg.items():
        assert v in autotune.SPACE[k], (k, v)

    def run(c):
        b = Batch()
        b.config(**c)
        for n, g, J, h in items:
            b.add_ising(Circuit(n, g), J, h)
        out = b.run()
        b.close()
        return out

    scale = np.array([np.abs(J).sum() + np.abs(h).sum() for _, _, J, h in items])
    assert np.all(np.abs(run(cfg) - run(dict(autotune.DEFAULT))) <= 1e-5 * scale)
    cfg2, rep2 = autotune.tune(items, sample_size=24, reps=1, max_sweeps=1)
    assert rep2["cached"] is True and cfg2 == cfg
    _, rep3 = autotune.tune(small_items(40, seed=22), sample_size=24, reps=1, max_sweeps=1)
    assert rep3["cached"] is False
