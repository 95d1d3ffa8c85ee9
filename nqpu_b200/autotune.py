"""Autotuner for the batched executor.

It picks, for one workload on one GPU model:
  * `tile_qubits`      - the tile shape of the larger circuits' passes (2^k
                         amplitudes per shared-memory tile, k = 10..13);
  * `small_max_qubits` - which circuits run whole in one CTA's shared memory
                         instead of as HBM pass tiles (5..13);
  * `queue_order`      - the qubit-block schedule of the work queue: small
                         circuits interleaved between the pass rounds of the
                         large ones (0), all first (1) or all last (2);
  * `ctas_per_sm`      - persistent CTAs per SM (1 or 2).

Method: coordinate descent from the library defaults.  Each candidate value of
one parameter is timed with the others fixed (device time of the graph replay,
median of `reps` runs after one warm run) on a stratified sample of the
workload (circuits sorted by qubit count and length, every k-th taken), the
best value is kept, and sweeps repeat until a full sweep changes nothing.
Every candidate's results are checked against the default configuration's
(within 1e-5 of the Hamiltonian's scale), so a faster but wrong schedule can
never win.  The choice is cached per GPU model and workload signature in a
JSON file (`NQPU_B200_CACHE`, default ~/.cache/nqpu_b200/autotune.json).
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from pathlib import Path

import numpy as np

from .batch import Batch
from .state import Circuit

SPACE = {
    "tile_qubits": (13, 12, 11),
    "small_max_qubits": (13, 12, 11, 10, 9),
    "queue_order": (0, 1, 2),
    "ctas_per_sm": (2, 1),
}
DEFAULT = {"tile_qubits": 13, "small_max_qubits": 13, "queue_order": 0, "ctas_per_sm": 2}


def cache_path() -> Path:
    env = os.environ.get("NQPU_B200_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "nqpu_b200" / "autotune.json"


def device_name() -> str:
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.get_device_name(0)
    except Exception:
        pass
    return "cuda"


def signature(items) -> str:
    """Workload signature: the histogram of (qubits, gate-count bucket)."""
    hist: dict[str, int] = {}
    for n, g, _J, _h in items:
        key = f"{n}:{len(g) // 64}"
        hist[key] = hist.get(key, 0) + 1
    blob = json.dumps(sorted(hist.items())).encode()
    return f"{len(items)}-" + hashlib.sha1(blob).hexdigest()[:16]


def stratified_sample(items, size: int) -> list[int]:
    """Indices of every k-th circuit in (qubits, length) order."""
    if size <= 0:
        return []
    order = sorted(range(len(items)), key=lambda i: (items[i][0], len(items[i][1]), i))
    if size >= len(order):
        return order
    step = len(order) / size
    return [order[int(j * step)] for j in range(size)]


def time_config(entries, cfg: dict, reps: int = 3):
    """Median device ms of the graph replay for `cfg`, and its results.
    `entries` = [(Circuit, J, h)]."""
    b = Batch()
    try:
        b.config(**cfg)
        for c, J, h in entries:
            b.add_ising(c, J, h)
        b.prepare()
        res = b.run()  # warm
        ms = []
        for _ in range(reps):
            res = b.run()
            ms.append(b.last_run_ms())
        return float(np.median(ms)), res
    finally:
        b.close()


def tune(items, sample_size: int = 1024, reps: int = 3, max_sweeps: int = 3, use_cache: bool = True,
         circuits=None, log=None):
    """Return (config, report).  `items` = [(n, gates, J, h)] as from
    `circuits.hea_batch`; `circuits` optionally holds prebuilt Circuit handles
    for the same items (index-aligned)."""
    key = f"{device_name()}|{signature(items)}|s{sample_size}"
    path = cache_path()
    cache = {}
    if use_cache and path.exists():
        try:
            cache = json.loads(path.read_text())
        except (OSError, ValueError):
            cache = {}
        if key in cache:
            return dict(cache[key]["config"]), {"cached": True, "key": key, **cache[key]}

    t0 = time.perf_counter()
    idx = stratified_sample(items, sample_size)
    entries = []
    for i in idx:
        n, g, J, h = items[i]
        c = circuits[i] if circuits is not None else Circuit(n, g)
        entries.append((c, J, h))
    scale = np.array([np.abs(items[i][2]).sum() + np.abs(items[i][3]).sum() for i in idx])

    best = dict(DEFAULT)
    best_ms, ref = time_config(entries, best, reps)
    trials = [{"config": dict(best), "ms": best_ms}]
    for _ in range(max_sweeps):
        changed = False
        for name, values in SPACE.items():
            for v in values:
                if v == best[name]:
                    continue
                cand = dict(best)
                cand[name] = v
                ms, res = time_config(entries, cand, reps)
                ok = bool(np.all(np.abs(res - ref) <= 1e-5 * scale))
                trials.append({"config": dict(cand), "ms": ms, "agrees": ok})
                if log:
                    log(f"autotune {cand} {ms:.3f} ms{'' if ok else ' (results differ: rejected)'}")
                if ok and ms < best_ms * 0.98:  # 2 % hysteresis against timing noise
                    best, best_ms, changed = cand, ms, True
        if not changed:
            break
    report = {"cached": False, "key": key, "config": best, "sample_ms": best_ms,
              "default_ms": trials[0]["ms"], "trials": len(trials), "sample": len(idx),
              "seconds": time.perf_counter() - t0}
    if use_cache:
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            cache[key] = {k: report[k] for k in ("config", "sample_ms", "default_ms", "trials", "sample")}
            path.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return dict(best), report
