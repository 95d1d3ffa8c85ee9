"""The multi-GPU replica path on CPU: two gloo ranks, each with its own
elapsed time, combine into one whole-job rate (units of all ranks over the
slowest rank's time), as bench.py --gpus N does over NCCL."""
import json
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from nqpu_b200 import replicas
    assert replicas.world() == (rank, rank, world)
    replicas.init("gloo", timeout_s=60)
    replicas.barrier()
    rate, t = replicas.replica_rate(units_per_rank=100.0, elapsed_s_local=1.0 + rank)
    m = replicas.max_over_ranks(float(rank) * 3.0)
    replicas.shutdown()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"rate": rate, "t": t, "m": m}, f)


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_combine_rate(tmp_path, world):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.spawn(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True)
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["t"] == pytest.approx(float(world))          # slowest rank: 1 + (world - 1)
        assert r["rate"] == pytest.approx(100.0 * world / world)  # 200 units / 2 s
        assert r["m"] == pytest.approx(3.0 * (world - 1))


def test_single_process_is_identity():
    from nqpu_b200 import replicas
    rate, t = replicas.replica_rate(50.0, 2.0)
    assert (rate, t) == (25.0, 2.0)
    assert replicas.max_over_ranks(1.5) == 1.5
