"""Host logic of bench.py's multi-rank runs, as world_size-2 gloo ranks on the CPU: every rank
reconstructs its own replica cloud (no data-path collective), the timing is the max over
ranks and the throughput counts all ranks' points; the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import bench
    w, r, local = bench.dist_env()
    dist = bench.dist_init(w, "gloo")
    cpu = torch.device("cpu")
    mx = bench.reduce_max(dist, [120.0, 135.5][rank], cpu)
    sm = bench.reduce_sum(dist, [1000.0, 2500.0][rank], cpu)

    class A:
        points, depth, steps, warmup, gpus = 10, 5, 1, 0, ws
    # the reference arm: rank != 0 returns at once without work or output
    ref_rc = bench.run_reference(A) if rank != 0 else 0
    q.put((rank, w, r, local, mx, sm, bench.replica_seed(rank), ref_rc))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [x[:4] for x in res] == [(0, 2, 0, 0), (1, 2, 1, 1)]
    assert all(x[4] == 135.5 for x in res)   # slowest rank's time
    assert all(x[5] == 3500.0 for x in res)  # all ranks' points
    assert res[0][6] != res[1][6]            # distinct replica clouds
    assert res[1][7] == 0


@pytest.mark.parametrize("ws", [1])
def test_single_rank_needs_no_process_group(ws, monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_env() == (1, 0, 0)
    assert bench.dist_init(ws, "gloo") is None
    assert bench.reduce_max(None, 2.5, None) == 2.5 and bench.reduce_sum(None, 4.0, None) == 4.0
