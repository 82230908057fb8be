"""Multi-GPU is replicas only: bench.py --gpus N runs N independent replicas,
joined by a gloo process group for the barrier and the max-over-ranks time.
These CPU tests run the same helpers as two gloo ranks on 127.0.0.1."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench

    ws, r, lr, pg = bench._dist()
    bench._barrier(pg)
    worst = bench._max(pg, 10.0 + rank)  # per-rank device time (ms)
    bench._barrier(pg)
    q.put((r, ws, lr, worst, ws * 1e3 / worst))
    pg.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time_and_aggregate():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2 and o[3] == 11.0 for o in out)  # every rank sees the slowest replica
    assert out[0][4] == pytest.approx(2 * 1e3 / 11.0)    # aggregate iterations/s over both replicas


def test_single_process_needs_no_group(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    ws, r, lr, pg = bench._dist()
    assert (ws, r, lr, pg) == (1, 0, 0, None)
    assert bench._max(pg, 3.5) == 3.5
