"""Replica bookkeeping of multi-GPU runs on CPU with the gloo backend, world size 2."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from nadvibs_b200 import replicas
    r, w, _ = replicas.init("gloo", timeout_s=30)
    replicas.barrier()
    m = replicas.max_over_ranks(1.0 + r)
    rate = replicas.aggregate_rate(10, 2.0 + 3.0 * r)
    replicas.shutdown()
    q.put((r, w, m, rate))


def test_two_rank_max_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, m, rate in res:
        assert w == 2 and m == 2.0
        assert rate == pytest.approx(2 * 10 / 5.0)   # 2 ranks * 10 steps / slowest 5 s


def test_single_process_is_a_no_op():
    from nadvibs_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(4, 2.0) == 2.0
