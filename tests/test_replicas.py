"""Host logic of the replica (one process per GPU) path, run as two gloo ranks on the CPU."""
import os
import socket

import torch.multiprocessing as mp

from bosss_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    w, r, _ = replicas.init("gloo", timeout_s=60)
    replicas.barrier(w)
    mx = replicas.max_over_ranks(1.5 + r, w)
    agg = replicas.aggregate(units=10.0 * (r + 1), seconds=2.0 + r, ws=w)
    part = list(replicas.shard(7, w, r))
    replicas.barrier(w)
    replicas.finalize(w)
    q.put((r, mx, agg, part))


def test_two_gloo_ranks():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, mx, agg, part in out:
        assert mx == 2.5                                  # max over ranks
        assert agg["units"] == 30.0 and agg["seconds"] == 3.0 and agg["per_s"] == 10.0
    assert out[0][3] == [0, 1, 2, 3] and out[1][3] == [4, 5, 6]


def test_single_process_is_a_no_op():
    assert replicas.max_over_ranks(3.0, 1) == 3.0
    assert replicas.aggregate(4.0, 2.0, 1)["per_s"] == 2.0
    assert list(replicas.shard(5, 1, 0)) == [0, 1, 2, 3, 4]
