"""The multi-rank path of the benchmark on the CPU: two processes joined with
gloo (as torchrun launches them, rendezvous on 127.0.0.1), each an
independent replica seeded by its rank.  The timing collectives give every
rank the slowest rank's time, the job value counts every rank's units, the
round-robin shard partitions the units, and the replicas' data differ."""
import multiprocessing as mp
import os
import socket

import numpy as np


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank),
                      LOCAL_RANK=str(rank))
    from maos_b200 import replicas
    from maos_b200.setup import screens
    try:
        ws, r, _ = replicas.init("gloo", timeout_s=60)
        scr = screens(64, 64, 1 / 32, 0.186, 30.0, [1.0], 1 + r)[0]  # this replica's own atmosphere
        step_s = 1.0 + r                                               # this replica's time
        mx = replicas.max_over_ranks(step_s, ws)
        tot = replicas.sum_over_ranks(float(scr.sum()), ws)
        replicas.barrier(ws)
        q.put((r, ws, mx, float(scr.sum()), tot, replicas.shard(list(range(7)), r, ws),
               replicas.job_value(10, 5, ws, mx)))
        replicas.finish(ws)
    except Exception as e:  # report instead of hanging the parent
        q.put(("error", repr(e)))


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(x[0] != "error" for x in res), res
    res.sort()
    (r0, ws0, mx0, s0, tot0, sh0, v0), (r1, ws1, mx1, s1, tot1, sh1, v1) = res
    assert (r0, r1, ws0, ws1) == (0, 1, 2, 2)
    assert mx0 == mx1 == 2.0                  # the slowest rank's time on every rank
    assert v0 == v1 == 10 * 5 * 2 / 2.0       # all ranks' units over that time
    assert np.isclose(tot0, s0 + s1) and tot0 == tot1
    assert s0 != s1                           # independent replicas
    assert sorted(sh0 + sh1) == list(range(7)) and not set(sh0) & set(sh1)
