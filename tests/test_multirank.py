"""Multi-rank host logic of bench.py on CPU: two gloo ranks agree on barriers and take the max
of their timings (the N-GPU bench runs one independent replica per rank)."""
import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    r, w, lr = bench.dist_env()
    d = bench.Dist(w)
    d.barrier()
    m = d.max(1.5 + r)
    d.close()
    q.put((r, w, lr, m))


def test_two_ranks_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [x[0] for x in res] == [0, 1]
    assert all(x[1] == 2 and x[3] == 2.5 for x in res)
