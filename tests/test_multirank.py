"""The N > 1 host path of bench.py on CPU ranks (gloo, world size 2): each
rank evaluates an independent replica (its own seeded basis), and the
timing reduction takes the max over ranks; no data-path collective."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench
    d = bench.Dist()
    sysm, params, e_floor = bench.setup_problem(64, d.rank)
    d.barrier()
    mx = d.max(10.0 * (rank + 1))
    sm = d.sum(rank + 1)
    out[rank] = (mx, sm, float(params.sum()), e_floor)
    d.close()


def test_two_rank_replicas_and_reductions():
    world = 2
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    assert res[0][1] == res[1][1] == 3.0
    assert res[0][2] != res[1][2]  # independent replicas
    assert res[0][3] == res[1][3] == -1.2
