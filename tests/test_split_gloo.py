"""The split evaluation's host logic (ecg_b200.split) over gloo ranks on
CPU: with the pair tiles divided between two ranks, each rank's H and S
after the exchange, its energy and its gradient are bit for bit those of
one rank doing everything (the same engine; the oracle computes the
matrices, see split_engine.py), and the tile ranges cover the list once,
in order, balanced."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, K, out):
    import datetime
    import sys
    for p in (os.path.join(ROOT, "atom-mol-nonbo_b200"), os.path.join(ROOT, "oracle"),
              os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from ecg_b200 import synth
        from ecg_b200.split import SplitEvaluation
        from split_engine import OracleEngine
        sysm, params = synth.config_basis(1, K=K)
        eng = OracleEngine(sysm, params, K)
        eng.o.last[:K] = 1.0
        ev = SplitEvaluation(eng)
        E, g, err, it = ev.energy_ib_adjoint(0, K, -1.1, 1e-12)
        out[rank] = (eng.H.copy(), eng.S.copy(), E, g.copy(), err, it)
    finally:
        dist.destroy_process_group()


def _run(world, K):
    port = _free_port()
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_worker, args=(world, port, K, out), nprocs=world, join=True)
        return dict(out)


def test_tile_ranges_cover_the_list():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "atom-mol-nonbo_b200"))
    from ecg_b200.split import tile_range
    for nt in (1, 7, 36, 7875):
        for w in (1, 2, 3, 8):
            rs = [tile_range(nt, r, w) for r in range(w)]
            assert rs[0][0] == 0 and sum(c for _, c in rs) == nt
            assert all(rs[i][0] + rs[i][1] == rs[i + 1][0] for i in range(w - 1))
            assert max(c for _, c in rs) - min(c for _, c in rs) <= 1


@pytest.mark.parametrize("K", [70, 97])
def test_two_ranks_match_one_rank_bit_for_bit(K):
    one = _run(1, K)[0]
    two = _run(2, K)
    for r in (0, 1):
        H, S, E, g, err, it = two[r]
        assert np.array_equal(H, one[0]) and np.array_equal(S, one[1])
        assert E == one[2] and (err, it) == (one[4], one[5])
        assert np.array_equal(g, one[3])
    # the exchange filled what each rank did not compute: its own tiles alone
    # would leave most of the strict lower triangle empty
    lo = np.tril_indices(K, -1)
    assert np.all(two[0][0][lo] != 0)
