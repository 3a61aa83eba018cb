"""The GPU side of the split evaluation (ecg_pair_tiles and the tile-range
entry points) on one GPU: two contexts stand for two ranks and exchange
their packed tiles and adjoint partials through device buffers (the copies
a collective would make), one after the other, with no collective.  Each
context then holds H and S bit for bit as one whole ComputeMatElem writes
them, and the energy and the gradient are bit for bit those of
ecg_energy_ib_adjoint."""
import numpy as np
import pytest
import torch

from ecg_b200 import Context
from ecg_b200.split import TILE_DOUBLES, tile_range
from gpu_util import problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cfg,K,world", [(1, 300, 2), (0, 257, 3)])
def test_tile_split_matches_the_whole_pass(cfg, K, world):
    sysm, params, lam, _ = problem(cfg, K)
    dev = torch.device("cuda:0")
    ones = np.ones(K, dtype=np.complex128)
    with Context(sysm, K) as ref:
        ref.set_params(params)
        ref.compute_mat_elem(1, K, lam)
        H0, S0, dS0, _, _ = ref.matrices(K)
        ref.set_vectors(K, last_eigvec=ones)
        E0, g0, err0, it0 = ref.energy_ib_adjoint(0, K, lam, 1e-12)
    ctxs = [Context(sysm, K) for _ in range(world)]
    try:
        nt = ctxs[0].pair_tiles(1, K)
        ranges = [tile_range(nt, r, world) for r in range(world)]
        bufs = []
        for ctx, (f, c) in zip(ctxs, ranges):
            ctx.set_params(params)
            ctx.compute_mat_elem_tiles(1, K, lam, f, c)
            b = torch.zeros(max(c, 1) * TILE_DOUBLES, dtype=torch.float64, device=dev)
            ctx.pack_tiles(1, K, f, c, b.data_ptr())
            ctx.sync()
            bufs.append(b)
        for r, ctx in enumerate(ctxs):
            for q, (f, c) in enumerate(ranges):
                if q != r:
                    ctx.unpack_tiles(1, K, f, c, bufs[q].data_ptr())
            H, S, dS, _, _ = ctx.matrices(K)
            assert np.array_equal(H, H0) and np.array_equal(S, S0) and np.array_equal(dS, dS0)
        pd = ctxs[0].adjoint_part_doubles()
        parts = []
        for ctx, (f, c) in zip(ctxs, ranges):
            ctx.set_vectors(K, last_eigvec=ones)
            E, err, it = ctx.energy_ia(1, K, lam, 1e-12, mat_elem_needed=False, specif_norm=0)
            assert (E, err, it) == (E0, err0, it0)
            p = torch.zeros(max(c, 1) * pd, dtype=torch.float64, device=dev)
            ctx.adjoint_tiles(0, K, E, f, c, p.data_ptr())
            ctx.sync()
            parts.append(p[:c * pd])
        full = torch.cat(parts)
        for ctx in ctxs:
            g = ctx.adjoint_finish(0, K, full.data_ptr())
            assert np.array_equal(g, g0)
    finally:
        for ctx in ctxs:
            ctx.close()
