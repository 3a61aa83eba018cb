"""One energy + gradient evaluation with its pair work split over the ranks
of a torch.distributed process group (one process and one context per GPU,
NCCL over NVLink on GPUs, gloo on CPU).

The reference deals (pair, term) units cyclically to its MPI ranks and sums
the H, S buffers and the gradient with MPI_ALLREDUCE (src/matform.f90:
170-213, src/workproc.f90:2129,2148).  Here each rank takes a contiguous,
balanced range of the 32 x 32 pair tiles of the lower triangle:

1. the rank computes its tiles of H and S (and every diagonal pair);
2. the packed tiles of all ranks are all-gathered and unpacked, so every
   rank holds the whole H and S, each entry computed once and bit for bit
   the single-GPU value;
3. every rank runs the LDL^H factorisation and the inverse iteration itself
   (replicated: they are not split);
4. the rank runs the fused adjoint pass over its tiles; the per-tile partial
   sums (not gradients) are all-gathered and summed in tile order, so the
   gradient is bit for bit the single-GPU one on every rank.

The engine carries out the per-rank work; `ContextEngine` drives a GPU
context through the C ABI.  Collectives are plain all-gathers of device
buffers; no rank reads another rank's memory directly.
"""
import numpy as np

TILE = 32
TILE_DOUBLES = 2 * TILE * TILE * 2  # H and S blocks of one tile, complex


def tile_range(ntiles, rank, nranks):
    """(first, count) of rank's contiguous share of ntiles tiles: counts
    differ by at most one, ranks in order."""
    base, rem = divmod(int(ntiles), int(nranks))
    first = rank * base + min(rank, rem)
    return first, base + (1 if rank < rem else 0)


class ContextEngine:
    """The per-rank steps on one GPU context (ecg_b200.Context)."""

    def __init__(self, ctx, device):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.device = device

    def zeros(self, n):
        return self.torch.zeros(int(n), dtype=self.torch.float64, device=self.device)

    def ntiles(self, nmin, nmax):
        return self.ctx.pair_tiles(nmin, nmax)

    def compute_tiles(self, nmin, nmax, lam, first, count):
        self.ctx.compute_mat_elem_tiles(nmin, nmax, lam, first, count)

    def pack(self, nmin, nmax, first, count, buf):
        self.ctx.pack_tiles(nmin, nmax, first, count, buf.data_ptr())
        self.ctx.sync()

    def unpack(self, nmin, nmax, first, count, buf):
        self.ctx.unpack_tiles(nmin, nmax, first, count, buf.data_ptr())

    def solve(self, nmin, nmax, lam, tol, max_iter):
        return self.ctx.energy_ia(nmin, nmax, lam, tol, max_iter=max_iter, mat_elem_needed=False, specif_norm=0)

    def part_doubles(self):
        return self.ctx.adjoint_part_doubles()

    def adjoint_tiles(self, nfru, nfa, E, first, count, buf):
        self.ctx.adjoint_tiles(nfru, nfa, E, first, count, buf.data_ptr())
        self.ctx.sync()

    def finish(self, nfru, nfa, buf):
        return self.ctx.adjoint_finish(nfru, nfa, buf.data_ptr())


class SplitEvaluation:
    """EnergyIB (fused adjoint form, src/workproc.f90:2063-2154) with the
    pair tiles split over the ranks of `group` (None: the default group)."""

    def __init__(self, engine, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.engine = engine
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)

    def _gather(self, local, per_unit, counts):
        """All-gather the ranks' buffers (padded to the largest count) and
        return the valid parts concatenated in rank order."""
        maxc = max(counts)
        gathered = self.engine.zeros(self.world * maxc * per_unit)
        self.dist.all_gather_into_tensor(gathered, local, group=self.group)
        parts = [gathered[r * maxc * per_unit:(r * maxc + counts[r]) * per_unit] for r in range(self.world)]
        return gathered, parts

    def energy_ib_adjoint(self, nfru, nfa, lam, tol, max_iter=20):
        """Returns (E, gradient, ErrorCode, NumIter) as
        Context.energy_ib_adjoint(nfru, nfa, ...) does."""
        if nfa - nfru < 1 or nfa < 2:
            raise ValueError("the split evaluation needs nfa >= 2")
        eng, nmin = self.engine, nfru + 1
        nt = eng.ntiles(nmin, nfa)
        ranges = [tile_range(nt, r, self.world) for r in range(self.world)]
        counts = [c for _, c in ranges]
        first, count = ranges[self.rank]
        # 1-2: own tiles of H and S, exchanged
        eng.compute_tiles(nmin, nfa, lam, first, count)
        buf = eng.zeros(max(counts) * TILE_DOUBLES)
        eng.pack(nmin, nfa, first, count, buf)
        _, parts = self._gather(buf, TILE_DOUBLES, counts)
        for r, (f, c) in enumerate(ranges):
            if r != self.rank and c > 0:
                eng.unpack(nmin, nfa, f, c, parts[r])
        # 3: replicated solve
        E, err, it = eng.solve(nmin, nfa, lam, tol, max_iter)
        if err == 1:
            return E, None, err, it
        # 4: adjoint partials of own tiles, gathered in tile order
        pd = eng.part_doubles()
        pbuf = eng.zeros(max(counts) * pd)
        eng.adjoint_tiles(nfru, nfa, E, first, count, pbuf)
        _, pparts = self._gather(pbuf, pd, counts)
        full = eng.zeros(nt * pd)
        o = 0
        for r in range(self.world):
            n = counts[r] * pd
            full[o:o + n] = pparts[r]
            o += n
        g = eng.finish(nfru, nfa, full)
        return E, g, err, it
