"""CPU engine for the split evaluation's host logic (ecg_b200.split), used by
the gloo tests: the oracle computes H and S; each rank keeps only its own
tiles (and the diagonal) before the exchange, so the rest of its matrices
can only come from the other ranks' packed tiles.  The adjoint stage is
stood in for by per-tile partial values that depend on the tile, the
energy and the eigenvector, and an order-sensitive finish, so a wrong tile
order or a missing range changes the result.  Test infrastructure."""
import numpy as np
import torch

import oracle as orc

TILE = 32


def tile_list(nmin, nmax):
    Rlo, Rhi = (nmin - 1) // TILE, (nmax + TILE - 1) // TILE
    return [(R, C) for R in range(Rlo, Rhi) for C in range(R + 1)]


class OracleEngine:
    def __init__(self, sysm, params, K):
        self.o = orc.Oracle(sysm, K)
        self.o.set_params(params)
        self.K = K
        self.H = np.zeros((K, K), dtype=np.complex128, order="F")
        self.S = np.zeros((K, K), dtype=np.complex128, order="F")

    def zeros(self, n):
        return torch.zeros(int(n), dtype=torch.float64)

    def ntiles(self, nmin, nmax):
        return len(tile_list(nmin, nmax))

    def _entries(self, nmin, nmax, first, count):
        for t, (R, C) in enumerate(tile_list(nmin, nmax)[first:first + count]):
            for ll in range(TILE):
                for lk in range(TILE):
                    k, l = R * TILE + lk, C * TILE + ll
                    if nmin - 1 <= k < nmax and l < k:
                        yield t, ll * TILE + lk, k, l

    def compute_tiles(self, nmin, nmax, lam, first, count):
        self.o.compute_mat_elem(nmin, nmax, lam)
        for k in range(nmin - 1, nmax):
            self.H[k, k] = self.o.H[k, k]
            self.S[k, k] = self.o.S[k, k]
        for _, _, k, l in self._entries(nmin, nmax, first, count):
            self.H[k, l] = self.o.H[k, l]
            self.S[k, l] = self.o.S[k, l]
            self.S[l, k] = self.o.S[l, k]

    def pack(self, nmin, nmax, first, count, buf):
        b = buf.numpy().view(np.complex128)
        for t, e, k, l in self._entries(nmin, nmax, first, count):
            b[t * 2 * TILE * TILE + e] = self.H[k, l]
            b[t * 2 * TILE * TILE + TILE * TILE + e] = self.S[k, l]

    def unpack(self, nmin, nmax, first, count, buf):
        b = buf.numpy().view(np.complex128)
        for t, e, k, l in self._entries(nmin, nmax, first, count):
            self.H[k, l] = b[t * 2 * TILE * TILE + e]
            s = b[t * 2 * TILE * TILE + TILE * TILE + e]
            self.S[k, l] = s
            self.S[l, k] = np.conj(s)

    def solve(self, nmin, nmax, lam, tol, max_iter):
        o = self.o
        o.H[:, :] = self.H
        o.S[:, :] = self.S
        o.c[:nmax] = o.last[:nmax]
        E, ra, it, err = o.ghepiis(nmin, nmax, lam, tol, max_iter, 0)
        return E, err, it

    def part_doubles(self):
        return 2 * TILE * 13

    def adjoint_tiles(self, nfru, nfa, E, first, count, buf):
        pd = self.part_doubles()
        w = np.abs(self.o.last[:nfa]).sum()
        for t in range(first, first + count):
            v = np.random.default_rng(t).standard_normal(pd) * E * w
            buf[(t - first) * pd:(t - first + 1) * pd] = torch.from_numpy(v)

    def finish(self, nfru, nfa, buf):
        acc = np.zeros(self.part_doubles())
        for chunk in buf.numpy().reshape(-1, self.part_doubles()):
            acc = acc * 0.9990234375 + chunk
        return acc
