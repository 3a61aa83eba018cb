"""Task list of the persistent LDL^H factorisation (ldlp.cu), checked on the
host: ecg_ldl_schedule returns the order in which the kernel's CTAs take
the tile tasks.  The list must hold every task of the factorisation once,
in an order where each task comes after the tasks it waits for (so the
kernel, whose CTAs are all resident, cannot deadlock), and executing it
task by task must give the LDL^H factor of the reference's recurrence
(src/linalg.f90:316-455): here in numpy, with the trailing updates in the
kernel's form conj(U(s, R))^T diag(d_s) U(s, C)."""
import ctypes as C

import numpy as np
import pytest

from ecg_b200 import _lib

NB = 64
D_, T_, B_ = 0, 1, 2


def schedule(n, workers):
    lib = _lib.load()
    cnt = C.c_longlong()
    assert lib.ecg_ldl_schedule(n, workers, None, 0, C.byref(cnt)) == 0
    out = np.zeros(cnt.value, dtype=np.uint32)
    assert lib.ecg_ldl_schedule(n, workers, C.c_void_p(out.ctypes.data), cnt.value, C.byref(cnt)) == 0
    return out


def decode(code):
    """(type, s, R, C, column half)."""
    code = int(code)
    return code >> 30, (code >> 20) & 511, (code >> 10) & 1023, code & 1023, (code >> 29) & 1


def split(s, r, c):
    """The updates of the two tile rows after panel s, except the chain's
    B(s, s+1, s+1), run as two column halves."""
    return r <= s + 2 and not (r == s + 1 and c == s + 1)


def expected_tasks(np_):
    t = set()
    for s in range(np_):
        t.add((D_, s, s, s, 0))
        for c in range(s + 1, np_):
            t.add((T_, s, s, c, 0))
        for r in range(s + 1, np_):
            for c in range(r, np_):
                t.add((B_, s, r, c, 0))
                if split(s, r, c):
                    t.add((B_, s, r, c, 1))
    return t


def upd(s, r, c):
    return [(B_, s, r, c, h) for h in ((0, 1) if split(s, r, c) else (0,))]


def deps(task):
    ty, s, r, c, _ = task
    if ty == D_:
        return upd(s - 1, s, s) if s > 0 else []
    if ty == T_:
        return [(D_, s, s, s, 0)] + (upd(s - 1, s, c) if s > 0 else [])
    d = [(T_, s, s, r, 0)]
    if c != r:
        d.append((T_, s, s, c, 0))
    if s > 0:
        d += upd(s - 1, r, c)
    return d


@pytest.mark.parametrize("n,workers", [(1, 1), (64, 4), (65, 2), (300, 296), (1000, 8), (4000, 296)])
def test_list_is_complete_and_topological(n, workers):
    lst = [decode(x) for x in schedule(n, workers)]
    np_ = (n + NB - 1) // NB
    assert len(lst) == len(set(lst)) and set(lst) == expected_tasks(np_)
    pos = {t: i for i, t in enumerate(lst)}
    for t in lst:
        for d in deps(t):
            assert pos[d] < pos[t], (t, d)


def test_chain_tasks_in_chain_order():
    """The chain CTA runs D(s), T(s, s+1), B(s, s+1, s+1) for s = 0, 1, ...
    in that order: the start order must list them in that same order, so
    that it stays a topological order of what each CTA actually runs (the
    kernel's no-deadlock argument)."""
    for n in (300, 4000):
        lst = [decode(x) for x in schedule(n, 296)]
        np_ = (n + NB - 1) // NB
        chain = []
        for s in range(np_):
            chain.append((D_, s, s, s, 0))
            if s + 1 < np_:
                chain += [(T_, s, s, s + 1, 0), (B_, s, s + 1, s + 1, 0)]
        pos = {t: i for i, t in enumerate(lst)}
        got = [pos[t] for t in chain]
        assert got == sorted(got)


def test_chain_tasks_lead_the_list():
    """The critical chain D(s) -> T(s, s+1) -> B(s, s+1, s+1) -> D(s+1)
    is taken early: every D(s+1) comes before the last update of panel s
    (the last few panels excepted, where little else is left to run)."""
    lst = [decode(x) for x in schedule(4000, 296)]
    pos = {t: i for i, t in enumerate(lst)}
    np_ = (4000 + NB - 1) // NB
    for s in range(np_ - 4):
        last_b = max(pos[(B_, s, r, c, 0)] for r in range(s + 1, np_) for c in range(r, np_))
        assert pos[(D_, s + 1, s + 1, s + 1, 0)] < last_b


def run_tasks(M, lst, complex_pivots=False):
    """Execute the task list on the Hermitian matrix M (numpy, sequential)."""
    n = M.shape[0]
    W = np.triu(M.conj().T).copy()   # working upper triangle W(r, c) = M(c, r)^*
    U = np.zeros_like(W)
    d = np.zeros(n, dtype=complex)
    for ty, s, r, c, h in lst:
        p0, p1 = s * NB, min(n, s * NB + NB)
        if ty == D_:
            Wb = W[p0:p1, p0:p1].copy()
            for q in range(p1 - p0):
                dq = Wb[q, q] if complex_pivots else Wb[q, q].real
                d[p0 + q] = dq
                u = Wb[q, q + 1:] / dq
                for i in range(q + 1, p1 - p0):
                    Wb[i, i:] -= np.conj(u[i - q - 1]) * Wb[q, i:]
                U[p0 + q, p0 + q + 1:p1] = u
                U[p0 + q, p0 + q] = 1.0
        elif ty == T_:
            c0, c1 = c * NB, min(n, c * NB + NB)
            L = U[p0:p1, p0:p1].conj().T
            wun = np.linalg.solve(L, W[p0:p1, c0:c1])
            U[p0:p1, c0:c1] = wun / d[p0:p1, None]
        else:
            r0, r1 = r * NB, min(n, r * NB + NB)
            c0, c1 = c * NB, min(n, c * NB + NB)
            if split(s, r, c):  # one column half of the tile
                c0, c1 = c0 + 32 * h, min(c1, c0 + 32 * h + 32)
            if c1 <= c0:
                continue
            upd = U[p0:p1, r0:r1].conj().T @ (d[p0:p1, None] * U[p0:p1, c0:c1])
            if r == c:
                upd = np.triu(upd, r0 - c0)  # keep global column >= global row
            W[r0:r1, c0:c1] -= upd
    return U, d


@pytest.mark.parametrize("n", [130, 300, 700])
def test_list_executes_to_the_ldlh_factor(n):
    rng = np.random.default_rng(n)
    X = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    M = X @ X.conj().T / n + np.diag(rng.uniform(-2.0, 2.0, n))   # Hermitian, indefinite
    lst = [decode(x) for x in schedule(n, 16)]
    U, d = run_tasks(M, lst)
    R = U.conj().T @ np.diag(d) @ U
    assert np.max(np.abs(R - M)) <= 1e-10 * np.max(np.abs(M))
    # the reference's row-by-row recurrence gives the same factor
    Ur = np.eye(n, dtype=complex)
    dr = np.zeros(n, dtype=complex)
    A = M.copy()
    for i in range(n):
        for j in range(i):
            x = A[i, j] - np.sum(np.conj(Ur[:j, i]) * dr[:j] * Ur[:j, j])
            Ur[j, i] = np.conj(x) / dr[j]
        dr[i] = (A[i, i] - np.sum(np.abs(Ur[:i, i]) ** 2 * dr[:i])).real
    assert np.max(np.abs(U - Ur)) <= 1e-9 * max(1.0, np.max(np.abs(Ur)))
    assert np.max(np.abs(d - dr)) <= 1e-9 * np.max(np.abs(dr))
