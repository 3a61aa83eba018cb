"""Failure paths of the bounded device waits, made to run out on purpose
without any fault: with the poll limit of the triangular solves set to 0,
a CTA that finds the panel it depends on unpublished gives up at once,
records the timeout and every other CTA stops waiting; the call returns
ECG_ECUDA (EcgError status -2), and after the limit is restored the next
call on the same context gives the same result as before."""
import numpy as np
import pytest

from ecg_b200 import Context, EcgError
from gpu_util import problem
from test_gpu_candidates import base_problem

pytestmark = pytest.mark.gpu
ECG_ECUDA = -2


def test_factorisation_wait_timeout_is_reported_and_the_context_recovers():
    """EnergyIA(1, K) factorises the whole matrix with the persistent tile
    kernel: with the poll limit at 0 the first task that finds a tile it
    depends on unfinished gives up, every CTA stops taking tasks, and the
    call reports ECG_ECUDA; the factorisation is deterministic, so the next
    call reproduces the first result bit for bit."""
    K = 400
    sysm, params, lam, _ = problem(1, K)
    ones = np.ones(K, dtype=np.complex128)
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K, last_eigvec=ones)
        E0, err0, it0 = ctx.energy_ia(1, K, lam, 1e-12)
        ctx.set_wait_limit(0)
        ctx.set_vectors(K, last_eigvec=ones)
        with pytest.raises(EcgError) as ei:
            ctx.energy_ia(1, K, lam, 1e-12)
        assert ei.value.status == ECG_ECUDA
        ctx.set_wait_limit(-1)
        ctx.set_vectors(K, last_eigvec=ones)
        E1, err1, it1 = ctx.energy_ia(1, K, lam, 1e-12)
    print(f"E before {E0:.15f} after {E1:.15f}")
    assert (err1, it1) == (err0, it0) and E1 == E0


def test_ghepiis_wait_timeout_is_reported_and_the_context_recovers():
    """EnergyIA(K, K) recomputes row K and extends the existing factor by
    one row (the bordered LDLHF, no waits), so the bounded waits that run
    out are those of GHEPIIS's cooperative triangular solves."""
    K = 400
    sysm, params, lam, _ = problem(1, K)
    ones = np.ones(K, dtype=np.complex128)
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K, last_eigvec=ones)
        ctx.energy_ia(1, K, lam, 1e-12)
        ctx.set_vectors(K, last_eigvec=ones)
        E0, err0, it0 = ctx.energy_ia(K, K, lam, 1e-12)
        ctx.set_wait_limit(0)
        ctx.set_vectors(K, last_eigvec=ones)
        with pytest.raises(EcgError) as ei:
            ctx.energy_ia(K, K, lam, 1e-12)
        assert ei.value.status == ECG_ECUDA
        ctx.set_wait_limit(-1)
        ctx.set_vectors(K, last_eigvec=ones)
        E1, err1, it1 = ctx.energy_ia(K, K, lam, 1e-12)
    print(f"E before {E0:.15f} after {E1:.15f}")
    assert (err1, it1) == (err0, it0) and E1 == E0


def test_candidate_solve_wait_timeout_is_reported_and_the_context_recovers():
    tol = 1e-12
    sysm, params, cands, o, lam, start = base_problem(1, 300, 40, 31, tol)
    K0 = 300
    with Context(sysm, K0 + 1) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K0, last_eigvec=np.ones(K0, dtype=np.complex128))
        ctx.energy_ia(1, K0, lam, tol)
        ctx.set_vectors(K0 + 1, last_eigvec=start)
        E0, err0, _, _ = ctx.eval_candidates(K0, cands, lam, tol)
        ctx.set_wait_limit(0)
        ctx.set_vectors(K0 + 1, last_eigvec=start)
        with pytest.raises(EcgError) as ei:
            ctx.eval_candidates(K0, cands, lam, tol)
        assert ei.value.status == ECG_ECUDA
        ctx.set_wait_limit(-1)
        ctx.set_vectors(K0 + 1, last_eigvec=start)
        E1, err1, _, _ = ctx.eval_candidates(K0, cands, lam, tol)
    assert np.array_equal(err0, err1)
    assert np.array_equal(E0[err0 != 1], E1[err1 != 1])
