"""Batched candidates with gradients (ecg_eval_candidates_grad): for every
candidate, the energy and the gradient EnergyIB(nbase, nbase+1)
(src/workproc.f90:2063-2154, nfo = 1) returns once the candidate is basis
function nbase+1 -- the energy + gradient that the optimisation of a newly
added function asks for (BasisEnlI's DRMNG loop, src/workproc.f90:4137-4170).
Checked against the oracle's EnergyIB per candidate (ComputeMatElemAndDeriv of
row K, GHEPIIS(K, K) on the base factor, the Glob_D contraction), against
the GPU's own one-call path (ecg_set_params + ecg_energy_ib_adjoint(nbase,
nbase+1)), and against central differences of the batched energies."""
import numpy as np
import pytest

import oracle as orc
from ecg_b200 import Context
from test_gpu_candidates import base_problem

pytestmark = pytest.mark.gpu
TOL_E = 1e-10
TOL_G = 1e-8  # max |g - g_ref| / max |g_ref| per candidate


def _gerr(g, gr):
    return float(np.max(np.abs(g - gr)) / np.max(np.abs(gr)))


@pytest.mark.parametrize("cfg,K0,B,seed", [(1, 200, 24, 21), (0, 150, 16, 22), (4, 90, 12, 23)])
def test_candidate_gradients_match_oracle_and_single_path(cfg, K0, B, seed):
    tol = 1e-12
    sysm, params, cands, o, lam, start = base_problem(cfg, K0, B, seed, tol)
    K = K0 + 1
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K0, last_eigvec=np.ones(K0, dtype=np.complex128))
        ctx.energy_ia(1, K0, lam, tol)
        ctx.set_vectors(K, last_eigvec=start)
        E, err, it, ra, g = ctx.eval_candidates_grad(K0, cands, lam, tol)
        single = []
        for j in range(B):
            ctx.set_params(cands[j:j + 1], first=K)
            ctx.set_vectors(K, last_eigvec=start)
            Es, gs, errs, _ = ctx.energy_ib_adjoint(K0, K, lam, tol)
            single.append((Es, gs, errs))
    # the oracle: the base factor of o, one EnergyIB(K0, K) per candidate
    od = orc.Oracle(sysm, K, max_nfo=1)
    od.H[:, :] = o.H
    od.S[:, :] = o.S
    od.diagS[:] = o.diagS
    od.invD[:] = o.invD
    worst_o = worst_s = 0.0
    for j in range(B):
        if err[j] == 1:
            continue
        od.set_params(np.vstack([params, cands[j:j + 1]]))
        od.last[:K] = start
        Eo, go, erro, _ = od.energy_ib(K0, K, lam, tol)
        Es, gs, errs = single[j]
        worst_o = max(worst_o, _gerr(g[j], go))
        worst_s = max(worst_s, _gerr(g[j], gs))
        assert abs(E[j] - Eo) <= TOL_E and abs(E[j] - Es) <= TOL_E, (j, E[j], Eo, Es)
        assert _gerr(g[j], go) <= TOL_G and _gerr(g[j], gs) <= TOL_G, (j, _gerr(g[j], go), _gerr(g[j], gs))
    print(f"cfg {cfg} K0 {K0} B {B}: codes {np.bincount(err, minlength=3)}; max rel grad diff vs oracle "
          f"{worst_o:.2e}, vs one-call adjoint path {worst_s:.2e}")


def test_candidate_gradient_finite_differences():
    """Central differences (h = 1e-6 relative) of the batched energies: the
    perturbed copies of one candidate go through the same call."""
    tol = 1e-12
    sysm, params, cands, o, lam, start = base_problem(1, 160, 4, 24, tol)
    K0, K = 160, 161
    npt = sysm.npt
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K0, last_eigvec=np.ones(K0, dtype=np.complex128))
        ctx.energy_ia(1, K0, lam, tol)
        ctx.set_vectors(K, last_eigvec=start)
        E, err, _, _, g = ctx.eval_candidates_grad(K0, cands, lam, tol)
        j = int(np.argmin(np.where(err == 0, E, np.inf)))
        c0 = cands[j]
        h = 1e-6 * np.abs(c0)
        pert = np.vstack([c0 + np.eye(npt)[m] * h[m] for m in range(npt)] +
                         [c0 - np.eye(npt)[m] * h[m] for m in range(npt)])
        ctx.set_vectors(K, last_eigvec=start)
        Ep, errp, _, _ = ctx.eval_candidates(K0, pert, lam, tol, max_iter=40)
    assert np.all(errp == 0)
    fd = (Ep[:npt] - Ep[npt:]) / (2 * h)
    gmax = np.max(np.abs(g[j]))
    # truncation and the energy's rounding over the step (64 eps |E| / h)
    bound = 1e-6 * gmax + 1e-5 * np.abs(g[j]) + 64 * np.finfo(np.float64).eps * abs(E[j]) / h
    print("analytic", g[j])
    print("fd      ", fd)
    print("|fd - analytic| / bound", np.abs(fd - g[j]) / bound)
    assert np.all(np.abs(fd - g[j]) <= bound)
