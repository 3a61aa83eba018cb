"""EnergyIB (src/workproc.f90:2063-2154) on the GPU: the plain drop-in that
forms Glob_D and the fused adjoint pass, against the oracle and against
central finite differences of the energy."""
import numpy as np
import pytest

import oracle as orc
from ecg_b200 import Context
from gpu_util import problem

pytestmark = pytest.mark.gpu
TOL_E = 1e-10
TOL_G = 1e-8   # max |g - g_oracle| / max |g_oracle|


def _gerr(g, go):
    return np.max(np.abs(g - go)) / np.max(np.abs(go))


@pytest.mark.parametrize("cfg,K,nfru", [(1, 160, 0), (1, 160, 110), (0, 200, 0), (4, 90, 0)])
def test_plain_and_adjoint_match_oracle(cfg, K, nfru):
    sysm, params, lam, o = problem(cfg, K, max_nfo=K)
    nfo = K - nfru
    o.last[:K] = 1.0
    if nfru:
        # the factor of the first nfru rows exists before a partial
        # gradient call (OptCycle keeps it from earlier evaluations)
        o.compute_mat_elem(1, nfru, lam)
        o.c[:nfru] = 1.0
        o.ghepiis(1, nfru, lam, 1e-12)
        o.last[:K] = 1.0
    Eo, go, erro, _ = o.energy_ib(nfru, K, lam, 1e-12)
    res = {}
    for mode in ("plain", "adjoint"):
        with Context(sysm, K, max_nfo=K) as ctx:
            ctx.set_params(params)
            ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
            if nfru:
                ctx.compute_mat_elem(1, nfru, lam)
                ctx.set_vectors(nfru, c=np.ones(nfru, dtype=np.complex128))
                ctx.ghepiis(1, nfru, lam, 1e-12)
                ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
            fn = ctx.energy_ib if mode == "plain" else ctx.energy_ib_adjoint
            E, g, err, it = fn(nfru, K, lam, 1e-12)
        res[mode] = (E, g)
        print(f"cfg {cfg} nfru {nfru} {mode}: dE={E - Eo:.2e} grad err={_gerr(g, go):.2e}")
        assert abs(E - Eo) <= TOL_E
        assert g.shape == (nfo * sysm.npt,)
        assert _gerr(g, go) <= TOL_G


def test_gradient_matches_finite_differences():
    """Central differences, h = 1e-6 relative, on seeded parameters (the
    reference's own check, commented out at src/workproc.f90:4174-4203)."""
    K = 80
    sysm, params, lam, _ = problem(1, K)
    rng = np.random.default_rng(5)
    picks = [(int(rng.integers(K)), int(rng.integers(sysm.npt))) for _ in range(12)]
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
        E, g, err, _ = ctx.energy_ib_adjoint(0, K, lam, 1e-12)
        for f, m in picks:
            h = 1e-6 * abs(params[f, m])
            es = []
            for s in (1, -1):
                p2 = params.copy()
                p2[f, m] += s * h
                ctx.set_params(p2)
                e2, _, _ = ctx.energy_ia(1, K, lam, 1e-12, max_iter=30)
                es.append(e2)
            fd = (es[0] - es[1]) / (2 * h)
            an = g[f * sysm.npt + m]
            print(f"f={f} m={m} analytic={an:.10e} fd={fd:.10e}")
            assert abs(fd - an) <= 1e-6 * np.max(np.abs(g)) + 1e-5 * abs(an)
