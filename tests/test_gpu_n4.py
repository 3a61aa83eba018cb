"""n = 4 (five particles: heavy particle + four electrons, 14 Y^+Y terms,
the n = 4 reading of the K = 10000 five-particle workload) through the whole path on the GPU against
the oracle: every stored element of H and S (ComputeMatElem + StoreHS,
src/matform.f90:11-51,119-230), the energy of GHEPIIS (src/linalg.f90:
1781-1926), and the EnergyIB gradient (src/workproc.f90:2063-2154) in the
plain and fused adjoint forms."""
import numpy as np
import pytest

from ecg_b200 import Context
from gpu_util import hs_ratio, problem

pytestmark = pytest.mark.gpu
TOL_E = 1e-10
TOL_G = 1e-8
K = 240


@pytest.fixture(scope="module")
def n4():
    sysm, params, lam, o = problem("4n4", K, max_nfo=K)
    assert sysm.n == 4 and sysm.T == 14
    return sysm, params, lam, o


def test_n4_hs_elements(n4):
    sysm, params, lam, o = n4
    o.compute_mat_elem(1, K, lam)
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, K, lam)
        H, S, dS, _, _ = ctx.matrices(K)
    r = hs_ratio(o, sysm, params, K, lam, "I", H, S, dS)
    print(f"n=4 K={K}: {r}")
    assert r["H"] <= 1 and r["S"] <= 1 and r["diagS"] <= 1


def test_n4_energy_and_gradient(n4):
    sysm, params, lam, o = n4
    o.last[:K] = 1.0
    Eo, go, erro, _ = o.energy_ib(0, K, lam, 1e-12)
    for mode in ("adjoint", "plain"):
        with Context(sysm, K, max_nfo=K) as ctx:
            ctx.set_params(params)
            ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
            fn = ctx.energy_ib_adjoint if mode == "adjoint" else ctx.energy_ib
            E, g, err, it = fn(0, K, lam, 1e-12)
        gerr = float(np.max(np.abs(g - go)) / np.max(np.abs(go)))
        print(f"n=4 {mode}: dE {E - Eo:.2e} grad err {gerr:.2e} codes {err}/{erro}")
        assert err in (0, 2) and abs(E - Eo) <= TOL_E
        assert gerr <= TOL_G
