"""GHEPIIS (src/linalg.f90:1781-1926) on the GPU: the reference's HD+ known
answers, agreement with the oracle, the bordered factorisation, and the
ErrorCode paths."""
import numpy as np
import pytest

import oracle as orc
from conftest import FIXTURES
from ecg_b200 import Context, System, synth
from gpu_util import problem

pytestmark = pytest.mark.gpu
TOL_E = 1e-10


@pytest.mark.parametrize("name", FIXTURES)
def test_energy_matches_stored(golden, name):
    f = golden(name)
    sysm = System(f["masses"], f["charges"], f["symmetry"])
    K = f["K"]
    with Context(sysm, K) as ctx:
        ctx.set_params(f["params"])
        ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
        E, err, it = ctx.energy_ia(1, K, f["energy"] * f["invit"], f["tol"])
    print(f"{name}: E={E:.16f} stored={f['energy']:.16f} diff={E - f['energy']:.2e} err={err} it={it}")
    assert err in (0, 2)
    assert abs(E - f["energy"]) <= TOL_E


@pytest.mark.parametrize("cfg,K", [(0, 300), (1, 300), (4, 150)])
def test_energy_matches_oracle(cfg, K):
    sysm, params, lam, o = problem(cfg, K)
    o.last[:K] = 1.0
    Eo, erro, ito = o.energy_ia(1, K, lam, 1e-12, specif_norm=0)
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
        E, err, it = ctx.energy_ia(1, K, lam, 1e-12, specif_norm=0)
        _, x = ctx.vectors(K)
    print(f"cfg {cfg}: E={E:.16f} oracle={Eo:.16f} diff={E - Eo:.2e} it={it}/{ito}")
    assert abs(E - Eo) <= TOL_E
    # eigenvector normalised x^H S x = 1; equal to the oracle's up to a phase
    xo = o.last[:K]
    ph = np.vdot(x, xo)
    ph /= abs(ph)
    assert np.max(np.abs(x * ph - xo)) <= 1e-6 * np.max(np.abs(xo))


def test_bordered_factorisation_matches_full():
    """GHEPIIS(k, n) with k > 1 reuses the first k-1 rows of the factor
    (the bordered LDLHF, src/linalg.f90:356-392) and gives the same energy."""
    sysm, params, lam, o = problem(1, 260)
    K = 260
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, K, lam)
        ctx.set_vectors(K, c=np.ones(K, dtype=np.complex128))
        E1, _, it1, e1 = ctx.ghepiis(1, K, lam, 1e-12)
        _, _, _, _, invD1 = ctx.matrices(K)
        # refactor rows 201..260 only, then rows 130..260 after a full factor of 1..200
        ctx.set_vectors(K, c=np.ones(K, dtype=np.complex128))
        E2, _, it2, e2 = ctx.ghepiis(201, K, lam, 1e-12)
        ctx.set_vectors(K, c=np.ones(K, dtype=np.complex128))
        E3, _, it3, e3 = ctx.ghepiis(130, K, lam, 1e-12)
        H, _, _, _, invD3 = ctx.matrices(K)
    assert abs(E2 - E1) <= TOL_E and abs(E3 - E1) <= TOL_E
    # pivots agree relative to the largest pivot (the last one is tiny by
    # design, lambda~ sits 1e-10 below the lowest eigenvalue)
    d1, d3 = 1.0 / invD1, 1.0 / invD3
    assert np.max(np.abs(d3 - d1)) <= 1e-12 * np.max(np.abs(d1))


def test_zero_pivot_reports_error_1():
    """lambda~ equal to the first normalised diagonal element gives an exact
    zero pivot (ErrorCode 1, src/linalg.f90:377-380), as in the oracle."""
    sysm, params = synth.config_basis(1, K=40)
    K = 40
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, K, 0.0)
        H, _, _, _, _ = ctx.matrices(K)
        h11 = H[0, 0].real
        ctx.compute_mat_elem(1, K, h11)
        lam_, ra, it, err = ctx.ghepiis(1, K, h11, 1e-12)
        # the context stays usable afterwards
        ctx.compute_mat_elem(1, K, -1.3)
        ctx.set_vectors(K, c=np.ones(K, dtype=np.complex128))
        _, _, _, err2 = ctx.ghepiis(1, K, -1.3, 1e-12, max_iter=5)
    o = orc.Oracle(sysm, K)
    o.set_params(params)
    o.compute_mat_elem(1, K, 0.0)
    h11o = o.H[0, 0].real
    o.compute_mat_elem(1, K, h11o)
    _, _, _, erro = o.ghepiis(1, K, h11o, 1e-12)
    assert err == 1 and erro == 1 and it == 0
    assert err2 in (0, 2)


def test_iteration_limit_reports_error_2():
    sysm, params, lam, _ = problem(1, 120)
    with Context(sysm, 120) as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, 120, -1.3)
        ctx.set_vectors(120, c=np.ones(120, dtype=np.complex128))
        _, ra, it, err = ctx.ghepiis(1, 120, -1.3, 1e-14, max_iter=1)
    assert err == 2 and it == 1 and ra > 1e-14
