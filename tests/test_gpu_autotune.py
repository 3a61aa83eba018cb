"""The pair-kernel autotuner: on the first large launch every shape of
k_pair_energy (warps per tile x register budget) and of k_adjoint (register
budget) is timed and the fastest kept; the shapes compute every element
with the same instructions, so the matrices and the gradient of the tuning
call equal, bit for bit, those of the calls after it."""
import numpy as np
import pytest

from ecg_b200 import Context
from gpu_util import problem

pytestmark = pytest.mark.gpu


def test_autotuned_shapes_give_identical_results():
    K = 800  # 325 pair tiles: above the tuning threshold of 256
    sysm, params, lam, _ = problem(1, K)
    ones = np.ones(K, dtype=np.complex128)
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        assert ctx.tuning()["pair_shape"] == -1
        ctx.set_vectors(K, last_eigvec=ones)
        E1, g1, e1, _ = ctx.energy_ib_adjoint(0, K, lam, 1e-12)  # tunes both kernels
        H1, S1, _, _, _ = ctx.matrices(K)
        t = ctx.tuning()
        print(t)
        assert 0 <= t["pair_shape"] < 4 and 0 <= t["adjoint_shape"] < 2
        assert all(x > 0 for x in t["pair_shape_ms"]) and all(x > 0 for x in t["adjoint_shape_ms"])
        ctx.set_vectors(K, last_eigvec=ones)
        E2, g2, e2, _ = ctx.energy_ib_adjoint(0, K, lam, 1e-12)
        H2, S2, _, _, _ = ctx.matrices(K)
    assert np.array_equal(np.tril(H1), np.tril(H2)) and np.array_equal(S1, S2)
    assert E1 == E2 and np.array_equal(g1, g2)
