"""The 'G' path on the GPU (EnergyGA / EnergyGAM / EnergyGB,
src/workproc.f90:1697-1950): the WHICH_EIGENVALUE-th eigenvalue of the
pencil with ZHEGVX(RANGE='I') semantics, found by inertia bisection and
inverse iteration.  Checked against the reference's stored HD+ energies
(WHICH_EIGENVALUE 1 and 2), against SciPy's generalised Hermitian solver on
the oracle's 'G' matrices, against the oracle's GHEPIIS at that eigenvalue,
and the EnergyGB gradient against the 'I' path's at the same eigenpair."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as orc
from ecg_b200 import Context, System, synth

pytestmark = pytest.mark.gpu
TOL_E = 1e-10


def scipy_eigs(o, K, idx):
    o.compute_mat_elem(1, K, 0.0, method="G")
    H = np.tril(o.H[:K, :K], -1)
    H = H + H.conj().T + np.diag(o.diagH[:K])
    S = np.tril(o.S[:K, :K], -1)
    S = S + S.conj().T + np.eye(K)
    return sl.eigh(H, S, eigvals_only=True, subset_by_index=[idx[0], idx[-1]])


@pytest.mark.parametrize("name", ["inout_1_500", "inout_2_500", "inout_1_1000", "inout_2_1000"])
def test_g_path_matches_stored(golden, name):
    f = golden(name)
    sysm = System(f["masses"], f["charges"], f["symmetry"])
    K, w = f["K"], f["which"]
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(f["params"])
        E, err, nf = ctx.energy_ga(1, K, which=w)
    print(f"{name}: which={w} E={E:.16f} stored={f['energy']:.16f} diff={E - f['energy']:.2e} "
          f"factorisations={nf}")
    assert err == 0
    assert abs(E - f["energy"]) <= TOL_E


@pytest.mark.parametrize("cfg,K", [(1, 200), (0, 160), (4, 120)])
def test_g_path_matches_oracle(cfg, K):
    """Eigenvalues 1..3 against SciPy (ZHEGVX semantics) to 1e-8 relative
    and against the oracle's GHEPIIS started at them to 1e-10."""
    sysm, params = synth.config_basis(cfg, K=K)
    o = orc.Oracle(sysm, K)
    o.set_params(params)
    ref = scipy_eigs(o, K, [0, 2])
    oi = orc.Oracle(sysm, K)
    oi.set_params(params)
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(params)
        for w in (1, 2, 3):
            E, err, nf = ctx.energy_ga(1, K, which=w, mat_elem_needed=(w == 1))
            lam = ref[w - 1] * (1.0 + 1e-10)
            oi.last[:K] = 1.0
            Eo, erro, _ = oi.energy_ia(1, K, lam, 1e-13, max_iter=40)
            print(f"cfg {cfg} K={K} which={w}: E={E:.15f} scipy={ref[w - 1]:.15f} GHEPIIS={Eo:.15f} "
                  f"factorisations={nf}")
            assert err == 0
            assert abs(E - ref[w - 1]) <= 1e-8 * max(1.0, abs(E))
            assert abs(E - Eo) <= TOL_E


def test_g_path_vector_and_single_function():
    """EnergyGAM's eigenvector satisfies c^H S c = 1 and H c = E S c; with one
    function E = Glob_diagH(1)."""
    sysm, params = synth.config_basis(1, K=150)
    K = 150
    o = orc.Oracle(sysm, K)
    o.set_params(params)
    o.compute_mat_elem(1, K, 0.0, method="G")
    H = np.tril(o.H[:K, :K], -1)
    H = H + H.conj().T + np.diag(o.diagH[:K])
    S = np.tril(o.S[:K, :K], -1)
    S = S + S.conj().T + np.eye(K)
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(params)
        E, err, _ = ctx.energy_ga(1, K, which=2, want_vector=True)
        c, _ = ctx.vectors(K)
        E1, err1, _ = ctx.energy_ga(1, 1, which=1)
    assert err == 0 and err1 == 0
    assert abs(np.vdot(c, S @ c).real - 1.0) <= 1e-10
    res = np.linalg.norm(H @ c - E * (S @ c)) / (np.linalg.norm(H, 1) * np.linalg.norm(c))
    print(f"EnergyGAM which=2: E={E:.15f} |c^H S c - 1|={abs(np.vdot(c, S @ c).real - 1):.1e} residual {res:.1e}")
    assert res <= 1e-9
    assert abs(E1 - o.diagH[0]) <= 1e-12 * abs(o.diagH[0])


@pytest.mark.parametrize("which", [1, 2])
def test_gb_gradient_matches_i_path(which):
    """EnergyGB's gradient (ZHEGVX eigenpair) equals EnergyIB's at the same
    eigenvalue (GHEPIIS at lambda~ next to it)."""
    sysm, params = synth.config_basis(1, K=120)
    K = 120
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(params)
        Eg, gg, err = ctx.energy_gb_adjoint(0, K, which=which)
    assert err == 0
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K, last_eigvec=np.ones(K, dtype=np.complex128))
        Ei, gi, erri, _ = ctx.energy_ib_adjoint(0, K, Eg * (1.0 + 1e-10), 1e-13, max_iter=40)
    d = np.max(np.abs(gg - gi)) / np.max(np.abs(gi))
    print(f"which={which}: E_G={Eg:.15f} E_I={Ei:.15f} max rel grad diff {d:.2e}")
    assert abs(Eg - Ei) <= TOL_E
    assert d <= 1e-7


@pytest.mark.parametrize("nfru", [0, 30])
def test_gb_plain_matches_adjoint(nfru):
    """EnergyGB through Glob_D (ecg_energy_gb) and through the fused adjoint
    pass: same eigenvalue, gradients within 1e-9 of the largest entry."""
    sysm, params = synth.config_basis(1, K=90)
    K = 90
    with Context(sysm, K, max_nfo=K, method="G") as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, K, 0.0)
        Ep, gp, errp = ctx.energy_gb(nfru, K, which=1)
        Ea, ga, erra = ctx.energy_gb_adjoint(nfru, K, which=1)
    d = np.max(np.abs(gp - ga)) / np.max(np.abs(ga))
    print(f"nfru={nfru}: E plain {Ep:.15f} adjoint {Ea:.15f}, max rel grad diff {d:.2e}")
    assert errp == 0 and erra == 0
    assert abs(Ep - Ea) <= 1e-12 * abs(Ea)
    assert d <= 1e-9
