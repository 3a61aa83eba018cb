"""The expectation-value pass on the GPU (ecg_expectation_values:
ExpectationValuesG's accumulation loop, src/workproc.f90:8159-8366, over
MatrixElementsForExpcVals, src/matelem.f90:949-1983) against the oracle's
restatement on the same eigenvector: every one of the 6np+9 sums, the
correlation functions and the particle densities.  The GPU evaluates the
same formulas in a different order, so the yardstick is the oracle's own
rounding error: both are compared with the oracle's x87 extended-precision
build of the same source, and the GPU must stay within 16 times the
double-precision oracle's distance from it (plus 1e-12 relative and 64
times the reference's rounding-error bound MEkl_e).  Some values lose many
digits to cancellation inside each pair term (the orbit-orbit term to about
1e-9 relative on the synthetic n = 3 basis, in the double-precision oracle
as much as on the GPU).  Also the full driver (ExpectationValuesG:
matrix elements, ZHEGVX-semantics eigenpair, pass) on the HD+ fixtures
against their stored energies, and size-independent identities at K=2000."""
import numpy as np
import pytest

import oracle as orc
from ecg_b200 import Context, System, expc, synth

pytestmark = pytest.mark.gpu


def close(gpu, ref, ext, label):
    """Per value: |gpu - ext| <= 16 |ref - ext| + 1e-12 |ext| + 64 (e_gpu + e_ref),
    ref the double-precision oracle, ext its extended-precision build."""
    vg, eg = gpu[0], gpu[1]
    vr, er = ref[0], ref[1]
    vx = ext[0]
    tol = 16 * np.abs(vr - vx) + 1e-12 * np.abs(vx) + 64 * (np.abs(eg) + np.abs(er)) + 1e-300
    ratio = np.abs(vg - vx) / tol
    k = int(np.argmax(ratio))
    print(f"{label}: worst |gpu - ext|/tol = {ratio[k]:.3f} at value {k}: gpu rel err "
          f"{abs(vg[k] - vx[k]) / abs(vx[k]):.1e}, oracle rel err {abs(vr[k] - vx[k]) / abs(vx[k]):.1e}; "
          f"max rel |gpu - ext| {np.max(np.abs(vg - vx) / np.maximum(np.abs(vx), 1e-300)):.2e}, "
          f"max rel |oracle - ext| {np.max(np.abs(vr - vx) / np.maximum(np.abs(vx), 1e-300)):.2e}")
    assert np.all(np.abs(vg - vx) <= tol)


def grid_close(g, r, x, label):
    """Grid values: |gpu - ext| <= 16 |ref - ext| + 1e-12 (largest |ext| of the row)."""
    scale = np.max(np.abs(x), axis=1, keepdims=True) + 1e-300
    tol = 16 * np.abs(r - x) + 1e-12 * scale
    print(f"{label}: max |gpu - ext| / row max = {np.max(np.abs(g - x) / scale):.2e}, "
          f"max |oracle - ext| / row max = {np.max(np.abs(r - x) / scale):.2e}")
    assert np.all(np.abs(g - x) <= tol)


@pytest.mark.parametrize("name", ["inout_1_500", "inout_2_500"])
def test_hdplus_expectation_values(golden, name):
    f = golden(name)
    sysm = System(f["masses"], f["charges"], f["symmetry"])
    K = f["K"]
    r = np.linspace(0.0, 12.0, 25)
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(f["params"])
        d = ctx.expectation_values_g(K, which=f["which"], cf_grid=r, dens_grid=r[:10])
        c, _ = ctx.vectors(K)
        gpu = ctx.expectation_values(K, d["E"], c, cf_grid=r, dens_grid=r[:10], raw=True)
    print(f"{name}: E={d['E']:.15f} <H>={d['H']:.15f} stored {f['energy']:.15f}")
    assert abs(d["H"] - f["energy"]) <= 1e-10
    assert abs(d["S"] - 1.0) <= 1e-10
    o = orc.Oracle(sysm, K)
    o.set_params(f["params"])
    o.compute_mat_elem(1, K, 0.0, method="G")
    ref = o.expectation_values(K, c, d["E"], cf_grid=r, dens_grid=r[:10])
    ext = o.expectation_values(K, c, d["E"], cf_grid=r, dens_grid=r[:10], extended=True)
    close(gpu, ref, ext, name)
    grid_close(gpu[2], ref[2], ext[2], name + " correlation functions")
    grid_close(gpu[3], ref[3], ext[3], name + " densities")


def case_basis(case, K):
    if isinstance(case, int):
        return synth.config_basis(case, K=K)
    if case == "n5":  # six particles, charge +5 and five electrons, one exchange
        sysm = System([12786.0, 1.0, 1.0, 1.0, 1.0, 1.0], [5.0, -1.0, -1.0, -1.0, -1.0, -1.0], "(1+P23)")
    else:
        sysm = synth.make_system(case)
    return sysm, synth.random_basis(sysm.n, K, 77)


@pytest.mark.parametrize("case,K,method", [(0, 150, 1), (1, 120, 1), (1, 60, 2), (4, 60, 1), (4, 30, 2),
                                           ("li_minus_like", 24, 1), ("li_minus_like", 10, 2), ("n5", 12, 1)])
def test_against_oracle(case, K, method):
    """n = 2 (two Y^+Y terms), 3 (four and six terms), 4 and 5;
    SymmAdaptMethod 1 and 2; a complex coefficient vector that is not an
    eigenvector, so no identity hides a wrong term; grids for both grid
    parts."""
    sysm, params = case_basis(case, K)
    rng = np.random.default_rng(100 + sysm.n)
    c = rng.normal(size=K) + 1j * rng.normal(size=K)
    E = -1.234
    r = np.linspace(0.1, 6.0, 7)
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, K, 0.0)
        gpu = ctx.expectation_values(K, E, c, method=method, cf_grid=r, dens_grid=r, raw=True)
        ctx.set_vectors(K, c=c)
        g2 = ctx.expectation_values(K, E, None, method=method, raw=True)
    assert np.array_equal(gpu[0], g2[0]) and np.array_equal(gpu[1], g2[1])
    o = orc.Oracle(sysm, K)
    o.set_params(params)
    o.compute_mat_elem(1, K, 0.0, method="G")
    ref = o.expectation_values(K, c, E, method=method, cf_grid=r, dens_grid=r)
    ext = o.expectation_values(K, c, E, method=method, cf_grid=r, dens_grid=r, extended=True)
    close(gpu, ref, ext, f"{case} n={sysm.n} T={sysm.T} K={K} method {method}")
    grid_close(gpu[2], ref[2], ext[2], "correlation functions")
    grid_close(gpu[3], ref[3], ext[3], "densities")


def test_single_pair_terms():
    """nbasis = 1 and 2: the diagonal factor 1/diagS and the off-diagonal
    factor 2/sqrt(diagS_i diagS_j) of src/workproc.f90:8165-8169."""
    sysm, params = synth.config_basis(1, K=2)
    c = np.array([0.7 - 0.2j, -0.4 + 0.9j])
    with Context(sysm, 2, method="G") as ctx:
        ctx.set_params(params)
        ctx.compute_mat_elem(1, 2, 0.0)
        for nb in (1, 2):
            gpu = ctx.expectation_values(nb, -0.5, c[:nb], raw=True)
            o = orc.Oracle(sysm, 2)
            o.set_params(params)
            o.compute_mat_elem(1, 2, 0.0, method="G")
            ref = o.expectation_values(nb, c, -0.5)
            ext = o.expectation_values(nb, c, -0.5, extended=True)
            close(gpu, ref, ext, f"nbasis {nb}")


def test_full_size_identities():
    """K = 2000, n = 3, four terms: the pass over 2,001,000 pairs on its own
    eigenvector reproduces c^H S c = 1, <H> = E, H = T + V, and
    drach_MV = drach_Darwin."""
    K = 2000
    sysm, params = synth.config_basis(3, K=K)
    with Context(sysm, K, method="G") as ctx:
        ctx.set_params(params)
        d = ctx.expectation_values_g(K, which=1)
    print(f"K={K}: E={d['E']:.15f} <H>={d['H']:.15f} S={d['S']:.15f} "
          f"H_e/H={d['H_e'] / abs(d['H']):.2e} drach_MV={d['drach_MV']:.12g} drach_Darwin={d['drach_Darwin']:.12g}")
    assert abs(d["S"] - 1.0) <= 1e-9 + 10 * d["S_e"]
    assert abs(d["H"] - d["E"]) <= 1e-9 * abs(d["E"]) + 10 * d["H_e"]
    assert abs(d["H"] - d["T"] - d["V"]) <= 1e-12 * abs(d["T"]) + 10 * (d["T_e"] + d["V_e"])
    assert abs(d["drach_MV"] - d["drach_Darwin"]) <= 1e-10 * abs(d["drach_MV"]) + 10 * d["drach_MV_e"]
