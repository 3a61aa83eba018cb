"""The oracle's restatement of the expectation-value pass (ExpectationValuesG,
src/workproc.f90:8159-8366, with MatrixElementsForExpcVals,
src/matelem.f90:949-1983) pinned without a reference fixture (the reference
ships no expectation values): on the optimised HD+ bases the sums must
reproduce the normalisation and the Rayleigh quotient of the eigenvector,
H = T + V, V from the 1/r values and the charges, Darwin from the delta(r)
values, the virial theorem, the Drachmanised delta(r) of the attractive
pairs close to the plain one, drach_MV equal to drach_Darwin (the
reference computes the same quantity along two code paths, :1675-1848 and
:1875-1929), and the correlation-function and density sum rules; for n = 3
with four symmetry terms, SymmAdaptMethod 1 and 2 agree on the
permutation-invariant operators."""
import numpy as np
import pytest
import scipy.linalg as sl

import oracle as orc
from ecg_b200 import System, expc, synth


def g_eigpair(o, K, which):
    """Eigenpair of the oracle's 'G' matrices, c^H S c = 1, and the
    Rayleigh quotient c^H H c (the accurate energy of that vector)."""
    o.compute_mat_elem(1, K, 0.0, method="G")
    H = np.tril(o.H[:K, :K], -1)
    H = H + H.conj().T + np.diag(o.diagH[:K])
    S = np.tril(o.S[:K, :K], -1)
    S = S + S.conj().T + np.eye(K)
    ev, V = sl.eigh(H, S, subset_by_index=[which - 1, which - 1])
    c = V[:, 0]
    return ev[0], c, np.vdot(c, H @ c).real, np.vdot(c, S @ c).real


@pytest.fixture(scope="module")
def hd_500(golden):
    out = {}
    for name in ("inout_1_500", "inout_2_500"):
        f = golden(name)
        sysm = System(f["masses"], f["charges"], f["symmetry"])
        K = f["K"]
        o = orc.Oracle(sysm, K)
        o.set_params(f["params"])
        E, c, rq, cSc = g_eigpair(o, K, f["which"])
        s, e, _, _ = o.expectation_values(K, c, rq)
        out[name] = (f, sysm, expc.unpack(s, e, sysm.n), rq, cSc)
    return out


@pytest.mark.parametrize("name", ["inout_1_500", "inout_2_500"])
def test_hdplus_identities(hd_500, name):
    f, sysm, d, rq, cSc = hd_500[name]
    n = sysm.n
    q0, q = sysm.charges[0], sysm.charges[1:]
    m = sysm.masses
    print(f"{name}: " + "  ".join(f"{k}={d[k]:.12g}" for k in expc.SCALAR_NAMES))
    assert abs(d["S"] - cSc) <= 1e-12
    assert abs(d["H"] - rq) <= 1e-12 * abs(rq)
    assert abs(d["H"] - f["energy"]) <= 1e-10
    assert abs(d["H"] - d["T"] - d["V"]) <= 1e-13
    V = q0 * sum(q[i] * d["rm"][i, i] for i in range(n)) + sum(
        q[i] * q[j] * d["rm"][i, j] for i in range(n) for j in range(i + 1, n))
    assert abs(V - d["V"]) <= 1e-13
    dar = sum((1 / m[0] ** 2 + 1 / m[i + 1] ** 2) * q0 * q[i] * d["deltar"][i, i] for i in range(n))
    dar += sum(q[i] * q[j] * d["deltar"][i, j] / m[i + 1] ** 2 for i in range(n) for j in range(n) if j != i)
    assert abs(-dar * np.pi / 2 - d["Darwin"]) <= 1e-13 * abs(d["Darwin"])
    assert abs(-d["V"] / d["T"] - 2) <= 1e-6                       # virial theorem
    assert abs(d["drach_MV"] - d["drach_Darwin"]) <= 1e-12 * abs(d["drach_MV"])
    # attractive pairs: the electron (coordinate 2) with particle 0 and with particle 1
    for (a, b) in ((1, 1), (0, 1)):
        rel = abs(d["drach_deltar"][a, b] / d["deltar"][a, b] - 1)
        print(f"  delta(r_{a + 1}{b + 1}) {d['deltar'][a, b]:.10f}  drachmanised {d['drach_deltar'][a, b]:.10f}")
        assert rel <= 2e-3
    for k in expc.SCALAR_NAMES:
        assert abs(d[k + "_e"]) <= 1e-11 * max(1.0, abs(d[k]))


def test_hdplus_report_format(hd_500):
    f, sysm, d, rq, cSc = hd_500["inout_1_500"]
    lines = expc.report_lines(d)
    assert len(lines) == 16
    assert lines[0].startswith("                       H=")
    assert lines[0][25:48].strip().startswith("-0.59789796")
    assert all(len(s) == 2 + 23 + 23 + 3 + 12 + 1 for s in lines)


def test_grid_sum_rules(golden):
    """Int 4 pi r^2 g_P(r) dr = <S> and Int 4 pi r^3 g_P(r) dr = <r_P> for
    the correlation functions; Int 4 pi r^2 rho_i(r) dr = <S> for the
    particle densities (first 60 functions of the HD+ basis, their own
    eigenvector)."""
    f = golden("inout_1_500")
    sysm = System(f["masses"], f["charges"], f["symmetry"])
    K = 60
    o = orc.Oracle(sysm, K)
    o.set_params(f["params"][:K])
    E, c, rq, cSc = g_eigpair(o, K, 1)
    r = np.linspace(0.0, 40.0, 4001)
    s, e, cf, dens = o.expectation_values(K, c, rq, cf_grid=r, dens_grid=r)
    d = expc.unpack(s, e, sysm.n)
    w = np.full(r.size, r[1] - r[0])
    w[0] = w[-1] = 0.5 * (r[1] - r[0])
    for P, (a, b) in enumerate([(0, 0), (0, 1), (1, 1)]):
        norm = np.sum(w * 4 * np.pi * r ** 2 * cf[P])
        mean = np.sum(w * 4 * np.pi * r ** 3 * cf[P])
        print(f"pair {P}: norm {norm:.10f}  <r> {mean:.8f} vs {d['r'][a, b]:.8f}")
        assert abs(norm - d["S"]) <= 1e-6
        assert abs(mean - d["r"][a, b]) <= 1e-5 * d["r"][a, b]
    for i in range(sysm.n + 1):
        norm = np.sum(w * 4 * np.pi * r ** 2 * dens[i])
        assert abs(norm - d["S"]) <= 1e-6


def test_symm_adapt_methods_agree():
    """n = 3, Y = (1+P12)(1+P34): H, S, T, V, MV and OO commute with the
    symmetry, so Y^+Y on the ket and Y on both sides give the same sums."""
    sysm, params = synth.config_basis(1, K=30)
    K = 30
    o = orc.Oracle(sysm, K)
    o.set_params(params)
    o.compute_mat_elem(1, K, 0.0, method="G")
    c = np.random.default_rng(3).normal(size=K) + 0.3j * np.random.default_rng(4).normal(size=K)
    s1, e1, _, _ = o.expectation_values(K, c, -1.1, method=1)
    s2, e2, _, _ = o.expectation_values(K, c, -1.1, method=2)
    d1, d2 = expc.unpack(s1, e1, sysm.n), expc.unpack(s2, e2, sysm.n)
    for k in ("H", "S", "T", "V", "MV", "Darwin", "OO"):
        tol = 1e-11 * abs(d1[k]) + 50 * (d1[k + "_e"] + d2[k + "_e"])
        print(f"{k}: method 1 {d1[k]:.15g}  method 2 {d2[k]:.15g}")
        assert abs(d1[k] - d2[k]) <= tol
