"""Seeded synthetic bases and candidate functions.

The reference ships optimised bases only for HD+ (n = 2, one symmetry term);
the larger systems it is benchmarked on here use seeded random bases with
this distribution per function k:

* diag(L_k) log-uniform in [0.05, 20] bohr^-1,
* L_k(i, j), i > j, uniform in [-0.5, 0.5] * L_k(j, j),
* B_k(i, j) = B_k(j, i) uniform in [-0.1, 0.1] * L_k(i, i) * L_k(j, j),

stored as the reference stores nonlinear parameters: (vech L, vech B) with
vech running over columns i and rows j >= i (src/matelem.f90:109-122).

Candidates follow GenerateTrialParam (src/workproc.f90:1375-1487): a parent
is drawn from the basis, then with probability p1 every parameter is scaled
by its own (s1 N(0,1) + 1) (method 1), else all parameters by one common
factor r = s2 N(0,1) + 1 redrawn while 0.8 < |r| < 1.2 (method 2).
"""
import numpy as np

__all__ = ["random_basis", "candidates", "vech_indices", "systems"]


def vech_indices(n):
    """(row, col) of each vech entry, column-major lower triangle."""
    return [(j, i) for i in range(n) for j in range(i, n)]


def random_basis(n, K, seed, row_scale=None):
    rng = np.random.default_rng(seed)
    idx = vech_indices(n)
    np_ = len(idx)
    out = np.empty((K, 2 * np_), dtype=np.float64)
    lo, hi = np.log(0.05), np.log(20.0)
    for k in range(K):
        d = np.exp(rng.uniform(lo, hi, size=n))
        L = np.diag(d)
        for i in range(n):
            for j in range(i + 1, n):
                L[j, i] = rng.uniform(-0.5, 0.5) * d[i]
        if row_scale is not None:
            L = L * np.asarray(row_scale)[:, None]
        dd = np.diag(L)
        B = np.zeros((n, n))
        for i in range(n):
            for j in range(i, n):
                B[j, i] = B[i, j] = rng.uniform(-0.1, 0.1) * dd[i] * dd[j]
        out[k, :np_] = [L[r, c] for r, c in idx]
        out[k, np_:] = [B[r, c] for r, c in idx]
    return out


def candidates(basis, B, seed, p1=0.7, s1=1.0, s2=3.0):
    """B trial functions from the basis rows (GENERATOR_PARAM p1, s1, s2)."""
    rng = np.random.default_rng(seed)
    K, npt = basis.shape
    out = np.empty((B, npt), dtype=np.float64)
    for b in range(B):
        k = int(rng.integers(0, K))
        if rng.uniform() < p1:
            out[b] = (s1 * rng.standard_normal(npt) + 1.0) * basis[k]
        else:
            r = s2 * rng.standard_normal() + 1.0
            while 0.8 < abs(r) < 1.2:
                r = s2 * rng.standard_normal() + 1.0
            out[b] = r * basis[k]
    return out


# e_floor: an energy below the lowest state of each system (the exact
# non-Born-Oppenheimer ground-state energies are about -0.527, -1.164 and
# -7.478 hartree), used as a first inverse-iteration shift.
SYSTEMS = {
    # heavy particle (+1, 1836.15) and two electrons, electron exchange
    "h_minus_like": dict(masses=[1836.15, 1.0, 1.0], charges=[1.0, -1.0, -1.0], symmetry="(1+P23)",
                         e_floor=-0.6),
    # two heavy particles (+1, 1836.15) and two electrons
    "h2_like": dict(masses=[1836.15, 1836.15, 1.0, 1.0], charges=[1.0, 1.0, -1.0, -1.0],
                    symmetry="(1+P12)(1+P34)", e_floor=-1.2),
    # heavy particle (+3, 12786) and three electrons (n = 3, six Y^+Y terms)
    "li_like": dict(masses=[12786.0, 1.0, 1.0, 1.0], charges=[3.0, -1.0, -1.0, -1.0],
                    symmetry="(1+P23)(1-P24)", e_floor=-7.6),
    # five particles (n = 4): heavy particle (+3, 12786) and four electrons,
    # exercising the n = 4 kernels
    "li_minus_like": dict(masses=[12786.0, 1.0, 1.0, 1.0, 1.0], charges=[3.0, -1.0, -1.0, -1.0, -1.0],
                          symmetry="(1+P23)(1+P45)(1-P24)", e_floor=-7.6),
}

# The benchmark configurations: system, basis size K, seed (1000 + index).
CONFIGS = {
    0: dict(system="h_minus_like", K=500, seed=1000),
    1: dict(system="h2_like", K=1500, seed=1001),
    2: dict(system="h2_like", K=4000, seed=1002),
    3: dict(system="h2_like", K=2000, seed=1003, candidates=256),
    4: dict(system="li_like", K=10000, seed=1004, mass_scaled=True),
}


# The K = 10000 workload is described as "5 particles: one heavy particle
# and three electrons, n = 4": that particle list is the n = 3 Li-like
# system of entry 4 above; the five-particle n = 4 reading is this one
# (heavy particle and four electrons), with the same seed, size and mass
# scaling.
CONFIG4_N4 = dict(system="li_minus_like", K=10000, seed=1004, mass_scaled=True)


def systems():
    """The physical systems of the benchmark configurations."""
    return SYSTEMS


def make_system(name):
    from .system import System
    d = SYSTEMS[name]
    return System(d["masses"], d["charges"], d["symmetry"])


def reduced_mass_scale(masses):
    """sqrt(mu_i / m_e) per pseudo-particle, mu_i = m0 m_i / (m0 + m_i)."""
    m = np.asarray(masses, dtype=np.float64)
    mu = m[0] * m[1:] / (m[0] + m[1:])
    return np.sqrt(mu)


def config_basis(index, K=None):
    """(system, params) of benchmark configuration `index` (or "4n4" for
    CONFIG4_N4); K overrides the basis size (the first K functions of the
    full basis are the same)."""
    cfg = CONFIG4_N4 if index == "4n4" else CONFIGS[index]
    sysm = make_system(cfg["system"])
    KK = cfg["K"] if K is None else K
    scale = reduced_mass_scale(SYSTEMS[cfg["system"]]["masses"]) if cfg.get("mass_scaled") else None
    return sysm, random_basis(sysm.n, KK, cfg["seed"], row_scale=scale)
