"""ctypes front end of the CPU oracle (liboracle.so, built from
ecg_oracle.c by the Makefile in this folder).

TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.
The product (libecgb200.so and the ecg_b200 package) never imports this.

The glue functions below restate EnergyIA / EnergyIAM / EnergyIB
(src/workproc.f90:1954-2154) on top of the C restatements of
ComputeMatElem(AndDeriv), GHEPIIS and the gradient contraction, and the
term list of ExpectationValuesG (src/workproc.f90:8175-8347) on top of the
C restatement of its accumulation loop.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def build():
    src = os.path.join(HERE, "ecg_oracle.c")
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(LIB)
        lib.orc_set_system.argtypes = [C.c_int, C.c_int, _dp, _dp, _ip, _ip]
        lib.orc_set_system.restype = C.c_int
        lib.orc_matrix_elements.argtypes = [_dp, _dp, _ip, _dp, _dp, _dp, C.c_int]
        lib.orc_compute_mat_elem.argtypes = [_dp, C.c_int, C.c_int, C.c_char, C.c_double, _dp, _dp, C.c_int, _dp, _dp]
        lib.orc_compute_mat_elem_and_deriv.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_char, C.c_double, _dp,
                                                       _dp, C.c_int, _dp, _dp, _dp, C.c_int]
        lib.orc_ldlhf.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, _dp]
        lib.orc_ldlhf.restype = C.c_int
        lib.orc_ldlhf_par.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, _dp]
        lib.orc_ldlhf_par.restype = C.c_int
        lib.orc_set_ldlhf_mode.argtypes = [C.c_int]
        lib.orc_term_magnitudes.argtypes = [_dp, C.c_int, _dp, _dp]
        lib.orc_ldlhs.argtypes = [C.c_int, _dp, C.c_int, _dp, _dp, _dp]
        lib.orc_vmmhmv.argtypes = [C.c_int, _dp, C.c_int, _dp]
        lib.orc_vmmhmv.restype = C.c_double
        lib.orc_ghepiis.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _dp, _dp, C.c_int, C.c_double, _dp, _dp,
                                    C.c_double, _dp, C.c_int, C.c_int, _dp, _ip]
        lib.orc_ghepiis.restype = C.c_int
        lib.orc_gradient_contract.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_int, _dp, C.c_double, _dp]
        lib.orc_set_masses.argtypes = [_dp]
        lib.orc_expc_matrix_elements.argtypes = [_dp, _dp, _ip, _ip, C.c_double, _dp, C.c_int, _dp, _dp, C.c_int,
                                                 _dp, _dp]
        lib.orc_expectation_values.argtypes = [_dp, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp, _dp, C.c_int,
                                               C.c_double, C.c_int, _dp, C.c_int, _dp, _dp, _dp, _dp, _dp]
        lib.orc_set_masses_ld.argtypes = [_dp]
        lib.orc_expectation_values_ld.argtypes = lib.orc_expectation_values.argtypes
        lib.orc_overlap_penalty.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp, _dp,
                                            C.c_int, _dp, C.c_int]
        lib.orc_overlap_penalty.restype = C.c_double
        lib.orc_set_threads.argtypes = [C.c_int]
        lib.orc_get_threads.restype = C.c_int
        lib.orc_set_threads(host_threads())
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def host_threads():
    """CPUs this process can use: its affinity mask, capped by a cgroup CPU
    quota when one is set (an OpenMP team larger than the quota
    oversubscribes the cores, which the parallel LDLHF branch's per-chunk
    barriers do not tolerate)."""
    n = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    try:
        quota, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(int(quota) // int(period))))
    except (OSError, ValueError):
        pass
    return max(1, n)


def set_threads(n):
    load().orc_set_threads(int(n))


def get_threads():
    return load().orc_get_threads()


def set_ldlhf_mode(mode):
    """LDLHF branch used by GHEPIIS: 0 serial, 1 parallel (the threads act
    as the MPI ranks), -1 as linalg_setparam picks it for the thread count
    (src/linalg.f90:113-121)."""
    load().orc_set_ldlhf_mode(int(mode))


class Oracle:
    """Oracle state for one system (mirrors the Glob_* arrays on the host)."""

    def __init__(self, system, ld, max_nfo=0):
        self.lib = load()
        self.sys = system
        self.n, self.np, self.npt = system.n, system.np, system.npt
        self.ld = ld
        mm = np.ascontiguousarray(system.mass_matrix_cm, dtype=np.float64)
        ch = np.ascontiguousarray(system.charges, dtype=np.float64)
        ym = np.ascontiguousarray(system.yhy_mats_cm, dtype=np.int32)
        yc = np.ascontiguousarray(system.yhy_coeffs, dtype=np.int32)
        self._keep = (mm, ch, ym, yc)
        assert self.lib.orc_set_system(self.n, system.T, _p(mm), _p(ch), ym.ctypes.data_as(_ip),
                                       yc.ctypes.data_as(_ip)) == 0
        self.H = np.zeros((ld, ld), dtype=np.complex128, order="F")
        self.S = np.zeros((ld, ld), dtype=np.complex128, order="F")
        self.diagS = np.zeros(ld)
        self.diagH = np.zeros(ld)
        self.invD = np.zeros(ld, dtype=np.complex128)
        self.c = np.zeros(ld, dtype=np.complex128)
        self.last = np.zeros(ld, dtype=np.complex128)
        self.max_nfo = max_nfo
        self.D = np.zeros((2 * self.npt, max(max_nfo, 1), ld), dtype=np.complex128, order="F") if max_nfo else None
        self.params = None

    def activate(self):
        """Re-install this system in the C globals (one system at a time)."""
        mm, ch, ym, yc = self._keep
        self.lib.orc_set_system(self.n, self.sys.T, _p(mm), _p(ch), ym.ctypes.data_as(_ip), yc.ctypes.data_as(_ip))

    def set_params(self, params):
        self.params = np.ascontiguousarray(params, dtype=np.float64)

    # MatrixElements with an explicit permutation matrix
    def matrix_elements(self, pk, pl, P, gradflag=0):
        pk = np.ascontiguousarray(pk, dtype=np.float64)
        pl = np.ascontiguousarray(pl, dtype=np.float64)
        Pcm = np.ascontiguousarray(np.asarray(P, dtype=np.int32).T).ravel()
        hs = np.zeros(2, dtype=np.complex128)
        dk = np.zeros(4 * self.np, dtype=np.complex128)
        dl = np.zeros(4 * self.np, dtype=np.complex128)
        self.lib.orc_matrix_elements(_p(pk), _p(pl), Pcm.ctypes.data_as(_ip), _p(hs), _p(dk), _p(dl), gradflag)
        return hs[0], hs[1], dk, dl

    def term_magnitudes(self, K):
        """(aH, aS): for k >= l, sum over the Y^+Y terms of |coef| |H_t(k,l)|
        and |coef| |S_t(k,l)| (lower triangles of K x K arrays)."""
        aH = np.zeros((K, K), order="F")
        aS = np.zeros((K, K), order="F")
        self.lib.orc_term_magnitudes(_p(self.params), K, _p(aH), _p(aS))
        return aH, aS

    def compute_mat_elem(self, nmin, nmax, approx_e, method="I"):
        self.lib.orc_compute_mat_elem(_p(self.params), nmin, nmax, method.encode(), approx_e, _p(self.H), _p(self.S),
                                      self.ld, _p(self.diagS), _p(self.diagH))

    def compute_mat_elem_and_deriv(self, nmin, nmax, nfru, approx_e, method="I"):
        self.lib.orc_compute_mat_elem_and_deriv(_p(self.params), nmin, nmax, nfru, method.encode(), approx_e,
                                                _p(self.H), _p(self.S), self.ld, _p(self.diagS), _p(self.diagH),
                                                _p(self.D), self.D.shape[1])

    def ghepiis(self, k, n, apprlambda, tol, max_iter=20, specif_norm=-1):
        """GHEPIIS on (H, invD, S) with start vector c; eigenvector -> last.
        Returns (lambda, RelAcc, NumIter, ErrorCode)."""
        w = np.zeros(self.ld, dtype=np.complex128)
        out = np.zeros(2)
        it = np.zeros(1, dtype=np.int32)
        err = self.lib.orc_ghepiis(k, n, _p(self.H), self.ld, _p(self.invD), _p(self.S), self.ld, apprlambda,
                                   _p(self.c), _p(w), tol, _p(self.last), max_iter, specif_norm, _p(out),
                                   it.ctypes.data_as(_ip))
        return out[0], out[1], int(it[0]), err

    # EnergyIA / EnergyIAM, src/workproc.f90:1954-2060
    def energy_ia(self, nmin, nmax, approx_e, tol, max_iter=20, mat_elem_needed=True, specif_norm=-1):
        if mat_elem_needed:
            self.compute_mat_elem(nmin, nmax, approx_e)
        if nmax == 1:
            return self.H[0, 0].real + approx_e, 0, 1
        self.c[:nmax] = self.last[:nmax]
        lam, ra, it, err = self.ghepiis(nmin, nmax, approx_e, tol, max_iter, specif_norm)
        return lam, err, it

    # EnergyIB, src/workproc.f90:2063-2154
    def energy_ib(self, nfru, nfa, approx_e, tol, max_iter=20, mat_elem_needed=True):
        nfo = nfa - nfru
        if mat_elem_needed:
            self.compute_mat_elem_and_deriv(nfru + 1, nfa, nfru, approx_e)
        if nfa == 1:
            E, err, it = self.H[0, 0].real + approx_e, 0, 1
            self.c[0] = 1.0
        else:
            self.c[:nfa] = self.last[:nfa]
            E, ra, it, err = self.ghepiis(nfru + 1, nfa, approx_e, tol, max_iter, 0)
            self.c[:nfa] = self.last[:nfa]
        g = np.zeros(nfo * self.npt)
        self.lib.orc_gradient_contract(nfo, nfa, nfru, _p(self.D), self.D.shape[1], _p(self.c), E, _p(g))
        return E, g, err, it

    # ComputeOverlapPenalty(AndAddGradient), src/workproc.f90:1491-1693
    def overlap_penalty(self, nfru, nfa, max_pen, thr2, WkGR=None, exact=False):
        """TotalPenalty from this oracle's Glob_S; with WkGR (npt * nfo
        array) the penalty gradient is added to it in place (needs Glob_D,
        as left by compute_mat_elem_and_deriv): the reference's formula, or
        with exact=True the derivative of the penalty."""
        wk = None
        if WkGR is not None:
            assert WkGR.dtype == np.float64 and WkGR.flags.c_contiguous
            wk = _p(WkGR)
        D = self.D if self.D is not None else np.zeros(1, dtype=np.complex128)
        ldo = self.D.shape[1] if self.D is not None else 1
        return self.lib.orc_overlap_penalty(nfru, nfa, max_pen, thr2, _p(self.S), self.ld, _p(self.diagS), _p(D),
                                            ldo, wk, int(exact))

    # ExpectationValuesG term lists, src/workproc.f90:8175-8347
    def expc_terms(self, method):
        """(Pbra, Pket, coef1, coef2, err_mult) for SymmAdaptMethod 1
        (identity bra, Y^+Y_t ket, YHYCoeff_t) or 2 (Y_k bra, Y_kk ket,
        YCoeff_k YCoeff_kk; k outer, kk inner)."""
        n, sysm = self.n, self.sys
        if method == 1:
            pb = [np.eye(n, dtype=np.int32)] * sysm.T
            pk = list(sysm.yhy_mats)
            c1 = [float(c) for c in sysm.yhy_coeffs]
            c2 = [1.0] * sysm.T
            em = 2
        elif method == 2:
            ny = len(sysm.y_coeffs)
            pb = [sysm.y_mats[k] for k in range(ny) for kk in range(ny)]
            pk = [sysm.y_mats[kk] for k in range(ny) for kk in range(ny)]
            c1 = [float(sysm.y_coeffs[k]) for k in range(ny) for kk in range(ny)]
            c2 = [float(sysm.y_coeffs[kk]) for k in range(ny) for kk in range(ny)]
            em = 3
        else:
            raise ValueError("SymmAdaptMethod is 1 or 2")

        def cm(mats):
            return np.ascontiguousarray(np.array([np.asarray(m).T for m in mats], dtype=np.int32)).ravel()
        return cm(pb), cm(pk), np.array(c1), np.array(c2), em

    def expectation_values(self, K, c, curr_energy, method=1, cf_grid=None, dens_grid=None, diagS=None,
                           extended=False):
        """The accumulation loop of ExpectationValuesG over functions 1..K
        with eigenvector c and Glob_CurrEnergy = curr_energy.  diagS defaults
        to this oracle's (set by compute_mat_elem).  Returns (sums, errs, cf,
        dens): 6np+9 values and error estimates in the MEkl order, cf np x
        ncf, dens (n+1) x ndens.  extended=True evaluates the same source in
        x87 extended precision (a more accurate value of the same sums)."""
        self.activate()
        m = np.ascontiguousarray(self.sys.masses, dtype=np.float64)
        (self.lib.orc_set_masses_ld if extended else self.lib.orc_set_masses)(_p(m))
        fn = self.lib.orc_expectation_values_ld if extended else self.lib.orc_expectation_values
        pb, pk, c1, c2, em = self.expc_terms(method)
        nt = len(c1)
        cf_grid = np.ascontiguousarray(cf_grid if cf_grid is not None else np.zeros(0), dtype=np.float64)
        dens_grid = np.ascontiguousarray(dens_grid if dens_grid is not None else np.zeros(0), dtype=np.float64)
        nv = 6 * self.np + 9
        sums, errs = np.zeros(nv), np.zeros(nv)
        cf = np.zeros((self.np, max(cf_grid.size, 1)), order="F")
        dens = np.zeros((self.n + 1, max(dens_grid.size, 1)), order="F")
        cc = np.ascontiguousarray(c[:K], dtype=np.complex128)
        dS = np.ascontiguousarray((self.diagS if diagS is None else diagS)[:K], dtype=np.float64)
        fn(_p(self.params), K, _p(cc), _p(dS), nt, pb.ctypes.data_as(_ip), pk.ctypes.data_as(_ip), _p(c1), _p(c2),
           em, curr_energy, cf_grid.size, _p(cf_grid), dens_grid.size, _p(dens_grid), _p(sums), _p(errs), _p(cf),
           _p(dens))
        return sums, errs, cf[:, :cf_grid.size], dens[:, :dens_grid.size]

    # BasisEnlI trial loop, src/workproc.f90:4054-4070
    def trial_loop(self, nbase, candidates, approx_e, tol, start, max_iter=20):
        """For each candidate: its parameters become function nbase+1 and
        EnergyIA(nbase+1, nbase+1, .true.) runs (ComputeMatElem of row K,
        then GHEPIIS(K, K) with the bordered LDLHF step).  Every trial starts
        from `start` (Glob_LastEigvector(1:K)).  Requires H, S and the
        LDL^H factor of the first nbase functions.  Returns arrays
        (E, ErrorCode, NumIter, RelAcc)."""
        K = nbase + 1
        base = np.array(self.params[:nbase], dtype=np.float64)
        cands = np.asarray(candidates, dtype=np.float64)
        out = np.zeros(len(cands)), np.zeros(len(cands), dtype=np.int32), np.zeros(len(cands), dtype=np.int32), \
            np.zeros(len(cands))
        for j, cnd in enumerate(cands):
            self.set_params(np.vstack([base, cnd[None, :]]))
            self.compute_mat_elem(K, K, approx_e)
            if K == 1:
                out[0][j], out[1][j], out[2][j], out[3][j] = self.H[0, 0].real + approx_e, 0, 1, 0.0
                continue
            self.c[:K] = start[:K]
            lam, ra, it, err = self.ghepiis(K, K, approx_e, tol, max_iter, -1)
            out[0][j], out[1][j], out[2][j], out[3][j] = lam, err, it, ra
        self.set_params(base)
        return out
