"""Host-side mirror of the reference's hot-path interface over the C ABI.

Method names follow the Fortran routines they replace (ComputeMatElem,
ComputeMatElemAndDeriv, GHEPIIS, EnergyIA/IAM, EnergyIB); indices are
1-based and inclusive as in the Fortran.  GHEPIIS error codes 1 (zero
pivot) and 2 (no convergence) are returned, as the reference returns them;
negative ABI statuses (bad arguments, CUDA failures) raise EcgError.
"""
import ctypes as C

import numpy as np

from . import _lib, expc
from ._lib import dptr, iptr

__all__ = ["Context", "EcgError", "probe_fp64_peak", "probe_fp64_tensor_peak"]


class EcgError(RuntimeError):
    def __init__(self, status, what):
        super().__init__(f"{what} failed with status {status}")
        self.status = status


def _check(status, what):
    if status < 0:
        raise EcgError(status, what)
    return status


class Context:
    """One basis on one GPU: device copies of Glob_NonlinParam, Glob_H,
    Glob_S, Glob_diagS, Glob_invD, Glob_c, Glob_LastEigvector, Glob_D."""

    def __init__(self, system, ld, max_nfo=0, method="I", device=0):
        self.lib = _lib.load()
        self.system = system
        self.ld = int(ld)
        self.npt = system.npt
        self.np = system.np
        mm = np.ascontiguousarray(system.mass_matrix_cm, dtype=np.float64)
        ch = np.ascontiguousarray(system.charges, dtype=np.float64)
        ym = np.ascontiguousarray(system.yhy_mats_cm, dtype=np.int32)
        yc = np.ascontiguousarray(system.yhy_coeffs, dtype=np.int32)
        h = C.c_void_p()
        _check(self.lib.ecg_ctx_create(system.n, dptr(mm), dptr(ch), system.T, iptr(ym), iptr(yc), self.ld,
                                       int(max_nfo), method.encode(), int(device), C.byref(h)), "ecg_ctx_create")
        self.h = h
        self.method = method

    # -- lifetime -----------------------------------------------------------
    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.ecg_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- data ---------------------------------------------------------------
    def set_params(self, params, first=1):
        """params: (count, npt) array of (vech L, vech B) rows."""
        p = np.ascontiguousarray(params, dtype=np.float64)
        if p.ndim != 2 or p.shape[1] != self.npt:
            raise ValueError(f"params must be (count, {self.npt})")
        _check(self.lib.ecg_set_params(self.h, dptr(p), int(first), p.shape[0]), "ecg_set_params")

    def set_params_device(self, ptr, first, count):
        """Glob_NonlinParam(:, first:first+count-1) from device memory at
        address ptr (npt x count doubles on the context's device)."""
        _check(self.lib.ecg_set_params_device(self.h, C.c_void_p(int(ptr)), int(first), int(count)),
               "ecg_set_params_device")

    def matrices(self, n):
        H = np.zeros((n, n), dtype=np.complex128, order="F")
        S = np.zeros((n, n), dtype=np.complex128, order="F")
        dS = np.zeros(n)
        dH = np.zeros(n)
        iD = np.zeros(n, dtype=np.complex128)
        _check(self.lib.ecg_get_matrices(self.h, n, H.ctypes.data_as(_lib._dp), S.ctypes.data_as(_lib._dp), n,
                                         dptr(dS), dptr(dH), iD.ctypes.data_as(_lib._dp)), "ecg_get_matrices")
        return H, S, dS, dH, iD

    def set_matrices(self, H=None, S=None, diagS=None, diagH=None):
        """Glob_H, Glob_S (n x n, the context's layout), Glob_diagS, Glob_diagH
        into the context (ecg_set_matrices)."""
        arrs = [None if a is None else np.asfortranarray(a, dtype=np.complex128) for a in (H, S)]
        n = next(a.shape[0] for a in arrs + [diagS, diagH] if a is not None)
        dS = None if diagS is None else np.ascontiguousarray(diagS, dtype=np.float64)
        dH = None if diagH is None else np.ascontiguousarray(diagH, dtype=np.float64)
        _check(self.lib.ecg_set_matrices(self.h, n, None if arrs[0] is None else arrs[0].ctypes.data_as(_lib._dp),
                                         None if arrs[1] is None else arrs[1].ctypes.data_as(_lib._dp), n,
                                         dptr(dS), dptr(dH)), "ecg_set_matrices")

    def store_swap(self, path, n, approx_energy=0.0):
        """StoreMatricesInSwapFile (src/workproc.f90:2244-2311): H and S of
        the first n functions to the reference's swap file."""
        from .inout import pack_swap, write_swap
        H, S, dS, dH, _ = self.matrices(n)
        write_swap(path, pack_swap(H, S, dH, self.method, approx_energy), dS)

    def read_swap(self, path, n, approx_energy=0.0):
        """ReadSwapFileAndDistributeData (src/workproc.f90:2158-2240): H and S
        of n functions from the reference's swap file into the context, the
        'I' layout shifted by approx_energy.  Returns False (and leaves the
        context alone) when the file holds another basis size."""
        from .inout import read_swap, unpack_swap
        got = read_swap(path, n)
        if got is None:
            return False
        P, dS = got
        H, S, dH = unpack_swap(P, self.method, approx_energy)
        self.set_matrices(H, S, dS, dH if self.method == "G" else None)
        return True

    def vectors(self, n):
        c = np.zeros(n, dtype=np.complex128)
        x = np.zeros(n, dtype=np.complex128)
        _check(self.lib.ecg_get_vectors(self.h, n, c.ctypes.data_as(_lib._dp), x.ctypes.data_as(_lib._dp)),
               "ecg_get_vectors")
        return c, x

    def set_vectors(self, n, c=None, last_eigvec=None):
        cc = None if c is None else np.ascontiguousarray(c, dtype=np.complex128)
        xx = None if last_eigvec is None else np.ascontiguousarray(last_eigvec, dtype=np.complex128)
        _check(self.lib.ecg_set_vectors(self.h, n, None if cc is None else cc.ctypes.data_as(_lib._dp),
                                        None if xx is None else xx.ctypes.data_as(_lib._dp)), "ecg_set_vectors")

    def deriv(self, nfo, nfa):
        D = np.zeros((nfa, nfo, 2 * self.npt), dtype=np.complex128)
        _check(self.lib.ecg_get_deriv(self.h, nfo, nfa, D.ctypes.data_as(_lib._dp)), "ecg_get_deriv")
        return np.transpose(D, (2, 1, 0))  # Glob_D(m, i, j)

    def gradient(self, nfo):
        g = np.zeros(nfo * self.npt)
        _check(self.lib.ecg_get_gradient(self.h, nfo, dptr(g)), "ecg_get_gradient")
        return g

    # -- reference routines -------------------------------------------------
    def compute_mat_elem(self, nmin, nmax, approx_energy):
        """ComputeMatElem(Nmin, Nmax) with StoreHS, src/matform.f90:119-230."""
        _check(self.lib.ecg_compute_mat_elem(self.h, nmin, nmax, float(approx_energy)), "ecg_compute_mat_elem")

    def compute_mat_elem_and_deriv(self, nmin, nmax, nfru, approx_energy):
        """ComputeMatElemAndDeriv(Nmin, Nmax) with StoreHSD, src/matform.f90:234-360."""
        _check(self.lib.ecg_compute_mat_elem_and_deriv(self.h, nmin, nmax, nfru, float(approx_energy)),
               "ecg_compute_mat_elem_and_deriv")

    def ghepiis(self, k, n, apprlambda, tol, max_iter=20, specif_norm=-1):
        """GHEPIIS, src/linalg.f90:1781-1926.  Returns (lambda, RelAcc,
        NumIter, ErrorCode)."""
        lam, ra, it = C.c_double(), C.c_double(), C.c_int()
        err = _check(self.lib.ecg_ghepiis(self.h, k, n, float(apprlambda), float(tol), int(max_iter),
                                          int(specif_norm), C.byref(lam), C.byref(ra), C.byref(it)), "ecg_ghepiis")
        return lam.value, ra.value, it.value, err

    def energy_ia(self, nmin, nmax, approx_energy, tol, max_iter=20, mat_elem_needed=True, specif_norm=-1):
        """EnergyIA (specif_norm=-1) / EnergyIAM (0), src/workproc.f90:1954-2060.
        Returns (E, ErrorCode, NumIter)."""
        e, it = C.c_double(), C.c_int()
        err = _check(self.lib.ecg_energy_ia(self.h, nmin, nmax, int(bool(mat_elem_needed)), float(approx_energy),
                                            float(tol), int(max_iter), int(specif_norm), C.byref(e), C.byref(it)),
                     "ecg_energy_ia")
        return e.value, err, it.value

    def _energy_ib(self, fn, name, nfru, nfa, approx_energy, tol, max_iter, mat_elem_needed, want_grad):
        e, it = C.c_double(), C.c_int()
        g = np.zeros((nfa - nfru) * self.npt) if want_grad else None
        err = _check(fn(self.h, nfru, nfa, int(bool(mat_elem_needed)), float(approx_energy), float(tol),
                        int(max_iter), C.byref(e), dptr(g), C.byref(it)), name)
        return e.value, g, err, it.value

    def energy_ib(self, nfru, nfa, approx_energy, tol, max_iter=20, mat_elem_needed=True, want_grad=True):
        """EnergyIB, src/workproc.f90:2063-2154 (plain: Glob_D formed and
        contracted).  Returns (E, gradient, ErrorCode, NumIter)."""
        return self._energy_ib(self.lib.ecg_energy_ib, "ecg_energy_ib", nfru, nfa, approx_energy, tol, max_iter,
                               mat_elem_needed, want_grad)

    def energy_ib_adjoint(self, nfru, nfa, approx_energy, tol, max_iter=20, mat_elem_needed=True, want_grad=True):
        """EnergyIB through the fused adjoint pass (no Glob_D)."""
        return self._energy_ib(self.lib.ecg_energy_ib_adjoint, "ecg_energy_ib_adjoint", nfru, nfa, approx_energy,
                               tol, max_iter, mat_elem_needed, want_grad)

    def energy_ga(self, nmin, nmax, which=1, want_vector=False, mat_elem_needed=True):
        """EnergyGA / EnergyGAM (src/workproc.f90:1697-1838) for a 'G'
        context: the which-th eigenvalue with ZHEGVX(RANGE='I') semantics.
        Returns (E, ErrorCode, number of LDL^H factorisations)."""
        e, nf = C.c_double(), C.c_int()
        err = _check(self.lib.ecg_energy_ga(self.h, int(nmin), int(nmax), int(bool(mat_elem_needed)), int(which),
                                            int(bool(want_vector)), C.byref(e), C.byref(nf)), "ecg_energy_ga")
        return e.value, err, nf.value

    def energy_gb(self, nfru, nfa, which=1, mat_elem_needed=True):
        """EnergyGB (src/workproc.f90:1841-1950), plain drop-in: Glob_D
        formed by ComputeMatElemAndDeriv, then contracted.  Needs a 'G'
        context with max_nfo >= nfa - nfru.  Returns (E, gradient, ErrorCode)."""
        e = C.c_double()
        g = np.zeros((nfa - nfru) * self.npt)
        err = _check(self.lib.ecg_energy_gb(self.h, int(nfru), int(nfa), int(bool(mat_elem_needed)), int(which),
                                            C.byref(e), dptr(g)), "ecg_energy_gb")
        return e.value, g, err

    def energy_gb_adjoint(self, nfru, nfa, which=1, mat_elem_needed=True):
        """EnergyGB (src/workproc.f90:1841-1950) through the fused adjoint
        pass.  Returns (E, gradient, ErrorCode)."""
        e = C.c_double()
        g = np.zeros((nfa - nfru) * self.npt)
        err = _check(self.lib.ecg_energy_gb_adjoint(self.h, int(nfru), int(nfa), int(bool(mat_elem_needed)),
                                                    int(which), C.byref(e), dptr(g)), "ecg_energy_gb_adjoint")
        return e.value, g, err

    def overlap_penalty(self, nfru, nfa, max_pair_overlap_penalty, overlap_threshold2, mode=0):
        """ComputeOverlapPenalty (mode 0) / ComputeOverlapPenaltyAndAddGradient
        (mode 1: the reference's gradient added to the context's gradient;
        mode 2: the exact derivative of the penalty instead),
        src/workproc.f90:1491-1693.  Returns (TotalPenalty, updated gradient
        or None)."""
        tp = C.c_double()
        g = np.zeros((nfa - nfru) * self.npt) if mode else None
        _check(self.lib.ecg_overlap_penalty(self.h, int(nfru), int(nfa), float(max_pair_overlap_penalty),
                                            float(overlap_threshold2), int(mode), C.byref(tp), dptr(g)),
               "ecg_overlap_penalty")
        return tp.value, g

    def expectation_values(self, nbasis, energy, c=None, method=1, cf_grid=None, dens_grid=None, raw=False):
        """The expectation-value pass of ExpectationValuesG
        (src/workproc.f90:8159-8366) over functions 1..nbasis with the
        eigenvector c (None: Glob_c, as left by energy_ga(want_vector=True))
        and Glob_CurrEnergy = energy.  method is SymmAdaptMethod (1: Y^+Y on
        the ket, 2: Y on bra and ket).  Returns a dict of named values and
        error bounds (see expc.unpack) plus "cf" (np x ncf) and "dens"
        ((n+1) x ndens) when grids are given; with raw=True the MEkl-ordered
        (values, errors, cf, dens) arrays instead."""
        sysm = self.system
        n = sysm.n
        nv = 6 * self.np + 9
        vals, errs = np.zeros(nv), np.zeros(nv)
        cfg = np.ascontiguousarray(cf_grid if cf_grid is not None else np.zeros(0), dtype=np.float64)
        dg = np.ascontiguousarray(dens_grid if dens_grid is not None else np.zeros(0), dtype=np.float64)
        cf = np.zeros((self.np, max(cfg.size, 1)), order="F")
        dens = np.zeros((n + 1, max(dg.size, 1)), order="F")
        masses = np.ascontiguousarray(sysm.masses, dtype=np.float64)
        ym = np.ascontiguousarray(sysm.y_mats_cm, dtype=np.int32)
        yc = np.ascontiguousarray(sysm.y_coeffs, dtype=np.int32)
        cc = None
        if c is not None:
            cc = np.ascontiguousarray(np.asarray(c)[:nbasis], dtype=np.complex128).view(np.float64)
        _check(self.lib.ecg_expectation_values(self.h, int(nbasis), dptr(masses), int(method), len(yc), iptr(ym),
                                               iptr(yc), float(energy), dptr(cc), cfg.size, dptr(cfg), dg.size,
                                               dptr(dg), dptr(vals), dptr(errs), dptr(cf), dptr(dens)),
               "ecg_expectation_values")
        cf, dens = cf[:, :cfg.size], dens[:, :dg.size]
        if raw:
            return vals, errs, cf, dens
        out = expc.unpack(vals, errs, n)
        if cfg.size:
            out["cf"] = cf
        if dg.size:
            out["dens"] = dens
        return out

    def expectation_values_g(self, nbasis, which=1, method=1, cf_grid=None, dens_grid=None):
        """ExpectationValuesG (src/workproc.f90:7785-8366) for a 'G'
        context: ComputeMatElem(1, nbasis), the which-th eigenpair (ZHEGVX
        semantics, c^H S c = 1), then the expectation-value pass with
        Glob_CurrEnergy = that eigenvalue.  Returns the dict of
        expectation_values with "E" added."""
        E, err, _ = self.energy_ga(1, nbasis, which=which, want_vector=True)
        if err != 0:
            raise EcgError(err, "ExpectationValuesG eigenproblem")
        out = self.expectation_values(nbasis, E, None, method, cf_grid, dens_grid)
        out["E"] = E
        return out

    def eval_candidates(self, nbase, candidates, approx_energy, tol, max_iter=20):
        """The BasisEnlI trial loop (src/workproc.f90:4054-4070) for a batch:
        for each row of `candidates` (count, npt), the energy of
        EnergyIA(nbase+1, nbase+1) with that function as basis function
        nbase+1.  Returns (E, ErrorCode, NumIter, RelAcc), one entry per
        candidate; the context's basis is left unchanged."""
        cand = np.ascontiguousarray(candidates, dtype=np.float64)
        if cand.ndim != 2 or cand.shape[1] != self.npt:
            raise ValueError(f"candidates must be (count, {self.npt})")
        cnt = cand.shape[0]
        E = np.zeros(cnt)
        err = np.zeros(cnt, dtype=np.int32)
        it = np.zeros(cnt, dtype=np.int32)
        ra = np.zeros(cnt)
        _check(self.lib.ecg_eval_candidates(self.h, int(nbase), cnt, dptr(cand), float(approx_energy), float(tol),
                                            int(max_iter), dptr(E), iptr(err), iptr(it), dptr(ra)),
               "ecg_eval_candidates")
        return E, err, it, ra

    def eval_candidates_grad(self, nbase, candidates, approx_energy, tol, max_iter=20):
        """eval_candidates plus, per candidate, the gradient EnergyIB(nbase,
        nbase+1) (src/workproc.f90:2063-2154) returns for it as function
        nbase+1.  Returns (E, ErrorCode, NumIter, RelAcc, grad (count, npt))."""
        cand = np.ascontiguousarray(candidates, dtype=np.float64)
        if cand.ndim != 2 or cand.shape[1] != self.npt:
            raise ValueError(f"candidates must be (count, {self.npt})")
        cnt = cand.shape[0]
        E = np.zeros(cnt)
        err = np.zeros(cnt, dtype=np.int32)
        it = np.zeros(cnt, dtype=np.int32)
        ra = np.zeros(cnt)
        g = np.zeros((cnt, self.npt))
        _check(self.lib.ecg_eval_candidates_grad(self.h, int(nbase), cnt, dptr(cand), float(approx_energy),
                                                 float(tol), int(max_iter), dptr(E), iptr(err), iptr(it), dptr(ra),
                                                 dptr(g)), "ecg_eval_candidates_grad")
        return E, err, it, ra, g

    def matrix_elements(self, pk, pl, terms, gradflag=0):
        """MatrixElements for a batch: returns H, S (count,) and Dk, Dl
        (count, 4np) complex (None when not requested)."""
        pk = np.ascontiguousarray(pk, dtype=np.float64)
        pl = np.ascontiguousarray(pl, dtype=np.float64)
        t = np.ascontiguousarray(terms, dtype=np.int32)
        cnt = t.size
        hs = np.zeros((cnt, 2), dtype=np.complex128)
        dk = np.zeros((cnt, 4 * self.np), dtype=np.complex128) if gradflag in (1, 3) else None
        dl = np.zeros((cnt, 4 * self.np), dtype=np.complex128) if gradflag in (2, 3) else None
        _check(self.lib.ecg_matrix_elements(self.h, cnt, dptr(pk), dptr(pl), iptr(t), int(gradflag),
                                            hs.ctypes.data_as(_lib._dp),
                                            None if dk is None else dk.ctypes.data_as(_lib._dp),
                                            None if dl is None else dl.ctypes.data_as(_lib._dp)),
               "ecg_matrix_elements")
        return hs[:, 0], hs[:, 1], dk, dl

    # -- diagnostics --------------------------------------------------------
    def launch_count(self):
        return int(self.lib.ecg_launch_count(self.h))

    def set_timing(self, on=True):
        _check(self.lib.ecg_set_timing(self.h, int(bool(on))), "ecg_set_timing")

    def stage_ms(self):
        ms = np.zeros(4)
        _check(self.lib.ecg_get_stage_ms(self.h, dptr(ms)), "ecg_get_stage_ms")
        return ms

    def sync(self):
        _check(self.lib.ecg_sync(self.h), "ecg_sync")

    def timer_start(self):
        _check(self.lib.ecg_timer_start(self.h), "ecg_timer_start")

    def timer_stop(self):
        ms = C.c_double()
        _check(self.lib.ecg_timer_stop(self.h, C.byref(ms)), "ecg_timer_stop")
        return ms.value

    # -- pair tiles split over ranks (see ecg_pair_tiles in ecg_abi.h) ------
    def pair_tiles(self, nmin, nmax):
        n = C.c_longlong()
        _check(self.lib.ecg_pair_tiles(self.h, int(nmin), int(nmax), C.byref(n)), "ecg_pair_tiles")
        return n.value

    def compute_mat_elem_tiles(self, nmin, nmax, approx_energy, first, count):
        _check(self.lib.ecg_compute_mat_elem_tiles(self.h, int(nmin), int(nmax), float(approx_energy), int(first),
                                                   int(count)), "ecg_compute_mat_elem_tiles")

    def pack_tiles(self, nmin, nmax, first, count, ptr):
        _check(self.lib.ecg_pack_tiles(self.h, int(nmin), int(nmax), int(first), int(count), C.c_void_p(int(ptr))),
               "ecg_pack_tiles")

    def unpack_tiles(self, nmin, nmax, first, count, ptr):
        _check(self.lib.ecg_unpack_tiles(self.h, int(nmin), int(nmax), int(first), int(count),
                                         C.c_void_p(int(ptr))), "ecg_unpack_tiles")

    def adjoint_part_doubles(self):
        n = C.c_longlong()
        _check(self.lib.ecg_adjoint_part_doubles(self.h, C.byref(n)), "ecg_adjoint_part_doubles")
        return n.value

    def adjoint_tiles(self, nfru, nfa, energy, first, count, ptr):
        _check(self.lib.ecg_adjoint_tiles(self.h, int(nfru), int(nfa), float(energy), int(first), int(count),
                                          C.c_void_p(int(ptr))), "ecg_adjoint_tiles")

    def adjoint_finish(self, nfru, nfa, ptr):
        g = np.zeros((nfa - nfru) * self.npt)
        _check(self.lib.ecg_adjoint_finish(self.h, int(nfru), int(nfa), C.c_void_p(int(ptr)), dptr(g)),
               "ecg_adjoint_finish")
        return g

    def tuning(self):
        """The autotuner's choices: dict(pair_shape, adjoint_shape,
        cand_row_shape, times_ms) (-1: not tuned yet)."""
        a, b, cc = C.c_int(), C.c_int(), C.c_int()
        t = np.zeros(6)
        _check(self.lib.ecg_get_tuning(self.h, C.byref(a), C.byref(b), C.byref(cc), dptr(t)), "ecg_get_tuning")
        return {"pair_shape": a.value, "adjoint_shape": b.value, "cand_row_shape": cc.value,
                "pair_shape_ms": t[:4].round(4).tolist(), "adjoint_shape_ms": t[4:].round(4).tolist()}

    def set_pivot_mode(self, mode):
        """LDL^H pivots: 0 real (default), 1 complex as the reference."""
        _check(self.lib.ecg_set_pivot_mode(self.h, int(mode)), "ecg_set_pivot_mode")

    def set_wait_limit(self, polls):
        """Poll limit of the bounded device waits (< 0: default)."""
        _check(self.lib.ecg_set_wait_limit(self.h, int(polls)), "ecg_set_wait_limit")

    def set_factor_mode(self, mode):
        """Whole-matrix LDL^H: 0 persistent tile kernel (default), 1 one launch per panel step."""
        _check(self.lib.ecg_set_factor_mode(self.h, int(mode)), "ecg_set_factor_mode")

    def factor_trace(self, n):
        """One traced persistent factorisation of the current matrix
        (ecg_factor_trace): an (records, 4) uint64 array."""
        cnt = C.c_longlong()
        np_ = (n + 63) // 64
        total = np_ + np_ * (np_ - 1) // 2 + (np_ - 1) * np_ * (np_ + 1) // 6
        total += sum(2 * (np_ - s - 2) for s in range(max(0, np_ - 2)))  # band updates in two halves
        out = np.zeros((total, 4), dtype=np.uint64)
        _check(self.lib.ecg_factor_trace(self.h, int(n), C.c_void_p(out.ctypes.data), out.size, C.byref(cnt)),
               "ecg_factor_trace")
        return out[:cnt.value]

    def io_bytes(self):
        a, b = C.c_longlong(), C.c_longlong()
        _check(self.lib.ecg_io_bytes(self.h, C.byref(a), C.byref(b)), "ecg_io_bytes")
        return a.value, b.value


def probe_fp64_peak(device=0):
    """Measured FP64 FMA throughput of the device in TFLOP/s."""
    lib = _lib.load()
    t = C.c_double()
    _check(lib.ecg_probe_fp64_peak(int(device), C.byref(t)), "ecg_probe_fp64_peak")
    return t.value


def probe_fp64_tensor_peak(device=0):
    """Measured FP64 tensor-core (mma.sync f64) throughput in TFLOP/s."""
    lib = _lib.load()
    t = C.c_double()
    _check(lib.ecg_probe_fp64_tensor_peak(int(device), C.byref(t)), "ecg_probe_fp64_tensor_peak")
    return t.value
