"""The reference's data file (inout.txt) and swap file, so that a GPU context
can start from, and write back, the reference's own checkpoints.

Data file: the keyword layout that ReadIOFile reads (src/workproc.f90:18-433)
and SaveResults writes (src/workproc.f90:436-571): system (PARTICLES,
MASSES, CHARGES, SYMMETRY), state (BASIS_SIZE, CURRENT_ENERGY,
WHICH_EIGENVALUE, tolerances, INVITPARAMETER, GENERATOR_PARAM), the history
line of the current basis size, the BBOP program, the history of every
basis size and one line of nonlinear parameters per basis function.
`write_inout` reproduces SaveResults' formats (Fortran D23.16 numbers,
fixed-width integers), so a file it writes reads back the same in the
reference.

Swap file: StoreMatricesInSwapFile / ReadSwapFileAndDistributeData
(src/workproc.f90:2158-2311) keep H and S between BBOP steps in an
unformatted stream (Intel form='binary', no record markers): the basis size
as a 4-byte integer, a K x K complex(8) matrix P (column-major) and
Glob_diagS(1:K).  P's lower triangle, diagonal included, is the normalised
H without the shift lambda~ (the 'I' layout plus lambda~ S; the 'G' layout's
strict lower triangle with Glob_diagH on the diagonal); its strict upper
triangle holds S's strict lower triangle transposed, P(j,i) = S(i,j), j < i.
`pack_swap` / `unpack_swap` convert between P and a context's layout
exactly as those two routines do.
"""
import struct
from dataclasses import dataclass, field

import numpy as np

__all__ = ["InOutFile", "read_inout", "write_inout", "fortran_d", "read_swap", "write_swap", "pack_swap",
           "unpack_swap"]

BBOP_ACTIONS = ("BASIS_ENL", "OPT_CYCLE", "FULL_OPT1", "EXPC_VALS", "ELIM_LCFN", "ELIM_LND1", "SEPR_LND1",
                "SEPR_FLCF", "DENSITIES", "SAVE_FILE")


def _num(tok):
    return float(tok.replace("D", "E").replace("d", "e"))


def fortran_d(v, w=23, d=16):
    """Fortran's Dw.d edit descriptor: 0.ddd...D+ee, right-justified in w."""
    v = float(v)
    if v == 0.0:
        s = "0." + "0" * d + "D+00"
    else:
        m, e = f"{abs(v):.{d - 1}E}".split("E")
        digits = m.replace(".", "")
        ex = int(e) + 1
        s = ("-" if v < 0 else "") + "0." + digits + ("D%+03d" % ex if abs(ex) < 100 else "%+04d" % ex)
    return s.rjust(w)


@dataclass
class InOutFile:
    """Contents of one data file (the Glob_* variables ReadIOFile sets)."""
    masses: np.ndarray                 # Glob_Mass(1:n+1)
    charges: np.ndarray                # (Glob_PseudoCharge0, Glob_PseudoCharge(1:n))
    symmetry: str                      # Glob_YOperatorString
    current_energy: float
    which_eigenvalue: int
    eigval_tol: float
    invit_parameter: float
    last_eigval_tol: float
    best_eigval_tol: float
    worst_eigval_tol: float
    generator_param: tuple             # (p1, s1, s2)
    bbop: list = field(default_factory=list)     # per step: token list as written
    history: list = field(default_factory=list)  # (energy, cycles, init_func, n_eval) per basis size
    params: np.ndarray = None          # K x npt (vech L, vech B) rows

    @property
    def n(self):
        return len(self.masses) - 1

    @property
    def basis_size(self):
        return 0 if self.params is None else self.params.shape[0]

    def system(self):
        from .system import System
        return System(list(self.masses), list(self.charges), self.symmetry)


def read_inout(path):
    """Parse a data file written by SaveResults (or by hand in its layout)."""
    with open(path) as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    pos = 0

    def field_line(key, count=None):
        nonlocal pos
        parts = lines[pos].split()
        pos += 1
        if parts[0] != key:
            raise ValueError(f"{path}:{pos}: expected {key}, found {parts[0]}")
        return parts[1:] if count is None else parts[1:1 + count]

    npart = int(field_line("PARTICLES")[0])
    n = npart - 1
    masses = np.array([_num(t) for t in field_line("MASSES", npart)])
    charges = np.array([_num(t) for t in field_line("CHARGES", npart)])
    symmetry = lines[pos].split(None, 1)[1].strip()
    if lines[pos].split()[0] != "SYMMETRY":
        raise ValueError(f"{path}:{pos + 1}: expected SYMMETRY")
    pos += 1
    K = int(field_line("BASIS_SIZE")[0])
    d = dict(current_energy=_num(field_line("CURRENT_ENERGY")[0]),
             which_eigenvalue=int(field_line("WHICH_EIGENVALUE")[0]),
             eigval_tol=_num(field_line("EIGVAL_TOLERANCE")[0]),
             invit_parameter=_num(field_line("INVITPARAMETER")[0]),
             last_eigval_tol=_num(field_line("LAST_EIGVAL_TOL")[0]),
             best_eigval_tol=_num(field_line("BEST_EIGVAL_TOL")[0]),
             worst_eigval_tol=_num(field_line("WORST_EIGVAL_TOL")[0]),
             generator_param=tuple(_num(t) for t in field_line("GENERATOR_PARAM", 3)))
    # "=====", the current size's history line, "====="  (ReadIOFile skips them)
    pos += 3
    bbop = []
    while lines[pos].split() and lines[pos].split()[0] in BBOP_ACTIONS:
        bbop.append(lines[pos].split())
        pos += 1
    if not lines[pos].strip().startswith("="):
        raise ValueError(f"{path}:{pos + 1}: expected the line after the BBOP program")
    pos += 1
    history = []
    for i in range(1, K + 1):
        p = lines[pos].split()
        if int(p[0]) != i:
            raise ValueError(f"{path}:{pos + 1}: history line {i} expected")
        history.append((_num(p[1]), int(p[2]), int(p[3]), int(p[4])))
        pos += 1
    pos += 1  # "====="
    npt = n * (n + 1)
    params = np.zeros((K, npt))
    for i in range(K):
        p = lines[pos].split()
        if int(p[0]) != i + 1:
            raise ValueError(f"{path}:{pos + 1}: parameters of function {i + 1} expected")
        params[i] = [_num(t) for t in p[1:1 + npt]]
        pos += 1
    return InOutFile(masses=masses, charges=charges, symmetry=symmetry, bbop=bbop, history=history,
                     params=params, **d)


def _bbop_line(tok):
    """One BBOP step in SaveResults' format for its action."""
    a = tok[0]
    D = fortran_d
    if a == "SAVE_FILE":
        return " %-9s %6d %s" % (a, int(tok[1]), tok[2])
    m = tok[1]
    if a == "BASIS_ENL":
        ints, fl = tok[2:7], tok[7:9]
        return " %s %s" % (a, m) + "".join(" %6d" % int(x) for x in ints) + "".join(" " + D(_num(x)) for x in fl)
    if a == "OPT_CYCLE":
        ints, fl = tok[2:9], tok[9:11]
        return " %s %s" % (a, m) + "".join(" %6d" % int(x) for x in ints) + "".join(" " + D(_num(x)) for x in fl)
    if a == "FULL_OPT1":
        return (" %s %s" % (a, m) + "".join(" %6d" % int(x) for x in tok[2:6]) +
                "".join(" " + D(_num(x)) for x in tok[6:8]) + "".join(" %6d" % int(x) for x in tok[8:10]) +
                " " + tok[10])
    if a == "EXPC_VALS":
        return " %s %s %6d" % (a, m, int(tok[2]))
    if a == "DENSITIES":
        return " %s %s %6d %s %s %s %s" % (a, m, int(tok[2]), tok[3], tok[4], tok[5], tok[6])
    if a in ("ELIM_LCFN", "ELIM_LND1"):
        return " %s %s %6d%s %s" % (a, m, int(tok[2]), D(_num(tok[3])), tok[4])
    if a in ("SEPR_LND1", "SEPR_FLCF"):
        return " %s %s %6d%s %s %s" % (a, m, int(tok[2]), D(_num(tok[3])), D(_num(tok[4])), tok[5])
    raise ValueError(f"unknown BBOP action {a}")


def write_inout(f, path):
    """Write `f` in SaveResults' layout (src/workproc.f90:436-571)."""
    D = fortran_d
    K = f.basis_size
    n = f.n
    out = [" %-9s%3d" % ("PARTICLES", n + 1),
           " MASSES" + "".join(" " + D(m) for m in f.masses),
           " CHARGES" + "".join(" " + D(q) for q in f.charges),
           " SYMMETRY %s" % f.symmetry.strip(),
           " BASIS_SIZE %6d" % K,
           " CURRENT_ENERGY   " + D(f.current_energy),
           " WHICH_EIGENVALUE %6d" % f.which_eigenvalue,
           " EIGVAL_TOLERANCE " + D(f.eigval_tol),
           " INVITPARAMETER   " + D(f.invit_parameter),
           " LAST_EIGVAL_TOL  " + D(f.last_eigval_tol),
           " BEST_EIGVAL_TOL  " + D(f.best_eigval_tol),
           " WORST_EIGVAL_TOL " + D(f.worst_eigval_tol),
           " GENERATOR_PARAM " + " ".join(D(x) for x in f.generator_param),
           " " + "=" * 30]
    e, cyc, ini, nev = f.history[K - 1] if K else (f.current_energy, 0, 0, 0)
    out.append(" %6d %s %6d %6d %7d" % (K, D(e), cyc, ini, nev))
    out.append(" " + "=" * 30)
    out += [_bbop_line(t) for t in f.bbop]
    out.append(" " + "=" * 30)
    out += [" %6d %s %6d %6d %7d" % (i + 1, D(h[0]), h[1], h[2], h[3]) for i, h in enumerate(f.history)]
    out.append(" " + "=" * 30)
    out += [" %6d" % (i + 1) + "".join(" " + D(x) for x in row) for i, row in enumerate(f.params)]
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


# ---------------------------------------------------------------------------
def read_swap(path, K):
    """(P, diagS) from a swap file written for basis size K, or None when the
    file holds another size or was emptied (ReadSwapFileAndDistributeData)."""
    with open(path, "rb") as fh:
        raw = fh.read()
    if len(raw) < 4 or struct.unpack("<i", raw[:4])[0] != K:
        return None
    need = 4 + 16 * K * K + 8 * K
    if len(raw) < need:
        return None
    P = np.frombuffer(raw, dtype=np.complex128, count=K * K, offset=4).reshape((K, K), order="F").copy()
    dS = np.frombuffer(raw, dtype=np.float64, count=K, offset=4 + 16 * K * K).copy()
    return P, dS


def write_swap(path, P, diagS):
    """StoreMatricesInSwapFile's stream: K, P (column-major), diagS."""
    K = P.shape[0]
    with open(path, "wb") as fh:
        fh.write(struct.pack("<i", K))
        fh.write(np.asfortranarray(P, dtype=np.complex128).tobytes(order="F"))
        fh.write(np.asarray(diagS[:K], dtype=np.float64).tobytes())


def pack_swap(H, S, diagH, method, approx_energy):
    """The swap matrix P from a context's H, S (K x K, its layout) and diagH,
    as StoreMatricesInSwapFile forms it."""
    K = H.shape[0]
    P = np.array(H, dtype=np.complex128, order="F")
    low = np.tril_indices(K, -1)
    P[low[1], low[0]] = S[low]  # P(j, i) = S(i, j), j < i
    if method == "G":
        P[np.diag_indices(K)] = diagH[:K]
    else:
        P[np.diag_indices(K)] = H[np.diag_indices(K)] + approx_energy
        P[low] = H[low] + approx_energy * S[low]
    return P


def unpack_swap(P, method, approx_energy):
    """(H, S, diagH) in a context's layout from the swap matrix P, as
    ReadSwapFileAndDistributeData forms them; upper triangles that the layout
    leaves unused are zero."""
    K = P.shape[0]
    low = np.tril_indices(K, -1)
    S = np.zeros((K, K), dtype=np.complex128, order="F")
    S[low] = P[low[1], low[0]]
    H = np.zeros((K, K), dtype=np.complex128, order="F")
    if method == "G":
        H[low] = P[low]
        diagH = P[np.diag_indices(K)].real.copy()
    else:
        S[low[1], low[0]] = np.conj(S[low])
        S[np.diag_indices(K)] = 1.0
        H[np.diag_indices(K)] = P[np.diag_indices(K)] - approx_energy
        H[low] = P[low] - approx_energy * S[low]
        diagH = np.zeros(K)
    return H, S, diagH
