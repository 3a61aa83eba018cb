"""Regenerate the known-answer fixtures in this folder from the reference's
example inputs.

The reference ships six optimised HD+ bases with the energy each one gives
(example_input/inout_{1,2}_{500,1000,1500}.txt).  This script reads those
keyword files -- the layout written by SaveResults, src/workproc.f90:436-571,
and read by ReadIOFile, src/workproc.f90:18-433 -- and stores the system, the
stored CURRENT_ENERGY, WHICH_EIGENVALUE, INVITPARAMETER, EIGVAL_TOLERANCE and
the K x npt nonlinear parameters in hdplus_fixtures.npz, and copies one of
the files (inout_2_500.txt) unchanged for the data-file reader/writer tests.

Run it with REFERENCE_ROOT set to the root of a checkout of the reference
(the folder holding example_input/).  The tests only read the .npz it writes.
"""
import os
import sys

import numpy as np

REF = os.environ.get("REFERENCE_ROOT")
HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = [f"inout_{w}_{k}" for w in (1, 2) for k in (500, 1000, 1500)]
TEXT_FIXTURE = "inout_2_500"


def _num(tok):
    return float(tok.replace("D", "E").replace("d", "e"))


def read_inout(path):
    with open(path) as fh:
        lines = fh.read().splitlines()
    hdr = {}
    for ln in lines:
        if ln.strip().startswith("="):
            break
        parts = ln.split()
        hdr[parts[0]] = parts[1:]
    npart = int(hdr["PARTICLES"][0])
    n = npart - 1
    npt = n * (n + 1)
    K = int(hdr["BASIS_SIZE"][0])
    # the basis is the last K lines of the file: "i vechL(1:np) vechB(1:np)"
    rows = [ln.split() for ln in lines[-K:]]
    params = np.array([[_num(t) for t in r[1:1 + npt]] for r in rows], dtype=np.float64)
    assert [int(r[0]) for r in rows] == list(range(1, K + 1))
    return dict(
        masses=np.array([_num(t) for t in hdr["MASSES"]]),
        charges=np.array([_num(t) for t in hdr["CHARGES"]]),
        symmetry=" ".join(hdr["SYMMETRY"]),
        K=K,
        energy=_num(hdr["CURRENT_ENERGY"][0]),
        which=int(hdr["WHICH_EIGENVALUE"][0]),
        tol=_num(hdr["EIGVAL_TOLERANCE"][0]),
        invit=_num(hdr["INVITPARAMETER"][0]),
        params=params,
    )


def main():
    if not REF:
        print("set REFERENCE_ROOT to the reference checkout (the folder holding example_input/)", file=sys.stderr)
        return 2
    out = {}
    for name in NAMES:
        d = read_inout(os.path.join(REF, "example_input", name + ".txt"))
        for key, val in d.items():
            out[f"{name}/{key}"] = np.asarray(val)
    dst = os.path.join(HERE, "hdplus_fixtures.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, os.path.getsize(dst), "bytes")
    # one data file verbatim, for the reader/writer round trip (SaveResults'
    # exact text layout)
    src = os.path.join(REF, "example_input", TEXT_FIXTURE + ".txt")
    dst = os.path.join(HERE, TEXT_FIXTURE + ".txt")
    with open(src) as fi, open(dst, "w") as fo:
        fo.write(fi.read())
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    sys.exit(main())
