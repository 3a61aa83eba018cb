"""Regenerate bench_k4000.json: the oracle's energy for the benchmark
workload (two heavy particles + two electrons, n = 3, T = 4, the first K =
4000 functions of the seed-1002 synthetic basis).

The shift lambda~ is set as an optimisation run sets it, CURRENT_ENERGY *
INVITPARAMETER (src/main.f90:52) with the example inputs' INVITPARAMETER
1.000001, from the lowest generalized eigenvalue of the oracle's H, S (SciPy
eigh).  The stored energy is then the oracle's EnergyIAM (ComputeMatElem,
GHEPIIS from a start vector of ones, SpecifNorm 0, EIGVAL_TOLERANCE 1e-12,
src/workproc.f90:2010-2060).  bench.py uses lambda~ from this file and checks
the GPU's energy for the unperturbed basis against the stored one.

Usage: python tests/golden/make_bench_fixture.py   (about a minute on 8 cores)
"""
import json
import os
import sys
import time

import numpy as np
import scipy.linalg as sl

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "atom-mol-nonbo_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as orc  # noqa: E402
from ecg_b200 import synth  # noqa: E402

INVIT_PARAMETER = 1.000001


def main(K=4000, cfg=2):
    t0 = time.time()
    sysm, params = synth.config_basis(cfg, K=K)
    o = orc.Oracle(sysm, K)
    o.set_params(params)
    o.compute_mat_elem(1, K, 0.0)
    H = np.tril(o.H[:K, :K]) + np.tril(o.H[:K, :K], -1).conj().T
    S = np.array(o.S[:K, :K])
    e_eigh = float(sl.eigh(H, S, eigvals_only=True, subset_by_index=[0, 0])[0])
    del H, S
    lam = e_eigh * INVIT_PARAMETER
    o.last[:K] = 1.0
    E, err, it = o.energy_ia(1, K, lam, 1e-12, max_iter=20, specif_norm=0)
    out = {"config": cfg, "system": synth.CONFIGS[cfg]["system"], "K": K, "seed": synth.CONFIGS[cfg]["seed"],
           "invit_parameter": INVIT_PARAMETER, "lambda_tilde": lam, "energy_oracle": E,
           "oracle_error_code": int(err), "oracle_iterations": int(it), "energy_scipy_eigh": e_eigh,
           "tol": 1e-12, "start_vector": "ones", "specif_norm": 0}
    dst = os.path.join(HERE, f"bench_k{K}.json")
    with open(dst, "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote", dst, out, f"{time.time() - t0:.1f} s")


if __name__ == "__main__":
    main()
