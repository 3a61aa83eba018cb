"""ecg_adjoint_gradient_noalloc: the adjoint gradient for callers that cannot
allocate device memory when they need it (a host that owns all GPU memory
through its own pool, an optimiser callback that must not fail or fragment
memory mid-run).  Checked against ecg_energy_ib_adjoint, the context path
that allocates its scratch, on two calls in a row (the second call reuses
the library's fixed scratch array left by the first).  The device buffers
here belong to the test, as they would belong to such a caller."""
import ctypes as C

import numpy as np
import pytest
import torch

from ecg_b200 import Context, _lib
from ecg_b200._lib import dptr, iptr
from gpu_util import problem

pytestmark = pytest.mark.gpu

TOL_G = 1e-8  # max |g - g_ref| / max |g_ref|, as in the other gradient tests
ECG_ELIMIT = -5


def _system_args(sysm):
    return (np.ascontiguousarray(sysm.mass_matrix_cm, dtype=np.float64),
            np.ascontiguousarray(sysm.charges, dtype=np.float64),
            np.ascontiguousarray(sysm.yhy_mats_cm, dtype=np.int32),
            np.ascontiguousarray(sysm.yhy_coeffs, dtype=np.int32))


def _noalloc(lib, sysm, args, params_d, c_d, ds_d, energy, nfru, nfa, grad_d, stream=None):
    mm, ch, ym, yc = args
    return lib.ecg_adjoint_gradient_noalloc(sysm.n, dptr(mm), dptr(ch), sysm.T, iptr(ym), iptr(yc),
                                            C.c_void_p(params_d.data_ptr()), C.c_void_p(c_d.data_ptr()),
                                            C.c_void_p(ds_d.data_ptr()), float(energy), nfru, nfa,
                                            C.c_void_p(grad_d.data_ptr()),
                                            None if stream is None else C.c_void_p(stream.cuda_stream))


def _context_reference(cfg, K, nfru):
    """Energy, gradient, eigenvector and diagS from the context path."""
    sysm, params, lam, _ = problem(cfg, K)
    ones = np.ones(K, dtype=np.complex128)
    with Context(sysm, K) as ctx:
        ctx.set_params(params)
        ctx.set_vectors(K, last_eigvec=ones)
        if nfru:
            ctx.compute_mat_elem(1, nfru, lam)
            ctx.set_vectors(nfru, c=ones[:nfru])
            ctx.ghepiis(1, nfru, lam, 1e-12)
            ctx.set_vectors(K, last_eigvec=ones)
        E, g_ref, err, _ = ctx.energy_ib_adjoint(nfru, K, lam, 1e-12)
        c, _ = ctx.vectors(K)
        _, _, dS, _, _ = ctx.matrices(K)
    assert err in (0, 2)
    return sysm, params, E, g_ref, c, dS


@pytest.mark.parametrize("cfg,K,nfru", [(1, 200, 0), (1, 200, 150), (4, 120, 0)])
def test_noalloc_gradient_matches_context_path(cfg, K, nfru):
    sysm, params, E, g_ref, c, dS = _context_reference(cfg, K, nfru)
    lib = _lib.load()
    args = _system_args(sysm)
    dev = torch.device("cuda:0")
    params_d = torch.from_numpy(np.ascontiguousarray(params).ravel()).to(dev)
    c_d = torch.from_numpy(np.ascontiguousarray(c).view(np.float64)).to(dev)
    ds_d = torch.from_numpy(dS).to(dev)
    grad_d = torch.empty((K - nfru) * sysm.npt, dtype=torch.float64, device=dev)
    for call in range(2):
        grad_d.fill_(float("nan"))  # every entry must be written by the call
        torch.cuda.synchronize()
        st = _noalloc(lib, sysm, args, params_d, c_d, ds_d, E, nfru, K, grad_d)
        torch.cuda.synchronize()
        assert st == 0
        g = grad_d.cpu().numpy()
        rel = np.max(np.abs(g - g_ref)) / np.max(np.abs(g_ref))
        print(f"cfg {cfg} K {K} nfru {nfru} call {call}: max rel diff vs context path {rel:.2e}")
        assert np.all(np.isfinite(g)) and rel <= TOL_G


def test_noalloc_on_a_caller_stream():
    """The intended use: the caller queues the call on its own stream and
    synchronises that stream before reading the gradient."""
    K, nfru = 160, 0
    sysm, params, E, g_ref, c, dS = _context_reference(1, K, nfru)
    lib = _lib.load()
    args = _system_args(sysm)
    dev = torch.device("cuda:0")
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        params_d = torch.from_numpy(np.ascontiguousarray(params).ravel()).to(dev, non_blocking=False)
        c_d = torch.from_numpy(np.ascontiguousarray(c).view(np.float64)).to(dev)
        ds_d = torch.from_numpy(dS).to(dev)
        grad_d = torch.full(((K - nfru) * sysm.npt,), float("nan"), dtype=torch.float64, device=dev)
    for call in range(2):
        with torch.cuda.stream(stream):
            grad_d.fill_(float("nan"))
        st = _noalloc(lib, sysm, args, params_d, c_d, ds_d, E, nfru, K, grad_d, stream=stream)
        assert st == 0
        stream.synchronize()
        g = grad_d.cpu().numpy()
        rel = np.max(np.abs(g - g_ref)) / np.max(np.abs(g_ref))
        print(f"caller stream, call {call}: max rel diff vs context path {rel:.2e}")
        assert np.all(np.isfinite(g)) and rel <= TOL_G


def test_noalloc_rejects_sizes_beyond_capacity():
    sysm, params, lam, _ = problem(1, 40)
    lib = _lib.load()
    args = _system_args(sysm)
    dev = torch.device("cuda:0")
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    st = _noalloc(lib, sysm, args, buf, buf, buf, -1.0, 0, 513, buf)
    assert st == ECG_ELIMIT
