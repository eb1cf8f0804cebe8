"""The allocation-free residual entry point (sddc_compresid_noalloc).

Some callers cannot call cudaMalloc -- a host that hands out the GPU's memory
from its own pool or budget, a plugin inside a framework that owns the
allocator.  For them the library offers one residual
evaluation that takes every input and output as caller-held device memory
and keeps its working memory in a fixed array inside the library.

This test calls it through the C ABI on two calls in a row and checks its
residual, gradients and running maxima against the regular entry point
(sddc_set_state + sddc_compresid) on the same case.  The file sorts last so
that a run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from helpers import case_channel, case_cylinder, case_periodic
from sddc_b200 import _native
from sddc_b200.solver import Params, Solver, lib

pytestmark = pytest.mark.gpu

_PD = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int)


def _bind():
    L = lib()
    L.sddc_noalloc_scratch_bytes.restype = ctypes.c_size_t
    L.sddc_noalloc_last_error.restype = ctypes.c_char_p
    L.sddc_noalloc_packed_sizes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t),
                                            ctypes.POINTER(ctypes.c_size_t)]
    L.sddc_noalloc_pack_tables.argtypes = [ctypes.c_int, ctypes.c_int, _PD, _PD, _PD, _PI, ctypes.c_int] + \
        [_PI, ctypes.c_int] * 7 + [_PD, _PI]
    L.sddc_compresid_noalloc.argtypes = [ctypes.POINTER(Params), _PD, _PD, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                         ctypes.c_void_p, _PD, ctypes.c_void_p]
    return L


def _p(a, t=_PD):
    return a.ctypes.data_as(t)


def _params(t, ph, precision):
    return Params(N=t.N, ncell=t.ncell, ncellglob=t.ncell, vismode=ph.vismode, artiv=ph.artiv, k_stage=3,
                  precision=precision, cells_per_cta=0, mu=0.0, eta0=0.0, dxcycl=ph.dxcycl, dycycl=ph.dycycl,
                  rinf=ph.rinf, pinf=ph.pinf, uinf=ph.uinf, vinf=ph.vinf, bxinf=ph.bxinf, byinf=ph.byinf)


def _packed(L, t):
    nm, nf = ctypes.c_size_t(), ctypes.c_size_t()
    assert L.sddc_noalloc_packed_sizes(t.N, t.ncell, ctypes.byref(nm), ctypes.byref(nf)) == 0
    met = np.zeros(nm.value)
    faces = np.zeros(nf.value, dtype=np.int32)
    ints = [np.ascontiguousarray(a, dtype=np.int32) for a in
            (t.ibfinter, t.ibfinl, t.ibfout, t.ibfwal, t.ibfsymp, t.ibfree)]
    cyc = np.asfortranarray(t.cyc2fpair, dtype=np.int32)
    if2c = np.asfortranarray(t.IF2C, dtype=np.int32)
    args = []
    for a in ints:
        args += [_p(a, _PI), len(a)]
    args += [_p(cyc, _PI), int(cyc.shape[0])]
    rc = L.sddc_noalloc_pack_tables(t.N, t.ncell, _p(np.asfortranarray(t.S1)), _p(np.asfortranarray(t.S2)),
                                    _p(np.asfortranarray(t.Jac)), _p(if2c, _PI), t.nface, *args, _p(met),
                                    _p(faces, _PI))
    assert rc == 0, L.sddc_noalloc_last_error()
    return met, faces


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("make", [case_cylinder, lambda: case_channel(N=5), case_periodic])
def test_noalloc_matches_regular_entry_point(make, precision):
    import torch

    torch.cuda.init()
    L = _bind()
    m, t, ph, Q = make()
    N, nc = t.N, t.ncell
    assert L.sddc_noalloc_scratch_bytes() == 16 << 20

    # the regular entry point, two evaluations in a row
    s = Solver(t, ph, precision=precision)
    s.set_state(Q)
    ref = []
    for _ in range(2):
        s.compresid()
        st = s.state(resid=True, nablaQs=True)
        mx = s.maxima()
        ref.append((st["resid"], st["nablaQs"], mx["eigvmax"], mx["umax"]))
    s.close()

    # caller-held device memory for every input and output
    met, faces = _packed(L, t)
    dev = torch.device("cuda")
    q_d = torch.from_numpy(np.asfortranarray(Q).ravel(order="F")).to(dev)
    met_d = torch.from_numpy(met).to(dev)
    faces_d = torch.from_numpy(faces).to(dev)
    res_d = torch.zeros(9 * N * N * nc, dtype=torch.float64, device=dev)
    grad_d = torch.zeros(18 * N * N * nc, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    p = _params(t, ph, precision)
    Lm, Mm = np.asfortranarray(t.Lmat), np.asfortranarray(t.Mmat)
    eig, um = 0.0, 0.0
    out = np.zeros(2)
    for call in range(2):
        free_before = torch.cuda.mem_get_info()[0]
        rc = L.sddc_compresid_noalloc(ctypes.byref(p), _p(Lm), _p(Mm), q_d.data_ptr(), met_d.data_ptr(),
                                      faces_d.data_ptr(), eig, um, res_d.data_ptr(), grad_d.data_ptr(),
                                      _p(out), None)
        assert rc == 0, L.sddc_noalloc_last_error()
        if call == 1:  # the first call may load the module that holds the array
            assert torch.cuda.mem_get_info()[0] == free_before
        resid = res_d.cpu().numpy().reshape((9, N, N, nc), order="F")
        grad = grad_d.cpu().numpy().reshape((9, 2, N, N, nc), order="F")
        r_res, r_grad, r_eig, r_um = ref[call]
        if precision == 0:
            assert np.array_equal(resid, r_res) and np.array_equal(grad, r_grad)
        else:
            rel = np.linalg.norm(resid - r_res) / np.linalg.norm(r_res)
            assert rel <= 1e-12
            assert np.allclose(grad, r_grad, rtol=1e-12, atol=1e-14)
        assert out[0] == r_eig and out[1] == r_um
        eig, um = float(out[0]), float(out[1])


def test_noalloc_rejects_oversize_case():
    L = _bind()
    m, t, ph, Q = case_cylinder()
    p = _params(t, ph, 0)
    p.ncell = 10 ** 6  # 1.15 GB of face traces at N = 4
    Lm, Mm = np.asfortranarray(t.Lmat), np.asfortranarray(t.Mmat)
    out = np.zeros(2)
    rc = L.sddc_compresid_noalloc(ctypes.byref(p), _p(Lm), _p(Mm), 1, 1, 1, 0.0, 0.0, 1, 1, _p(out), None)
    assert rc == -1
    assert b"too large" in L.sddc_noalloc_last_error()
