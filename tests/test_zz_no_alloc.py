"""h2g_calcrk_noalloc: CalcRK! for callers that cannot allocate device memory (their memory
belongs to a pool such as CUDA.jl's, or they run a loop that must not stall on cudaMalloc /
cudaFree).  The entry point allocates nothing; its
reduction scratch is a fixed array inside the library.  It must return the same residual as the
handle-based h2g_calcrk, on two calls in a row (the shared scratch keeps the last call's
contents), and refuse grids larger than its scratch.

This file is collected last so that a failure here does not hide any other test's result."""
import ctypes as C

import numpy as np
import pytest

import h2_b200
from h2_b200 import _lib as L
from conftest import mode3_model

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda()


@pytest.mark.parametrize("case", [dict(NX=40), dict(NX=41, NY=37), dict(NX=40, is_steady=False, dt=1e-4)],
                         ids=["mode3", "odd", "transient"])
def test_calcrk_noalloc_matches_calcrk(oracle, case):
    import torch
    prob = mode3_model(oracle, **case)
    w = prob.wk
    rng = np.random.default_rng(5)
    w["theta"][1:-1, 1:-1, 1:-1] += rng.standard_normal(tuple(n - 2 for n in prob.shape))
    steady = prob.is_steady
    # the existing entry point (handle based)
    s = h2_b200.Solver(*prob.shape)
    s.set_grid(prob.ZC, prob.dZ, prob.dx, prob.dy, prob.dt, prob.HC, steady)
    s.set_fields(w["lam"], w["mask"], None if steady else w["rho"], None if steady else w["cp"])
    s.set_rhs(w["b"])
    s.set_theta(w["theta"])
    r_ref, res_ref = s.calc_rk()
    s.close()
    # the allocation-free entry point on device arrays the caller owns
    lib = L.load()
    d = {n: _dev(torch, w[n]) for n in ("theta", "b", "lam", "mask", "rho", "cp")}
    zc = torch.from_numpy(prob.ZC.copy()).cuda()
    dz = torch.from_numpy(prob.dZ.copy()).cuda()
    r = torch.zeros_like(d["theta"])
    HC = np.ascontiguousarray(prob.HC, dtype=np.float64)
    torch.cuda.synchronize()
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    for call in range(2):
        if call == 1:
            r.fill_(123.0)  # stale values must be overwritten on the interior
            torch.cuda.synchronize()
        res = C.c_double(0.0)
        st = lib.h2g_calcrk_noalloc(*prob.shape, ptr(d["theta"]), ptr(d["b"]), ptr(d["lam"]), ptr(d["mask"]),
                                    ptr(d["rho"]), ptr(d["cp"]), ptr(zc), ptr(dz), prob.dx, prob.dy, prob.dt,
                                    HC.ctypes.data_as(C.POINTER(C.c_double)), int(steady), ptr(r), C.byref(res),
                                    None)
        assert st == 0
        got = r.cpu().numpy().reshape(prob.shape, order="F")
        assert np.array_equal(got[1:-1, 1:-1, 1:-1], r_ref[1:-1, 1:-1, 1:-1])
        assert abs(res.value - res_ref) <= 1e-13 * res_ref


def test_calcrk_noalloc_rejects_oversized_grid():
    lib = L.load()
    HC = np.zeros(6)
    res = C.c_double(-1.0)
    one = C.c_void_p(16)  # never dereferenced: the size check comes first
    st = lib.h2g_calcrk_noalloc(10, 1002, 102, one, one, one, one, one, one, one, one, 1e-5, 1e-5, 1.0,
                                HC.ctypes.data_as(C.POINTER(C.c_double)), 1, one, C.byref(res), None)
    assert st == L.H2G_BAD_ARG and res.value == -1.0
