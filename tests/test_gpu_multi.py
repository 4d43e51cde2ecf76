"""K right-hand sides on one operator (h2g_create_multi / h2g_pbicgstab_multi): the batch members
of one grid size solved together give bit for bit the results of their lone solves -- iterations,
initial and final residuals and every theta value -- including a last group of fewer than the
right-hand sides a thread holds, and after one of them has stopped early.  The API rejects what
it does not implement."""
import numpy as np
import pytest

import h2_b200
from h2_b200 import _lib as L
from h2_b200 import batch as B

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,size", [(6, 32), (9, 24)], ids=["6x32^2", "9x24^2"])
def test_multi_equals_lone_solves(n, size):
    members = B.draw_batch(n, 2000, sizes=(size,))
    lone = B.BatchSolver(members)
    multi = B.MultiBatchSolver(members)
    try:
        lone.restore()
        lone_res = lone.solve_sequential(tol=1e-8)
        lone_th = lone.thetas()
        multi.restore()
        st, res = multi.solve(tol=1e-8)
        assert st == 0
        for a, b_ in zip(lone_res, res):
            assert a.isconverged and b_.isconverged
            assert (a.itr, a.res0, a.res) == (b_.itr, b_.res0, b_.res)
        for a, b_ in zip(lone_th, multi.thetas()):
            assert np.array_equal(a, b_)
        # a second solve from the restored start gives the same bits again
        multi.restore()
        st2, res2 = multi.solve(tol=1e-8)
        assert [(r.itr, r.res) for r in res2] == [(r.itr, r.res) for r in res]
    finally:
        lone.close()
        multi.close()


def test_multi_maxitr_cap():
    """A cap of 30 iterations stops the members that have not converged by then with the status
    and residual of their lone solves; those that converged earlier stopped at their own count."""
    members = B.draw_batch(3, 3000, sizes=(24,))
    lone = B.BatchSolver(members)
    multi = B.MultiBatchSolver(members)
    try:
        lone.restore()
        lone_res = lone.solve_sequential(tol=1e-8, maxItr=30)
        multi.restore()
        st, res = multi.solve(tol=1e-8, maxItr=30)
        for a, b_ in zip(lone_res, res):
            assert (a.itr, a.res, a.status) == (b_.itr, b_.res, b_.status)
        for a, b_ in zip(lone.thetas(), multi.thetas()):
            assert np.array_equal(a, b_)
    finally:
        lone.close()
        multi.close()


def test_multi_api_rejects():
    lib = L.load()
    h = h2_b200.Solver(26, 26, 32)
    assert lib.h2g_set_rhs_multi(h.h, None) == L.H2G_BAD_ARG  # not a multi handle
    h.close()
    import ctypes as C
    out = C.c_void_p()
    assert lib.h2g_create_multi(26, 26, 32, 0, C.byref(out)) == L.H2G_BAD_ARG
    assert lib.h2g_create_multi(26, 26, 32, 65, C.byref(out)) == L.H2G_BAD_ARG
    members = B.draw_batch(2, 4000, sizes=(24,))
    multi = B.MultiBatchSolver(members)
    try:
        ms = multi.groups[0][1]
        outs = (L.Result * 2)()
        assert lib.h2g_pbicgstab_multi(ms.h, 1e-8, 100, 0, outs) == L.H2G_UNSUPPORTED
        assert lib.h2g_pbicgstab_multi(ms.h, 1e-8, 100, 1, None) == L.H2G_BAD_ARG
    finally:
        multi.close()
