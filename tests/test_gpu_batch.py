"""h2g_batch_solve: members solved concurrently give exactly the results of lone solves (the
kernels are deterministic), and match the oracle on the same heat maps."""
import numpy as np
import pytest

from h2_b200 import batch as B
from h2_b200 import model as M

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch():
    ms = B.draw_batch(6, 1000, sizes=(24, 32, 40))
    bs = B.BatchSolver(ms)
    yield bs
    bs.close()


def test_batch_equals_sequential(small_batch):
    bs = small_batch
    bs.restore()
    st, res = bs.solve(tol=1e-8)
    assert st == 0 and all(r.isconverged and r.status == 0 for r in res)
    th_batch = [s.get_theta() for s in bs.solvers]
    bs.restore()
    seq = bs.solve_sequential(tol=1e-8)
    for r, q, s, tb in zip(res, seq, bs.solvers, th_batch):
        assert (r.itr, r.res0, r.res) == (q.itr, q.res0, q.res)
        assert np.array_equal(s.get_theta(), tb)


def test_batch_members_match_oracle(oracle, small_batch):
    bs = small_batch
    bs.restore()
    st, res = bs.solve(tol=1e-8)
    assert st == 0
    _, ZC, _ = M.zgrid(B.NZ)
    for q in (0, 3):
        m = bs.members[q]
        ID = oracle.fill_id(m.nx, m.nx, B.NZ)
        hs = B.heat_map(m, ID, ZC, oracle.pitch(m.nx), oracle.pitch(m.nx))
        prob = oracle.build_mode3(m.nx, m.nx, B.NZ, ID=ID, hsrc=hs)
        conv, itr, res0, _ = oracle.pbicgstab(prob, tol=1e-8, maxItr=20000, smoother="gs")
        assert conv
        assert abs(res[q].res0 - res0) <= 1e-12 * res0
        assert abs(res[q].itr - itr) <= max(1, 0.1 * itr)
        assert np.abs(bs.solvers[q].get_theta() - prob.wk["theta"]).max() <= 1e-3


def test_batch_rejects_duplicates(small_batch):
    import ctypes as C

    from h2_b200 import _lib as L
    s = small_batch.solvers[0]
    hs = (C.c_void_p * 2)(s.h.value, s.h.value)
    outs = (L.Result * 2)()
    assert L.load().h2g_batch_solve(2, hs, 0, 1e-8, 100, 1, 2, outs) == L.H2G_BAD_ARG


@pytest.mark.parametrize("method", ["cg", "sor"])
def test_batch_other_methods_equal_sequential(method):
    """h2g_batch_solve with CG and with solveSOR! (omega = 1): each member gets the results of its
    lone solve through the single-solve call."""
    ms = B.draw_batch(3, 1000, sizes=(24, 32))
    bs = B.BatchSolver(ms)
    try:
        tol, maxItr = (1e-8, 20000) if method == "cg" else (1e-4, 400)
        bs.restore()
        st, res = bs.solve(method=method, tol=tol, maxItr=maxItr)
        th = [s.get_theta() for s in bs.solvers]
        bs.restore()
        seq = bs.solve_sequential(method=method, tol=tol, maxItr=maxItr)
        for r, q, s, t in zip(res, seq, bs.solvers, th):
            assert (r.itr, r.res0, r.res, r.status) == (q.itr, q.res0, q.res, q.status)
            assert np.array_equal(s.get_theta(), t)
        if method == "cg":
            assert all(r.isconverged for r in res)
        with pytest.raises(ValueError):
            bs.solvers[0].solve("sor")
    finally:
        bs.close()
