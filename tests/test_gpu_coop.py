"""The cooperative preconditioner (k_precond_coop: the first pass and the 9 colour passes of
Preconditioner! in one launch, a bounded grid barrier between passes) against the oracle and
against the ten-launch path.

Within one colour every update is independent, so the one-launch form must give exactly the bits
of the separate passes: the preconditioner is compared with `array_equal` to the oracle on the
model grids and the hand-built boxes (grids smaller than the launch, odd sizes, one plane, every
boundary type, transient) for one and two planes per thread; whole PBiCGSTAB and CG solves equal
the ten-launch solves bit for bit.  A zero wait budget makes the barriers give up: the solve ends
with H2G_TIMEOUT and the handle keeps working.
"""
import ctypes

import numpy as np
import pytest

import h2_b200
from h2_b200 import _lib as L
from conftest import mode3_model
from test_gpu_boxes import GRIDS, box_problem
from test_gpu_kernels import CASES, make_solver, random_interior

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_coop_preconditioner_bit_exact(oracle, case):
    prob = mode3_model(oracle, **case)
    s = make_solver(prob)
    s.set_coop(1)
    assert s.coop()
    bb = random_interior(prob.shape, 31)
    ref = oracle.preconditioner(prob, bb, "gs")
    for planes in (1, 2):
        s.set_tuning(8, planes)
        assert np.array_equal(s.preconditioner(bb, "gs"), ref), planes
    # smoother :none stays a copy
    assert np.array_equal(s.preconditioner(bb, "none"), oracle.preconditioner(prob, bb, "none"))
    s.close()


@pytest.mark.parametrize("transient", [False, True], ids=["steady", "transient"])
@pytest.mark.parametrize("grid", GRIDS, ids=["x".join(map(str, g)) for g in GRIDS])
def test_coop_preconditioner_boxes(oracle, grid, transient):
    prob = box_problem(oracle, *grid, seed=sum(grid) + 7, transient=transient)
    s = make_solver(prob)
    s.set_coop(1)
    bb = random_interior(prob.shape, 9)
    ref = oracle.preconditioner(prob, bb, "gs")
    for planes in (1, 2):
        s.set_tuning(8, planes)
        assert np.array_equal(s.preconditioner(bb, "gs"), ref), planes
    s.close()


@pytest.mark.parametrize("method", ["pbicgstab", "cg"])
@pytest.mark.parametrize("nx,ny", [(40, 40), (41, 37)], ids=["40x40", "41x37"])
def test_coop_solve_identical(oracle, method, nx, ny):
    """Same iterations, residual history and field bits as the ten-launch solve; the launch count
    shows the one-launch preconditioner ran."""
    prob = mode3_model(oracle, nx, ny)
    out = []
    for coop in (0, 1):
        s = make_solver(prob)
        s.set_coop(coop)
        assert s.coop() == bool(coop)
        hist = np.zeros(20000)
        st, res = s.solve(method, tol=1e-8, maxItr=20000, smoother="gs", hist=hist)
        assert st == 0 and res.isconverged
        out.append((res.itr, hist[:res.itr].copy(), s.get_theta(), res.launches))
        s.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
    itr = out[1][0]
    if method == "pbicgstab":  # 2 preconditioners + 2 CalcAX + 1 update per iteration
        assert out[1][3] == 2 + 5 * itr
    else:  # CalcAX + update + preconditioner + dot + p update
        assert out[1][3] == 2 + 1 + 1 + 5 * itr


def test_coop_timeout_is_reported(oracle):
    """A zero wait budget: the barriers give up, the solve and the single preconditioner call
    report H2G_TIMEOUT, and with the default budget back the same handle gives the bits of a
    fresh solve."""
    prob = mode3_model(oracle, 40)
    ref = make_solver(prob)
    st, rr = ref.solve("pbicgstab", tol=1e-8, maxItr=20000, smoother="gs")
    assert st == 0
    s = make_solver(prob)
    s.set_coop(1)
    s.snapshot()
    s.set_wait_limit(0)
    res = L.Result()
    st = L.load().h2g_pbicgstab(s.h, 1e-8, 200, 1, 0, None, ctypes.byref(res))
    assert st == L.H2G_TIMEOUT and res.status == L.H2G_TIMEOUT and not res.isconverged
    with pytest.raises(h2_b200.H2GError) as e:
        s.preconditioner(random_interior(prob.shape, 1), "gs")
    assert e.value.status == L.H2G_TIMEOUT
    s.set_wait_limit(2_000_000_000)
    s.snapshot(restore=True)
    st, res = s.solve("pbicgstab", tol=1e-8, maxItr=20000, smoother="gs")
    assert st == 0 and (res.itr, res.res) == (rr.itr, rr.res)
    assert np.array_equal(s.get_theta(), ref.get_theta())
    s.close()
    ref.close()


def test_coop_controls(oracle):
    prob = mode3_model(oracle, 40)
    lib = L.load()
    s = make_solver(prob)
    assert lib.h2g_set_coop(s.h, 2) == L.H2G_BAD_ARG
    assert lib.h2g_set_coop(None, 1) == L.H2G_BAD_ARG
    assert lib.h2g_get_coop(s.h, None) == L.H2G_BAD_ARG
    s.set_coop(1)
    s.set_sweep(1, 2, False)  # the fused sweep replaces the colour passes: no cooperative launch
    assert not s.coop()
    s.set_coop(1)  # and back: forcing the cooperative launch clears a forced fused sweep
    assert s.coop() and not s.sweep()[0]
    s.close()
    m = make_solver(prob, precision="mixed")
    assert lib.h2g_set_coop(m.h, 1) == L.H2G_UNSUPPORTED
    m.close()


def test_coop_batch_members(oracle):
    """h2g_batch_solve with handles that ask for the cooperative launch: with two solves in flight
    they run the colour passes, alone the cooperative launch; both equal the lone solves."""
    from h2_b200 import batch as B
    members = B.draw_batch(4, 5000, sizes=(24, 32))
    bs = B.BatchSolver(members)
    try:
        bs.restore()
        lone = bs.solve_sequential(tol=1e-8)
        lone_th = bs.thetas()
        for s in bs.solvers:
            s.set_coop(1)
        for threads in (2, 1):
            bs.restore()
            st, res = bs.solve(tol=1e-8, threads=threads)
            assert st == 0
            for a, b_ in zip(lone, res):
                assert (a.itr, a.res) == (b_.itr, b_.res)
            for a, b_ in zip(lone_th, bs.thetas()):
                assert np.array_equal(a, b_)
            per_itr = 5 if threads == 1 else 2 * 10 + 3
            assert all(r.launches == 2 + per_itr * r.itr for r in res), threads
    finally:
        bs.close()
