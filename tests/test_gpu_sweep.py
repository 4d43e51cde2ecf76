"""The fused RB-GS sweep (k_rb_sweep: both colours of a sweep in one launch, planes staged in
shared memory by TMA, z-marching in chunks, ping-pong output) against the oracle and against the
colour passes, through the C ABI.

Within one colour every update is independent, so the fused sweep must give exactly the bits of
two colour passes: the 5-sweep preconditioner is compared with `array_equal` to the oracle (FP64)
and to the colour-pass path (FP32), for several z-chunk counts, both dd sources, the model grids
and the hand-built boxes (tiny, odd, one plane, every boundary type, transient).  Whole solves with
the fused sweep must equal the colour-pass solves bit for bit, iteration count included.  The
bounded waits of the kernel are exercised with a zero budget: the solve ends with H2G_TIMEOUT and
the handle keeps working.
"""
import ctypes

import numpy as np
import pytest

import h2_b200
from conftest import mode3_model
from test_gpu_boxes import GRIDS, box_problem
from test_gpu_kernels import CASES, make_solver, random_interior

pytestmark = pytest.mark.gpu

H2G_TIMEOUT = 6
VARIANTS = [(1, False), (2, True), (3, False), (7, True)]


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_fused_preconditioner_bit_exact(oracle, case):
    prob = mode3_model(oracle, **case)
    s = make_solver(prob)
    bb = random_interior(prob.shape, 31)
    ref = oracle.preconditioner(prob, bb, "gs")
    for chunks, dd in VARIANTS:
        s.set_sweep(1, chunks, dd)
        assert s.sweep()[0]
        assert np.array_equal(s.preconditioner(bb, "gs"), ref), (chunks, dd)
    s.set_sweep(0)
    assert not s.sweep()[0]
    assert np.array_equal(s.preconditioner(bb, "gs"), ref)
    s.close()


@pytest.mark.parametrize("transient", [False, True], ids=["steady", "transient"])
@pytest.mark.parametrize("grid", GRIDS, ids=["x".join(map(str, g)) for g in GRIDS])
def test_fused_preconditioner_boxes(oracle, grid, transient):
    """Grids smaller than one tile, odd sizes, NZ = 1 (a chunk count above NZ is clamped), every
    boundary type; the transient boxes take the full 13-term dd (a_p0 per cell)."""
    prob = box_problem(oracle, *grid, seed=sum(grid) + 3, transient=transient)
    s = make_solver(prob)
    bb = random_interior(prob.shape, 5)
    ref = oracle.preconditioner(prob, bb, "gs")
    for chunks, dd in VARIANTS:
        s.set_sweep(1, chunks, dd)
        assert np.array_equal(s.preconditioner(bb, "gs"), ref), (chunks, dd)
    s.close()


def test_fused_fp32_equals_colour_passes(oracle):
    """The FP32 smoother of H2G_MIXED: fused and colour-pass sweeps give the same bits."""
    prob = mode3_model(oracle, 41, 37)
    s = make_solver(prob, precision="mixed")
    bb = random_interior(prob.shape, 8)
    s.set_sweep(0)
    ref = s.preconditioner(bb, "gs")
    pref = oracle.preconditioner(prob, bb, "gs")
    assert np.abs(ref - pref).max() <= 2e-6 * np.abs(pref).max()
    for chunks, dd in VARIANTS:
        s.set_sweep(1, chunks, dd)
        assert np.array_equal(s.preconditioner(bb, "gs"), ref), (chunks, dd)
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("method", ["pbicgstab", "cg"])
def test_fused_solve_identical(oracle, method, precision):
    """A whole solve with fused sweeps equals the colour-pass solve: same iterations, same
    residual history, same field bits."""
    prob = mode3_model(oracle, 40)
    out = []
    for fused in (0, 1):
        s = make_solver(prob, precision=precision)
        s.set_sweep(fused, 2, False)
        hist = np.zeros(20000)
        st, res = s.solve(method, tol=1e-8, maxItr=20000, smoother="gs", hist=hist)
        assert st == 0 and res.isconverged
        out.append((res.itr, hist[:res.itr].copy(), s.get_theta()))
        s.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_fused_solve_matches_oracle(oracle):
    """PBiCGSTAB with the fused sweep forced, against the oracle's FP64 solve (the solve-level
    tolerances of the other solver tests: 1e-3 K, iterations within 10 %)."""
    prob = mode3_model(oracle, 41, 37)
    ref = mode3_model(oracle, 41, 37)
    conv, itr, res0, _ = oracle.pbicgstab(ref, tol=1e-8, maxItr=20000, smoother="gs")
    assert conv
    s = make_solver(prob)
    s.set_sweep(1, 3, False)
    st, res = s.solve("pbicgstab", tol=1e-8, maxItr=20000, smoother="gs")
    assert st == 0 and res.isconverged
    assert abs(res.itr - itr) <= max(2, itr // 10)
    assert abs(res.res0 - res0) <= 1e-12 * res0
    assert np.abs(s.get_theta() - ref.wk["theta"]).max() <= 1e-3
    s.close()


def test_fused_wait_timeout_is_reported(oracle):
    """A zero wait budget makes every bounded wait of the fused sweep give up at once: the
    kernel drains its copies and returns, the solve and the single preconditioner call report
    H2G_TIMEOUT, and with the default budget back the same handle solves normally."""
    prob = mode3_model(oracle, 40)
    s = make_solver(prob)
    s.set_sweep(1, 2, False)
    s.snapshot()
    s.set_wait_limit(0)
    # through the C ABI: the status is returned and copied into the result
    from h2_b200 import _lib as L
    res = L.Result()
    st = L.load().h2g_pbicgstab(s.h, 1e-8, 200, 1, 0, None, ctypes.byref(res))
    assert st == H2G_TIMEOUT and res.status == H2G_TIMEOUT and not res.isconverged
    # the Python mirror raises it, as it does every hard error
    with pytest.raises(h2_b200.H2GError) as e:
        s.solve("pbicgstab", tol=1e-8, maxItr=200, smoother="gs")
    assert e.value.status == H2G_TIMEOUT
    with pytest.raises(h2_b200.H2GError) as e:
        s.preconditioner(random_interior(prob.shape, 1), "gs")
    assert e.value.status == H2G_TIMEOUT
    s.set_wait_limit(2_000_000_000)
    s.snapshot(restore=True)
    st, res = s.solve("pbicgstab", tol=1e-8, maxItr=20000, smoother="gs")
    assert st == 0 and res.isconverged
    s.close()


def test_bench_hook_fused_sweep(oracle):
    """The benchmark hook runs one fused launch per sweep when the handle uses the fused path."""
    prob = mode3_model(oracle, 40)
    s = make_solver(prob)
    s.set_sweep(1, 2, False)
    assert s.sweep() == (True, 2, False)
    assert s.bench_kernel(0, 3) == 3
    s.set_sweep(0)
    assert s.bench_kernel(0, 3) == 6
    s.close()


def test_sweep_controls_reject_bad_arguments(oracle):
    """h2g_set_sweep and h2g_set_wait_limit check their arguments on the host (H2G_BAD_ARG)."""
    from h2_b200 import _lib as L
    prob = mode3_model(oracle, 40)
    s = make_solver(prob)
    lib = L.load()
    assert lib.h2g_set_sweep(s.h, 2, 1, 0) == L.H2G_BAD_ARG
    assert lib.h2g_set_sweep(s.h, 1, 0, 0) == L.H2G_BAD_ARG
    assert lib.h2g_set_sweep(s.h, 1, 256, 0) == L.H2G_BAD_ARG
    assert lib.h2g_set_sweep(s.h, 1, 2, 5) == L.H2G_BAD_ARG
    assert lib.h2g_set_wait_limit(s.h, -1) == L.H2G_BAD_ARG
    assert lib.h2g_set_sweep(None, 0, 1, 0) == L.H2G_BAD_ARG
    s.set_sweep(1, 200, True)  # more chunks than planes: clamped to NZ
    assert s.sweep() == (True, 30, True)
    s.close()
