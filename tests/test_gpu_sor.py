"""GPU solveSOR!/resSOR (NonUniform.jl:680-743, 1004-1051) against the oracle.

Within one colour pass every updated cell reads only cells of the other colour, so the RB-SOR
iterate does not depend on the order of the updates: the GPU field must equal the oracle's bit
for bit after any number of passes.  Only the residual sums (a reduction) differ in rounding.
"""
import io

import numpy as np
import pytest

import h2_b200
from conftest import mode3_model
from test_gpu_kernels import make_solver

pytestmark = pytest.mark.gpu


def test_sor_passes_bit_exact(oracle):
    """300 passes with omega = 1.5 (not converged): identical field, residuals to rounding."""
    prob = mode3_model(oracle, 20)
    ref = mode3_model(oracle, 20)
    n_r, res0_r, hist_r = oracle.solve_sor(ref, omega=1.5, tol=1e-3, maxItr=300)
    assert n_r == -300
    s = make_solver(prob)
    hist = np.zeros(300)
    st, res = s.sor(omega=1.5, tol=1e-3, maxItr=300, hist=hist)
    assert st == h2_b200._lib.H2G_NOT_CONVERGED and not res.isconverged and res.itr == 300
    assert abs(res.res0 - res0_r) <= 1e-13 * res0_r
    assert np.allclose(hist, hist_r, rtol=1e-12, atol=0)
    assert np.array_equal(s.get_theta(), ref.wk["theta"])
    s.close()


def test_sor_converges_like_oracle(oracle):
    """omega = 1.95 to 1e-6 on 20x20x30: the oracle needs 8552 passes."""
    prob = mode3_model(oracle, 20)
    ref = mode3_model(oracle, 20)
    n_r, res0_r, hist_r = oracle.solve_sor(ref, omega=1.95, tol=1e-6, maxItr=20000)
    assert n_r > 0
    s = make_solver(prob)
    hist = np.zeros(20000)
    st, res = s.sor(omega=1.95, tol=1e-6, maxItr=20000, hist=hist)
    assert st == 0 and res.isconverged
    # the stop test compares a reduced sum with tol: rounding can move the crossing by a pass
    assert abs(res.itr - n_r) <= 1, (res.itr, n_r)
    assert hist[res.itr - 1] < 1e-6 <= hist[res.itr - 2]
    th = s.get_theta()
    if res.itr == n_r:
        assert np.array_equal(th, ref.wk["theta"])
    else:
        assert np.abs(th - ref.wk["theta"]).max() <= 1e-3
    s.close()


def test_sor_oneshot_and_log(oracle, capfd):
    """h2g_SolveSOR with host arrays: theta in place, the reference's log lines on stdout and F."""
    prob = mode3_model(oracle, 20)
    w = prob.wk
    theta = np.asfortranarray(w["theta"].copy())
    F = io.StringIO()
    conv, itr, res0 = h2_b200.solveSOR(theta, w["lam"], w["b"], w["mask"], w["rho"], w["cp"], (prob.dx, prob.dy, 1.0),
                                       prob.dt, 1.5, prob.ZC, prob.dZ, prob.HC, F, 1e-3, "gpu", maxItr=40,
                                       is_steady=True, verbose=True)
    assert not conv and itr == 40 and res0 > 0
    out = capfd.readouterr().out.splitlines()
    assert out[0].startswith("Initial residual = ")
    assert len([ln for ln in out if len(ln) == 35 and ln[:10].strip().isdigit()]) == 40
    lines = F.getvalue().splitlines()
    assert len(lines) == 40 and lines[0][:10] == "%10d" % 1
    ref = mode3_model(oracle, 20)
    oracle.solve_sor(ref, omega=1.5, tol=1e-3, maxItr=40)
    assert np.array_equal(theta, ref.wk["theta"])
    h2_b200.load().h2g_release_cached()


def test_sor_bad_omega(oracle):
    prob = mode3_model(oracle, 20)
    s = make_solver(prob)
    with pytest.raises(h2_b200.H2GError):
        s.sor(omega=2.0, tol=1e-3, maxItr=10)
    with pytest.raises(h2_b200.H2GError):
        s.sor(omega=1.0, tol=1e-3, maxItr=0)
    s.close()
