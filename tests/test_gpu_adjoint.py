"""Steady adjoint (h2g_adjoint): J = (sum_silicon V theta^8)^(1/8), gradients with respect to the
per-cell heat source and the 13 conductivity log-scales, checked against the oracle's FP64
forward and adjoint solves with a numpy restatement of the gradient, and against central finite
differences of GPU forward solves."""
import numpy as np
import pytest

import h2_b200
from h2_b200 import adjoint as A
from h2_b200 import model as M

pytestmark = pytest.mark.gpu

P = 8.0
NX = 40


def _model(beta, hsrc=None, ID=None):
    _, ZC, _ = M.zgrid(30)
    return M.build_mode3(NX, NX, 30, ID=ID, hsrc=hsrc, lam_scale=A.lam_scale(beta, ZC))


def _solver(m):
    s = h2_b200.Solver(*m.shape)
    w = m.wk
    s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
    s.set_fields(w.lam, w.mask)
    s.set_rhs(w.b)
    s.set_theta(w.theta)
    return s


def _oracle_problem(oracle, m, theta, b):
    wk = {n: np.zeros(m.shape, order="F") for n in oracle._WK_NAMES}
    for n, src in (("mask", m.wk.mask), ("rho", m.wk.rho), ("lam", m.wk.lam), ("cp", m.wk.cp),
                   ("hsrc", m.wk.hsrc)):
        wk[n][...] = src
    wk["theta"][...] = theta
    wk["b"][...] = b
    return oracle.Problem(m.NX, m.NY, m.NZ, m.dx, m.dy, m.dt, True, m.Z, m.ZC, m.dZ, m.HC, m.bcs, m.ID, wk)


@pytest.fixture(scope="module")
def case():
    beta = A.draw_beta(7)
    m = _model(beta)
    w = A.silicon_weights(m.ID, m.dx, m.dy, m.dZ)
    s = _solver(m)
    J, gh, gl, rf, ra = A.steady_gradient(s, w, P, tol=1e-12)
    th = s.get_theta()
    s.close()
    return dict(beta=beta, m=m, w=w, J=J, gh=gh, gl=gl, rf=rf, ra=ra, theta=th)


def test_adjoint_matches_oracle(oracle, case):
    from oracle import adjoint as OA
    m, w = case["m"], case["w"]
    assert case["rf"].isconverged and case["ra"].isconverged
    fwd = _oracle_problem(oracle, m, m.wk.theta, m.wk.b)
    assert oracle.pbicgstab(fwd, tol=1e-12, maxItr=20000, smoother="gs")[0]
    th = fwd.wk["theta"]
    assert np.abs(case["theta"] - th).max() <= 1e-6
    J = OA.objective(th, w, P)
    assert abs(case["J"] - J) <= 1e-12 * J
    g = OA.adj_rhs(th, w, P)
    adj = _oracle_problem(oracle, m, np.zeros(m.shape, order="F"), g)
    assert oracle.pbicgstab(adj, tol=1e-12, maxItr=20000, smoother="gs")[0]
    gh, gl = OA.gradients(m.wk.lam, m.wk.mask, th, adj.wk["theta"], m.dx, m.dy, m.ZC, m.dZ)
    assert np.abs(case["gh"] - gh).max() <= 1e-6 * np.abs(gh).max()
    assert np.abs(case["gl"] - gl).max() <= 1e-6 * np.abs(gl).max()
    pg, pr = A.params_gradient(case["gl"], m.ZC), A.params_gradient(gl, m.ZC)
    assert np.allclose(pg, pr, rtol=1e-6, atol=1e-9 * np.abs(pr).max())
    # more heat anywhere raises J: -A is an M-matrix, so la = A^-1 g <= 0 and dJ/dhsrc >= 0
    assert (case["gh"][1:-1, 1:-1, 1:-1] >= -1e-30).all()


def _J_of(beta, hsrc=None):
    m = _model(beta, hsrc=hsrc)
    s = _solver(m)
    st, res = s.solve("pbicgstab", tol=1e-13, maxItr=20000, smoother="gs")
    assert st == 0
    th = s.get_theta()
    s.close()
    w = A.silicon_weights(m.ID, m.dx, m.dy, m.dZ)
    return float(np.sum(np.where(w != 0, w * th ** P, 0.0))) ** (1.0 / P)


def test_params_gradient_finite_differences(case):
    beta, m = case["beta"], case["m"]
    grad = A.params_gradient(case["gl"], m.ZC)
    h = 1e-4
    scale = np.abs(grad).max()
    for j in (A.NBANDS, 2, 4, 5, 11):  # global, bottom die, power-grid band, ..., heatsink
        e = np.zeros(A.NPARAMS)
        e[j] = h
        fd = (_J_of(beta + e) - _J_of(beta - e)) / (2 * h)
        assert abs(fd - grad[j]) <= 1e-4 * scale + 1e-4 * abs(grad[j]), (j, fd, grad[j])


def test_hsrc_gradient_finite_differences(case):
    m = case["m"]
    rng = np.random.default_rng(11)
    v = np.where(np.isin(m.ID, (2, 7)), rng.random(m.shape), 0.0)
    v = np.asfortranarray(v * 1e8)
    eps = 1e-2
    base = m.wk.hsrc
    fd = (_J_of(case["beta"], hsrc=base + eps * v) - _J_of(case["beta"], hsrc=base - eps * v)) / (2 * eps)
    ad = float(np.sum(case["gh"] * v))
    assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def test_mixed_precision_gradient(case):
    """The same gradients from a handle whose solves use the FP32 preconditioner (H2G_MIXED):
    both solves still converge on the FP64 true residual (to 1e-9: the FP32 smoother's noise
    keeps the mixed solver from much tighter tolerances), so the gradients agree with the FP64
    ones to about that tolerance."""
    m = case["m"]
    w = m.wk
    s = h2_b200.Solver(*m.shape, precision="mixed")
    s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
    s.set_fields(w.lam, w.mask)
    s.set_rhs(w.b)
    s.set_theta(w.theta)
    J, gh, gl, rf, ra = A.steady_gradient(s, case["w"], P, tol=1e-9)
    s.close()
    assert rf.isconverged and ra.isconverged
    assert abs(J - case["J"]) <= 1e-9 * case["J"]
    assert np.abs(gh - case["gh"]).max() <= 1e-4 * np.abs(case["gh"]).max()
    assert np.abs(gl - case["gl"]).max() <= 1e-4 * np.abs(case["gl"]).max()
