"""The adjoint-gradient checker (oracle/adjoint.py) against central finite differences of the
oracle's own FP64 solves, on a small Mode-3 model: pins the gradient formula the GPU adjoint is
compared with, independently of the GPU."""
import numpy as np
import pytest

from oracle import adjoint as OA

P = 8.0


def _weights(prob):
    from h2_b200.adjoint import silicon_weights
    return silicon_weights(prob.ID, prob.dx, prob.dy, prob.dZ)


def _solve(oracle, prob):
    prob.wk["b"][...] = 0.0
    oracle.calRHS(prob)
    prob.wk["theta"][1:-1, 1:-1, 1:-1] = 300.0
    assert oracle.pbicgstab(prob, tol=1e-14, maxItr=20000, smoother="gs")[0]
    return prob.wk["theta"].copy(order="F")


def test_gradient_formula_matches_finite_differences(oracle):
    prob = oracle.build_mode3(8, 8, 30, calrhs=False)
    w = _weights(prob)
    th = _solve(oracle, prob)
    g = OA.adj_rhs(th, w, P)
    adj = oracle.build_mode3(8, 8, 30, ID=prob.ID, calrhs=False)
    adj.wk["theta"][...] = 0.0
    adj.wk["b"][...] = g
    assert oracle.pbicgstab(adj, tol=1e-14, maxItr=20000, smoother="gs")[0]
    gh, gl = OA.gradients(prob.wk["lam"], prob.wk["mask"], th, adj.wk["theta"], prob.dx, prob.dy, prob.ZC,
                          prob.dZ)
    rng = np.random.default_rng(4)
    inner = np.argwhere(np.isin(prob.ID[2:-2, 2:-2, 2:-2], (2, 7))) + 2
    cells = [tuple(c) for c in inner[rng.choice(len(inner), 4, replace=False)]]
    for c in cells:
        # ln(lambda_c): scale one interior cell's conductivity (no guard copies it)
        fd = []
        for sgn in (1, -1):
            p2 = oracle.build_mode3(8, 8, 30, ID=prob.ID, calrhs=False)
            p2.wk["lam"][c] *= np.exp(sgn * 1e-4)
            fd.append(OA.objective(_solve(oracle, p2), w, P))
        d = (fd[0] - fd[1]) / 2e-4
        assert abs(d - gl[c]) <= 1e-4 * abs(gl[c]) + 1e-6 * np.abs(gl).max(), (c, d, gl[c])
        # heat source of that cell
        fd = []
        for sgn in (1, -1):
            p2 = oracle.build_mode3(8, 8, 30, ID=prob.ID, calrhs=False)
            p2.wk["hsrc"][c] += sgn * 1e9
            fd.append(OA.objective(_solve(oracle, p2), w, P))
        d = (fd[0] - fd[1]) / 2e9
        assert d == pytest.approx(gh[c], rel=1e-4)
