"""Transient adjoint (h2g_adjoint_transient): J on theta after nt implicit steps, gradients with
respect to the heat source and the conductivity log-scales, with checkpointed recomputation.
Checked for independence of the checkpoint spacing, against central finite differences of GPU
forward runs, and against an FP64 reference gradient built from the oracle's solves."""
import numpy as np
import pytest

import h2_b200
from h2_b200 import adjoint as A
from h2_b200 import model as M

pytestmark = pytest.mark.gpu

P = 8.0
NX = 24
DT = 1e-4


def _model(beta=None, hsrc=None):
    _, ZC, _ = M.zgrid(30)
    scale = None if beta is None else A.lam_scale(beta, ZC)
    return M.build_mode3(NX, NX, 30, is_steady=False, dt=DT, hsrc=hsrc, lam_scale=scale)


def _solver(m):
    w = m.wk
    s = h2_b200.Solver(*m.shape)
    s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, False)
    s.set_fields(w.lam, w.mask, w.rho, w.cp)
    s.set_rhs(w.b)
    s.set_theta(w.theta)
    s.set_hsrc(w.hsrc)
    return s


def _weights(m):
    return A.silicon_weights(m.ID, m.dx, m.dy, m.dZ)


def _J_forward(m, nt):
    s = _solver(m)
    st, res, stats = s.transient(m.bcs, nt, tol=1e-13, smoother="gs")
    assert st == 0
    th = s.get_theta()
    s.close()
    w = _weights(m)
    return float(np.sum(np.where(w != 0, w * th ** P, 0.0))) ** (1.0 / P)


def _adjoint(m, nt, k):
    s = _solver(m)
    out = A.transient_gradient(s, m.bcs, nt, _weights(m), P, tol=1e-12, checkpoint_every=k)
    th = s.get_theta()
    s.close()
    return out, th


def test_checkpoint_spacing_does_not_matter():
    m = _model(A.draw_beta(3))
    (J1, gh1, gl1, r1), th1 = _adjoint(m, 6, 1)
    (J2, gh2, gl2, _), th2 = _adjoint(m, 6, 4)
    (J6, gh6, gl6, _), th6 = _adjoint(m, 6, 6)
    assert J1 == J2 == J6
    for a, b in ((gh1, gh2), (gh1, gh6), (gl1, gl2), (gl1, gl6), (th1, th2), (th1, th6)):
        assert np.array_equal(a, b)
    assert r1.outer == 6 and r1.itr > 0
    # theta is left at the final state of the forward run
    s = _solver(m)
    s.transient(m.bcs, 6, tol=1e-12, smoother="gs")
    assert np.array_equal(s.get_theta(), th1)
    s.close()


def test_transient_gradients_finite_differences():
    nt = 8
    beta = A.draw_beta(5)
    m = _model(beta)
    (J, gh, gl, _), _ = _adjoint(m, nt, 3)
    assert abs(J - _J_forward(m, nt)) <= 1e-12 * J
    grad = A.params_gradient(gl, m.ZC)
    scale = np.abs(grad).max()
    h = 1e-4
    for j in (A.NBANDS, 2, 4):
        e = np.zeros(A.NPARAMS)
        e[j] = h
        fd = (_J_forward(_model(beta + e), nt) - _J_forward(_model(beta - e), nt)) / (2 * h)
        assert abs(fd - grad[j]) <= 1e-4 * scale + 1e-4 * abs(grad[j]), (j, fd, grad[j])
    rng = np.random.default_rng(3)
    v = np.asfortranarray(np.where(np.isin(m.ID, (2, 7)), rng.random(m.shape), 0.0) * 1e8)
    eps = 1e-2
    fd = (_J_forward(_model(beta, m.wk.hsrc + eps * v), nt) - _J_forward(_model(beta, m.wk.hsrc - eps * v), nt)) / (
        2 * eps)
    ad = float(np.sum(gh * v))
    assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def _dbdtheta(prob):
    """Per-cell d b / d theta of calRHS! (RHS.jl:140-186, NonUniform.jl:87-90)."""
    MX, MY, MZ = prob.shape
    dz = prob.dZ[None, None, 1:-1]
    w = prob.wk
    d = -(w["rho"] * w["cp"])[1:-1, 1:-1, 1:-1] * prob.dx * prob.dy * dz / prob.dt
    area = [prob.dy * dz, prob.dy * dz, prob.dx * dz, prob.dx * dz, prob.dx * prob.dy, prob.dx * prob.dy]
    for f, (typ, _t, _q, h, _ta) in enumerate(prob.bcs):
        if typ != 2:
            continue
        ax, plus = f // 2, f % 2
        sl = [slice(None)] * 3
        sl[ax] = -1 if plus else 0
        a = np.broadcast_to(area[f], d.shape)[tuple(sl)]
        d[tuple(sl)] += (h * a) if plus else -(h * a)
    out = np.zeros(prob.shape, order="F")
    out[1:-1, 1:-1, 1:-1] = d
    return out


def test_transient_gradient_matches_oracle(oracle):
    from oracle import adjoint as OA
    nt = 3
    m = _model()
    (J, gh, gl, _), _ = _adjoint(m, nt, 2)
    prob = oracle.build_mode3(NX, NX, 30, is_steady=False, dt=DT, calrhs=False)
    w = prob.wk
    states = []
    for _ in range(nt):
        w["b"][...] = 0.0
        oracle.calRHS(prob)
        assert oracle.pbicgstab(prob, tol=1e-13, maxItr=20000, smoother="gs")[0]
        states.append(w["theta"].copy(order="F"))
    wt = _weights(m)
    Jr = OA.objective(states[-1], wt, P)
    assert abs(J - Jr) <= 1e-10 * Jr
    lam = OA.adj_rhs(states[-1], wt, P)
    d = _dbdtheta(prob)
    ghr = np.zeros(prob.shape, order="F")
    glr = np.zeros(prob.shape, order="F")
    adj = oracle.build_mode3(NX, NX, 30, is_steady=False, dt=DT, calrhs=False)
    for q in range(nt - 1, -1, -1):
        adj.wk["theta"][...] = 0.0
        adj.wk["b"][...] = lam
        assert oracle.pbicgstab(adj, tol=1e-13, maxItr=20000, smoother="gs")[0]
        mu = adj.wk["theta"].copy(order="F")
        g1, g2 = OA.gradients(w["lam"], w["mask"], states[q], mu, prob.dx, prob.dy, prob.ZC, prob.dZ)
        ghr += g1
        glr += g2
        lam = np.asfortranarray(d * mu)
    assert np.abs(gh - ghr).max() <= 1e-6 * np.abs(ghr).max()
    assert np.abs(gl - glr).max() <= 1e-6 * np.abs(glr).max()
