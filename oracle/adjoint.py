"""Numpy restatement of the steady adjoint gradient (the checker of h2g_adjoint).

TEST INFRASTRUCTURE ONLY (imported by tests/).  Given the oracle's arrays (lambda, mask,
theta with its physical guards) and the adjoint field la (zero guards) it forms, per interior
cell c, the derivative of la^T A theta with respect to ln lambda_c from the face conductances of
CalcAX! (NonUniform.jl:478-486: lambda_f (common.jl:35) times area over distance):

    dJ/dln(lambda_c) = -sum_f c_f w_f (theta_q - theta_c)(la_c - la_q)
    w_f = lambda_q / (lambda_c + lambda_q) for an unmasked neighbour q, 1 for a guard
    dJ/dhsrc_c = -dx dy dz_k la_c
"""
import numpy as np


def lam_f(a, b, ma, mb):
    return 2.0 * a * b / (a + b) * (2.0 - np.floor((ma + mb) / 2.0))


def objective(theta, w, p):
    return float(np.sum(np.where(w != 0, w * theta ** p, 0.0))) ** (1.0 / p)


def adj_rhs(theta, w, p):
    J = objective(theta, w, p)
    return np.asfortranarray(np.where(w != 0, w * theta ** (p - 1.0) * J ** (1.0 - p), 0.0))


def gradients(lam, mask, theta, la, dx, dy, ZC, dZ):
    MX, MY, MZ = lam.shape
    inner = (slice(1, -1),) * 3
    lc, mc, tc, ac = lam[inner], mask[inner], theta[inner], la[inner]
    k = np.arange(1, MZ - 1)
    dz = dZ[k][None, None, :]
    dzm = (ZC[k] - ZC[k - 1])[None, None, :]
    dzp = (ZC[k + 1] - ZC[k])[None, None, :]
    G = np.zeros_like(lc)
    faces = [((slice(0, -2), slice(1, -1), slice(1, -1)), dy * dz / dx),
             ((slice(2, None), slice(1, -1), slice(1, -1)), dy * dz / dx),
             ((slice(1, -1), slice(0, -2), slice(1, -1)), dx * dz / dy),
             ((slice(1, -1), slice(2, None), slice(1, -1)), dx * dz / dy),
             ((slice(1, -1), slice(1, -1), slice(0, -2)), dx * dy / dzm),
             ((slice(1, -1), slice(1, -1), slice(2, None)), dx * dy / dzp)]
    for sl, geo in faces:
        lq, mq, tq = lam[sl], mask[sl], theta[sl]
        aq = la[sl] * mq
        with np.errstate(invalid="ignore", divide="ignore"):
            cf = np.nan_to_num(lam_f(lq, lc, mq, mc)) * geo
            wf = np.where(mq == 0, 1.0, lq / (lc + lq))
        G -= np.where(cf != 0, cf * wf * (tq - tc) * (ac - aq), 0.0)
    G *= mc
    out = np.zeros_like(lam)
    out[inner] = G
    gh = np.zeros_like(lam)
    gh[inner] = -(dx * dy * dz) * ac * mc
    return np.asfortranarray(gh), np.asfortranarray(out)
