"""Differentiation of the steady solve (no reference counterpart): gradients of a smooth
maximum of the temperature over the silicon layers,

    J = (sum_{silicon cells c} V_c theta_c^p)^(1/p),   p = 8,

with respect to the per-cell heat source and to the conductivities, by one adjoint solve on the
GPU (h2g_adjoint).  The conductivity parameters are 13 log-scales: one per z-band between the
layer planes zm0 .. zm12 of the stack (modelA.jl:18-30) and one global factor; a cell of band b
has lambda = lambda_material * exp(beta_b + beta_global).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .nonuniform import Solver, _ptr, smoother_selector

# layer planes of the stack [m] (modelA.jl:18-30)
ZM = np.array([0.0, 0.05e-3, 0.1e-3, 0.195e-3, 0.2e-3, 0.25e-3, 0.345e-3, 0.35e-3, 0.4e-3, 0.495e-3, 0.5e-3,
               0.55e-3, 0.6e-3])
NBANDS = len(ZM) - 1
NPARAMS = NBANDS + 1
SILICON_IDS = (2, 7)


def band_of_plane(ZC: np.ndarray) -> np.ndarray:
    """Band index (0..11) of every plane k by its centre ZC[k]; -1 for the guard planes."""
    b = np.searchsorted(ZM, ZC, side="right") - 1
    b[(ZC < ZM[0]) | (ZC > ZM[-1])] = -1
    b[0] = b[-1] = -1
    return np.minimum(b, NBANDS - 1)


def lam_scale(beta: np.ndarray, ZC: np.ndarray) -> np.ndarray:
    """Per-plane conductivity factor exp(beta_band + beta_global) (1 on guard planes)."""
    beta = np.asarray(beta, dtype=np.float64)
    b = band_of_plane(ZC)
    out = np.ones(ZC.size)
    inner = b >= 0
    out[inner] = np.exp(beta[b[inner]] + beta[NBANDS])
    return out


def draw_beta(seed: int = 7) -> np.ndarray:
    """Parameters perturbed +-20 % log-uniformly: beta ~ U[ln 0.8, ln 1.2]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.uniform(np.log(0.8), np.log(1.2), NPARAMS)


def silicon_weights(ID: np.ndarray, dx: float, dy: float, dZ: np.ndarray) -> np.ndarray:
    """w_c = V_c on the silicon cells (ID 2 and 7), 0 elsewhere (Fortran order)."""
    V = (dx * dy) * np.asarray(dZ)[None, None, :]
    w = np.where(np.isin(ID, SILICON_IDS), V, 0.0)
    w[0], w[-1] = 0.0, 0.0
    w[:, 0], w[:, -1] = 0.0, 0.0
    w[:, :, 0], w[:, :, -1] = 0.0, 0.0
    return np.asfortranarray(w)


def params_gradient(dJ_dlnlam: np.ndarray, ZC: np.ndarray) -> np.ndarray:
    """dJ/dbeta: the per-cell log-conductivity gradient summed over each band, and over all."""
    per_plane = dJ_dlnlam.sum(axis=(0, 1))
    b = band_of_plane(ZC)
    g = np.zeros(NPARAMS)
    for k in range(ZC.size):
        if b[k] >= 0:
            g[b[k]] += per_plane[k]
    g[NBANDS] = g[:NBANDS].sum()
    return g


def steady_gradient(s: Solver, weights: np.ndarray, p: float = 8.0, tol: float = 1e-10, maxItr: int = 20_000,
                    smoother: str = "gs"):
    """h2g_adjoint on a prepared handle (grid, fields, b, theta set).  Returns
    (J, dJ_dhsrc, dJ_dlnlam, forward Result, adjoint Result); theta of the handle is left at the
    forward solution."""
    w = np.asfortranarray(weights, dtype=np.float64)
    J = C.c_double()
    gh = np.zeros(s.shape, order="F")
    gl = np.zeros(s.shape, order="F")
    rf, ra = L.Result(), L.Result()
    st = s.lib.h2g_adjoint(s.h, _ptr(s._arr(w, "weights")), float(p), float(tol), int(maxItr),
                           smoother_selector(smoother), C.byref(J), _ptr(gh), _ptr(gl), C.byref(rf), C.byref(ra))
    L.check(st)
    return J.value, gh, gl, rf, ra


def transient_gradient(s: Solver, bcs, nt: int, weights: np.ndarray, p: float = 8.0, tol: float = 1e-10,
                       maxItr: int = 20_000, smoother: str = "gs", checkpoint_every: int = 0):
    """h2g_adjoint_transient: J on theta after nt implicit steps of the transient model (grid set
    with is_steady=False, rho and cp, hsrc set) and its gradients summed over the steps.
    checkpoint_every = 0 picks ceil(sqrt(nt)).  Returns (J, dJ_dhsrc, dJ_dlnlam, Result)."""
    from .nonuniform import bc_array
    k = int(checkpoint_every) or max(1, int(np.ceil(np.sqrt(nt))))
    w = np.asfortranarray(weights, dtype=np.float64)
    J = C.c_double()
    gh = np.zeros(s.shape, order="F")
    gl = np.zeros(s.shape, order="F")
    res = L.Result()
    st = s.lib.h2g_adjoint_transient(s.h, bc_array(bcs), int(nt), _ptr(s._arr(w, "weights")), float(p), float(tol),
                                     int(maxItr), smoother_selector(smoother), k, C.byref(J), _ptr(gh), _ptr(gl),
                                     C.byref(res))
    L.check(st)
    return J.value, gh, gl, res
