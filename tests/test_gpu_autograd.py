"""The differentiable steady solve (h2_b200.autograd.HotspotNorm, a torch.autograd.Function over
h2g_adjoint) on the 40x40x30 Mode-3 model: J and its gradients through backward() against central
finite differences of GPU forward solves, and torch.autograd.gradcheck on a three-parameter
restriction (one heat-source direction and two log-conductivity directions, constant per z-band).
Solves run to 1e-12, so the difference quotients carry about 1e-7 relative error."""
import numpy as np
import pytest
import torch

import h2_b200
from h2_b200 import adjoint as A
from h2_b200 import autograd as AG
from h2_b200 import model as M

pytestmark = pytest.mark.gpu

P = 8.0


@pytest.fixture(scope="module")
def problem():
    m = M.build_mode3(40, 40, 30)
    w = m.wk
    s = h2_b200.Solver(*m.shape)
    s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
    prob = AG.HotspotProblem(s, w.lam, w.mask, w.theta, m.bcs, A.silicon_weights(m.ID, m.dx, m.dy, m.dZ), P,
                             tol=1e-12)
    yield m, prob
    s.close()


def _directions(m, seed):
    """A heat-source direction on the silicon cells and a log-conductivity direction constant on
    each z-band of the stack (the 13-parameter mapping; a field of per-cell values would exceed the
    library's 127 distinct conductivities)."""
    rng = np.random.default_rng(seed)
    inner = (slice(1, -1),) * 3
    dh = np.zeros(m.shape)
    dh[inner] = rng.uniform(0.0, 1.0, (m.NX, m.NY, m.NZ)) * 1e10 * np.isin(m.ID[inner], (2, 7))
    band = A.band_of_plane(m.ZC)
    per_band = rng.uniform(-1.0, 1.0, A.NBANDS) * 0.1
    dl = np.zeros(m.shape)
    dl[inner] = np.where(band >= 0, per_band[np.maximum(band, 0)], 0.0)[None, None, 1:-1]
    return dh, dl


def test_backward_matches_central_differences(problem):
    m, prob = problem
    h0 = torch.tensor(np.ascontiguousarray(m.wk.hsrc), dtype=torch.float64, requires_grad=True)
    l0 = torch.zeros(m.shape, dtype=torch.float64, requires_grad=True)
    J = AG.hotspot_norm(h0, l0, prob)
    J.backward()
    dh, dl = _directions(m, 3)
    for d_h, d_l in ((dh, 0 * dl), (0 * dh, dl)):
        eps = 1e-4
        th, tl = torch.from_numpy(d_h), torch.from_numpy(d_l)
        with torch.no_grad():
            jp = AG.hotspot_norm(h0 + eps * th, l0 + eps * tl, prob).item()
            jm = AG.hotspot_norm(h0 - eps * th, l0 - eps * tl, prob).item()
        fd = (jp - jm) / (2 * eps)
        an = float((h0.grad * th).sum() + (l0.grad * tl).sum())
        assert abs(an - fd) <= 1e-5 * abs(fd), (an, fd)
    # the forward value without gradients equals the adjoint call's J
    with torch.no_grad():
        assert abs(AG.hotspot_norm(h0, l0, prob).item() - J.item()) <= 1e-12 * J.item()
    assert not h0.grad[0].any() and not l0.grad[:, :, -1].any()  # guards carry no gradient


def test_gradcheck_three_parameters(problem):
    m, prob = problem
    dh, dl = _directions(m, 5)
    _, ZC, _ = M.zgrid(30)
    band = np.zeros(m.shape)
    band[1:-1, 1:-1, 1:-1] = (A.band_of_plane(ZC) == 4)[None, None, 1:-1]  # one z-band of the stack
    h_base = torch.tensor(np.ascontiguousarray(m.wk.hsrc), dtype=torch.float64)
    dirs = [torch.from_numpy(d) for d in (dh, dl, band)]

    def f(a):
        return AG.hotspot_norm(h_base + a[0] * dirs[0], a[1] * dirs[1] + a[2] * dirs[2], prob)

    a = torch.tensor([0.3, 0.2, -0.1], dtype=torch.float64, requires_grad=True)
    assert torch.autograd.gradcheck(f, (a,), eps=1e-4, atol=1e-9, rtol=1e-5, nondet_tol=1e-12)
