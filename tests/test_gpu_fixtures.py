"""GPU results at the workload's own sizes against committed oracle fixtures (tests/golden/, made
by tests/golden/make_golden.py with the oracle: OpenMP reductions, FP64):

* three members of the 64-member batch (one each of 120^2, 180^2 and 240^2 x 30, their seeded
  hotspot heat maps), solved together by h2g_batch_solve to 1e-8;
* the steady adjoint at 240x240x30 (J and both gradient fields at 4096 sampled cells, their
  per-plane sums) to 1e-10;
* the FP64 PBiCGSTAB solve at 480x480x60 to 1e-8.

Tolerances are the north star's: temperature within 1e-3 K, FP64 iteration counts within 10 %
(the oracle's own count moves by several percent with the summation order of its OpenMP
reductions), gradients within 1e-6 of their largest magnitude.
"""
import numpy as np
import pytest

import h2_b200
from conftest import golden
from h2_b200 import adjoint as A
from h2_b200 import batch as B
from h2_b200 import model as M

pytestmark = pytest.mark.gpu


def _at(a, ijk):
    ijk = np.asarray(ijk)
    return a[ijk[:, 0], ijk[:, 1], ijk[:, 2]]


def _check_field(th, fx):
    inner = th[1:-1, 1:-1, 1:-1]
    assert np.abs(_at(th, fx["sample_ijk"]) - np.asarray(fx["sample_theta"])).max() <= 1e-3
    assert abs(inner.min() - fx["theta_min"]) <= 1e-3 and abs(inner.max() - fx["theta_max"]) <= 1e-3


def test_batch_members_match_oracle_fixture():
    fx = golden("oracle_batch3.json")
    allm = B.draw_batch(fx["batch"], fx["seed0"])
    members = [allm[f["index"]] for f in fx["members"]]
    assert [m.nx for m in members] == [f["nx"] for f in fx["members"]] == list(B.SIZES)
    bs = B.BatchSolver(members)
    try:
        bs.restore()
        st, res = bs.solve(tol=1e-8)
        assert st == 0
        for r, s, f in zip(res, bs.solvers, fx["members"]):
            assert r.isconverged and f["isconverged"]
            assert abs(r.res0 - f["res0"]) <= 1e-12 * f["res0"]
            assert abs(r.itr - f["itr"]) <= max(2, 0.1 * f["itr"]), (r.itr, f["itr"])
            _check_field(s.get_theta(), f)
    finally:
        bs.close()


def test_steady_adjoint_240_matches_oracle_fixture():
    fx = golden("oracle_adjoint_240.json")
    m = M.build_mode3(240, 240, 30)
    w = m.wk
    s = h2_b200.Solver(*m.shape)
    try:
        s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
        s.set_fields(w.lam, w.mask)
        s.set_rhs(w.b)
        s.set_theta(w.theta)
        wts = A.silicon_weights(m.ID, m.dx, m.dy, m.dZ)
        J, gh, gl, rf, ra = A.steady_gradient(s, wts, fx["p"], tol=fx["epsilon"])
        assert rf.isconverged and ra.isconverged
        assert abs(J - fx["J"]) <= 1e-10 * fx["J"]
        assert abs(rf.itr - fx["forward_itr"]) <= 0.1 * fx["forward_itr"]
        assert abs(ra.itr - fx["adjoint_itr"]) <= 0.1 * fx["adjoint_itr"]
        assert np.abs(_at(s.get_theta(), fx["sample_ijk"]) - np.asarray(fx["sample_theta"])).max() <= 1e-6
        ijk = fx["sample_ijk"]
        assert np.abs(_at(gh, ijk) - np.asarray(fx["sample_gh"])).max() <= 1e-6 * fx["gh_absmax"]
        assert np.abs(_at(gl, ijk) - np.asarray(fx["sample_gl"])).max() <= 1e-6 * fx["gl_absmax"]
        ph, pl = np.asarray(fx["gh_plane_sum"]), np.asarray(fx["gl_plane_sum"])
        assert np.abs(gh.sum(axis=(0, 1)) - ph).max() <= 1e-6 * np.abs(ph).max()
        assert np.abs(gl.sum(axis=(0, 1)) - pl).max() <= 1e-6 * np.abs(pl).max()
    finally:
        s.close()


def test_fp64_480x60_matches_oracle_fixture():
    fx = golden("oracle_480x60_1e-8.json")
    m = M.build_mode3(fx["NX"], fx["NY"], fx["NZ"])
    w = m.wk
    s = h2_b200.Solver(*m.shape)
    try:
        s.set_grid(m.ZC, m.dZ, m.dx, m.dy, m.dt, m.HC, True)
        s.set_fields(w.lam, w.mask)
        s.set_rhs(w.b)
        s.set_theta(w.theta)
        st, res = s.solve("pbicgstab", tol=fx["epsilon"], maxItr=20000, smoother="gs")
        assert st == 0 and res.isconverged and fx["isconverged"]
        assert abs(res.res0 - fx["res0"]) <= 1e-12 * fx["res0"]
        assert abs(res.itr - fx["itr"]) <= 0.1 * fx["itr"], (res.itr, fx["itr"])
        _check_field(s.get_theta(), fx)
    finally:
        s.close()
