"""GPU calRHS! (NonUniform.jl:57-91, RHS.jl:23-192) and the time loop of main()
(heat3ds.jl:123-151) against the oracle."""
import numpy as np
import pytest

import h2_b200
from conftest import mode3_model
from test_gpu_kernels import make_solver

pytestmark = pytest.mark.gpu

# every boundary type on some face, with non-zero heat flux and theta_inf != theta
MIXED_BCS = [
    (2, 0.0, 0.0, 7.5, 310.0),     # x-: convection
    (1, 0.0, 2.5e4, 0.0, 0.0),     # x+: heat flux
    (1, 0.0, -1.0e4, 0.0, 0.0),    # y-: heat flux
    (2, 0.0, 0.0, 12.0, 290.0),    # y+: convection
    (0, 300.0, 0.0, 0.0, 0.0),     # z-: isothermal (no RHS term)
    (2, 0.0, 0.0, 5.0, 300.0),     # z+: convection
]


def _rand_theta(prob, seed):
    rng = np.random.default_rng(seed)
    th = prob.wk["theta"]
    th[1:-1, 1:-1, 1:-1] = 300.0 + 40.0 * rng.random((prob.NX, prob.NY, prob.NZ))


@pytest.mark.parametrize("steady", [True, False])
@pytest.mark.parametrize("bcs", ["mode3", "mixed"])
@pytest.mark.parametrize("zero_b", [True, False])
def test_calrhs_bit_exact(oracle, steady, bcs, zero_b):
    prob = oracle.build_mode3(18, 14, 30, is_steady=steady, dt=1e-4, calrhs=False)
    if bcs == "mixed":
        prob.bcs = MIXED_BCS
    _rand_theta(prob, 7)
    rng = np.random.default_rng(3)
    b0 = np.zeros(prob.shape, order="F")
    if not zero_b:
        b0[1:-1, 1:-1, 1:-1] = rng.standard_normal((prob.NX, prob.NY, prob.NZ))
    prob.wk["b"][...] = b0
    oracle.calRHS(prob)
    s = make_solver(prob, is_steady=steady)
    s.set_hsrc(prob.wk["hsrc"])
    s.set_rhs(b0)
    s.calrhs(prob.bcs, zero_b=zero_b)
    b = s.get_rhs()
    assert np.array_equal(b, prob.wk["b"])
    s.close()


def test_calrhs_bad_bc(oracle):
    prob = mode3_model(oracle, 12)
    s = make_solver(prob)
    bad = list(prob.bcs)
    bad[2] = (9, 0.0, 0.0, 0.0, 0.0)
    with pytest.raises(h2_b200.H2GError):
        s.calrhs(bad)
    s.close()


def test_transient_steps_match_oracle(oracle):
    """Three implicit steps (dt = 1e-4 s) of the transient Mode-3 model from theta = 300 K:
    per step b is rebuilt from b = 0, the solve starts from the previous theta."""
    nt, tol = 3, 1e-8
    prob = oracle.build_mode3(20, 20, 30, is_steady=False, dt=1e-4, calrhs=False)
    ref = oracle.build_mode3(20, 20, 30, is_steady=False, dt=1e-4, calrhs=False)
    s = make_solver(prob, is_steady=False)
    s.set_hsrc(prob.wk["hsrc"])
    st, res, stats = s.transient(prob.bcs, nt, tol=tol, smoother="gs")
    assert st == 0 and res.isconverged and res.outer == nt
    w = ref.wk
    for step in range(nt):
        w["b"][...] = 0.0
        oracle.calRHS(ref)
        conv, itr, _, _ = oracle.pbicgstab(ref, tol=tol, maxItr=20000, smoother="gs")
        assert conv
        inner = w["theta"][1:-1, 1:-1, 1:-1]
        assert abs(stats[step, 3] - itr) <= max(1, 0.1 * itr)
        assert abs(stats[step, 0] - inner.min()) <= 1e-3
        assert abs(stats[step, 1] - inner.max()) <= 1e-3
        assert abs(stats[step, 2] - np.sqrt((inner * inner).sum())) <= 1e-9 * stats[step, 2]
    assert np.abs(s.get_theta() - w["theta"]).max() <= 1e-3
    # theta rises from 300 K under the heat source
    assert stats[0, 1] > 300.0 and stats[-1, 1] >= stats[0, 1]
    s.close()
