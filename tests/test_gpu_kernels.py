"""GPU kernels vs the oracle, one kernel at a time, through the C ABI.

FP64 kernels follow the reference's per-cell arithmetic exactly (tabulated face conductances,
no FMA contraction), so CalcAX, CalcRK's residual vector, one RB-SOR colour pass and the
5-sweep preconditioner must be bit-identical to the oracle.  Only reductions differ in order:
||r|| is checked to 1e-13 relative.  FP32 kernels (mixed precision) are checked to 2e-6
relative to the FP64 oracle.
"""
import numpy as np
import pytest

import h2_b200
from conftest import mode3_model

pytestmark = pytest.mark.gpu


def make_solver(prob, precision="fp64", is_steady=None):
    steady = prob.is_steady if is_steady is None else is_steady
    s = h2_b200.Solver(*prob.shape, precision=precision)
    s.set_grid(prob.ZC, prob.dZ, prob.dx, prob.dy, prob.dt, prob.HC, steady)
    w = prob.wk
    s.set_fields(w["lam"], w["mask"], None if steady else w["rho"], None if steady else w["cp"])
    s.set_rhs(w["b"])
    s.set_theta(w["theta"])
    return s


def random_interior(shape, seed):
    rng = np.random.default_rng(seed)
    x = np.zeros(shape, order="F")
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal((shape[0] - 2, shape[1] - 2, shape[2] - 2)) * 10.0
    return x


# Mode 3 (convective sides/top, isothermal bottom); the symmetric variant (adiabatic faces);
# an odd-sized grid; a transient grid (rho*cp term).
CASES = [
    dict(NX=40, NY=40),
    dict(NX=40, NY=40, symmetric=True),
    dict(NX=41, NY=37),
    dict(NX=40, NY=40, is_steady=False, dt=1e-4),
]


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_calcax_bit_exact(oracle, case):
    prob = mode3_model(oracle, **case)
    s = make_solver(prob)
    for seed in (1, 2):
        x = random_interior(prob.shape, seed)
        ref = oracle.calc_ax(prob, x)
        got = s.calc_ax(x)
        assert np.array_equal(got[1:-1, 1:-1, 1:-1], ref[1:-1, 1:-1, 1:-1])
        assert not got[0].any() and not got[-1].any()
    s.close()


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_calcrk_bit_exact(oracle, case):
    prob = mode3_model(oracle, **case)
    th = prob.wk["theta"].copy(order="F")
    th[1:-1, 1:-1, 1:-1] += random_interior(prob.shape, 7)[1:-1, 1:-1, 1:-1]
    prob.wk["theta"][...] = th
    s = make_solver(prob)
    r_ref, res_ref = oracle.calc_rk(prob)
    r, res = s.calc_rk()
    assert np.array_equal(r[1:-1, 1:-1, 1:-1], r_ref[1:-1, 1:-1, 1:-1])
    assert abs(res - res_ref) <= 1e-13 * res_ref
    s.close()


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
@pytest.mark.parametrize("color", [0, 1])
@pytest.mark.parametrize("omega", [1.0, 1.6])
def test_rbsor_pass_bit_exact(oracle, case, color, omega):
    prob = mode3_model(oracle, **case)
    s = make_solver(prob)
    x = random_interior(prob.shape, 11)
    b = random_interior(prob.shape, 12)
    xr = x.copy(order="F")
    oracle.rbsor_core(prob, xr, b, color, omega=omega)
    got = s.rbsor_pass(x.copy(order="F"), b, color, omega)
    assert np.array_equal(got, xr)
    s.close()


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_preconditioner_bit_exact(oracle, case):
    prob = mode3_model(oracle, **case)
    s = make_solver(prob)
    bb = random_interior(prob.shape, 21)
    ref = oracle.preconditioner(prob, bb, "gs")
    got = s.preconditioner(bb, "gs")
    assert np.array_equal(got, ref)
    got_none = s.preconditioner(bb, "none")
    assert np.array_equal(got_none, oracle.preconditioner(prob, bb, "none"))
    s.close()


def test_fp32_kernels_close_to_fp64(oracle):
    """FP32 operator (difference form, H2G_MIXED_IR) and FP32 preconditioner (H2G_MIXED) vs the
    FP64 oracle; H2G_MIXED applies CalcAX in FP64, bit-identical to the reference."""
    prob = mode3_model(oracle, 40)
    x = random_interior(prob.shape, 3)
    ref = oracle.calc_ax(prob, x)[1:-1, 1:-1, 1:-1]
    s_ir = make_solver(prob, precision="mixed_ir")
    got = s_ir.calc_ax(x)[1:-1, 1:-1, 1:-1]
    assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max()
    s_ir.close()
    s = make_solver(prob, precision="mixed")
    assert np.array_equal(s.calc_ax(x)[1:-1, 1:-1, 1:-1], ref)
    bb = random_interior(prob.shape, 4)
    pref = oracle.preconditioner(prob, bb, "gs")
    pgot = s.preconditioner(bb, "gs")
    assert np.abs(pgot - pref).max() <= 2e-5 * np.abs(pref).max()
    s.close()


def test_nonfinite_and_unsupported_fields(oracle):
    prob = mode3_model(oracle, 20)
    s = h2_b200.Solver(*prob.shape)
    s.set_grid(prob.ZC, prob.dZ, prob.dx, prob.dy, prob.dt, prob.HC, True)
    lam = prob.wk["lam"].copy(order="F")
    lam[5, 5, 5] = np.nan
    with pytest.raises(h2_b200.H2GError) as e:
        s.set_fields(lam, prob.wk["mask"])
    assert e.value.status == 3  # H2G_NONFINITE
    mask = prob.wk["mask"].copy(order="F")
    mask[5, 5, 5] = 0.5
    with pytest.raises(h2_b200.H2GError) as e:
        s.set_fields(prob.wk["lam"], mask)
    assert e.value.status == 7  # H2G_UNSUPPORTED
    s.close()


def test_most_materials(oracle):
    """127 distinct conductivities, the most a 7-bit material key holds: CalcAX and the 5-sweep
    preconditioner stay bit-identical to the oracle.  A 128th distinct value is rejected on the
    host (H2G_UNSUPPORTED) before any solve."""
    prob = mode3_model(oracle, 20)
    lam = prob.wk["lam"]
    have = len(np.unique(lam))
    rng = np.random.default_rng(3)
    inner = np.argwhere(prob.wk["mask"] == 1.0)
    pick = inner[rng.choice(len(inner), 128 - have, replace=False)]
    vals = rng.uniform(0.5, 400.0, len(pick))
    for (i, j, k), v in zip(pick[:-1], vals[:-1]):
        lam[i, j, k] = v
    assert len(np.unique(lam)) == 127
    s = make_solver(prob)
    x = random_interior(prob.shape, 5)
    assert np.array_equal(s.calc_ax(x)[1:-1, 1:-1, 1:-1], oracle.calc_ax(prob, x)[1:-1, 1:-1, 1:-1])
    bb = random_interior(prob.shape, 6)
    assert np.array_equal(s.preconditioner(bb, "gs"), oracle.preconditioner(prob, bb, "gs"))
    i, j, k = pick[-1]
    lam[i, j, k] = vals[-1]
    with pytest.raises(h2_b200.H2GError) as e:
        s.set_fields(lam, prob.wk["mask"])
    assert e.value.status == 7  # H2G_UNSUPPORTED
    s.close()


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_calcax_symmetric(oracle, case):
    """(A x, y) = (x, A y) to rounding on the GPU operator (test_symmetry.jl:11-81 restated): the
    adjoint solves rely on it.  Vectors with zero guards, as every Krylov vector."""
    prob = mode3_model(oracle, **case)
    s = make_solver(prob)
    x = random_interior(prob.shape, 21)
    y = random_interior(prob.shape, 22)
    ax, ay = s.calc_ax(x), s.calc_ax(y)
    l, r = float(np.sum(ax * y)), float(np.sum(x * ay))
    assert abs(l - r) <= 1e-12 * max(abs(l), abs(r))
    s.close()
