"""Kernels and solves on hand-built boxes against the oracle: tiny and odd grid sizes (one cell
wide, a half-row spanning two warps), odd and small NZ (the two-planes-per-thread colour pass
then has a last plane pair with one plane outside the grid), a non-uniform Z grid, five
materials at random, and all three boundary types on the six faces (isothermal at two
temperatures, convection at two coefficients, heat flux, adiabatic).  Every launch shape of the
colour pass must give the oracle's bits."""
import numpy as np
import pytest

from test_gpu_kernels import make_solver, random_interior

pytestmark = pytest.mark.gpu

GRIDS = [(1, 1, 3), (6, 5, 7), (3, 2, 5), (33, 31, 9), (65, 4, 4), (70, 9, 1)]
SHAPES = [(8, 2), (2, 1), (16, 2), (4, 1)]


def box_problem(O, NX, NY, NZ, seed, transient=False):
    """A box with random materials and mixed boundary conditions, set up with the oracle's own
    boundary routine (apply_boundary_conditions! / set_BC_coef) and calRHS!."""
    MX, MY, MZ = NX + 2, NY + 2, NZ + 2
    shape = (MX, MY, MZ)
    rng = np.random.default_rng(seed)
    dz = rng.uniform(2e-6, 2e-5, NZ)
    zf = np.concatenate([[0.0], np.cumsum(dz)])
    ZC = np.empty(MZ)
    ZC[0], ZC[-1] = zf[0], zf[-1]  # guards on the faces, as genZ!
    ZC[1:-1] = 0.5 * (zf[1:] + zf[:-1])
    dZ = np.concatenate([[dz[0]], dz, [dz[-1]]])
    Z = np.concatenate([[2 * zf[0] - zf[min(1, NZ)]], zf, [2 * zf[-1] - zf[-2]]])
    wk = {n: O.zeros(shape) for n in O._WK_NAMES}
    mats = np.array([0.4, 1.5, 50.0, 149.0, 386.0])
    wk["lam"][...] = mats[rng.integers(0, len(mats), shape)]
    wk["rho"][...] = rng.uniform(1e3, 9e3, shape)
    wk["cp"][...] = rng.uniform(300.0, 900.0, shape)
    wk["mask"][...] = 1.0
    wk["theta"][...] = 300.0
    bcs = [O.isothermal_bc(300.0), O.convection_bc(5.0, 290.0), O.heat_flux_bc(2.0e4), O.adiabatic_bc(),
           O.isothermal_bc(320.0), O.convection_bc(12.0, 300.0)]
    bca = O.bc_array(bcs)
    L = O.lib()
    L.h2o_apply_bc(MX, MY, MZ, bca, O._p(wk["theta"]), O._p(wk["lam"]), O._p(wk["rho"]), O._p(wk["cp"]),
                   O._p(wk["mask"]))
    HC = np.zeros(6)
    L.h2o_set_bc_coef(bca, O._p(HC))
    wk["hsrc"][1:-1, 1:-1, 1:-1] = rng.uniform(0.0, 1.0e12, (NX, NY, NZ))
    ID = np.zeros(shape, dtype=np.uint8, order="F")
    prob = O.Problem(NX, NY, NZ, 1.0e-5, 1.3e-5, 1.0e-4 if transient else 1.0, not transient, Z, ZC, dZ, HC, bcs,
                     ID, wk)
    O.calRHS(prob)
    return prob


@pytest.mark.parametrize("transient", [False, True], ids=["steady", "transient"])
@pytest.mark.parametrize("grid", GRIDS, ids=["x".join(map(str, g)) for g in GRIDS])
def test_box_kernels_bit_exact(oracle, grid, transient):
    prob = box_problem(oracle, *grid, seed=sum(grid), transient=transient)
    s = make_solver(prob)
    x = random_interior(prob.shape, 1)
    assert np.array_equal(s.calc_ax(x)[1:-1, 1:-1, 1:-1], oracle.calc_ax(prob, x)[1:-1, 1:-1, 1:-1])
    r, res = s.calc_rk()
    r_ref, res_ref = oracle.calc_rk(prob)
    assert np.array_equal(r[1:-1, 1:-1, 1:-1], r_ref[1:-1, 1:-1, 1:-1])
    assert abs(res - res_ref) <= 1e-13 * res_ref
    b = random_interior(prob.shape, 2)
    bb = random_interior(prob.shape, 3)
    pre_ref = oracle.preconditioner(prob, bb, "gs")
    for rows, planes in SHAPES:
        s.set_tuning(rows, planes)
        for color, omega in ((0, 1.0), (1, 1.0), (0, 1.7)):
            xr = x.copy(order="F")
            oracle.rbsor_core(prob, xr, b, color, omega=omega)
            assert np.array_equal(s.rbsor_pass(x.copy(order="F"), b, color, omega), xr), (rows, planes, color)
        assert np.array_equal(s.preconditioner(bb, "gs"), pre_ref), (rows, planes)
    s.close()


BOX_SOLVES = [(6, 5, 7), (33, 31, 9), (70, 9, 1)]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("method", ["pbicgstab", "cg"])
@pytest.mark.parametrize("grid", BOX_SOLVES, ids=["x".join(map(str, g)) for g in BOX_SOLVES])
def test_box_solve(oracle, grid, method, precision):
    """The solve on a box converges to the oracle's field (1e-3 K); in FP64 also like the oracle
    (iterations within 10 %, at least 2).  Mixed precision runs the FP32 colour pass on the same
    odd plane counts and confirms convergence on the FP64 true residual."""
    prob = box_problem(oracle, *grid, seed=7)
    ref = box_problem(oracle, *grid, seed=7)
    fn = oracle.pbicgstab if method == "pbicgstab" else oracle.cg
    conv, itr, res0, _ = fn(ref, tol=1e-10, maxItr=20000, smoother="gs")
    assert conv
    s = make_solver(prob, precision=precision)
    tol = 1e-10 if precision == "fp64" else 1e-9
    st, res = s.solve(method, tol=tol, maxItr=20000, smoother="gs")
    assert st == 0 and res.isconverged
    assert abs(res.res0 - res0) <= 1e-12 * res0
    if precision == "fp64":
        assert abs(res.itr - itr) <= max(2, itr // 10), (res.itr, itr)
    assert np.abs(s.get_theta() - ref.wk["theta"]).max() <= 1e-3
    s.close()


@pytest.mark.parametrize("grid", BOX_SOLVES, ids=["x".join(map(str, g)) for g in BOX_SOLVES])
def test_box_sor_bit_exact(oracle, grid):
    """solveSOR! (omega = 1.5, 25 passes, not converged) on a box: the field equals the oracle's
    bit for bit (the colour pass with its residual sum, k_sor_pass, on odd plane counts too)."""
    prob = box_problem(oracle, *grid, seed=9)
    ref = box_problem(oracle, *grid, seed=9)
    n_r, res0_r, hist_r = oracle.solve_sor(ref, omega=1.5, tol=1e-30, maxItr=25)
    assert n_r == -25
    s = make_solver(prob)
    hist = np.zeros(25)
    st, res = s.sor(omega=1.5, tol=1e-30, maxItr=25, hist=hist)
    assert not res.isconverged and res.itr == 25
    assert abs(res.res0 - res0_r) <= 1e-13 * res0_r
    assert np.allclose(hist, hist_r, rtol=1e-12, atol=0)
    assert np.array_equal(s.get_theta(), ref.wk["theta"])
    s.close()


@pytest.mark.parametrize("transient", [False, True], ids=["steady", "transient"])
@pytest.mark.parametrize("grid", GRIDS, ids=["x".join(map(str, g)) for g in GRIDS])
def test_box_calrhs_bit_exact(oracle, grid, transient):
    """calRHS! on a box with every boundary type and a random temperature field."""
    prob = box_problem(oracle, *grid, seed=11, transient=transient)
    rng = np.random.default_rng(5)
    prob.wk["theta"][1:-1, 1:-1, 1:-1] = 300.0 + 40.0 * rng.random(grid)
    prob.wk["b"][...] = 0.0
    oracle.calRHS(prob)
    s = make_solver(prob)
    s.set_hsrc(prob.wk["hsrc"])
    s.calrhs(prob.bcs, zero_b=True)
    assert np.array_equal(s.get_rhs(), prob.wk["b"])
    s.close()


@pytest.mark.parametrize("grid", [(6, 5, 7), (33, 31, 9)], ids=["6x5x7", "33x31x9"])
def test_box_time_loop(oracle, grid):
    """Four implicit steps (dt = 1e-4 s) of the time loop on a box with every boundary type:
    b rebuilt from zero each step, the solve from the previous field, against the oracle's loop."""
    nt, tol = 4, 1e-10
    prob = box_problem(oracle, *grid, seed=13, transient=True)
    ref = box_problem(oracle, *grid, seed=13, transient=True)
    s = make_solver(prob)
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
        assert abs(stats[step, 3] - itr) <= max(2, 0.1 * itr)
        assert abs(stats[step, 0] - inner.min()) <= 1e-3 and abs(stats[step, 1] - inner.max()) <= 1e-3
    assert np.abs(s.get_theta() - w["theta"]).max() <= 1e-3
    s.close()


def test_box_steady_adjoint(oracle):
    """h2g_adjoint on a box with every boundary type (heat-flux and convective guards carry
    lambda = 0, isothermal guards a copy of their neighbour's): J and both gradient fields against
    the oracle's FP64 forward and adjoint solves with the numpy restatement of the gradient."""
    from oracle import adjoint as OA

    from h2_b200 import adjoint as A
    grid, P = (33, 31, 9), 8.0
    prob = box_problem(oracle, *grid, seed=17)
    w = np.zeros(prob.shape, order="F")
    w[1:-1, 1:-1, 1:-1] = (prob.dx * prob.dy) * prob.dZ[None, None, 1:-1]
    s = make_solver(prob)
    J, gh, gl, rf, ra = A.steady_gradient(s, w, P, tol=1e-12)
    assert rf.isconverged and ra.isconverged
    th = s.get_theta()
    s.close()
    fwd = box_problem(oracle, *grid, seed=17)
    assert oracle.pbicgstab(fwd, tol=1e-12, maxItr=20000, smoother="gs")[0]
    th_ref = fwd.wk["theta"]
    assert np.abs(th - th_ref).max() <= 1e-6
    J_ref = OA.objective(th_ref, w, P)
    assert abs(J - J_ref) <= 1e-12 * J_ref
    adj = box_problem(oracle, *grid, seed=17)
    adj.wk["theta"][...] = 0.0
    adj.wk["b"][...] = OA.adj_rhs(th_ref, w, P)
    assert oracle.pbicgstab(adj, tol=1e-12, maxItr=20000, smoother="gs")[0]
    w_ = prob.wk
    gh_ref, gl_ref = OA.gradients(w_["lam"], w_["mask"], th_ref, adj.wk["theta"], prob.dx, prob.dy, prob.ZC,
                                  prob.dZ)
    assert np.abs(gh - gh_ref).max() <= 1e-6 * np.abs(gh_ref).max()
    assert np.abs(gl - gl_ref).max() <= 1e-6 * np.abs(gl_ref).max()


def singular_box(O, NX, NY, NZ, seed=21):
    """A steady box with every face adiabatic and a heat source: A is singular (pure Neumann)
    and the system has no solution (the net heat input is not zero)."""
    p = box_problem(O, NX, NY, NZ, seed)
    MX, MY, MZ = p.shape
    w = p.wk
    rng = np.random.default_rng(seed)
    w["lam"][...] = np.array([0.4, 1.5, 50.0, 149.0, 386.0])[rng.integers(0, 5, p.shape)]
    w["mask"][...] = 1.0
    w["theta"][...] = 300.0
    w["b"][...] = 0.0
    p.bcs = [O.adiabatic_bc()] * 6
    O.lib().h2o_apply_bc(MX, MY, MZ, O.bc_array(p.bcs), O._p(w["theta"]), O._p(w["lam"]), O._p(w["rho"]),
                         O._p(w["cp"]), O._p(w["mask"]))
    p.HC[...] = 0.0
    O.calRHS(p)
    return p


@pytest.mark.parametrize("method", ["pbicgstab", "cg"])
@pytest.mark.parametrize("grid", [(6, 5, 7), (33, 31, 9)], ids=["6x5x7", "33x31x9"])
def test_box_singular_system(oracle, grid, method):
    """No solution: the oracle runs to maxItr without converging.  The GPU solve ends within
    maxItr with a failure status: NOT_CONVERGED after maxItr iterations, or BREAKDOWN or
    NONFINITE earlier if its rounding takes it there first."""
    ref = singular_box(oracle, *grid)
    fn = oracle.pbicgstab if method == "pbicgstab" else oracle.cg
    conv, itr, res0, _ = fn(ref, tol=1e-10, maxItr=500, smoother="gs")
    assert not conv and itr == 500
    s = make_solver(singular_box(oracle, *grid))
    st, res = s.solve(method, tol=1e-10, maxItr=500, smoother="gs")
    assert st in (1, 2, 3) and st == res.status and not res.isconverged
    assert res.itr <= 500 and (st != 1 or res.itr == 500)
    assert abs(res.res0 - res0) <= 1e-12 * res0
    s.close()
