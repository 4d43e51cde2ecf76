"""The stencil-class coefficient source of the FP64 kernels (k_class_insert / k_class_assign /
k_class_coef; coefficient source 2 of the colour pass, the first pass and CalcAX).

Every class row is written by cell_coef itself, so the class source must give exactly the bits
of the key tables: CalcAX and the 5-sweep preconditioner are compared with `array_equal` to the
oracle on the model grids and on boxes with random materials, every boundary type, transient
grids (dd then comes from the per-cell array) and masked interior cells; whole solves equal the
key-table solves bit for bit.  Grids with more distinct stencils than 16-bit class indices, or
H2G_CLS=0, keep the key tables.
"""
import numpy as np
import pytest

import h2_b200
from conftest import mode3_model
from test_gpu_boxes import GRIDS, box_problem
from test_gpu_kernels import CASES, make_solver, random_interior

pytestmark = pytest.mark.gpu


@pytest.fixture
def class_source(monkeypatch):
    monkeypatch.setenv("H2G_RB_DD", "2")
    monkeypatch.setenv("H2G_AX_DD", "2")
    monkeypatch.delenv("H2G_CLS", raising=False)


def _check_kernels(oracle, prob, seed):
    s = make_solver(prob)
    assert s.tuning()[2:] == (2, 2)  # the class table is built and used by both kernels
    x = random_interior(prob.shape, seed)
    assert np.array_equal(s.calc_ax(x)[1:-1, 1:-1, 1:-1], oracle.calc_ax(prob, x)[1:-1, 1:-1, 1:-1])
    for planes in (1, 2):
        s.set_tuning(8, planes)
        assert np.array_equal(s.preconditioner(x, "gs"), oracle.preconditioner(prob, x, "gs")), planes
    s.close()


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_class_kernels_bit_exact(oracle, class_source, case):
    _check_kernels(oracle, mode3_model(oracle, **case), 3)


@pytest.mark.parametrize("transient", [False, True], ids=["steady", "transient"])
@pytest.mark.parametrize("grid", GRIDS, ids=["x".join(map(str, g)) for g in GRIDS])
def test_class_kernels_boxes(oracle, class_source, grid, transient):
    _check_kernels(oracle, box_problem(oracle, *grid, seed=sum(grid) + 11, transient=transient), 4)


def test_class_kernels_masked_cells(oracle, class_source):
    """Interior cells with mask 0 are never updated (no class) and double lambda_f of their
    neighbours' faces."""
    prob = box_problem(oracle, 33, 31, 9, seed=21)
    rng = np.random.default_rng(5)
    m = prob.wk["mask"]
    inner = (slice(1, -1),) * 3
    m[inner] = np.where(rng.uniform(size=m[inner].shape) < 0.1, 0.0, 1.0)
    _check_kernels(oracle, prob, 6)


@pytest.mark.parametrize("method", ["pbicgstab", "cg"])
def test_class_solve_identical(oracle, monkeypatch, method):
    prob = mode3_model(oracle, 41, 37)
    out = []
    for src in ("1", "2"):
        monkeypatch.setenv("H2G_RB_DD", src)
        monkeypatch.setenv("H2G_AX_DD", src)
        s = make_solver(prob)
        assert s.tuning()[2:] == (int(src), int(src))
        hist = np.zeros(20000)
        st, res = s.solve(method, tol=1e-8, maxItr=20000, smoother="gs", hist=hist)
        assert st == 0 and res.isconverged
        out.append((res.itr, hist[:res.itr].copy(), s.get_theta()))
        s.close()
    assert out[0][0] == out[1][0]
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])


def test_classes_disabled_or_too_many(oracle, monkeypatch):
    """H2G_CLS=0, or more distinct (plane, stencil keys) pairs than 16-bit class indices hold: the
    table is not built, a forced class source falls back to dd read from the array, and results
    stay those of the oracle."""
    monkeypatch.setenv("H2G_RB_DD", "2")
    monkeypatch.setenv("H2G_AX_DD", "2")
    monkeypatch.setenv("H2G_CLS", "0")
    prob = mode3_model(oracle, 40)
    s = make_solver(prob)
    assert s.tuning()[2:] == (1, 1)
    s.close()
    monkeypatch.delenv("H2G_CLS")
    # 70 x 70 x 20 cells of 40 random conductivities: about 98 000 distinct stencils
    prob = box_problem(oracle, 70, 70, 20, seed=8)
    rng = np.random.default_rng(9)
    prob.wk["lam"][...] = rng.choice(np.linspace(1.0, 400.0, 40), prob.shape)
    oracle.calRHS(prob)
    s = make_solver(prob)
    assert s.tuning()[2:] == (1, 1)
    x = random_interior(prob.shape, 2)
    assert np.array_equal(s.calc_ax(x)[1:-1, 1:-1, 1:-1], oracle.calc_ax(prob, x)[1:-1, 1:-1, 1:-1])
    s.close()


def test_operator_rebuilt_when_inputs_change(oracle):
    """One handle given new conductivity values (same key layout), new boundary coefficients, the
    first fields again and the same fields twice: every CalcAX and preconditioner equals the
    oracle's for the inputs of that moment.  A build is skipped only when nothing changed."""
    import copy
    a = mode3_model(oracle, 40)
    a2 = copy.deepcopy(a)
    a2.wk["lam"][...] = a2.wk["lam"] * 1.5
    a3 = copy.deepcopy(a)
    a3.HC = a3.HC * 2.0
    x = random_interior(a.shape, 17)
    s = make_solver(a)

    def check(prob):
        assert np.array_equal(s.calc_ax(x)[1:-1, 1:-1, 1:-1], oracle.calc_ax(prob, x)[1:-1, 1:-1, 1:-1])
        assert np.array_equal(s.preconditioner(x, "gs"), oracle.preconditioner(prob, x, "gs"))

    check(a)
    s.set_fields(a2.wk["lam"], a2.wk["mask"])
    check(a2)
    s.set_fields(a.wk["lam"], a.wk["mask"])
    check(a)
    s.set_grid(a3.ZC, a3.dZ, a3.dx, a3.dy, a3.dt, a3.HC, True)
    check(a3)
    s.set_grid(a.ZC, a.dZ, a.dx, a.dy, a.dt, a.HC, True)
    s.set_fields(a.wk["lam"], a.wk["mask"])
    s.set_fields(a.wk["lam"], a.wk["mask"])
    check(a)
    s.close()


@pytest.mark.parametrize("case", CASES, ids=["mode3", "adiabatic", "odd", "transient"])
def test_fp32_smoother_classes_equal_key_tables(oracle, monkeypatch, case):
    """The FP32 smoother of the mixed handles with its own class rows (FP32 copies written by
    cell_coef<float>) gives the bits of the FP32 key tables, for 1 and 2 planes per thread."""
    prob = mode3_model(oracle, **case)
    bb = random_interior(prob.shape, 23)
    out = {}
    for src in ("1", "2"):
        monkeypatch.setenv("H2G_RB_DD", src)
        s = make_solver(prob, precision="mixed")
        assert s.tuning()[2] == int(src)
        out[src] = []
        for planes in (1, 2):
            s.set_tuning(8, planes)
            out[src].append(s.preconditioner(bb, "gs"))
        s.close()
    for a, b_ in zip(out["1"], out["2"]):
        assert np.array_equal(a, b_)


@pytest.mark.parametrize("transient", [False, True], ids=["steady", "transient"])
def test_fp32_smoother_classes_boxes(oracle, monkeypatch, transient):
    prob = box_problem(oracle, 33, 31, 9, seed=41, transient=transient)
    bb = random_interior(prob.shape, 3)
    res = []
    for src in ("1", "2"):
        monkeypatch.setenv("H2G_RB_DD", src)
        s = make_solver(prob, precision="mixed")
        res.append(s.preconditioner(bb, "gs"))
        s.close()
    assert np.array_equal(res[0], res[1])


def test_mixed_solve_identical_across_sources(oracle, monkeypatch):
    prob = mode3_model(oracle, 41, 37)
    out = []
    for src in ("1", "2"):
        monkeypatch.setenv("H2G_RB_DD", src)
        monkeypatch.setenv("H2G_AX_DD", src)
        s = make_solver(prob, precision="mixed")
        st, res = s.solve("pbicgstab", tol=1e-8, maxItr=20000, smoother="gs")
        assert st == 0 and res.isconverged
        out.append((res.itr, res.outer, res.res, s.get_theta()))
        s.close()
    assert out[0][:3] == out[1][:3]
    assert np.array_equal(out[0][3], out[1][3])
