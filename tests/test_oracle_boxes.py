"""The oracle on the hand-built boxes of the GPU box tests (no GPU): the operator is symmetric
with every boundary type, steady and transient (test_symmetry.jl:11-81 restated on boxes; the
adjoint relies on it), and PBiCGSTAB and CG reach the same field."""
import numpy as np
import pytest

from test_gpu_boxes import GRIDS, box_problem


def _interior(shape, rng):
    x = np.zeros(shape, order="F")
    x[1:-1, 1:-1, 1:-1] = rng.standard_normal(tuple(n - 2 for n in shape))
    return x


@pytest.mark.parametrize("transient", [False, True], ids=["steady", "transient"])
@pytest.mark.parametrize("grid", GRIDS, ids=["x".join(map(str, g)) for g in GRIDS])
def test_box_operator_symmetric(oracle, grid, transient):
    prob = box_problem(oracle, *grid, seed=sum(grid), transient=transient)
    rng = np.random.default_rng(31)
    for _ in range(2):
        x, y = _interior(prob.shape, rng), _interior(prob.shape, rng)
        axy = float(np.sum(oracle.calc_ax(prob, x) * y))
        xay = float(np.sum(x * oracle.calc_ax(prob, y)))
        assert abs(axy - xay) <= 1e-12 * max(abs(axy), abs(xay)), (axy, xay)


@pytest.mark.parametrize("grid", [(6, 5, 7), (33, 31, 9)], ids=["6x5x7", "33x31x9"])
def test_box_krylov_methods_agree(oracle, grid):
    a = box_problem(oracle, *grid, seed=7)
    b = box_problem(oracle, *grid, seed=7)
    assert oracle.pbicgstab(a, tol=1e-12, maxItr=20000, smoother="gs")[0]
    assert oracle.cg(b, tol=1e-12, maxItr=20000, smoother="gs")[0]
    assert np.abs(a.wk["theta"] - b.wk["theta"]).max() <= 1e-6
