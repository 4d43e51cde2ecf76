"""Launch-shape tuning of the colour pass: every block height and planes-per-thread choice gives
bit-identical results (the pass has no reduction); the tuner picks an allowed shape and caches
it per grid."""
import os

import numpy as np
import pytest

import h2_b200
from conftest import mode3_model
from test_gpu_kernels import make_solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_heights_give_identical_solves(oracle, precision):
    prob = mode3_model(oracle, 40)
    ref = None
    for rows, planes in ((2, 2), (4, 2), (8, 2), (16, 2), (4, 1), (8, 1)):
        s = make_solver(prob, precision=precision)
        s.set_tuning(rows, planes)
        st, res = s.solve("pbicgstab", tol=1e-8, maxItr=20000, smoother="gs")
        assert st == 0
        out = (res.itr, res.res0, res.res, s.get_theta())
        pre = s.preconditioner(prob.wk["b"])
        if ref is None:
            ref = out + (pre,)
        else:
            assert out[:3] == ref[:3]
            assert np.array_equal(out[3], ref[3]) and np.array_equal(pre, ref[4])
        s.close()


def test_tuner_choice_is_cached(oracle):
    prob = mode3_model(oracle, 32)
    s1 = make_solver(prob)
    r1 = s1.autotune()
    assert r1[0] in (2, 4, 8, 16) and r1[1] in (1, 2)
    s2 = make_solver(prob)
    assert s2.autotune() == r1
    with pytest.raises(h2_b200.H2GError):
        s2.set_tuning(3)
    with pytest.raises(h2_b200.H2GError):
        s2.set_tuning(4, 3)
    s2.set_tuning(0)  # tune again: the cached choice comes back
    assert s2.autotune() == r1
    s1.close()
    s2.close()


def test_dd_source_gives_identical_results(oracle, monkeypatch):
    """dd summed per cell or read from the per-cell array, in CalcAX and in the colour pass."""
    prob = mode3_model(oracle, 40)
    x = np.zeros(prob.shape, order="F")
    x[1:-1, 1:-1, 1:-1] = np.random.default_rng(1).standard_normal((prob.NX, prob.NY, prob.NZ))
    outs = []
    for dd in ("0", "1"):
        monkeypatch.setenv("H2G_AX_DD", dd)
        monkeypatch.setenv("H2G_RB_DD", dd)
        s = make_solver(prob)
        st, res = s.solve("pbicgstab", tol=1e-8, maxItr=20000, smoother="gs")
        assert st == 0
        outs.append((res.itr, res.res, s.get_theta(), s.calc_ax(x)))
        s.close()
    assert outs[0][:2] == outs[1][:2]
    assert np.array_equal(outs[0][2], outs[1][2]) and np.array_equal(outs[0][3], outs[1][3])
    assert os.environ.get("H2G_AX_DD") == "1" and os.environ.get("H2G_RB_DD") == "1"


def test_forced_choices_restrict_the_tuner(oracle, monkeypatch):
    """A forced plane count or dd source is kept and the other choices are tuned around it."""
    prob = mode3_model(oracle, 32)
    for planes, dd in (("1", None), ("2", "0"), ("1", "1"), ("2", "2")):
        monkeypatch.setenv("H2G_RB_PLANES", planes)
        if dd is None:
            monkeypatch.delenv("H2G_RB_DD", raising=False)
        else:
            monkeypatch.setenv("H2G_RB_DD", dd)
        s = make_solver(prob)
        rows, p, rb_dd, _ = s.tuning()
        assert rows in (2, 4, 8, 16) and p == int(planes)
        if dd is not None:
            assert rb_dd == int(dd)
        s.close()
