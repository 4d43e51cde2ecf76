"""The GPU geometry fill (fillID!, src/modelA.jl:545-556) and the host set-up of h2_b200.model
against the oracle: the material-ID field and every WorkBuffers array are bit-identical."""
import numpy as np
import pytest

from conftest import mode3_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("NX,NY,NZ", [(40, 40, 30), (41, 37, 30), (120, 120, 30), (240, 240, 30), (180, 180, 30)])
def test_fill_id_bit_exact(oracle, NX, NY, NZ):
    from h2_b200 import model
    got = model.fill_id(NX, NY, NZ)
    ref = oracle.fill_id(NX, NY, NZ)
    assert np.array_equal(got, ref), np.argwhere(got != ref)[:10]


def test_fill_id_refined_z(oracle):
    """NZ = 60 (the refined Z grid of the 480^2 x 60 configuration) at a small XY size."""
    from h2_b200 import model
    assert np.array_equal(model.fill_id(48, 48, 60), oracle.fill_id(48, 48, 60))


@pytest.mark.parametrize("kw", [dict(), dict(symmetric=True), dict(is_steady=False, dt=1e-4)])
def test_build_mode3_bit_exact(oracle, kw):
    from h2_b200 import model
    m = model.build_mode3(40, 40, 30, **kw)
    ref = mode3_model(oracle, 40, **kw)
    for n_ref, n_got in [("theta", "theta"), ("b", "b"), ("mask", "mask"), ("rho", "rho"), ("lam", "lam"),
                         ("cp", "cp"), ("hsrc", "hsrc")]:
        assert np.array_equal(getattr(m.wk, n_got), ref.wk[n_ref]), n_ref
    assert np.array_equal(m.HC, ref.HC) and np.array_equal(m.ZC, ref.ZC) and np.array_equal(m.dZ, ref.dZ)
    assert (m.dx, m.dy) == (ref.dx, ref.dy)
