"""Host side of the gradient parametrisation (no GPU): the z-band of every plane, the per-plane
conductivity factors and the reduction of a per-cell dJ/d ln(lambda) to the 13 parameters use
one mapping; checked through a functional that is linear in ln(lambda), whose parameter
gradient the reduction must give exactly."""
import numpy as np

from h2_b200 import adjoint as A


def _zc(oracle, nz=30):
    return oracle.genz(nz)[1]


def test_bands_cover_the_stack(oracle):
    for nz in (30, 60):
        ZC = _zc(oracle, nz)
        b = A.band_of_plane(ZC)
        assert b[0] == -1 and b[-1] == -1
        inner = b[1:-1]
        assert (inner >= 0).all() and (np.diff(inner) >= 0).all()
        assert set(inner) == set(range(A.NBANDS))
        for k in range(1, ZC.size - 1):
            assert A.ZM[b[k]] <= ZC[k] <= A.ZM[b[k] + 1]


def test_lam_scale_and_draw(oracle):
    ZC = _zc(oracle)
    beta = A.draw_beta(3)
    assert beta.shape == (A.NPARAMS,)
    assert (beta >= np.log(0.8)).all() and (beta <= np.log(1.2)).all()
    s = A.lam_scale(beta, ZC)
    b = A.band_of_plane(ZC)
    assert s[0] == 1.0 and s[-1] == 1.0
    assert np.allclose(s[1:-1], np.exp(beta[b[1:-1]] + beta[A.NBANDS]), rtol=0, atol=0)


def test_params_gradient_is_the_chain_rule(oracle):
    """J(beta) = sum_c G_c ln(lambda_c(beta)) with lambda_c = lambda0_c * lam_scale(beta)[k]:
    dJ/dbeta from params_gradient(G) equals central differences of J (J is linear in beta)."""
    ZC = _zc(oracle)
    rng = np.random.default_rng(4)
    shape = (9, 8, ZC.size)
    G = np.zeros(shape)
    G[1:-1, 1:-1, 1:-1] = rng.standard_normal((7, 6, ZC.size - 2))
    lam0 = rng.uniform(0.5, 400.0, shape)

    def J(beta):
        return float(np.sum(G * np.log(lam0 * A.lam_scale(beta, ZC)[None, None, :])))

    beta = A.draw_beta(5)
    g = A.params_gradient(G, ZC)
    h = 1e-3
    for j in range(A.NPARAMS):
        e = np.zeros(A.NPARAMS)
        e[j] = h
        fd = (J(beta + e) - J(beta - e)) / (2 * h)
        assert abs(fd - g[j]) <= 1e-8 * max(1.0, abs(g[j])), (j, fd, g[j])


def test_silicon_weights(oracle):
    NX, NZ = 12, 30
    ID = oracle.fill_id(NX, NX, NZ)
    _, _, dZ = oracle.genz(NZ)
    dx = oracle.pitch(NX)
    w = A.silicon_weights(ID, dx, dx, dZ)
    sil = np.isin(ID, A.SILICON_IDS)
    sil[0], sil[-1], sil[:, 0], sil[:, -1], sil[:, :, 0], sil[:, :, -1] = (False,) * 6
    assert w.flags.f_contiguous
    assert (w[~sil] == 0).all()
    k = np.nonzero(sil)[2]
    assert np.array_equal(w[sil], (dx * dx) * dZ[k])
