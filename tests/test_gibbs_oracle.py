"""The oracle's Gibbs penalties (GibbsPenalty.inl with the Quadratic and Relative Difference potentials):
derivatives against finite differences (test_priors.cxx style), Gibbs Quadratic against QuadraticPrior."""
import numpy as np
import pytest

from stir_b200 import _abi

TEST_PACK_WEIGHTS = np.array([[[0, 1, 0], [1, 0, 1], [0, 1, 0]]], np.float32)  # OSMAPOSL_test_PM_QPweights.par


def _image(seed, shape=(5, 6, 7)):
    return np.random.default_rng(seed).uniform(0.5, 2.0, shape).astype(np.float32)


def _weights(oracle_lib, kind):
    if kind == "default":
        return oracle_lib.gibbs_default_weights((2.0, 3.0, 3.0))
    if kind == "2D":
        return oracle_lib.gibbs_default_weights((2.0, 3.0, 3.0), only_2D=True)
    if kind == "test_pack":
        return TEST_PACK_WEIGHTS
    rng = np.random.default_rng(5)  # a symmetric 5x3x5 neighbourhood
    w = rng.uniform(0, 1, (5, 3, 5)).astype(np.float32)
    w = (w + w[::-1, ::-1, ::-1]) / 2
    w[2, 1, 2] = 0
    return w.astype(np.float32)


@pytest.mark.parametrize("potential", [1, 2])
@pytest.mark.parametrize("kind", ["default", "2D", "test_pack", "5x3x5"])
def test_gibbs_derivatives_vs_finite_differences(oracle_lib, potential, kind):
    O = oracle_lib
    x = _image(11)
    w = _weights(O, kind)
    kappa = np.random.default_rng(3).uniform(0.5, 1.5, x.shape).astype(np.float32)
    beta, gamma, eps = 0.7, 2.0, 0.01
    args = dict(kappa=kappa, gamma=gamma, epsilon=eps)
    g = O.gibbs("gradient", potential, beta, w, x, **args)
    d = O.gibbs("hessian_diagonal", potential, beta, w, x, **args)
    h = 1e-2
    for idx in [(0, 0, 0), (2, 3, 4), (4, 5, 6), (1, 2, 3)]:
        xp, xm = x.astype(np.float64).copy(), x.astype(np.float64).copy()
        xp[idx] += h
        xm[idx] -= h
        vp = O.gibbs("value", potential, beta, w, xp.astype(np.float32), **args)
        vm = O.gibbs("value", potential, beta, w, xm.astype(np.float32), **args)
        assert abs((vp - vm) / (2 * h) - g[idx]) <= 2e-3 * max(1.0, np.abs(g).max())
        gp = O.gibbs("gradient", potential, beta, w, xp.astype(np.float32), **args)
        gm = O.gibbs("gradient", potential, beta, w, xm.astype(np.float32), **args)
        assert abs((gp[idx] - gm[idx]) / (2 * h) - d[idx]) <= 5e-3 * max(1.0, np.abs(d).max())
        # the Hessian row of voxel idx = H e_idx (symmetric weights and potential)
        e = np.zeros_like(x)
        e[idx] = 1
        row = O.gibbs("hessian", potential, beta, w, x, voxel=idx, **args)
        col = O.gibbs("hessian_times_input", potential, beta, w, x, input_image=e, **args)
        assert np.allclose(row, col, rtol=1e-5, atol=1e-6 * np.abs(col).max())
        assert abs(row[idx] - d[idx]) <= 1e-5 * max(1.0, abs(d[idx]))
    # H v against the directional difference of the gradient
    v = np.random.default_rng(8).uniform(-1, 1, x.shape).astype(np.float32)
    hv = O.gibbs("hessian_times_input", potential, beta, w, x, input_image=v, **args)
    hs = 1e-3
    gp = O.gibbs("gradient", potential, beta, w, (x + hs * v).astype(np.float32), **args).astype(np.float64)
    gm = O.gibbs("gradient", potential, beta, w, (x - hs * v).astype(np.float32), **args).astype(np.float64)
    assert np.linalg.norm((gp - gm) / (2 * hs) - hv) / np.linalg.norm(hv) < 2e-2
    # gradient times input is <gradient, input>
    gti = O.gibbs("gradient_times_input", potential, beta, w, x, input_image=v, **args)
    assert abs(gti - float(g.astype(np.float64).ravel() @ v.astype(np.float64).ravel())) <= 1e-5 * abs(gti)


def test_gibbs_quadratic_is_quadratic_prior(oracle_lib):
    """GibbsQuadraticPenalty's gradient (2 beta sum w (c - n) / 2) is QuadraticPrior's (beta sum w (c - n)) with the
    same weights, and so is the value: equal up to rounding (QuadraticPrior multiplies w (c - n) in float, the Gibbs
    penalty in double)."""
    O = oracle_lib
    x = _image(12, (6, 7, 8))
    vox = (2.0, 3.0, 3.0)
    kappa = np.random.default_rng(4).uniform(0.5, 1.5, x.shape).astype(np.float32)
    w = O.gibbs_default_weights(vox)
    p = _abi.Prior(type=_abi.PRIOR_QUADRATIC, penalisation_factor=0.5)
    for k in (None, kappa):
        gg = O.gibbs("gradient", 1, 0.5, w, x, kappa=k)
        qg = O.prior_gradient(p, x, vox, kappa=k)
        assert np.max(np.abs(gg - qg)) <= 1e-6 * np.abs(qg).max()
        assert abs(O.gibbs("value", 1, 0.5, w, x, kappa=k) - O.prior_value(p, x, vox, kappa=k)) <= 1e-7 * abs(
            O.prior_value(p, x, vox, kappa=k))


def test_gibbs_zero_penalisation_factor(oracle_lib):
    O = oracle_lib
    x = _image(13)
    w = O.gibbs_default_weights((2.0, 2.0, 2.0))
    assert O.gibbs("value", 2, 0.0, w, x) == 0.0
    assert not O.gibbs("gradient", 2, 0.0, w, x).any()
    base = np.ones_like(x)
    assert np.array_equal(O.gibbs("hessian_times_input", 2, 0.0, w, x, input_image=x, out=base), base)


def test_gibbs_default_weights(oracle_lib):
    w = oracle_lib.gibbs_default_weights((2.0, 2.0, 2.0))
    assert w.shape == (3, 3, 3) and w[1, 1, 1] == 0
    assert np.isclose(w[1, 1, 0], 1.0) and np.isclose(w[1, 0, 0], 1 / np.sqrt(2)) and np.isclose(w[0, 0, 0], 1 / np.sqrt(3))
    w2 = oracle_lib.gibbs_default_weights((2.0, 2.0, 2.0), only_2D=True)
    assert w2.shape == (1, 3, 3) and np.array_equal(w2[0], w[1])
