"""The SSD filter likelihood (BINDER/src/cpu/SSDLikelihoodFilter.cpp with the log-space E-step of
Registration.cpp:331-470: M fixed-image feature channels predicted from F moving-image features
by an M x F coefficient matrix that EM refits, and a variance per channel) on the GPU against the
FP64 oracle, whose likelihood and parameter update are pinned to the reference's compiled class
(tests/test_oracle.py).  Tolerances: posterior weights in FP32, parameter sums in FP64."""
import math

import numpy as np
import pytest
from scipy import ndimage as ndi

pytestmark = pytest.mark.gpu

SIGMA = math.sqrt(9.0 / (8.0 * math.pi))


def feature_case(shape=(12, 10, 9), M=2, F=3, rfa=0, seed=0, disp=0.6):
    """Smooth random moving-image features at the nodes, fixed-image channels that are a linear
    mix of them sampled through a smooth warp, plus noise."""
    from binder_b200 import phantoms
    from binder_b200.utils import initialize_fourier_domain_smoothing
    rng = np.random.default_rng(seed)
    Fn = M if rfa else F
    feats = np.stack([ndi.gaussian_filter(rng.normal(0, 1, shape), 1.5) * 6.0 + f
                      for f in range(Fn)], -1)
    mix = np.eye(M, Fn) if rfa else rng.normal(0.0, 1.0, (M, Fn))
    grid = phantoms.identity_positions(shape)
    warp = grid + phantoms.smooth_random_field(shape, 0.8, 3.0, rng)
    moved = np.stack([ndi.map_coordinates(feats[..., f], np.moveaxis(warp, -1, 0), order=1,
                                          mode="nearest") for f in range(Fn)], -1)
    vox = moved @ mix.T + rng.normal(0.0, 0.3, shape + (M,))
    d0 = (grid + phantoms.smooth_random_field(shape, disp, 3.0, rng)).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, len(shape)).astype(np.float32)
    coeff = rng.normal(0.0, 1.0, (M, F))
    sigma = rng.random(M) * 1.5 + 0.5
    return dict(shape=shape, M=M, F=F, Fn=Fn, rfa=rfa, nodes=feats.reshape(-1, Fn),
                voxels=vox.reshape(-1, M), grid=grid, d0=d0, D=D, gamma=(0.8, 0.6, 1.1),
                coeff=coeff, sigma=sigma, alpha0=2.0, beta0=0.5)


def new_reg(core, c):
    shape = c["shape"]
    reg = core.Registration(c["d0"], 1, c["grid"], c["grid"], *shape, *shape, 3,
                            float(np.prod(shape)))
    reg.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, c["D"])
    reg.setSSDLikelihoodFilter(c["coeff"], 1, c["sigma"], c["nodes"], c["voxels"], c["rfa"],
                               c["alpha0"], c["beta0"], c["M"], c["F"])
    return reg


def oracle_iteration(oracle, c, p, d, update=True):
    shape = c["shape"]
    mll, dream, acc = oracle.ssdf_estep(d, c["nodes"], c["voxels"], p, shape, shape)
    cost = oracle.ssdf_update(p, c["nodes"], shape, acc, update)
    lpt, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA, shape)
    return mll, dream, cost, lpt, final


def params(oracle, c):
    return oracle.ssdf_params(c["coeff"], c["sigma"], c["rfa"], c["alpha0"], c["beta0"])


@pytest.mark.parametrize("rfa,M,F", [(0, 2, 3), (1, 3, 3), (0, 1, 1), (0, 3, 6)])
def test_one_em_iteration_matches_oracle(core, oracle, rfa, M, F):
    c = feature_case(M=M, F=F, rfa=rfa, seed=10 * M + F + rfa)
    reg = new_reg(core, c)
    assert reg.EM(1, -1e30, 1, 0) == 1
    p = params(oracle, c)
    mll, dream, cost, lpt, final = oracle_iteration(oracle, c, p, c["d0"].astype(np.float64))
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)
    coeff, sigma = reg.ssd_filter_parameters()
    np.testing.assert_allclose(coeff, np.array(p.coeff[:M * F]).reshape(M, F), rtol=1e-4,
                               atol=1e-5)
    np.testing.assert_allclose(sigma, np.array(p.sigma[:M]), rtol=1e-4)
    np.testing.assert_allclose(reg.get_likelihood_parameters(), coeff.ravel(), rtol=1e-6)
    st = reg.iteration_stats()[0]
    assert st[0] == pytest.approx(mll, rel=1e-6)
    assert st[1] == pytest.approx(cost, rel=1e-4, abs=1e-6)
    assert st[2] == pytest.approx(lpt, rel=2e-4)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)


def test_three_iterations_track_oracle(core, oracle):
    c = feature_case(M=2, F=2, seed=7)
    reg = new_reg(core, c)
    assert reg.EM(3, -1e30, 1, 0) == 3
    p = params(oracle, c)
    d = c["d0"].astype(np.float64)
    mlps = []
    for _ in range(3):
        mll, _, cost, lpt, d = oracle_iteration(oracle, c, p, d)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), d, rtol=0,
                               atol=1e-3)
    coeff, sigma = reg.ssd_filter_parameters()
    np.testing.assert_allclose(coeff, np.array(p.coeff[:4]).reshape(2, 2), rtol=1e-3, atol=1e-4)
    np.testing.assert_allclose(sigma, np.array(p.sigma[:2]), rtol=1e-3)


def test_without_parameter_updates(core, oracle):
    """update_likelihood_parameters = 0: coefficients and variances stay, the cost is that of the
    given variances."""
    c = feature_case(M=2, F=3, seed=3)
    reg = new_reg(core, c)
    assert reg.EM(1, -1e30, 0, 0) == 1
    coeff, sigma = reg.ssd_filter_parameters()
    np.testing.assert_array_equal(coeff, c["coeff"])
    np.testing.assert_array_equal(sigma, c["sigma"])
    p = params(oracle, c)
    mll, dream, cost, _, _ = oracle_iteration(oracle, c, p, c["d0"].astype(np.float64), False)
    st = reg.iteration_stats()[0]
    assert st[0] == pytest.approx(mll, rel=1e-6)
    assert st[1] == pytest.approx(cost, rel=1e-9)
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)


def test_2d_image(core, oracle):
    from binder_b200 import phantoms
    from binder_b200.utils import initialize_fourier_domain_smoothing
    rng = np.random.default_rng(21)
    shape2, M, F = (26, 22), 2, 2
    feats = np.stack([ndi.gaussian_filter(rng.normal(0, 1, shape2), 1.5) * 6.0 + f
                      for f in range(F)], -1)
    vox = feats @ rng.normal(0, 1, (M, F)).T + rng.normal(0, 0.3, shape2 + (M,))
    grid = phantoms.identity_positions(shape2)
    d0 = (grid + phantoms.smooth_random_field(shape2, 0.6, 3.0, rng)).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape2, True, 2, 2).astype(np.float32)
    c = dict(shape=shape2 + (1,), M=M, F=F, rfa=0, nodes=feats.reshape(-1, F),
             voxels=vox.reshape(-1, M), grid=grid, D=D, gamma=(0.8, 0.6, 1.0),
             coeff=rng.normal(0, 1, (M, F)), sigma=np.array([1.0, 2.0]), alpha0=2.0, beta0=0.5)
    nx, ny = shape2
    reg = core.Registration(d0, 1, grid, grid, nx, ny, 1, nx, ny, 1, 3, float(nx * ny))
    reg.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, D)
    reg.setSSDLikelihoodFilter(c["coeff"], 1, c["sigma"], c["nodes"], c["voxels"], 0,
                               c["alpha0"], c["beta0"], M, F)
    assert reg.EM(1, -1e30, 1, 0) == 1
    p = params(oracle, c)
    mll, dream, cost, lpt, final = oracle_iteration(oracle, c, p, d0.astype(np.float64))
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)
    coeff, sigma = reg.ssd_filter_parameters()
    np.testing.assert_allclose(coeff, np.array(p.coeff[:M * F]).reshape(M, F), rtol=1e-4,
                               atol=1e-5)
    np.testing.assert_allclose(sigma, np.array(p.sigma[:M]), rtol=1e-4)
    assert reg.iteration_stats()[0][0] == pytest.approx(mll, rel=1e-6)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)


def test_reset_and_errors(core):
    from binder_b200._lib import BinderError
    c = feature_case(M=2, F=3, seed=1)
    reg = new_reg(core, c)
    reg.EM(2, -1e30, 1, 0)
    assert not np.array_equal(reg.ssd_filter_parameters()[1], c["sigma"])
    reg.reset()
    coeff, sigma = reg.ssd_filter_parameters()
    np.testing.assert_array_equal(coeff, c["coeff"])
    np.testing.assert_array_equal(sigma, c["sigma"])
    # the sampler runs with this likelihood (its checks: tests/test_gpu_filter_sampler.py)
    m, cv = reg.sampler(1, 1, 2, 0, 1, 1, 1, 1)
    assert np.all(np.isfinite(m)) and np.all(np.isfinite(cv))
    with pytest.raises(BinderError, match="sigma must be positive"):
        reg.setSSDLikelihoodFilter(c["coeff"], 1, [1.0, -1.0], c["nodes"], c["voxels"], 0, 2.0,
                                   0.5, 2, 3)
    V = int(np.prod(c["shape"]))
    with pytest.raises(BinderError, match="1 <= M, F <= 8"):
        reg.setSSDLikelihoodFilter(np.ones((9, 1)), 1, np.ones(9), np.ones(V), np.ones(V * 9), 0,
                                   2.0, 0.5, 9, 1)
