"""The SSD likelihood (BINDER/src/cpu/SSDLikelihood.cpp with the log-space E-step of
Registration.cpp:331-470) on the GPU against the FP64 oracle's restatement.  Tolerances: posterior
weights in FP32 (log2 table, exp2 relative to the voxel's largest term), parameter sums in FP64."""
import math

import numpy as np
import pytest

from test_gpu_parity import make_case

pytestmark = pytest.mark.gpu

SIGMA = math.sqrt(9.0 / (8.0 * math.pi))


def ssd_case(seed, shape=(12, 14, 10), bins=16):
    c = make_case(shape=shape, K=bins, L=bins, seed=seed)
    c["bins"] = bins
    return c


def new_reg(core, c, shift_scale, sigma2=4.0, scale=0.9, shift=0.5):
    shape = c["shape"]
    reg = core.Registration(c["d0"], 1, c["grid"], c["grid"], *shape, *shape, 3,
                            float(np.prod(shape)))
    reg.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, c["D"])
    reg.setSSDLikelihood(c["bins"], 1, sigma2, shift_scale, scale, shift, c["v"], c["u"], 1.0, 1.0)
    return reg


def params(oracle, shift_scale, sigma2=4.0, scale=0.9, shift=0.5):
    # with shiftScale 0 the likelihood ignores shift and scale, which stay as given (the reference
    # reports them so: tests/golden/em_ref.npz)
    return oracle.SSDParams(shift_scale, sigma2, shift, scale, 1.0, 1.0)


@pytest.mark.parametrize("shift_scale", [0, 1])
def test_one_em_iteration_matches_oracle(core, oracle, shift_scale):
    c = ssd_case(seed=40 + shift_scale)
    shape, B = c["shape"], c["bins"]
    reg = new_reg(core, c, shift_scale)
    assert reg.EM(1, -1e30, 1, 0) == 1
    p = params(oracle, shift_scale)
    mll, dream, hist = oracle.ssd_estep(c["d0"].astype(np.float64), c["u"], c["v"], p, shape,
                                        shape, B, B)
    lpl = oracle.ssd_update(hist, B, B, p, True)
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)
    got = reg.ssd_parameters()
    assert got["sigma_sq"] == pytest.approx(p.sigma2, rel=1e-4)
    if shift_scale:
        assert got["shift"] == pytest.approx(p.shift, abs=1e-4)
        assert got["scale"] == pytest.approx(p.scale, rel=1e-4)
        np.testing.assert_allclose(reg.get_likelihood_parameters(), [p.scale, p.shift],
                                   rtol=1e-4, atol=1e-4)
    st = reg.iteration_stats()[0]
    assert st[0] == pytest.approx(mll, rel=1e-6)
    assert st[1] == pytest.approx(lpl, rel=1e-4, abs=1e-6)
    lpt, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA, shape)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)


@pytest.mark.parametrize("shift_scale", [0, 1])
def test_em_run_matches_oracle(core, oracle, shift_scale):
    c = ssd_case(seed=50 + shift_scale, shape=(14, 12, 16))
    shape, B = c["shape"], c["bins"]
    reg = new_reg(core, c, shift_scale)
    assert reg.EM(8, -1e30, 1, 0) == 8
    p = params(oracle, shift_scale)
    it, final_o, stats_o = oracle.ssd_em(c["d0"], c["grid"], c["u"], c["v"], p, c["D"],
                                         c["gamma"], SIGMA, shape, shape, B, B,
                                         float(np.prod(shape)), 8, -1e30)
    assert it == 8
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final_o, rtol=0,
                               atol=2e-3)
    np.testing.assert_allclose(reg.iteration_stats()[:, 3], stats_o[:, 3], rtol=1e-5)
    got = reg.ssd_parameters()
    assert got["sigma_sq"] == pytest.approx(p.sigma2, rel=1e-3)
    assert got["shift"] == pytest.approx(p.shift, abs=1e-3)
    assert got["scale"] == pytest.approx(p.scale, rel=1e-3)


def test_small_sigma_does_not_underflow(core, oracle):
    """sigma^2 = 0.05 bins^2: many neighbourhoods have every likelihood below FP32's range in
    linear space; the log-space E-step keeps every voxel and matches the oracle."""
    c = ssd_case(seed=60)
    shape, B = c["shape"], c["bins"]
    reg = new_reg(core, c, 0, sigma2=0.05)
    reg.EM(1, -1e30, 0, 0)
    assert reg.state()["degenerate"] == 0
    p = params(oracle, 0, sigma2=0.05)
    mll, dream, _ = oracle.ssd_estep(c["d0"].astype(np.float64), c["u"], c["v"], p, shape, shape,
                                     B, B)
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=2e-4)
    assert reg.iteration_stats()[0][0] == pytest.approx(mll, rel=1e-5)


def test_reset_and_rejections(core):
    c = ssd_case(seed=61)
    reg = new_reg(core, c, 1)
    reg.EM(3, -1e30, 1, 0)
    a = reg.get_final_locations_as_numpy_array().copy()
    reg.reset()
    assert reg.ssd_parameters() == {"sigma_sq": 4.0, "shift": 0.5, "scale": 0.9}
    reg.EM(3, -1e30, 1, 0)
    # the same run again; the cross-CTA FP32 histogram sums are atomics, so equal to round-off
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array(), a, rtol=0, atol=1e-5)
    # the sampler runs with this likelihood (its checks: tests/test_gpu_ssd_sampler.py)
    m, cv = reg.sampler(1, 1, 2, 0, 1, 1, 1, 1)
    assert np.all(np.isfinite(m)) and np.all(np.isfinite(cv))
    with pytest.raises(core.BinderError):
        new_reg(core, ssd_case(seed=62, bins=80), 0)
