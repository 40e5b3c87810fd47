"""B-spline orders 1 and 2 (BINDER/src/cpu/Spline.cpp; the reference's CPU backend) through the C ABI
/ _core mirror against the FP64 oracle run with the same order.  Tolerances as in the cubic
parity tests."""
import math

import numpy as np
import pytest

from test_gpu_parity import make_case

pytestmark = pytest.mark.gpu

SIGMA = {1: 0.4, 2: math.sqrt(8.0 / (9.0 * math.pi)), 3: math.sqrt(9.0 / (8.0 * math.pi))}


@pytest.fixture
def ordered(oracle):
    yield oracle
    oracle.set_spline_order(3)


def new_reg(core, c, order):
    shape = c["shape"]
    reg = core.Registration(c["d0"], 1, c["grid"], c["grid"], *shape, *shape, order,
                            float(np.prod(shape)))
    reg.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, c["D"])
    reg.setMILikelihood(2.0, c["theta"], c["K"], c["L"], 1, c["v"], c["u"])
    return reg


@pytest.mark.parametrize("order", [1, 2])
def test_one_em_iteration_matches_oracle(core, ordered, order):
    oracle = ordered
    oracle.set_spline_order(order)
    c = make_case(seed=10 + order)
    shape, K, L = c["shape"], c["K"], c["L"]
    reg = new_reg(core, c, order)
    assert reg.EM(1, -1e30, 1, 0) == 1
    mll, dream, hist, deg = oracle.estep(c["d0"].astype(np.float64), c["u"], c["v"],
                                         c["theta"].astype(np.float64), shape, shape, K, L)
    assert deg == 0
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)
    theta = oracle.theta_map(hist, K, L, 2.0)
    np.testing.assert_allclose(reg.get_likelihood_parameters(), theta, rtol=1e-4, atol=1e-7)
    st = reg.iteration_stats()[0]
    assert st[0] == pytest.approx(mll, rel=1e-6)
    lpt, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA[order], shape)
    assert st[2] == pytest.approx(lpt, rel=2e-4)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)


@pytest.mark.parametrize("order", [1, 2])
def test_em_run_matches_oracle_and_mi(core, ordered, order):
    oracle = ordered
    oracle.set_spline_order(order)
    c = make_case(shape=(14, 12, 16), seed=20 + order)
    shape, K, L = c["shape"], c["K"], c["L"]
    reg = new_reg(core, c, order)
    assert reg.EM(10, -1e30, 1, 0) == 10
    final_g = reg.get_final_locations_as_numpy_array().astype(np.float64).ravel()
    it, final_o, theta_o, stats_o = oracle.em(c["d0"], c["grid"], c["u"], c["v"], c["theta"], 2.0,
                                             c["D"], c["gamma"], SIGMA[order], shape, shape, K, L,
                                             float(np.prod(shape)), 10, -1e30)
    np.testing.assert_allclose(final_g, final_o, rtol=0, atol=2e-3)
    np.testing.assert_allclose(reg.iteration_stats()[:, 3], stats_o[:, 3], rtol=1e-5)
    _, _, h_g, _ = oracle.estep(final_g, c["u"], c["v"], theta_o, shape, shape, K, L)
    _, _, h_o, _ = oracle.estep(final_o, c["u"], c["v"], theta_o, shape, shape, K, L)
    mi_g, mi_o = oracle.mutual_information(h_g, K, L), oracle.mutual_information(h_o, K, L)
    assert abs(mi_g - mi_o) <= 1e-3 * abs(mi_o)


@pytest.mark.parametrize("order", [1, 2])
def test_sampler_matches_oracle_draw_for_draw(core, ordered, order):
    oracle = ordered
    oracle.set_spline_order(order)
    c = make_case(seed=30 + order)
    shape, K, L = c["shape"], c["K"], c["L"]
    reg = new_reg(core, c, order)
    mean_g, cov_g = reg.sampler(555, 1, 4, 0, 1, 1, 1, 1)
    mean_o, cov_o, _, _, _, capped = oracle.sampler(
        c["d0"], np.zeros_like(c["d0"]), c["grid"], c["u"], c["v"], c["theta"], 2.0, c["D"],
        c["gamma"], SIGMA[order], [1, 1, 1], [1, 1, 1], shape, shape, K, L, 555, 1, 4,
        sample_gamma=0, sample_gamma_every=1)
    assert capped == 0
    assert np.quantile(np.abs(mean_g.ravel() - mean_o), 0.99) < 1e-3
    assert np.median(np.abs(cov_g.ravel() - cov_o)) < 1e-4


def test_unsupported_order_is_rejected(core):
    c = make_case()
    with pytest.raises(core.BinderError) as e:
        core.Registration(c["d0"], 1, c["grid"], c["grid"], *c["shape"], *c["shape"], 4, 10.0)
    assert e.value.status == 3
