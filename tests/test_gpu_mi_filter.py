"""The MI filter likelihood (MILikelihoodFilter.cpp: M channels of bins, the weight of a node the
product of the channels' theta entries, one joint histogram per channel) through the C ABI / _core
mirror against the FP64 oracle, whose likelihood and parameter update are pinned to the reference's
compiled class (tests/test_oracle.py).  Tolerances as in the MI parity tests."""
import math

import numpy as np
import pytest

from test_gpu_parity import make_case

pytestmark = pytest.mark.gpu

SIGMA = math.sqrt(9.0 / (8.0 * math.pi))


def filter_case(shape=(12, 10, 9), K=8, L=6, M=3, seed=0):
    """make_case's pair with M channels: channel 0 is its bins, the others shifted copies mixed
    with noise, laid out [..., M] and flattened as a caller of the reference would."""
    c = make_case(shape=shape, K=K, L=L, seed=seed)
    rng = np.random.default_rng(seed + 100)
    V = int(np.prod(shape))
    vch = [c["v"].ravel()] + [np.where(rng.random(V) < 0.3, rng.integers(0, K, V),
                                       np.roll(c["v"].ravel(), 7 * m)) for m in range(1, M)]
    uch = [c["u"].ravel()] + [np.where(rng.random(V) < 0.3, rng.integers(0, L, V),
                                       np.roll(c["u"].ravel(), 5 * m)) for m in range(1, M)]
    c["vf"] = np.stack(vch, -1).astype(np.int32).ravel()
    c["uf"] = np.stack(uch, -1).astype(np.int32).ravel()
    th = rng.random((M, K, L)) + 0.05
    c["thf"] = (th / th.sum(-1, keepdims=True)).astype(np.float32)
    c["M"] = M
    return c


def new_filter_reg(core, c):
    shape = c["shape"]
    reg = core.Registration(c["d0"], 1, c["grid"], c["grid"], *shape, *shape, 3,
                            float(np.prod(shape)))
    reg.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, c["D"])
    reg.setMILikelihoodFilter(2.0, c["thf"], 1, c["vf"], c["uf"], c["K"], c["L"], c["M"])
    return reg


def oracle_iteration(oracle, c, d, theta):
    shape, K, L, M = c["shape"], c["K"], c["L"], c["M"]
    mll, dream, hist, deg = oracle.estep_filter(d, c["uf"], c["vf"], theta, shape, shape, K, L, M)
    th = oracle.theta_map(hist, M * K, L, 2.0)
    lpt, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA, shape)
    return mll, dream, th, lpt, final, deg


@pytest.mark.parametrize("M", [1, 2, 3, 8])
def test_one_em_iteration_matches_oracle(core, oracle, M):
    c = filter_case(M=M, K=8 if M < 8 else 6, L=6 if M < 8 else 5, seed=M)
    reg = new_filter_reg(core, c)
    assert reg.EM(1, -1e30, 1, 0) == 1
    mll, dream, th, lpt, final, deg = oracle_iteration(
        oracle, c, c["d0"].astype(np.float64), c["thf"].astype(np.float64))
    assert deg == 0
    st = reg.iteration_stats()[0]
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)
    got_th = reg.get_likelihood_parameters()
    assert got_th.size == M * c["K"] * c["L"]
    np.testing.assert_allclose(got_th, th, rtol=1e-4, atol=1e-6)
    assert st[0] == pytest.approx(mll, rel=1e-6)
    assert st[1] == pytest.approx(oracle.dirichlet_cost(th, M * c["K"], c["L"], 2.0), rel=1e-5)
    assert st[2] == pytest.approx(lpt, rel=2e-4)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)


def test_three_iterations_track_oracle(core, oracle):
    c = filter_case(M=2, seed=4)
    reg = new_filter_reg(core, c)
    assert reg.EM(3, -1e30, 1, 0) == 3
    d, th = c["d0"].astype(np.float64), c["thf"].astype(np.float64)
    for _ in range(3):
        _, _, th, _, d, _ = oracle_iteration(oracle, c, d, th)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), d, rtol=0,
                               atol=1e-3)
    np.testing.assert_allclose(reg.get_likelihood_parameters(), th, rtol=1e-3, atol=1e-5)


def test_one_channel_equals_mi(core):
    """M = 1 is the MI likelihood (the filter kernel against the MI kernel)."""
    c = filter_case(M=1, seed=9)
    a = new_filter_reg(core, c)
    b = core.Registration(c["d0"], 1, c["grid"], c["grid"], *c["shape"], *c["shape"], 3,
                          float(np.prod(c["shape"])))
    b.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, c["D"])
    b.setMILikelihood(2.0, c["thf"][0], c["K"], c["L"], 1, c["vf"], c["uf"])
    assert a.EM(2, -1e30, 1, 0) == b.EM(2, -1e30, 1, 0) == 2
    np.testing.assert_allclose(a.get_final_locations_as_numpy_array(),
                               b.get_final_locations_as_numpy_array(), rtol=0, atol=1e-4)
    np.testing.assert_allclose(a.get_likelihood_parameters(), b.get_likelihood_parameters(),
                               rtol=1e-4, atol=1e-6)


def test_2d_image(core, oracle):
    from test_gpu_2d import make_case2d
    c = make_case2d(shape=(30, 26), K=8, L=6, seed=3)
    rng = np.random.default_rng(5)
    M, K, L = 2, c["K"], c["L"]
    V = int(np.prod(c["shape"]))
    c["vf"] = np.stack([c["v"].ravel(), rng.integers(0, K, V)], -1).astype(np.int32).ravel()
    c["uf"] = np.stack([c["u"].ravel(), rng.integers(0, L, V)], -1).astype(np.int32).ravel()
    th = rng.random((M, K, L)) + 0.05
    thf = (th / th.sum(-1, keepdims=True)).astype(np.float32)
    nx, ny = c["shape"]
    reg = core.Registration(c["d0"], 1, c["grid"], c["grid"], nx, ny, 1, nx, ny, 1, 3,
                            float(nx * ny))
    reg.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, c["D"])
    reg.setMILikelihoodFilter(2.0, thf, 1, c["vf"], c["uf"], K, L, M)
    assert reg.EM(1, -1e30, 1, 0) == 1
    vs = c["vshape"]
    mll, dream, hist, _ = oracle.estep_filter(c["d0"].astype(np.float64), c["uf"], c["vf"],
                                              thf.astype(np.float64), vs, vs, K, L, M)
    _, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA, vs)
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)
    np.testing.assert_allclose(reg.get_likelihood_parameters(),
                               oracle.theta_map(hist, M * K, L, 2.0), rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)
    assert reg.iteration_stats()[0][0] == pytest.approx(mll, rel=1e-6)


def test_reset_and_errors(core):
    from binder_b200._lib import BinderError
    c = filter_case(M=2, seed=1)
    reg = new_filter_reg(core, c)
    th0 = reg.get_likelihood_parameters().copy()
    np.testing.assert_array_equal(th0, c["thf"].ravel())
    reg.EM(2, -1e30, 1, 0)
    assert not np.array_equal(reg.get_likelihood_parameters(), th0)
    reg.reset()
    np.testing.assert_array_equal(reg.get_likelihood_parameters(), th0)
    # the sampler runs with this likelihood (its checks: tests/test_gpu_filter_sampler.py)
    m, cv = reg.sampler(1, 1, 2, 0, 1, 1, 1, 1)
    assert np.all(np.isfinite(m)) and np.all(np.isfinite(cv))
    bad = c["uf"].copy()
    bad[17] = c["L"]
    with pytest.raises(BinderError, match="binned_voxels value 6 outside"):
        reg.setMILikelihoodFilter(2.0, c["thf"], 1, c["vf"], bad, c["K"], c["L"], 2)
    with pytest.raises(BinderError, match="channels"):
        reg.setMILikelihoodFilter(2.0, np.ones((9, 2, 2), np.float32) / 2, 1, c["vf"], c["uf"],
                                  2, 2, 9)
    V = int(np.prod(c["shape"]))
    with pytest.raises(ValueError, match="at least"):
        reg.setMILikelihoodFilter(2.0, c["thf"], 1, c["vf"], c["uf"][:V], c["K"], c["L"], 2)
