"""The sampler with the filter likelihoods (Registration.cpp:515-642 driving
MILikelihoodFilter.cpp: M channels, channel m of voxel / node i read at [i + m]).

1. The draws of theta against the oracle: with order-1 splines at integer positions every
   voxel's categorical draw is its own node, so each channel's counts are the joint histogram of
   its (node bin, voxel bin) at the identity, and theta after two sweeps must equal the oracle's
   Dirichlet draw (Philox, the same counters) over the M * K rows of those counts.
2. The whole sampler against the reference's own Registration::sampler with the MI filter
   likelihood in distribution: 32 GPU chains from the positions of
   tests/golden/sampler_mi_filter_ref.npz (32 reference chains, every switch on) agree in their
   chain means, covariances and final theta within Monte Carlo error.
3. The same two checks for the SSD filter likelihood (SSDLikelihoodFilter.cpp), with
   reg_across_features 1 (sigmas drawn) and 0 (coefficients drawn too)."""
import numpy as np
import pytest

from conftest import golden
from sampler_stats import UPPER, agrees, summary

pytestmark = pytest.mark.gpu


def _registration(core, d0, grid, shape, D, gamma, v, u, theta, alpha, order=3):
    V = int(np.prod(shape))
    M, K, L = theta.shape
    reg = core.Registration(d0.astype(np.float32), 1, grid.astype(np.float32),
                            grid.astype(np.float32), *shape, *shape, order, float(V))
    reg.setNonLinearTransformation(*[float(x) for x in gamma], 1, 1, 1, 1, 1, 1,
                                   D.astype(np.float32))
    reg.setMILikelihoodFilter(alpha, theta.astype(np.float32), 1, v, u, K, L, M)
    return reg


def test_mi_filter_theta_draw_matches_oracle(core, oracle):
    from binder_b200 import phantoms
    from binder_b200.utils import bin_signal_robust, initialize_fourier_domain_smoothing
    shape, M, B, alpha = (12, 14, 10), 2, 8, 2.0
    pair = phantoms.make_pair(shape, 13, bins=B, n_objects=8, axes=(2.0, 5.0), rms=1.0,
                              spacing=3.0)
    v, _ = bin_signal_robust(pair.moving, B)
    v = np.append(v.astype(np.int32).ravel(), 3)
    u = np.append(pair.u.astype(np.int32).ravel(), 5)
    rng = np.random.default_rng(3)
    theta = rng.random((M, B, B)) + 0.1
    theta /= theta.sum(2, keepdims=True)
    grid = phantoms.identity_positions(shape)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3)
    reg = _registration(core, grid, grid, shape, D, (0.8, 0.6, 1.1), v, u, theta, alpha, order=1)
    seed = 4711
    reg.sampler(seed, 0, 2, 0, 1, 1, 1, 0)
    got = np.asarray(reg.get_likelihood_parameters(), np.float64)
    V = int(np.prod(shape))
    counts = np.zeros((M, B, B))
    for m in range(M):
        np.add.at(counts[m], (v[m:m + V], u[m:m + V]), 1.0)
    want, capped = oracle.dirichlet_sample(counts, M * B, B, alpha, seed, 1)
    assert capped == 0
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=1e-9)


def test_mi_filter_sampler_matches_reference_in_distribution(core):
    g = golden("sampler_mi_filter_ref.npz")
    shape = tuple(int(s) for s in g["shape"])
    V = int(np.prod(shape))
    grid = np.stack(np.indices(shape), -1).astype(np.float64)
    reg = _registration(core, g["d0"], grid, shape, g["D"], g["gamma"], g["v"], g["u"],
                        g["theta"], float(g["alpha"]))
    means, covs, pars = [], [], []
    for ch in range(int(g["chains"])):
        reg.reset()  # every chain starts from the given positions and theta
        reg.set_chain(ch)
        m, cv = reg.sampler(9000 + ch, int(g["N_b"]), int(g["N_s"]), 1, 1, 1, 1, 1)
        means.append(np.asarray(m, np.float64).reshape(V, 3))
        covs.append(np.asarray(cv, np.float64).reshape(V, 9)[:, UPPER])
        pars.append(np.asarray(reg.get_likelihood_parameters(), np.float64))
    m, c, p = np.asarray(means), np.asarray(covs), np.asarray(pars)
    C, Cr = len(m), int(g["chains"])
    zm = (m.mean(0) - g["mean_mean"]) / np.sqrt(m.var(0, ddof=1) / C + g["mean_var"] / Cr)
    zc = (c.mean(0) - g["cov_mean"]) / np.sqrt(c.var(0, ddof=1) / C + g["cov_var"] / Cr)
    assert agrees(zm), summary(zm)
    assert agrees(zc), summary(zc)
    zp = (p.mean(0) - g["params_mean"]) / np.sqrt(p.var(0, ddof=1) / C + g["params_var"] / Cr)
    assert agrees(zp), summary(zp)


# ---- the SSD filter likelihood (SSDLikelihoodFilter.cpp: M voxel channels, F node features) ----
def _ssdf_registration(core, d0, grid, shape, D, gamma, fn, fv, coeff, sigma, rfa, order=3):
    V = int(np.prod(shape))
    M, F = np.asarray(coeff).shape
    reg = core.Registration(d0.astype(np.float32), 1, grid.astype(np.float32),
                            grid.astype(np.float32), *shape, *shape, order, float(V))
    reg.setNonLinearTransformation(*[float(x) for x in gamma], 1, 1, 1, 1, 1, 1,
                                   D.astype(np.float32))
    reg.setSSDLikelihoodFilter(coeff, 1, sigma, fn if not rfa else fn[:, :M], fv, rfa, 1.0, 1.0,
                               M, F)
    return reg


def _ssdf_case(shape=(12, 14, 10), seed=17):
    from scipy import ndimage
    from binder_b200 import phantoms
    pair = phantoms.make_pair(shape, seed, bins=16, n_objects=8, axes=(2.0, 5.0), rms=1.0,
                              spacing=3.0)
    mv, fx = pair.moving.astype(np.float64), pair.fixed.astype(np.float64)
    fn = np.stack([mv, ndimage.gaussian_filter(mv, 1.0)], -1).reshape(-1, 2)
    fv = np.stack([fx, ndimage.gaussian_filter(fx, 1.0)], -1).reshape(-1, 2)
    return fn, fv


@pytest.mark.parametrize("rfa", [1, 0])
def test_ssd_filter_parameter_draw_matches_oracle(core, oracle, rfa):
    """order-1 splines at integer positions: every voxel draws its own node, so the sweep's
    accumulators are known; coefficients and sigmas after two sweeps against the oracle's
    restatement of sample_parameters applied twice"""
    from binder_b200 import phantoms
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape = (12, 14, 10)
    fn, fv = _ssdf_case(shape)
    grid = phantoms.identity_positions(shape)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3)
    coeff, sigma = np.eye(2), np.array([0.05, 0.08])
    reg = _ssdf_registration(core, grid, grid, shape, D, (0.8, 0.6, 1.1), fn, fv, coeff, sigma,
                             rfa, order=1)
    seed = 2024
    reg.sampler(seed, 0, 2, 0, 1, 1, 1, 0)
    got_c, got_s = reg.ssd_filter_parameters()
    V, M = int(np.prod(shape)), 2
    nodes = fn if not rfa else fn[:, :M]
    acc = (np.ones(V), np.ascontiguousarray(fv.T).ravel(),
           np.ascontiguousarray((fv * fv).T).ravel(), np.zeros(1 + 2 * M))
    p = oracle.ssdf_params(coeff, sigma, rfa, 1.0, 1.0)
    for sweep in range(2):
        assert oracle.ssdf_sample(p, nodes, shape, acc, seed, sweep) == 0
    want_c = np.array([p.coeff[q] for q in range(4)]).reshape(2, 2)
    want_s = np.array([p.sigma[m] for m in range(2)])
    np.testing.assert_allclose(got_s, want_s, rtol=1e-10)
    np.testing.assert_allclose(got_c, want_c, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("rfa", [1, 0])
def test_ssd_filter_sampler_matches_reference_in_distribution(core, rfa):
    g = golden("sampler_ssd_filter_ref.npz")
    shape = tuple(int(s) for s in g["shape"])
    V = int(np.prod(shape))
    grid = np.stack(np.indices(shape), -1).astype(np.float64)
    reg = _ssdf_registration(core, g["d0"], grid, shape, g["D"], g["gamma"], g["fn"], g["fv"],
                             g["coeff"], g["sigma"], rfa)
    means, covs, pars = [], [], []
    for ch in range(int(g["chains"])):
        reg.reset()
        reg.set_chain(ch)
        m, cv = reg.sampler(9000 + ch, int(g["N_b"]), int(g["N_s"]), 1, 1, 1, 1, 1)
        means.append(np.asarray(m, np.float64).reshape(V, 3))
        covs.append(np.asarray(cv, np.float64).reshape(V, 9)[:, UPPER])
        pars.append(reg.ssd_filter_parameters()[0].ravel())
    m, c, p = np.asarray(means), np.asarray(covs), np.asarray(pars)
    C, Cr = len(m), int(g["chains"])
    k = f"r{rfa}_"
    zm = (m.mean(0) - g[k + "mean_mean"]) / np.sqrt(m.var(0, ddof=1) / C + g[k + "mean_var"] / Cr)
    zc = (c.mean(0) - g[k + "cov_mean"]) / np.sqrt(c.var(0, ddof=1) / C + g[k + "cov_var"] / Cr)
    assert agrees(zm), summary(zm)
    assert agrees(zc), summary(zc)
    if not rfa:
        zp = (p.mean(0) - g[k + "params_mean"]) / np.sqrt(p.var(0, ddof=1) / C +
                                                          g[k + "params_var"] / Cr)
        assert np.all(np.abs(zp) < 4.5), zp
