"""The sampler with the SSD likelihood (Registration.cpp:515-642 driving SSDLikelihood.cpp).

1. The parameter draw against the oracle: with order-1 splines at integer positions every
   voxel's categorical draw is its own node (one non-zero weight), so the sweep's counts are the
   joint histogram of (node bin, voxel bin) at the identity, and the drawn sigma^2, shift and
   scale after two sweeps must equal the oracle's restatement (oracle/binder_oracle.c
   orc_ssd_sample, Philox-driven) applied twice to those counts, to FP64 accuracy.
2. The whole sampler against the reference's own Registration::sampler with the SSD likelihood
   in distribution: 32 GPU chains from the positions of tests/golden/sampler_ssd_ref.npz (32
   reference chains, every switch on) agree in their chain means, covariances and final
   (scale, shift) within Monte Carlo error (the z-score bounds of tests/sampler_stats.py)."""
import numpy as np
import pytest

from conftest import golden
from sampler_stats import UPPER, agrees, summary

pytestmark = pytest.mark.gpu


def _registration(core, d0, grid, shape, D, gamma, v, u, bins, ssd, order=3):
    V = int(np.prod(shape))
    reg = core.Registration(d0.astype(np.float32), 1, grid.astype(np.float32),
                            grid.astype(np.float32), *shape, *shape, order, float(V))
    reg.setNonLinearTransformation(*[float(x) for x in gamma], 1, 1, 1, 1, 1, 1,
                                   D.astype(np.float32))
    sigma2, shift_scale, scale, shift, a0, b0 = ssd
    reg.setSSDLikelihood(bins, 1, sigma2, int(shift_scale), scale, shift, v, u, a0, b0)
    return reg


@pytest.mark.parametrize("shift_scale", [0, 1])
def test_ssd_parameter_draw_matches_oracle(core, oracle, shift_scale):
    from binder_b200 import phantoms
    from binder_b200.utils import bin_signal_robust, initialize_fourier_domain_smoothing
    shape, bins = (12, 14, 10), 16
    pair = phantoms.make_pair(shape, 11, bins=bins, n_objects=8, axes=(2.0, 5.0), rms=1.0,
                              spacing=3.0)
    v, _ = bin_signal_robust(pair.moving, bins)
    v, u = v.astype(np.int32), pair.u.astype(np.int32)
    grid = phantoms.identity_positions(shape)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3)
    ssd = (4.0, shift_scale, 1.0, 0.0, 1.0, 1.0)
    reg = _registration(core, grid, grid, shape, D, (0.8, 0.6, 1.1), v, u, bins, ssd, order=1)
    seed = 31337
    reg.sampler(seed, 0, 2, 0, 1, 1, 1, 0)
    got = reg.ssd_parameters()
    counts = np.zeros((bins, bins))
    np.add.at(counts, (v.ravel(), u.ravel()), 1.0)
    p = oracle.SSDParams(shift_scale, 4.0, 0.0, 1.0, 1.0, 1.0)
    for sweep in range(2):
        assert oracle.ssd_sample(counts, bins, bins, p, seed, sweep) == 0
    assert got["sigma_sq"] == pytest.approx(p.sigma2, rel=1e-12)
    assert got["shift"] == pytest.approx(p.shift, rel=1e-12, abs=1e-12)
    assert got["scale"] == pytest.approx(p.scale, rel=1e-12)
    if shift_scale:
        assert got["scale"] != 1.0 and got["shift"] != 0.0  # the draw moved them


def test_ssd_sampler_matches_reference_in_distribution(core):
    g = golden("sampler_ssd_ref.npz")
    shape = tuple(int(s) for s in g["shape"])
    V = int(np.prod(shape))
    bins = int(g["bins"])
    grid = np.stack(np.indices(shape), -1).astype(np.float64)
    reg = _registration(core, g["d0"], grid, shape, g["D"], g["gamma"], g["v"], g["u"], bins,
                        tuple(g["ssd"]))
    means, covs, pars = [], [], []
    for ch in range(int(g["chains"])):
        reg.reset()  # every chain starts from the given positions and parameters
        reg.set_chain(ch)
        m, cv = reg.sampler(9000 + ch, int(g["N_b"]), int(g["N_s"]), 1, 1, 1, 1, 1)
        means.append(np.asarray(m, np.float64).reshape(V, 3))
        covs.append(np.asarray(cv, np.float64).reshape(V, 9)[:, UPPER])
        scale, shift = reg.get_likelihood_parameters()
        pars.append((scale, shift))
    m, c, p = np.asarray(means), np.asarray(covs), np.asarray(pars, np.float64)
    C, Cr = len(m), int(g["chains"])
    zm = (m.mean(0) - g["mean_mean"]) / np.sqrt(m.var(0, ddof=1) / C + g["mean_var"] / Cr)
    zc = (c.mean(0) - g["cov_mean"]) / np.sqrt(c.var(0, ddof=1) / C + g["cov_var"] / Cr)
    assert agrees(zm), summary(zm)
    assert agrees(zc), summary(zc)
    zp = (p.mean(0) - g["params_mean"]) / np.sqrt(p.var(0, ddof=1) / C + g["params_var"] / Cr)
    assert np.all(np.abs(zp) < 4.5), zp
