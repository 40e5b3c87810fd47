"""Fixture for the sampler's parity in distribution: the reference's own Registration::sampler
(BINDER/src/cpu/Registration.cpp:515-642, compiled unmodified in oracle/_ref) run as 32 independent
chains from the same positions and theta, every sampling switch on.

Draws cannot match draw for draw (the reference uses std::mt19937 streams, this project Philox), so
the fixture holds per-voxel chain statistics: the mean over chains of each chain's sampler mean
and covariance, and their variance over chains.  A sampler whose chains follow the same Markov
kernel from the same start has the same expected chain mean and covariance whatever its random
numbers, so the difference of the two across-chain means divided by its standard error is a
z-score per voxel (tests/test_oracle.py and tests/test_gpu_sampler_reference.py).

Run from the repository root:  python tests/golden/make_sampler_golden.py        (MI)
                               python tests/golden/make_sampler_golden.py ssd    (SSD)
                               python tests/golden/make_sampler_golden.py mi_filter
                               python tests/golden/make_sampler_golden.py ssd_filter
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from binder_b200 import phantoms  # noqa: E402
from binder_b200.utils import bin_signal_robust, initialize_fourier_domain_smoothing  # noqa: E402
from oracle import pyoracle  # noqa: E402

SHAPE, K, L = (12, 14, 10), 16, 12
CHAINS, N_B, N_S = 32, 20, 200
SEED0 = 1000
UPPER = [0, 1, 2, 4, 5, 8]  # xx, xy, xz, yy, yz, zz of a row-major 3x3


def case():
    rng = np.random.default_rng(20261204)
    pair = phantoms.make_pair(SHAPE, 7, bins=L, n_objects=10, axes=(2.0, 6.0), rms=1.0,
                              spacing=3.0)
    v, _ = bin_signal_robust(pair.moving, K)
    grid = phantoms.identity_positions(SHAPE)
    d0 = grid + phantoms.smooth_random_field(SHAPE, 0.6, 3.0, rng)
    theta = rng.random((K, L)) + 0.05
    theta /= theta.sum(1, keepdims=True)
    D = initialize_fourier_domain_smoothing(SHAPE, True, 2, 3)
    return dict(d0=d0, grid=grid, u=pair.u.astype(np.int32), v=v.astype(np.int32), theta=theta,
                D=D, gamma=np.array([0.8, 0.6, 1.1]))


def chain_stats(means, covs):
    """per-voxel mean over chains and variance over chains (ddof 1) of the chain means [C, V, 3]
    and of the upper-triangle covariances [C, V, 6]"""
    m, c = np.asarray(means), np.asarray(covs)
    return m.mean(0), m.var(0, ddof=1), c.mean(0), c.var(0, ddof=1)


def main():
    R = pyoracle.ref_lib()
    assert R is not None, "oracle/_ref/libbinder_ref.so is needed (make -C oracle)"
    c = case()
    V = int(np.prod(SHAPE))
    means, covs = [], []
    # the reference prints every sweep on stdout
    saved = os.dup(1)
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    try:
        for ch in range(CHAINS):
            m, cv, _ = pyoracle.ref_sampler(R, c["d0"], c["grid"], c["D"], c["gamma"], SHAPE,
                                            c["v"], c["u"], 2.0, c["theta"], SEED0 + ch, N_B, N_S)
            means.append(m.reshape(V, 3))
            covs.append(cv.reshape(V, 9)[:, UPPER])
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    mm, mv, cm, cvv = chain_stats(means, covs)
    np.savez_compressed(os.path.join(HERE, "sampler_ref.npz"), shape=np.array(SHAPE), K=K, L=L,
                        chains=CHAINS, N_b=N_B, N_s=N_S, alpha=2.0, d0=c["d0"], u=c["u"],
                        v=c["v"], theta=c["theta"], D=c["D"], gamma=c["gamma"], mean_mean=mm,
                        mean_var=mv, cov_mean=cm, cov_var=cvv)
    print("sampler_ref.npz:", CHAINS, "chains of", N_B + N_S, "sweeps on", SHAPE)


# the SSD likelihood's case: the same positions, prior and field as case(), both images in 16
# intensity bins (the SSD likelihood compares bin values), (sigmaSq, shiftScale, scale, shift,
# alpha_0, beta_0) = (4, 1, 1, 0, 1, 1) (run_BINDER's alpha_0 = beta_0 = 1)
SSD_BINS = 16
SSD_PARAMS = (4.0, 1, 1.0, 0.0, 1.0, 1.0)


def case_ssd():
    c = case()
    pair = phantoms.make_pair(SHAPE, 7, bins=SSD_BINS, n_objects=10, axes=(2.0, 6.0), rms=1.0,
                              spacing=3.0)
    v, _ = bin_signal_robust(pair.moving, SSD_BINS)
    c.update(u=pair.u.astype(np.int32), v=v.astype(np.int32))
    return c


def main_ssd():
    """sampler_ssd_ref.npz: the reference's sampler with the SSD likelihood (SSDLikelihood.cpp:
    147-300), 32 chains from case_ssd(), every switch on; also each chain's final (scale, shift)"""
    R = pyoracle.ref_lib()
    assert R is not None, "oracle/_ref/libbinder_ref.so is needed (make -C oracle)"
    c = case_ssd()
    V = int(np.prod(SHAPE))
    means, covs, pars = [], [], []
    saved = os.dup(1)
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    try:
        for ch in range(CHAINS):
            m, cv, par, _ = pyoracle.ref_sampler_ssd(R, c["d0"], c["grid"], c["D"], c["gamma"],
                                                     SHAPE, c["v"], c["u"], SSD_BINS, SSD_PARAMS,
                                                     SEED0 + ch, N_B, N_S)
            means.append(m.reshape(V, 3))
            covs.append(cv.reshape(V, 9)[:, UPPER])
            pars.append(par)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    mm, mv, cm, cvv = chain_stats(means, covs)
    pars = np.asarray(pars)
    np.savez_compressed(os.path.join(HERE, "sampler_ssd_ref.npz"), shape=np.array(SHAPE),
                        bins=SSD_BINS, ssd=np.array(SSD_PARAMS), chains=CHAINS, N_b=N_B, N_s=N_S,
                        d0=c["d0"], u=c["u"], v=c["v"], D=c["D"], gamma=c["gamma"],
                        mean_mean=mm, mean_var=mv, cov_mean=cm, cov_var=cvv,
                        params_mean=pars.mean(0), params_var=pars.var(0, ddof=1))
    print("sampler_ssd_ref.npz:", CHAINS, "chains of", N_B + N_S, "sweeps on", SHAPE)


# the MI filter likelihood's case: M = 2 channels of 8 bins, channel m of voxel (node) i read
# at [i + m] (MILikelihoodFilter.cpp:46-68), one bin array each with one extra entry
FILTER_M, FILTER_BINS = 2, 8


def case_mi_filter():
    c = case()
    rng = np.random.default_rng(20261205)
    pair = phantoms.make_pair(SHAPE, 7, bins=FILTER_BINS, n_objects=10, axes=(2.0, 6.0),
                              rms=1.0, spacing=3.0)
    v, _ = bin_signal_robust(pair.moving, FILTER_BINS)
    c["v"] = np.append(v.astype(np.int32).ravel(), 0)
    c["u"] = np.append(pair.u.astype(np.int32).ravel(), 0)
    theta = rng.random((FILTER_M, FILTER_BINS, FILTER_BINS)) + 0.05
    c["theta"] = theta / theta.sum(2, keepdims=True)
    return c


def main_mi_filter():
    """sampler_mi_filter_ref.npz: the reference's sampler with the MI filter likelihood
    (MILikelihoodFilter.cpp:102-175), 32 chains from case_mi_filter(), every switch on; also
    each chain's final theta"""
    R = pyoracle.ref_lib()
    assert R is not None, "oracle/_ref/libbinder_ref.so is needed (make -C oracle)"
    c = case_mi_filter()
    V = int(np.prod(SHAPE))
    means, covs, pars = [], [], []
    saved = os.dup(1)
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    try:
        for ch in range(CHAINS):
            m, cv, par = pyoracle.ref_sampler_filter(
                R, c["d0"], c["grid"], c["D"], c["gamma"], SHAPE, SEED0 + ch, N_B, N_S,
                mi=(2.0, c["theta"], c["v"], c["u"]))
            means.append(m.reshape(V, 3))
            covs.append(cv.reshape(V, 9)[:, UPPER])
            pars.append(par)
    finally:
        os.dup2(saved, 1)
        os.close(saved)
    mm, mv, cm, cvv = chain_stats(means, covs)
    pars = np.asarray(pars)
    np.savez_compressed(os.path.join(HERE, "sampler_mi_filter_ref.npz"), shape=np.array(SHAPE),
                        M=FILTER_M, K=FILTER_BINS, L=FILTER_BINS, alpha=2.0, chains=CHAINS,
                        N_b=N_B, N_s=N_S, d0=c["d0"], u=c["u"], v=c["v"], theta=c["theta"],
                        D=c["D"], gamma=c["gamma"], mean_mean=mm, mean_var=mv, cov_mean=cm,
                        cov_var=cvv, params_mean=pars.mean(0), params_var=pars.var(0, ddof=1))
    print("sampler_mi_filter_ref.npz:", CHAINS, "chains of", N_B + N_S, "sweeps on", SHAPE)


def case_ssd_filter():
    """the SSD filter likelihood's case: F = 2 node features (the moving image and its Gaussian
    smoothing, sigma 1) and M = 2 voxel channels (the same of the fixed image), identity
    coefficients, sigma 0.05 per channel, alpha_0 = beta_0 = 1"""
    from scipy import ndimage
    c = case()
    pair = phantoms.make_pair(SHAPE, 7, bins=16, n_objects=10, axes=(2.0, 6.0), rms=1.0,
                              spacing=3.0)
    mv, fx = pair.moving.astype(np.float64), pair.fixed.astype(np.float64)
    c["fn"] = np.stack([mv, ndimage.gaussian_filter(mv, 1.0)], -1).reshape(-1, 2)
    c["fv"] = np.stack([fx, ndimage.gaussian_filter(fx, 1.0)], -1).reshape(-1, 2)
    c["coeff"] = np.eye(2)
    c["sigma"] = np.array([0.05, 0.05])
    return c


def main_ssd_filter():
    """sampler_ssd_filter_ref.npz: the reference's sampler with the SSD filter likelihood
    (SSDLikelihoodFilter.cpp:168-463), 32 chains each with reg_across_features 1 (sigma drawn)
    and 0 (coefficients drawn too), every switch on; also each chain's final coefficients"""
    R = pyoracle.ref_lib()
    assert R is not None, "oracle/_ref/libbinder_ref.so is needed (make -C oracle)"
    c = case_ssd_filter()
    V = int(np.prod(SHAPE))
    out = dict(shape=np.array(SHAPE), chains=CHAINS, N_b=N_B, N_s=N_S, d0=c["d0"], fn=c["fn"],
               fv=c["fv"], coeff=c["coeff"], sigma=c["sigma"], D=c["D"], gamma=c["gamma"])
    for rfa in (1, 0):
        means, covs, pars = [], [], []
        saved = os.dup(1)
        os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
        try:
            for ch in range(CHAINS):
                m, cv, par = pyoracle.ref_sampler_filter(
                    R, c["d0"], c["grid"], c["D"], c["gamma"], SHAPE, SEED0 + ch, N_B, N_S,
                    ssd=(c["coeff"], c["sigma"], c["fn"], c["fv"], rfa, 1.0, 1.0))
                means.append(m.reshape(V, 3))
                covs.append(cv.reshape(V, 9)[:, UPPER])
                pars.append(par)
        finally:
            os.dup2(saved, 1)
            os.close(saved)
        mm, mv, cm, cvv = chain_stats(means, covs)
        pars = np.asarray(pars)
        out.update({f"r{rfa}_mean_mean": mm, f"r{rfa}_mean_var": mv, f"r{rfa}_cov_mean": cm,
                    f"r{rfa}_cov_var": cvv, f"r{rfa}_params_mean": pars.mean(0),
                    f"r{rfa}_params_var": pars.var(0, ddof=1)})
    np.savez_compressed(os.path.join(HERE, "sampler_ssd_filter_ref.npz"), **out)
    print("sampler_ssd_filter_ref.npz: 2 x", CHAINS, "chains of", N_B + N_S, "sweeps on", SHAPE)


if __name__ == "__main__":
    # no argument: the MI fixture; "ssd" / "mi_filter" / "ssd_filter": the other likelihoods'
    {"ssd": main_ssd, "mi_filter": main_mi_filter,
     "ssd_filter": main_ssd_filter}.get((sys.argv[1:] or [""])[0], main)()
