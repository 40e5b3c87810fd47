"""Host-side helpers that produce the engine's inputs, restated from the reference's Python layer.

``initialize_fourier_domain_smoothing`` builds the per-coefficient eigenvalues D of the DCT-domain
prior (BINDER/utils.py:270-365) and ``bin_signal_robust`` the integer intensity bins
(BINDER/utils.py:20-82); ``bin_signal`` is BINDER/utils.py:12-16.
"""
from __future__ import annotations

import numpy as np


def initialize_fourier_domain_smoothing(size, DCT=True, finite_difference_order=2,
                                        number_of_dimensions=3, return_full_matrix=False,
                                        voxel_size=np.ones(3)):
    """Eigenvalues of the finite-difference penalty: D[k] = (sum_a (2 - 2cos(pi k_a / N_a)) / h_a^2)
    ** order for the DCT, or the periodic (2 pi k_a / N_a) version for the FFT half-spectrum."""
    size = [int(s) for s in size][:number_of_dimensions]
    vs = np.asarray(voxel_size, dtype=np.float64)
    order = finite_difference_order

    def term(k, n, h, dct):
        ang = (np.pi if dct else 2.0 * np.pi) * k / n
        return (2.0 - 2.0 * np.cos(ang)) / h ** 2

    if DCT:
        ranges = [np.arange(2 * n if return_full_matrix else n) for n in size]
        grids = np.meshgrid(*ranges, indexing="ij")
        D = sum(term(g, n, vs[a], True) for a, (g, n) in enumerate(zip(grids, size)))
        D = D ** order
        crop = D[tuple(slice(0, n) for n in size)]
        return (crop, D) if return_full_matrix else crop
    grids = np.meshgrid(*[np.arange(n) for n in size], indexing="ij")
    D = sum(term(g, n, vs[a], False) for a, (g, n) in enumerate(zip(grids, size))) ** order
    half = D.shape[number_of_dimensions - 1] // 2 + 1
    crop = D[..., :half]
    return (crop, D) if return_full_matrix else crop


def bin_signal(signal, number_of_bins):
    lo, hi = np.min(signal), np.max(signal)
    width = (hi - lo) / (number_of_bins - 1)
    return np.round((signal - lo) / width).astype(np.int32)


def bin_signal_robust(signal, number_of_bins, lower_percentile=0.01, higher_percentile=0.99,
                      intensity_bins=None):
    """Floor-bin the signal between robust percentiles taken from a 1000-bin histogram; values
    below / above the range go to the first / last bin.  Returns (bins int32, bin_edges)."""
    signal = np.asarray(signal)
    if intensity_bins is not None:
        edges = np.asarray(intensity_bins)
        b = np.digitize(signal, edges).astype(np.int32) - 1
        b[signal <= edges[0]] = 0
        b[signal >= edges[-1]] = number_of_bins - 1
        return b, edges
    hist, edges = np.histogram(signal, 1000)
    cdf = np.cumsum(hist / np.sum(hist))

    def robust(p):
        add = 0.0
        while True:
            idx = np.where(cdf <= p + add)[0]
            if idx.size:
                return edges[idx[-1]]
            add += 0.01

    lo, hi = robust(lower_percentile), robust(higher_percentile)
    width = (hi - lo) / (number_of_bins - 1)
    out_edges = np.linspace(lo, hi, number_of_bins + 1)
    b = np.floor((signal - lo) / width).astype(np.int32)
    b[signal < lo] = 0
    b[signal > hi] = number_of_bins - 1
    return b, out_edges
