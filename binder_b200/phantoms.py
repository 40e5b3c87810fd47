"""Seeded synthetic image pairs standing in for the benchmark datasets (none are public).

Fixed image: a sum of random ellipsoids (ellipses in 2D) with uniform intensities, Gaussian blur
and additive noise.  Moving image: the fixed image warped by a smooth random field drawn from the
DCT-domain prior's spectrum (correlation length set by `spacing`, scaled to a target RMS
displacement), then passed through a random monotone intensity LUT.  Both are binned with the
reference's robust binning.  Everything is numpy/scipy on the host and fully determined by `seed`.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy import fft as sfft
from scipy import ndimage

from .utils import bin_signal_robust, initialize_fourier_domain_smoothing


@dataclass
class Pair:
    fixed: np.ndarray
    moving: np.ndarray
    field: np.ndarray          # true displacement used to make `moving` [*shape, ndim]
    u: np.ndarray              # fixed bins (int32)
    v: np.ndarray              # moving bins (int32)
    bins: int


def ellipsoid_phantom(shape, n_objects, axes, blur, noise, rng):
    shape = tuple(int(s) for s in shape)
    grids = np.meshgrid(*[np.arange(s, dtype=np.float32) for s in shape], indexing="ij")
    img = np.zeros(shape, np.float32)
    for _ in range(n_objects):
        c = [rng.uniform(0, s) for s in shape]
        a = [rng.uniform(axes[0], axes[1]) for _ in shape]
        val = rng.uniform(0.0, 1.0)
        r = sum(((g - ci) / ai) ** 2 for g, ci, ai in zip(grids, c, a))
        img[r <= 1.0] += val
    if blur > 0:
        img = ndimage.gaussian_filter(img, blur)
    img = img + rng.normal(0.0, noise, shape).astype(np.float32)
    return img.astype(np.float32)


def smooth_random_field(shape, rms, spacing, rng):
    """Displacement field [*shape, ndim] from the DCT prior's spectrum: coefficients N(0,1) scaled
    by 1/(1 + (spacing/pi)^4 D) with second-order D, transformed back and scaled to `rms`."""
    shape = tuple(int(s) for s in shape)
    nd = len(shape)
    D = initialize_fourier_domain_smoothing(shape, True, 2, nd)
    filt = 1.0 / (1.0 + (spacing / np.pi) ** 4 * D)
    comps = []
    for _ in range(nd):
        c = rng.standard_normal(shape) * filt
        comps.append(sfft.idctn(c, norm="ortho"))
    f = np.stack(comps, axis=-1)
    cur = np.sqrt(np.mean(np.sum(f ** 2, axis=-1)))
    return (f * (rms / max(cur, 1e-12))).astype(np.float32)


def monotone_lut(img, knots, rng):
    lo, hi = float(img.min()), float(img.max())
    xs = np.linspace(lo, hi, knots)
    ys = np.sort(rng.uniform(0.0, 1.0, knots))
    ys[0], ys[-1] = 0.0, 1.0
    return np.interp(img, xs, ys).astype(np.float32)


def make_pair(shape, seed, bins=64, n_objects=None, axes=None, blur=None, noise=0.02,
              rms=3.0, spacing=5.0, knots=8) -> Pair:
    shape = tuple(int(s) for s in shape)
    rng = np.random.default_rng(seed)
    nd = len(shape)
    if n_objects is None:
        n_objects = 12 if nd == 2 else 40
    if axes is None:
        axes = (5.0, 40.0) if nd == 2 else (4.0, 50.0)
    if blur is None:
        blur = 1.5 if nd == 2 else 1.0
    fixed = ellipsoid_phantom(shape, n_objects, axes, blur, noise, rng)
    field = smooth_random_field(shape, rms, spacing, rng)
    grid = np.meshgrid(*[np.arange(s, dtype=np.float32) for s in shape], indexing="ij")
    coords = [g + field[..., a] for a, g in enumerate(grid)]
    warped = ndimage.map_coordinates(fixed, coords, order=1, mode="nearest").astype(np.float32)
    moving = monotone_lut(warped, knots, rng)
    u, _ = bin_signal_robust(fixed, bins)
    v, _ = bin_signal_robust(moving, bins)
    return Pair(fixed, moving, field, u.astype(np.int32), v.astype(np.int32), bins)


def identity_positions(shape):
    """Voxel positions in node-grid coordinates for same-geometry images: [*shape, ndim]."""
    return np.stack(np.indices(shape, dtype=np.float64), axis=-1)
