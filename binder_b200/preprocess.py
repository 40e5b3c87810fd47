"""The registration driver's preprocessing and output steps on the GPU.

``FastRegistration`` (BINDER/FastRegistration.py) bins both images with ``utils.bin_signal_robust``
(or ``utils.bin_signal``), may shift the voxel positions by the difference of the two masks'
centres of mass, and ``utils.save_warped_image`` resamples the moving image through the final
positions.  These run here on the device with the same arithmetic; the arrays may be numpy
arrays of any shape (flattened in C order).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._core import _out
from ._lib import check, lib


def _signal(signal):
    a = np.asarray(signal)
    if a.dtype == np.float32:
        return np.ascontiguousarray(a), 0
    return np.ascontiguousarray(a, dtype=np.float64), 1


def bin_signal_robust(signal, number_of_bins, lower_percentile=0.01, higher_percentile=0.99):
    """``utils.bin_signal_robust`` (BINDER/utils.py:20-82) without ``intensity_bins``: returns
    (binned int32 array of the signal's shape, bin edges).  float32 signals are binned in
    float32 and every other dtype in float64, as numpy computes it."""
    a, is_double = _signal(signal)
    binned = np.empty(a.shape, np.int32)
    edges = np.empty(int(number_of_bins) + 1, np.float64)
    check(lib().binder_bin_signal_robust(a.ctypes.data, is_double, a.size, int(number_of_bins),
                                         float(lower_percentile), float(higher_percentile),
                                         binned.ctypes.data, edges.ctypes.data))
    return binned, edges.astype(a.dtype)


def bin_signal(signal, number_of_bins):
    """``utils.bin_signal`` (BINDER/utils.py:12-17)."""
    a, is_double = _signal(signal)
    binned = np.empty(a.shape, np.int32)
    check(lib().binder_bin_signal(a.ctypes.data, is_double, a.size, int(number_of_bins),
                                  binned.ctypes.data))
    return binned


def center_of_mass_nonzero(bins):
    """``scipy.ndimage.center_of_mass(bins > 0)`` of a 2-D or 3-D bin volume (index space)."""
    b = np.ascontiguousarray(bins, dtype=np.int32)
    shape = b.shape + (1,) * (3 - b.ndim)
    out = np.zeros(3, np.float64)
    check(lib().binder_center_of_mass(b.reshape(-1), *shape, out))
    return out[:b.ndim]


def warp_image(moving_image, deformed_position, order=1):
    """The resampling of ``utils.save_warped_image`` (BINDER/utils.py:222-227): the moving image
    sampled at the deformed positions [..., 3] (index space), order 0, 1 or 3, zero outside,
    clipped as skimage clips.  Returns an array of the positions' spatial shape."""
    im = np.ascontiguousarray(moving_image, dtype=np.float64)
    pos = np.ascontiguousarray(deformed_position, dtype=np.float64)
    if im.ndim != 3 or pos.shape[-1] != 3:
        raise ValueError("moving_image must be 3-D and deformed_position [..., 3]")
    M = pos.size // 3
    out = _out(M, np.float64)
    check(lib().binder_warp_image(im.reshape(-1), *im.shape, pos.reshape(-1), M, int(order), out))
    return out.reshape(pos.shape[:-1])
