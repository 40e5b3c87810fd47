"""Parity in distribution of a sampler against the reference's chain statistics
(tests/golden/sampler_ref.npz, written by tests/golden/make_sampler_golden.py).

z = (across-chain mean here - the reference's) / sqrt(var_here / C_here + var_ref / C_ref) per
voxel and component, for the chain means and for the upper-triangle chain covariances.  For
samplers with the same kernel z is close to Student-t with ~60 degrees of freedom: E[z^2] ~ 1.03
and |z| > 4.5 at about 1e-5 per entry (neighbouring voxels are correlated, so the test bounds the
average and the tail loosely).
"""
import numpy as np

from conftest import golden

UPPER = [0, 1, 2, 4, 5, 8]  # xx, xy, xz, yy, yz, zz of a row-major 3x3
MEAN_Z2_MAX = 1.5
TAIL_Z, TAIL_FRAC = 4.5, 0.005


def fixture():
    g = golden("sampler_ref.npz")
    return {k: g[k] for k in g.files}


def zscores(g, means, covs):
    """means [C, V, 3], covs [C, V, 6] of C chains here -> (z of the means, z of the covs)"""
    m, c = np.asarray(means), np.asarray(covs)
    C, Cr = len(m), int(g["chains"])
    zm = (m.mean(0) - g["mean_mean"]) / np.sqrt(m.var(0, ddof=1) / C + g["mean_var"] / Cr)
    zc = (c.mean(0) - g["cov_mean"]) / np.sqrt(c.var(0, ddof=1) / C + g["cov_var"] / Cr)
    return zm, zc


def summary(z):
    return float(np.mean(z ** 2)), float(np.mean(np.abs(z) > TAIL_Z))


def agrees(z):
    z2, tail = summary(z)
    return z2 < MEAN_Z2_MAX and tail < TAIL_FRAC
