"""The GPU sampler against the reference's own Registration::sampler in distribution: 32 GPU chains
from the same positions and theta as the 32 reference chains in tests/golden/sampler_ref.npz,
every sampling switch on.  Chain means and covariances agree within Monte Carlo error (the
z-score bounds of tests/sampler_stats.py)."""
import numpy as np
import pytest

from sampler_stats import UPPER, agrees, fixture, summary, zscores

pytestmark = pytest.mark.gpu


def gpu_chains(core, g, chains=32, seed0=9000):
    shape = tuple(int(s) for s in g["shape"])
    V = int(np.prod(shape))
    K, L = int(g["K"]), int(g["L"])
    grid = np.stack(np.indices(shape), -1).astype(np.float32)
    reg = core.Registration(g["d0"].astype(np.float32), 1, grid, grid, *shape, *shape, 3, float(V))
    reg.setNonLinearTransformation(*[float(x) for x in g["gamma"]], 1, 1, 1, 1, 1, 1,
                                   g["D"].astype(np.float32))
    reg.setMILikelihood(float(g["alpha"]), g["theta"].astype(np.float32), K, L, 1, g["v"], g["u"])
    means, covs = [], []
    for ch in range(chains):
        reg.reset()  # every chain starts from the given positions and theta
        reg.set_chain(ch)
        m, cv = reg.sampler(seed0 + ch, int(g["N_b"]), int(g["N_s"]), 1, 1, 1, 1, 1)
        means.append(np.asarray(m, np.float64).reshape(V, 3))
        covs.append(np.asarray(cv, np.float64).reshape(V, 9)[:, UPPER])
    return means, covs


def test_gpu_sampler_matches_reference_in_distribution(core):
    g = fixture()
    zm, zc = zscores(g, *gpu_chains(core, g))
    assert agrees(zm), summary(zm)
    assert agrees(zc), summary(zc)


def test_gpu_chain_batch_matches_reference_in_distribution(core):
    """The same check with the 32 chains run as one batch (sampler_chains)."""
    g = fixture()
    shape = tuple(int(s) for s in g["shape"])
    V = int(np.prod(shape))
    K, L = int(g["K"]), int(g["L"])
    grid = np.stack(np.indices(shape), -1).astype(np.float32)
    reg = core.Registration(g["d0"].astype(np.float32), 1, grid, grid, *shape, *shape, 3, float(V))
    reg.setNonLinearTransformation(*[float(x) for x in g["gamma"]], 1, 1, 1, 1, 1, 1,
                                   g["D"].astype(np.float32))
    reg.setMILikelihood(float(g["alpha"]), g["theta"].astype(np.float32), K, L, 1, g["v"], g["u"])
    means, covs = reg.sampler_chains(4242, 32, int(g["N_b"]), int(g["N_s"]), 1, 1, 1, 1, 1,
                                     pooled=False)
    zm, zc = zscores(g, means.reshape(32, V, 3), covs.reshape(32, V, 9)[:, :, UPPER])
    assert agrees(zm), summary(zm)
    assert agrees(zc), summary(zc)
