"""Edge cases of the GPU path against the FP64 oracle: ragged grid sizes (partial tiles, axis lengths
that are not multiples of 4 or 16), the general E-step kernel (K > 64 bins), the smallest bin
counts, positions that are not finite or lie far outside the node grid, and a 1-voxel-thin axis."""
import math

import numpy as np
import pytest

from test_gpu_parity import make_case, new_reg

pytestmark = pytest.mark.gpu

SIGMA = math.sqrt(9.0 / (8.0 * math.pi))


def one_iteration(core, oracle, c, positions=None, atol_dream=5e-5, atol_final=2e-4):
    shape, K, L = c["shape"], c["K"], c["L"]
    d = c["d0"] if positions is None else positions
    reg = new_reg(core, c, d)
    assert reg.EM(1, -1e30, 1, 0) == 1
    mll, dream, hist, deg = oracle.estep(np.asarray(d, np.float64), c["u"], c["v"],
                                         c["theta"].astype(np.float64), shape, shape, K, L)
    theta = oracle.theta_map(hist, K, L, 2.0)
    _, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA, shape)
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=atol_dream)
    np.testing.assert_allclose(reg.get_likelihood_parameters(), theta, rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=atol_final)
    assert reg.iteration_stats()[0][0] == pytest.approx(mll, rel=1e-6)
    return reg, deg


@pytest.mark.parametrize("shape", [(7, 5, 9), (17, 3, 33), (130, 6, 5), (2, 2, 2)])
def test_ragged_grids_match_oracle(core, oracle, shape):
    c = make_case(shape=shape, K=8, L=6, seed=sum(shape))
    _, deg = one_iteration(core, oracle, c)
    assert deg == 0


@pytest.mark.parametrize("K,L", [(96, 40), (200, 64)])
def test_many_bins_general_kernel(core, oracle, K, L):
    """K > 64 takes the general E-step kernel (theta and histogram in shared memory, one
    atomic per neighbour)."""
    c = make_case(shape=(12, 10, 14), K=K, L=L, seed=K)
    one_iteration(core, oracle, c)


def test_two_bins(core, oracle):
    c = make_case(shape=(9, 8, 7), K=2, L=2, seed=2)
    one_iteration(core, oracle, c)


def test_degenerate_positions(core, oracle):
    """Non-finite positions and positions far outside the grid keep their place and count as
    degenerate; every other voxel is unaffected."""
    c = make_case(shape=(10, 9, 8), seed=5)
    d = c["d0"].copy()
    d[0, 0, 0] = (np.nan, 1.0, 1.0)
    d[1, 2, 3] = (np.inf, 0.0, 0.0)
    d[4, 4, 4] = (2e6, 3.0, 3.0)
    reg = new_reg(core, c, d)
    reg.EM(1, -1e30, 1, 0)
    assert reg.state()["degenerate"] == 3
    ok = np.ones(c["shape"], bool)
    ok[0, 0, 0] = ok[1, 2, 3] = ok[4, 4, 4] = False
    clean = c["d0"].astype(np.float64)
    _, dream, _, _ = oracle.estep(clean, c["u"], c["v"], c["theta"].astype(np.float64),
                                  c["shape"], c["shape"], c["K"], c["L"])
    got = reg.get_dream_locations().reshape(c["shape"] + (3,))
    np.testing.assert_allclose(got[ok], dream.reshape(c["shape"] + (3,))[ok], rtol=0, atol=5e-5)


def test_far_outside_uses_bin_zero(core, oracle):
    """A voxel 5 nodes outside the grid sees only nodes with bin 0 (MILikelihood.cpp:46-48); its
    posterior follows theta[0] and the oracle agrees."""
    c = make_case(shape=(10, 9, 8), seed=6)
    d = c["d0"].copy()
    d[2, 2, 2] = (-5.5, 4.0, 4.0)
    d[7, 7, 7] = (3.0, 14.2, 2.0)
    one_iteration(core, oracle, c, positions=d)


def test_thin_axis(core, oracle):
    """A 3D volume with a 2-voxel axis: the DCT pass along it is a 2 x 2 transform."""
    c = make_case(shape=(14, 2, 12), K=8, L=8, seed=7)
    one_iteration(core, oracle, c)


@pytest.mark.parametrize("shape", [(33, 1), (1, 40), (37, 5), (3, 130)])
def test_thin_images_match_oracle(core, oracle, shape):
    """2D images with a 1-pixel axis: (nx, 1) runs the prior scaling on a unit-stride axis."""
    from test_gpu_2d import make_case2d, new_reg2d
    c = make_case2d(shape=shape, K=8, L=6, seed=sum(shape))
    vshape, K, L = c["vshape"], c["K"], c["L"]
    reg = new_reg2d(core, c)
    assert reg.EM(1, -1e30, 1, 0) == 1
    mll, dream, hist, deg = oracle.estep(c["d0"].astype(np.float64), c["u"], c["v"],
                                         c["theta"].astype(np.float64), vshape, vshape, K, L)
    lpt, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA, vshape)
    st = reg.iteration_stats()[0]
    np.testing.assert_allclose(reg.get_dream_locations(), dream, rtol=0, atol=5e-5)
    np.testing.assert_allclose(reg.get_likelihood_parameters(), oracle.theta_map(hist, K, L, 2.0),
                               rtol=1e-4, atol=1e-6)
    assert st[2] == pytest.approx(lpt, rel=2e-4)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)


@pytest.mark.parametrize("shape", [(12, 14, 10), (17, 3, 33), (7, 5, 9)])
def test_persistent_passes_match_oracle(core, oracle, shape, monkeypatch):
    """The persistent tensor-core pass kernel (BINDER_B200_PERSISTENT=1: all components in one
    launch, one CTA per SM, double-buffered TMEM accumulator, cp.async-staged A chunks) gives the
    oracle's M-step like the default per-tile kernel."""
    monkeypatch.setenv("BINDER_B200_PERSISTENT", "1")
    c = make_case(shape=shape, K=8, L=6, seed=sum(shape) + 1)
    one_iteration(core, oracle, c)
