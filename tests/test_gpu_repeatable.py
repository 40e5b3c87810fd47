"""EM is bitwise repeatable: the single-pass E-step merges its per-CTA fixed-point histograms as
exact 64-bit integer sums and adds the per-CTA log-likelihood partials in CTA order, so two runs
of the same registration (the same object after reset, or a second object on the same inputs)
give identical positions, likelihood parameters, log-likelihoods and Dirichlet costs, bit for bit.
The deformation prior's cost (a reported statistic, fed back nowhere) is summed over the DCT
tiles with FP64 atomics and is compared to 1e-12 relative."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (48, 40, 44)
BINS = 64


def _reg(core, pair, grid=0):
    from binder_b200 import phantoms
    from binder_b200.utils import initialize_fourier_domain_smoothing
    V = int(np.prod(SHAPE))
    x = phantoms.identity_positions(SHAPE).astype(np.float32)
    D = initialize_fourier_domain_smoothing(SHAPE, True, 2, 3).astype(np.float32)
    r = core.Registration(x, 1, x, x, *SHAPE, *SHAPE, 3, float(np.count_nonzero(pair.u)))
    r.setNonLinearTransformation(1e-4 * V, 1e-4 * V, 1e-4 * V, 1, 1, 1, 1, 1, 1, D)
    r.setMILikelihood(2.0, np.full((BINS, BINS), 1 / BINS, np.float32), BINS, BINS, 1, pair.v,
                      pair.u)
    if grid:
        r.set_estep_grid(grid)
    return r


def _run(r, iters=25):
    it = r.EM(iters, -1e300, 1, 0)
    return (it, r.get_final_locations_as_numpy_array().copy(),
            np.asarray(r.get_likelihood_parameters()).copy(), r.iteration_stats().copy())


def _bits_equal(x, y):
    x, y = np.ascontiguousarray(x), np.ascontiguousarray(y)
    assert x.shape == y.shape
    assert np.array_equal(x.view(np.uint8), y.view(np.uint8))


def _same(a, b):
    assert a[0] == b[0]
    _bits_equal(a[1], b[1])  # positions
    _bits_equal(a[2], b[2])  # theta
    _bits_equal(a[3][:, :2], b[3][:, :2])  # mll, Dirichlet cost per iteration
    np.testing.assert_allclose(a[3][:, 2:], b[3][:, 2:], rtol=1e-12, atol=0)


@pytest.mark.parametrize("grid", [0, 37])
def test_em_bitwise_repeatable(core, grid):
    from binder_b200 import phantoms
    pair = phantoms.make_pair(SHAPE, 515, bins=BINS)
    r = _reg(core, pair, grid)
    first = _run(r)
    r.reset()
    _same(first, _run(r))
    _same(first, _run(_reg(core, pair, grid)))
