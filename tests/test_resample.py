"""Resampling between resolutions (FastRegistration.move_resolution): the spectral up-sampling of
NonLinearTransformation::up_sample against the reference's own output, and the order-1 resize
(skimage.transform.resize semantics) against its scipy.ndimage restatement.  FP64 on the GPU."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden


def _matrix(core, kind, n, m):
    from binder_b200._lib import lib
    out = np.zeros(m * n)
    assert lib().binder_resample_matrix(kind, n, m, out) == 0
    return out.reshape(m, n)


@pytest.mark.parametrize("n,m", [(40, 10), (41, 11), (160, 40), (10, 20), (11, 21), (7, 7),
                                 (5, 2), (3, 1), (1, 4), (2, 7)])
def test_linear_resize_matrix_matches_scipy(core, n, m):
    """The per-axis matrix (host arithmetic, no GPU) equals scipy applied to unit vectors."""
    from scipy import ndimage as ndi
    M = _matrix(core, 1, n, m)
    cols = []
    for j in range(n):
        x = np.eye(n)[j]
        if m < n:
            x = ndi.gaussian_filter(x, (n / m - 1) / 2, mode="mirror")
        cols.append(ndi.zoom(x, m / n, order=1, mode="mirror", grid_mode=True))
    np.testing.assert_allclose(M, np.stack(cols, 1), rtol=0, atol=1e-15)


@pytest.mark.parametrize("n,m", [(6, 12), (7, 13), (9, 17), (5, 5)])
def test_upsample_matrix_matches_oracle(core, oracle, n, m):
    U = _matrix(core, 0, n, m)
    # a 1-D field along x (ny = nz = 1 is not a 2D case for the oracle: use a 3D line)
    f = np.random.default_rng(n * m).standard_normal((n, 1, 2, 3))
    out = oracle.up_sample(f, (n, 1, 2), (m, 1, 2))
    np.testing.assert_allclose(np.einsum("on,nyzc->oyzc", U, f), out, rtol=0, atol=1e-13)


@pytest.mark.gpu
def test_up_sample_matches_reference_golden(core):
    g = golden("upsample_ref.npz")
    for k in range(int(g["ncases"])):
        f = g[f"field{k}"]
        o = tuple(int(s) for s in g[f"oshape{k}"])
        out = core.NonLinearTransformation.up_sample(f.ravel(), *f.shape[:3], *o, 1)
        assert out.shape == g[f"out{k}"].shape
        np.testing.assert_allclose(out, g[f"out{k}"], rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_up_sample_rejects_shrinking(core):
    with pytest.raises(core.BinderError):
        core.NonLinearTransformation.up_sample(np.zeros(8 * 8 * 8 * 3), 8, 8, 8, 4, 8, 8, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,oshape,scale", [
    ((40, 48, 40), (10, 12, 10), 0.25),      # first level of resolutions [4, ...]: shrink 4x
    ((20, 24, 20), (40, 48, 40), 2.0),       # coarse -> fine
    ((27, 25, 30), (14, 13, 15), 0.5),       # odd sizes, ceil(n / 2)
    ((64, 50), (128, 100), 2.0),             # 2D image
])
def test_resize_linear_matches_restatement(core, oracle, shape, oshape, scale):
    rng = np.random.default_rng(sum(shape))
    from binder_b200 import phantoms
    f = phantoms.identity_positions(shape) + rng.normal(0, 0.7, shape + (len(shape),))
    out = core.resize_linear(f, oshape, scale)
    ref = oracle.resize_linear(f, oshape, scale)
    assert out.shape == ref.shape
    np.testing.assert_allclose(out, ref, rtol=0, atol=1e-11 * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("shape,fshape", [((20, 24, 16), (5, 6, 4)), ((18, 14, 1), (6, 7, 1))])
def test_add_displacement_equals_resized_start(core, shape, fshape):
    """Registration.add_displacement (the positions moved by the order-1 resize of a coarse
    field, on the device) equals a registration created at identity + resize_linear(field), and
    keeps theta; a 2D registration takes a field with fz == 1."""
    rng = np.random.default_rng(3)
    N = 2 if shape[2] == 1 else 3
    grid = np.stack(np.indices(shape), -1).astype(np.float32)[..., :N]
    field = rng.normal(0.0, 1.5, fshape + (N,)).astype(np.float32)
    up = core.resize_linear(field.reshape(fshape[:N] + (N,)).astype(np.float64), shape[:N])
    up = up.reshape(shape + (N,))
    V = int(np.prod(shape))
    K = 8
    bins = rng.integers(0, K, V).astype(np.int32)

    def make(start):
        r = core.Registration(start, 1, grid, grid, *shape, *shape, 3, float(V))
        r.setMILikelihood(2.0, np.full((K, K), 1.0 / K, np.float32), K, K, 1, bins, bins)
        return r

    a = make(grid)
    a.add_displacement(field)
    b = make((grid + up.astype(np.float32)).astype(np.float32))
    np.testing.assert_allclose(a.get_final_locations_as_numpy_array(),
                               b.get_final_locations_as_numpy_array(), rtol=0, atol=2e-5)
    np.testing.assert_array_equal(a.get_likelihood_parameters(), np.full(K * K, 1.0 / K,
                                                                         np.float32))
