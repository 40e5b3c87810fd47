"""The registration driver's preprocessing and output steps on the GPU (binder_b200.preprocess)
against the reference's own binning functions (golden fixtures), scipy's centre of mass, and the
restatement of skimage's warp on scipy.ndimage."""
import numpy as np
import pytest

from conftest import golden


def test_warp_restatement_identity(oracle):
    rng = np.random.default_rng(0)
    im = rng.random((6, 7, 5))
    pos = np.stack(np.indices(im.shape), -1).astype(np.float64)
    for order in (0, 1):
        np.testing.assert_array_equal(oracle.warp_image(im, pos, order), im)
    # the cubic spline interpolates its samples
    np.testing.assert_allclose(oracle.warp_image(im, pos, 3), im, rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_bin_signal_robust_matches_reference_golden(core):
    from binder_b200 import preprocess as pp
    g = golden("preprocess_ref.npz")
    for name in g["names"]:
        sig, nb = g[f"{name}_signal"], int(g[f"{name}_bins"])
        b, e = pp.bin_signal_robust(sig, nb)
        assert b.dtype == np.int32 and b.shape == sig.shape
        assert np.array_equal(b, g[f"{name}_robust"]), name          # bit-exact
        assert np.array_equal(e, g[f"{name}_edges"]), name
        assert np.array_equal(pp.bin_signal(sig, nb), g[f"{name}_plain"]), name


@pytest.mark.gpu
def test_bin_signal_robust_full_size_matches_restatement(core):
    from binder_b200 import phantoms, preprocess as pp
    from binder_b200.utils import bin_signal_robust
    pair = phantoms.make_pair((160, 192, 160), 20260001, bins=64)
    img = pair.moving.astype(np.float64) * 2.5 - 0.3
    b, e = pp.bin_signal_robust(img, 64)
    br, er = bin_signal_robust(img, 64)
    assert np.array_equal(b, br) and np.array_equal(e, er)
    b32, _ = pp.bin_signal_robust(pair.moving, 64)                   # float32 arithmetic
    assert np.array_equal(b32, bin_signal_robust(pair.moving, 64)[0])


@pytest.mark.gpu
def test_binning_errors(core):
    from binder_b200 import preprocess as pp
    with pytest.raises(core.BinderError):
        pp.bin_signal_robust(np.full(100, 3.0), 8)
    with pytest.raises(core.BinderError):
        pp.bin_signal(np.full(100, 3.0), 8)
    with pytest.raises(core.BinderError):
        pp.center_of_mass_nonzero(np.zeros((4, 4, 4), np.int32))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(40, 36, 30), (64, 50)])
def test_center_of_mass_matches_scipy(core, shape):
    from scipy import ndimage as ndi
    from binder_b200 import preprocess as pp
    rng = np.random.default_rng(len(shape))
    bins = (rng.random(shape) > 0.6).astype(np.int32) * rng.integers(1, 9, shape)
    bins[: shape[0] // 3] = 0
    got = pp.center_of_mass_nonzero(bins)
    want = np.array(ndi.center_of_mass(bins > 0))
    np.testing.assert_array_equal(got, want)                          # exact


@pytest.mark.gpu
@pytest.mark.parametrize("order", [0, 1, 3])
def test_warp_image_matches_restatement(core, oracle, order):
    from binder_b200 import phantoms, preprocess as pp
    rng = np.random.default_rng(7 + order)
    shape = (48, 40, 36)
    im = phantoms.ellipsoid_phantom(shape, 10, (3.0, 12.0), 1.0, 0.02, rng).astype(np.float64) + 0.5
    pos = phantoms.identity_positions(shape) + \
        phantoms.smooth_random_field(shape, 2.0, 3.0, rng).astype(np.float64)
    pos[:3] -= 4.0          # some samples leave the image: zero fill and the clip rule
    got = pp.warp_image(im, pos, order)
    want = oracle.warp_image(im, pos, order)
    if order == 0:
        # nearest neighbour: equal except where a coordinate sits on a half-integer
        frac = np.abs(np.modf(pos)[0])
        ok = np.all(np.abs(frac - 0.5) > 1e-9, axis=-1)
        np.testing.assert_array_equal(got[ok], want[ok])
    else:
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)


@pytest.mark.gpu
def test_warp_cubic_far_outside_and_small(core, oracle):
    """Order 3 on a small image at points inside, at the edge, beyond the 12-sample padding the
    spline prefilter uses, and non-finite ones; the input range excludes 0 (clip widening)."""
    from binder_b200 import preprocess as pp
    rng = np.random.default_rng(3)
    im = rng.random((9, 7, 11)) * 5.0 + 1.0
    pos = np.concatenate([
        rng.uniform(-3.0, np.array(im.shape) + 2.0, (400, 3)),
        np.array([[-11.5, 3.0, 3.0], [-12.7, 2.2, 4.1], [3.0, 20.3, 5.0], [-30.0, 1.0, 1.0],
                  [8.9, 6.9, 10.9], [0.0, 0.0, 0.0], [4.0, 3.0, 33.9]])])
    got = pp.warp_image(im, pos, 3)
    want = oracle.warp_image(im, pos, 3)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-12)
    # non-finite and huge coordinates give the fill value (scipy gives NaN, or overflows)
    bad = np.array([[np.nan, 1.0, 1.0], [2.0, np.inf, 2.0], [1e300, 0.0, 0.0]])
    assert np.all(pp.warp_image(im, bad, 3) == 0.0)
