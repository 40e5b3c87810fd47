"""binder_jacobian_determinant_3d_noalloc (the Jacobian staged through a fixed device array, no
cudaMalloc) against binder_jacobian_determinant_3d, both called through the C ABI.

The file name sorts last so that it also runs after every other test has used the device; it must
pass that way and alone in a fresh process.  The two calls in a row differ in shape and in sign
of the determinants, so a summary or a J left over from the previous call would show."""
import ctypes as C

import numpy as np
import pytest

MAX_VOXELS = 1 << 19


def _field(shape, rms, seed):
    from binder_b200 import phantoms
    rng = np.random.default_rng(seed)
    f = phantoms.identity_positions(shape) + \
        phantoms.smooth_random_field(shape, rms, 2.0, rng).astype(np.float64)
    return np.ascontiguousarray(f, dtype=np.float64)


def _allocating(L, check, f, shape, vs):
    J = np.full(int(np.prod(shape)), np.nan)
    check(L.binder_jacobian_determinant_3d(f, *shape, *vs, J))
    return J


def _noalloc(L, check, f, shape, vs):
    J = np.full(int(np.prod(shape)), np.nan)
    mm = (C.c_double * 2)(np.nan, np.nan)
    neg = C.c_longlong(-1)
    check(L.binder_jacobian_determinant_3d_noalloc(f, *shape, *vs, J, mm, C.byref(neg)))
    return J, (mm[0], mm[1]), neg.value


@pytest.mark.gpu
def test_noalloc_matches_allocating_entry_point_on_two_calls(core):
    from binder_b200._lib import check, lib
    L = lib()
    cases = [
        ((48, 40, 36), _field((48, 40, 36), 3.0, 11), (1.0, 1.0, 1.0)),    # folds: J < 0 somewhere
        ((20, 24, 28), _field((20, 24, 28), 0.05, 12), (1.5, 1.0, 0.8)),   # no folds, smaller grid
    ]
    negatives = []
    for shape, f, vs in cases:
        Jr = _allocating(L, check, f, shape, vs)
        J, (jmin, jmax), neg = _noalloc(L, check, f, shape, vs)
        assert np.array_equal(J, Jr)                      # FP64, bit-identical
        assert (jmin, jmax) == (Jr.min(), Jr.max())
        assert neg == int((Jr < 0).sum())
        negatives.append(neg)
    assert negatives[0] > 0 and negatives[1] == 0


@pytest.mark.gpu
def test_noalloc_largest_grid_then_rejection_then_small(core):
    from binder_b200._lib import BinderError, check, lib
    L = lib()
    assert L.binder_jacobian_noalloc_max_voxels() == MAX_VOXELS
    shape = (64, 64, 128)                                  # exactly the limit
    f = _field(shape, 1.5, 13)
    J, (jmin, jmax), neg = _noalloc(L, check, f, shape, (1.0, 1.0, 1.0))
    Jr = _allocating(L, check, f, shape, (1.0, 1.0, 1.0))
    assert np.array_equal(J, Jr)
    assert (jmin, jmax, neg) == (Jr.min(), Jr.max(), int((Jr < 0).sum()))
    # one voxel past the limit, and a grid well past it: rejected before any device work
    for big in ((1, 1, MAX_VOXELS + 1), (80, 80, 82)):
        fb = np.zeros(int(np.prod(big)) * 3)
        with pytest.raises(BinderError, match="no-allocation limit"):
            check(L.binder_jacobian_determinant_3d_noalloc(fb, *big, 1.0, 1.0, 1.0,
                                                             np.zeros(int(np.prod(big))), None,
                                                             None))
    # and the entry point still works afterwards
    small = (9, 10, 11)
    fs = _field(small, 0.7, 14)
    J2, _, _ = _noalloc(L, check, fs, small, (1.0, 2.0, 0.5))
    assert np.array_equal(J2, _allocating(L, check, fs, small, (1.0, 2.0, 0.5)))


def test_noalloc_rejects_oversized_grid(core):
    """The size check comes before any CUDA call, so it holds without a device too."""
    from binder_b200._lib import lib
    L = lib()
    # exactly one voxel past the limit (64 x 64 x 128 + 1), and 80 x 80 x 82 (524,800 voxels)
    for big in ((1, 1, MAX_VOXELS + 1), (80, 80, 82)):
        assert int(np.prod(big)) > MAX_VOXELS
        st = L.binder_jacobian_determinant_3d_noalloc(np.zeros(int(np.prod(big)) * 3), *big,
                                                      1.0, 1.0, 1.0, np.zeros(int(np.prod(big))),
                                                      None, None)
        assert st == 1
        assert b"no-allocation limit of 524288 voxels" in L.binder_last_error()
