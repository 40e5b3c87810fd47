"""A batch of registrations of uneven sizes in one graph per EM chunk (RegistrationBatch) against
the same pairs registered one by one: the same iteration counts and final positions within 1e-4
voxels (the batch's E-steps run on 16 CTAs, whose fixed-point histogram scale differs from the
default grid's, so theta can differ in its last bits)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(20, 24, 16), (32, 28, 36), (16, 16, 16), (40, 24, 32), (24, 40, 20)]


def _pairs():
    from binder_b200 import phantoms
    return [phantoms.make_pair(s, 4242 + i, bins=32, n_objects=12, axes=(3.0, 10.0), rms=1.5,
                               spacing=4.0) for i, s in enumerate(SHAPES)]


def _reg(core, pair, grid=0):
    from binder_b200 import phantoms
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape = pair.u.shape
    V = int(np.prod(shape))
    x = phantoms.identity_positions(shape).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3).astype(np.float32)
    r = core.Registration(x, 1, x, x, *shape, *shape, 3, float(np.count_nonzero(pair.u)))
    r.setNonLinearTransformation(1e-4 * V, 1e-4 * V, 1e-4 * V, 1, 1, 1, 1, 1, 1, D)
    r.setMILikelihood(2.0, np.full((32, 32), 1 / 32, np.float32), 32, 32, 1, pair.v, pair.u)
    if grid:
        r.set_estep_grid(grid)
    return r


def test_batch_matches_individual_registrations(core):
    pairs = _pairs()
    solo = []
    for p in pairs:
        r = _reg(core, p)
        it = r.EM(60, 1e-5, 1, 0)
        solo.append((it, r.get_final_locations_as_numpy_array().copy()))
    regs = [_reg(core, p, grid=16) for p in pairs]
    batch = core.RegistrationBatch(regs)
    its = batch.EM(60, 1e-5, 1)
    assert batch.last_ms > 0
    for (it, fin), it_b, r in zip(solo, its, regs):
        assert it_b == it
        np.testing.assert_allclose(r.get_final_locations_as_numpy_array(), fin, rtol=0, atol=1e-4)
    # a second run of the same pairs, restored to their start, gives the same iteration counts
    for r in regs:
        r.reset()
    its2 = core.RegistrationBatch(regs).EM(60, 1e-5, 1)
    assert list(its2) == list(its)
