"""The MI E-step with FP16 per-thread bin columns (set_histogram_precision(1)) against the FP32
columns and the FP64 oracle (BINDER/src/cpu/Registration.cpp:219-330 restated in oracle/).

The FP16 mode stages theta multiplied by 2^12 and keeps the normaliser S and the axis moments in
FP32, so S and the moments are exactly 2^12 times those of the FP32 mode and the dream locations
(moment / S) must come out bit for bit the same; only each voxel's per-bin mass, and hence the
histogram and theta, carries the FP16 rounding (2^-11 relative per addition, unbiased)."""
import numpy as np
import pytest

from test_gpu_parity import make_case, new_reg

pytestmark = pytest.mark.gpu


def _one_iteration(core, c, hp):
    reg = new_reg(core, c)
    reg.set_histogram_precision(hp)
    assert reg.EM(1, -1e30, 1, 0) == 1
    return (np.asarray(reg.get_dream_locations(), np.float64),
            np.asarray(reg.get_likelihood_parameters(), np.float64),
            np.asarray(reg.get_final_locations_as_numpy_array(), np.float64).ravel(),
            reg.iteration_stats()[0])


@pytest.mark.parametrize("shape,K,L,seed", [((40, 36, 44), 64, 64, 3), ((21, 17, 30), 32, 24, 4)])
def test_fp16_columns_against_fp32_columns_and_oracle(core, oracle, shape, K, L, seed):
    c = make_case(shape=shape, K=K, L=L, seed=seed, disp=1.5)
    dream32, theta32, final32, st32 = _one_iteration(core, c, 0)
    dream16, theta16, final16, st16 = _one_iteration(core, c, 1)
    # the normaliser and the moments are the FP32 mode's times 2^12: same dream locations, and
    # the M-step, which reads only them, gives the same positions
    assert np.array_equal(dream16, dream32)
    assert np.array_equal(final16, final32)
    # log-likelihood: log(2^12 S) - ln 2^12 against log(S), FP32 logs in an FP64 sum
    assert st16[0] == pytest.approx(st32[0], rel=1e-6)
    # theta from the FP16-rounded masses: within 2e-3 relative of the FP32 columns' theta where
    # theta > 1e-3 (a cell sums many voxels' masses, each off by at most a few 2^-12)
    big = theta32 > 1e-3
    rel = np.abs(theta16[big] - theta32[big]) / theta32[big]
    assert rel.max() < 2e-3, rel.max()
    assert np.abs(theta16 - theta32).max() < 2e-4
    # and against the FP64 oracle's E-step and MAP update
    _, dream, hist, deg = oracle.estep(c["d0"].astype(np.float64), c["u"], c["v"],
                                       c["theta"].astype(np.float64), shape, shape, K, L)
    theta = oracle.theta_map(hist, K, L, 2.0)
    assert deg == 0
    np.testing.assert_allclose(dream16, dream, rtol=0, atol=5e-5)
    big = theta > 1e-3
    assert (np.abs(theta16[big] - theta[big]) / theta[big]).max() < 2e-3


def test_fp16_columns_em_run_is_repeatable_and_close(core):
    """Ten iterations each way: the FP16 run is bitwise repeatable (the CTA histograms still merge
    in fixed order) and ends within FP32-level distance of the FP32 run's positions."""
    c = make_case(shape=(36, 40, 32), K=64, L=64, seed=5, disp=1.5)
    runs = []
    for hp in (1, 1, 0):
        reg = new_reg(core, c)
        reg.set_histogram_precision(hp)
        assert reg.EM(10, -1e30, 1, 0) == 10
        runs.append((np.asarray(reg.get_final_locations_as_numpy_array(), np.float64).ravel(),
                     np.asarray(reg.get_likelihood_parameters(), np.float64),
                     reg.iteration_stats()[:, 3]))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    assert np.abs(runs[0][0] - runs[2][0]).max() < 2e-3
    np.testing.assert_allclose(runs[0][2], runs[2][2], rtol=1e-4)


def test_histogram_precision_rejects_other_values(core):
    from binder_b200._lib import BinderError
    c = make_case()
    reg = new_reg(core, c)
    for bad in (-1, 2):
        with pytest.raises(BinderError, match="histogram precision"):
            reg.set_histogram_precision(bad)
