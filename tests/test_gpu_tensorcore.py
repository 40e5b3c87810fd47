"""The tcgen05 tensor-core DCT passes against the FP32 CUDA-core passes, the reference's golden
smoothing output and the FP64 oracle.  Stated tolerances: 3xTF32 keeps FP32-level accuracy (same
bounds as the FP32 path); one TF32 product per pass is checked at 2e-3 relative to the field's
scale; the BF16 split (three kind::f16 products, ~16-bit operands) at 2e-4 and one BF16 product
at 2e-2 relative to the field's scale."""
import math

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

PREC_FP32, PREC_TF32X3, PREC_TF32, PREC_BF16X3, PREC_BF16 = 0, 1, 2, 3, 4


def smooth(core, g, prec):
    shape = g["field"].shape[:3]
    t = core.NonLinearTransformation(*g["gamma"], 1, 1, 1, 1, 1, 1, g["D"], *shape, 1,
                                     float(g["sigma"]), 0.0)
    t.set_precision(prec)
    return t.smooth_deformation(g["field"])


def test_tensorcore_tf32x3_smoothing_matches_reference(core):
    g = golden("smoothing_ref.npz")
    cost, out = smooth(core, g, PREC_TF32X3)
    np.testing.assert_allclose(out, g["out"], rtol=0, atol=2e-6)
    assert cost == pytest.approx(float(g["cost"]), rel=1e-5)


def test_tensorcore_tf32_smoothing_error_bound(core):
    g = golden("smoothing_ref.npz")
    cost, out = smooth(core, g, PREC_TF32)
    scale = np.abs(g["out"]).max()
    assert np.abs(out - g["out"]).max() < 2e-3 * scale
    assert cost == pytest.approx(float(g["cost"]), rel=5e-3)


@pytest.mark.parametrize("prec,bound", [(PREC_BF16X3, 2e-4), (PREC_BF16, 2e-2)])
def test_tensorcore_bf16_smoothing_error_bound(core, prec, bound):
    g = golden("smoothing_ref.npz")
    cost, out = smooth(core, g, prec)
    scale = np.abs(g["out"]).max()
    err = np.abs(out - g["out"]).max() / scale
    print(f"precision {prec}: max error {err:.2e} of the field's scale, cost rel "
          f"{abs(cost / float(g['cost']) - 1):.2e}")
    assert err < bound
    assert cost == pytest.approx(float(g["cost"]), rel=5 * bound)


@pytest.mark.parametrize("shape", [(20, 24, 18), (33, 17, 40), (64, 48, 96)])
def test_tensorcore_bf16x3_matches_cuda_cores_on_odd_sizes(core, shape):
    from binder_b200.utils import initialize_fourier_domain_smoothing
    rng = np.random.default_rng(sum(shape) + 1)
    field = rng.standard_normal(shape + (3,)).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3)
    outs = {}
    for prec in (PREC_FP32, PREC_BF16X3):
        t = core.NonLinearTransformation(2.0, 3.0, 4.0, 1, 1, 1, 1, 1, 1, D, *shape, 1, 0.6, 0.0)
        t.set_precision(prec)
        outs[prec] = t.smooth_deformation(field)
    scale = np.abs(outs[PREC_FP32][1]).max()
    assert np.abs(outs[PREC_BF16X3][1] - outs[PREC_FP32][1]).max() < 2e-4 * scale
    assert outs[PREC_BF16X3][0] == pytest.approx(outs[PREC_FP32][0], rel=1e-3)


@pytest.mark.parametrize("shape", [(20, 24, 18), (33, 17, 40), (64, 48, 96)])
def test_tensorcore_matches_cuda_cores_on_odd_sizes(core, shape):
    from binder_b200.utils import initialize_fourier_domain_smoothing
    rng = np.random.default_rng(sum(shape))
    field = rng.standard_normal(shape + (3,)).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3)
    outs = {}
    for prec in (PREC_FP32, PREC_TF32X3):
        t = core.NonLinearTransformation(2.0, 3.0, 4.0, 1, 1, 1, 1, 1, 1, D, *shape, 1, 0.6, 0.0)
        t.set_precision(prec)
        outs[prec] = t.smooth_deformation(field)
    np.testing.assert_allclose(outs[PREC_TF32X3][1], outs[PREC_FP32][1], rtol=0, atol=5e-6)
    assert outs[PREC_TF32X3][0] == pytest.approx(outs[PREC_FP32][0], rel=1e-5)


def test_tensorcore_em_matches_oracle(core, oracle):
    from test_gpu_parity import SIGMA_CUBIC, make_case, new_reg
    c = make_case(shape=(14, 12, 16), seed=1)
    shape, K, L = c["shape"], c["K"], c["L"]
    reg = new_reg(core, c)
    reg.set_precision(PREC_TF32X3)
    assert reg.EM(12, -1e30, 1, 0) == 12
    final_g = reg.get_final_locations_as_numpy_array().astype(np.float64).ravel()
    it, final_o, theta_o, stats_o = oracle.em(c["d0"], c["grid"], c["u"], c["v"], c["theta"], 2.0,
                                             c["D"], c["gamma"], SIGMA_CUBIC, shape, shape, K, L,
                                             float(np.prod(shape)), 12, -1e30)
    np.testing.assert_allclose(final_g, final_o, rtol=0, atol=2e-3)
    np.testing.assert_allclose(reg.iteration_stats()[:, 3], stats_o[:, 3], rtol=1e-5)
    assert reg.state()["flags"] == 0


def test_tensorcore_bf16x3_em_matches_oracle(core, oracle):
    from test_gpu_parity import SIGMA_CUBIC, make_case, new_reg
    c = make_case(shape=(14, 12, 16), seed=1)
    shape, K, L = c["shape"], c["K"], c["L"]
    reg = new_reg(core, c)
    reg.set_precision(PREC_BF16X3)
    assert reg.EM(12, -1e30, 1, 0) == 12
    final_g = reg.get_final_locations_as_numpy_array().astype(np.float64).ravel()
    it, final_o, theta_o, stats_o = oracle.em(c["d0"], c["grid"], c["u"], c["v"], c["theta"], 2.0,
                                             c["D"], c["gamma"], SIGMA_CUBIC, shape, shape, K, L,
                                             float(np.prod(shape)), 12, -1e30)
    np.testing.assert_allclose(final_g, final_o, rtol=0, atol=2e-3)
    np.testing.assert_allclose(reg.iteration_stats()[:, 3], stats_o[:, 3], rtol=1e-4)
    assert reg.state()["flags"] == 0


def test_tensorcore_sampler_prior_covariance(core):
    """Prior sampling through the fused tensor-core pass (noise in the TMEM epilogue)."""
    from test_oracle import _prior_covariance
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape, gamma, sigma = (3, 5, 4), 5.0, 0.34
    cov = _prior_covariance(shape, gamma, sigma, 2)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3)
    t = core.NonLinearTransformation(gamma, gamma, gamma, 1, 1, 1, 1, 1, 1, D, *shape, 1, sigma,
                                     0.0)
    t.set_precision(PREC_TF32X3)
    s = t.sampleDeformationField(np.zeros(shape + (3,)), 100000)
    x = s[..., 0].astype(np.float64).reshape(-1, np.prod(shape), order="F")
    np.testing.assert_allclose(x.T @ x / x.shape[0], cov, rtol=1e-3, atol=1e-3)
