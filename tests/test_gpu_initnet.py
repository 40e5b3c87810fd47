"""The learned initialiser's hand-written kernels (tcgen05 BF16 GEMMs, im2col, pooling, Adam)
against FP64: the GEMM exactly (BF16 operands, FP32 accumulation), the whole network against the
FP64 oracle of the same network (oracle/netoracle.py, rounding where the kernels round) within the
spread BF16 rounding flips give, and its training."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _net(core, batch, size, seed=0):
    from binder_b200.initnet import InitNet
    return InitNet(batch, size, seed)


def _layer_slices():
    from oracle import netoracle as N
    out, o = [], 0
    for ci, co, _, _ in N.LAYERS:
        out.append((slice(o, o + 27 * ci * co), slice(o + 27 * ci * co, o + 27 * ci * co + co)))
        o += 27 * ci * co + co
    return out


@pytest.mark.parametrize("M,N,K", [(300, 16, 64), (1000, 128, 448), (17, 3, 128),
                                   (128, 1728, 8192), (64, 96, 64)])
def test_gemm_bf16_matches_fp64(core, M, N, K):
    """The tcgen05 BF16 GEMM every convolution runs on: exact BF16 operands, so the only error is
    FP32 accumulation (TMEM) against FP64: 1e-5 of the row scale; K = 8192 runs split over CTAs
    with atomic accumulation."""
    import ctypes as C
    from binder_b200._lib import check, lib
    from oracle import netoracle as N_
    rng = np.random.default_rng(M + N + K)
    A = N_.bf16(rng.standard_normal((M, K))).astype(np.float32)
    B = N_.bf16(rng.standard_normal((N, K))).astype(np.float32)
    Ab = np.ascontiguousarray((A.view(np.uint32) >> 16).astype(np.uint16))
    Bb = np.ascontiguousarray((B.view(np.uint32) >> 16).astype(np.uint16))
    Cg = np.empty((M, N), np.float32)
    check(lib().binder_gemm_bf16(Ab.ctypes.data, Bb.ctypes.data, Cg.ctypes.data, M, N, K))
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    scale = np.sqrt(K)
    assert np.abs(Cg - ref).max() < 1e-5 * scale


def _sensitivity(p, x, t, eps, reps=2, seed=0):
    """largest relative change of any layer's weight gradient of the FP64 oracle (rounding as the
    kernels round) when the parameters move by a relative eps: the spread BF16 rounding-boundary
    flips give to results that agree to FP32 accuracy"""
    from oracle import netoracle as N
    rng = np.random.default_rng(seed)
    _, _, g0 = N.forward_backward(p, x, t, round=True)
    worst = np.zeros(len(_layer_slices()))
    for _ in range(reps):
        _, _, g1 = N.forward_backward(p * (1 + eps * rng.standard_normal(p.size)), x, t,
                                      round=True)
        for i, (w, _) in enumerate(_layer_slices()):
            worst[i] = max(worst[i], np.linalg.norm(g1[w] - g0[w]) / np.linalg.norm(g0[w]))
    return worst


@pytest.mark.parametrize("batch,size", [(1, 8), (2, 16)])
def test_initnet_forward_and_gradients_match_oracle(core, batch, size):
    """The whole network (im2col, GEMMs, leaky ReLU, pooling, up-sampling, skip, MSE) against the
    FP64 oracle rounding where the kernels round.  With BF16 activations a difference at FP32
    level flips roundings, and in networks this small the flips spread to several per cent of a
    gradient; the bound is therefore the oracle's own spread under a 1e-5 relative parameter
    perturbation (three times it, at least 2e-2), with cosine similarity above 0.99."""
    from oracle import netoracle as N
    net = _net(core, batch, size, seed=1)
    rng = np.random.default_rng(size)
    p = net.get_parameters()
    # a larger head than the initialisation's, so every layer's gradient is well above round-off
    for w, _ in _layer_slices()[-1:]:
        p[w] *= 30.0
    net.set_parameters(p)
    x = rng.random((batch, size, size, size, 2)).astype(np.float32)
    c = size // 4
    t = (rng.standard_normal((batch, c, c, c, 3)) * 0.5).astype(np.float32)
    out_g = net.predict(x)
    loss_g, g = net.gradients(x, t)
    p64 = p.astype(np.float64)
    out_o, loss_o, g_o = N.forward_backward(p64, x, t, round=True)
    spread = _sensitivity(p64, x, t, 1e-5)
    scale = np.abs(out_o).max()
    assert np.abs(out_g - out_o).max() < 2e-2 * scale
    assert loss_g == pytest.approx(loss_o, rel=1e-2)
    for i, (w, b) in enumerate(_layer_slices()):
        ref = g_o[w]
        err = np.linalg.norm(g[w] - ref) / np.linalg.norm(ref)
        cos = float(g[w] @ ref / (np.linalg.norm(g[w]) * np.linalg.norm(ref)))
        print(f"layer {i}: W gradient error {err:.2e} (oracle spread {spread[i]:.2e}), "
              f"cosine {cos:.5f}")
        assert err < max(3 * spread[i], 2e-2), (i, err, spread[i])
        assert cos > 0.99, (i, cos)


def test_initnet_training_lowers_the_loss(core):
    net = _net(core, 2, 16, seed=2)
    rng = np.random.default_rng(7)
    x = rng.random((2, 16, 16, 16, 2)).astype(np.float32)
    t = np.zeros((2, 4, 4, 4, 3), np.float32)
    t[..., 0] = x[:, ::4, ::4, ::4, 0] - 0.5  # a target the input determines
    losses = [net.train_step(x, t, 1e-3) for _ in range(60)]
    assert losses[-1] < 0.2 * losses[0], losses[::10]
    # parameters round-trip through the ABI
    p = net.get_parameters()
    net.set_parameters(p)
    assert np.array_equal(net.get_parameters(), p)
