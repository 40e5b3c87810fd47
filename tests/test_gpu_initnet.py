"""The learned initialiser's hand-written kernels (tcgen05 BF16 GEMMs, im2col, pooling, Adam)
against the FP64 oracle of the same network (oracle/netoracle.py, rounding where the kernels
round), and its training and use.  Tolerances: forward output within 1e-2 of its scale, every
layer's weight and bias gradients within 3e-2 relative L2 error (FP32 accumulation over up to
2 x 64^3 products against FP64, with BF16 operands whose rounding can flip where a value sits on a
rounding boundary)."""
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


@pytest.mark.parametrize("batch,size", [(1, 8), (2, 16)])
def test_initnet_forward_and_gradients_match_oracle(core, batch, size):
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
    out_o, loss_o, g_o = N.forward_backward(p.astype(np.float64), x, t, round=True)
    scale = np.abs(out_o).max()
    assert np.abs(out_g - out_o).max() < 1e-2 * scale
    assert loss_g == pytest.approx(loss_o, rel=1e-2)
    for i, (w, b) in enumerate(_layer_slices()):
        for sl, name in ((w, "W"), (b, "b")):
            ref = g_o[sl]
            err = np.linalg.norm(g[sl] - ref) / max(np.linalg.norm(ref), 1e-30)
            assert err < 3e-2, (i, name, err)


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
