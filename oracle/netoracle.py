"""FP64 CPU restatement of the learned initialiser's network (TEST INFRASTRUCTURE ONLY): forward
pass, mean-squared-error loss and the gradient of every parameter, by numpy.  With round=True it
rounds where the GPU kernels round (BF16 network input, BF16 weights, BF16 activations after each
leaky ReLU / pooling / skip sum, BF16 output gradients as GEMM operands), so the GPU gradients can
be compared with it at FP32-accumulation accuracy; with round=False it is the exact FP64 network,
whose gradients a finite-difference test checks.

Layout (binder_initnet_* in include/binder_b200.h): activations [B, S, S, S, C] channels last;
per layer W [Cout, 27 * Cin] (tap = (dx * 3 + dy) * 3 + dz over offsets -1..1, then Cin) and
b [Cout], concatenated in forward order.
"""
from __future__ import annotations

import numpy as np

SLOPE = 0.1
# (Cin, Cout, level, leaky ReLU): level l has spatial size S / 2^l
LAYERS = [(2, 16, 0, 1), (16, 16, 0, 1), (16, 32, 1, 1), (32, 32, 1, 1), (32, 64, 2, 1),
          (64, 64, 2, 1), (64, 128, 3, 1), (128, 128, 3, 1), (128, 64, 2, 1), (64, 64, 2, 1),
          (64, 3, 2, 0)]


def bf16(a):
    """round to BF16 (nearest, ties to even) and back, as FP64"""
    a32 = np.ascontiguousarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(in_channels=2):
    """the layer table for a network with `in_channels` input channels"""
    return [(in_channels,) + LAYERS[0][1:]] + LAYERS[1:]


def unpack(params, in_channels=2):
    """[(W [Cout, 27 Cin], b [Cout]), ...] from the flat parameter vector"""
    out, o = [], 0
    for cin, cout, _, _ in layers(in_channels):
        W = np.asarray(params[o:o + 27 * cin * cout], np.float64).reshape(cout, 27 * cin)
        o += 27 * cin * cout
        b = np.asarray(params[o:o + cout], np.float64)
        o += cout
        out.append((W, b))
    assert o == len(params)
    return out


def im2col(x):
    """[B, S, S, S, C] -> [B, S, S, S, 27, C]: the 27 neighbours (zero outside), tap-major"""
    S = x.shape[1]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))
    return np.stack([xp[:, a:a + S, b:b + S, c:c + S, :]
                     for a in range(3) for b in range(3) for c in range(3)], axis=4)


def col2im(dcol):
    """adjoint of im2col: [B, S, S, S, 27, C] -> [B, S, S, S, C]"""
    S = dcol.shape[1]
    dxp = np.zeros((dcol.shape[0], S + 2, S + 2, S + 2, dcol.shape[-1]))
    t = 0
    for a in range(3):
        for b in range(3):
            for c in range(3):
                dxp[:, a:a + S, b:b + S, c:c + S, :] += dcol[:, :, :, :, t, :]
                t += 1
    return dxp[:, 1:-1, 1:-1, 1:-1, :]


def pool(x):
    B, S, _, _, C = x.shape
    return x.reshape(B, S // 2, 2, S // 2, 2, S // 2, 2, C).mean(axis=(2, 4, 6))


def pool_back(dy):
    return np.repeat(np.repeat(np.repeat(dy, 2, 1), 2, 2), 2, 3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 1), 2, 2), 2, 3)


def up_back(dy):
    B, T, _, _, C = dy.shape
    return dy.reshape(B, T // 2, 2, T // 2, 2, T // 2, 2, C).sum(axis=(2, 4, 6))


def forward_backward(params, x, target=None, round=True):
    """(output [B, S/4, S/4, S/4, 3], loss, gradient [n params]) of the network on input x
    [B, S, S, S, 2]; loss and gradient are None without a target"""
    R = bf16 if round else (lambda a: np.asarray(a, np.float64))
    lay = unpack(params, x.shape[-1])
    cache = []

    def conv(i, xin):
        W, b = lay[i]
        _, _, _, act = LAYERS[i]
        col = im2col(xin)
        z = col.reshape(col.shape[:4] + (-1,)) @ R(W).T + b
        y = R(np.where(z > 0, z, SLOPE * z)) if act else z
        cache.append((i, xin, col, z))
        return y

    x0 = R(x)
    a0 = conv(0, x0)
    e0 = conv(1, a0)
    p0 = R(pool(e0))
    a1 = conv(2, p0)
    e1 = conv(3, a1)
    p1 = R(pool(e1))
    a2 = conv(4, p1)
    e2 = conv(5, a2)
    p2 = R(pool(e2))
    a3 = conv(6, p2)
    e3 = conv(7, a3)
    u3 = up(e3)
    d2a = conv(8, u3)
    s2 = R(d2a + e2)
    d2b = conv(9, s2)
    out = conv(10, d2b)
    if target is None:
        return out, None, None
    n = out.size
    diff = out - np.asarray(target, np.float64)
    loss = float((diff * diff).sum() / n)
    grads = [None] * len(LAYERS)
    by_layer = {c[0]: c for c in cache}

    def back(i, dy, want_dx=True):
        _, xin, col, z = by_layer[i]
        W, _ = lay[i]
        act = LAYERS[i][3]
        dz = np.where(z > 0, dy, SLOPE * dy) if act else dy
        dzr = R(dz)
        flat = col.reshape(-1, col.shape[4] * col.shape[5])
        gW = dzr.reshape(-1, dz.shape[-1]).T @ flat
        gb = dz.reshape(-1, dz.shape[-1]).sum(0)
        grads[i] = (gW, gb)
        if not want_dx:
            return None
        dcol = (dzr @ R(W)).reshape(dz.shape[:4] + (27, xin.shape[-1]))
        return col2im(dcol)

    d_out = 2.0 * diff / n
    d_d2b = back(10, d_out)
    d_s2 = back(9, d_d2b)
    d_u3 = back(8, d_s2)
    d_e3 = up_back(d_u3)
    d_a3 = back(7, d_e3)
    d_p2 = back(6, d_a3)
    d_e2 = pool_back(d_p2) + d_s2
    d_a2 = back(5, d_e2)
    d_p1 = back(4, d_a2)
    d_e1 = pool_back(d_p1)
    d_a1 = back(3, d_e1)
    d_p0 = back(2, d_a1)
    d_e0 = pool_back(d_p0)
    d_a0 = back(1, d_e0)
    back(0, d_a0, want_dx=False)
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return out, loss, flat
