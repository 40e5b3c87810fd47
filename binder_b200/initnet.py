"""Learned initialiser of the registration (no counterpart in the reference).

A 3D convolutional encoder-decoder (channels 16-32-64-128) predicts, from a moving / fixed image
pair, the displacement on the grid of every 4th voxel; up-sampled to the full grid it seeds the
positions the EM starts from -- the reference's own hook for an initial deformation is the
final_locations argument of Registration (BINDER/FastRegistration.py:443-450).  The registration
has the last word: it runs to convergence from the seeded positions exactly as from the identity.

The network trains and runs on the library's hand-written kernels (binder_initnet_* in
include/binder_b200.h).  Training pairs are generated by this package itself, the way the
benchmark's phantoms are: random-ellipsoid phantoms warped by prior-sampled deformations, then
registered by the plain method (FP32 DCT passes, from the identity, to convergence) -- the
network learns the field the method itself converges to.

Recipe of the shipped checkpoint (binder_b200/data/initnet_seeded_64.npz: BF16 convolution
weights, FP32 biases):
    python -m binder_b200.initnet --seeded --pairs 2048 --steps 8000 --batch 8 --lr 5e-4 \
        --warmup 500 --evaluate 16 --out initnet_seeded_64.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import functools
import time

import numpy as np

from ._lib import check, lib

SIZE = 64             # training / inference grid (voxels per side)
COARSE = 4            # output spacing (voxels)
BINS = 64
GAMMA_INIT = 1e-6     # run_BINDER's default gamma, scaled as FastRegistration.py:412-417
ALPHA = 2.0
CONVERGENCE = 2.5e-5  # run_BINDER's default EM convergence threshold
MAX_EM = 400


class InitNet:
    """ctypes front of binder_initnet_*: batch x size^3 x 2 FP32 input (moving, fixed), batch x
    (size/4)^3 x 3 FP32 output (displacement in voxels)."""

    def __init__(self, batch=4, size=SIZE, seed=0, in_channels=2):
        self.batch, self.size, self.in_channels = int(batch), int(size), int(in_channels)
        self._h = C.c_void_p()
        check(lib().binder_initnet_create(C.byref(self._h), self.batch, self.size,
                                          self.in_channels, int(seed)))
        n = C.c_longlong(0)
        check(lib().binder_initnet_parameter_count(self._h, C.byref(n)))
        self.nparam = int(n.value)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binder_initnet_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self._h = C.c_void_p()

    def _in(self, x):
        x = np.ascontiguousarray(x, np.float32)
        if x.size != self.batch * self.size ** 3 * self.in_channels:
            raise ValueError(f"input must hold {self.batch} x {self.size}^3 x "
                             f"{self.in_channels} values")
        return x

    def _tgt(self, t):
        c = self.size // COARSE
        t = np.ascontiguousarray(t, np.float32)
        if t.size != self.batch * c ** 3 * 3:
            raise ValueError(f"target must hold {self.batch} x {c}^3 x 3 values")
        return t

    def get_parameters(self):
        out = np.empty(self.nparam, np.float32)
        check(lib().binder_initnet_get_parameters(self._h, out.ctypes.data))
        return out

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, np.float32).ravel()
        if p.size != self.nparam:
            raise ValueError(f"expected {self.nparam} parameters")
        check(lib().binder_initnet_set_parameters(self._h, p.ctypes.data))

    def predict(self, x):
        x = self._in(x)
        c = self.size // COARSE
        out = np.empty((self.batch, c, c, c, 3), np.float32)
        check(lib().binder_initnet_predict(self._h, x.ctypes.data, out.ctypes.data))
        return out

    def train_step(self, x, target, lr):
        x, t = self._in(x), self._tgt(target)
        loss = C.c_double(0)
        check(lib().binder_initnet_train_step(self._h, x.ctypes.data, t.ctypes.data, float(lr),
                                              C.byref(loss), None))
        return loss.value

    def gradients(self, x, target):
        x, t = self._in(x), self._tgt(target)
        g = np.empty(self.nparam, np.float32)
        loss = C.c_double(0)
        check(lib().binder_initnet_gradients(self._h, x.ctypes.data, t.ctypes.data,
                                             C.byref(loss), g.ctypes.data))
        return loss.value, g

    def _weight_mask(self):
        """True at the parameters that are convolution weights (False at the biases)"""
        from .initnet_layers import layer_table
        mask = np.zeros(self.nparam, bool)
        o = 0
        for cin, cout in layer_table(self.in_channels):
            mask[o:o + 27 * cin * cout] = True
            o += 27 * cin * cout + cout
        return mask

    def save(self, path, bf16_weights=False):
        """an .npz checkpoint; bf16_weights stores the convolution weights as BF16 -- exactly the
        operands the kernels use, so inference is unchanged -- at half the size"""
        p = self.get_parameters()
        meta = dict(size=self.size, in_channels=self.in_channels)
        if bf16_weights:
            m = self._weight_mask()
            u = p.view(np.uint32).astype(np.uint64)
            bits = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)
            np.savez_compressed(path, weights_bf16=bits[m], biases=p[~m], **meta)
        else:
            np.savez_compressed(path, params=p, **meta)

    def load(self, path):
        z = np.load(path)
        if int(z["size"]) != self.size or int(z["in_channels"]) != self.in_channels:
            raise ValueError("checkpoint was trained for another grid size or input")
        if "params" in z.files:
            self.set_parameters(z["params"])
            return
        m = self._weight_mask()
        p = np.empty(self.nparam, np.float32)
        p[m] = (z["weights_bf16"].astype(np.uint32) << 16).view(np.float32)
        p[~m] = z["biases"]
        self.set_parameters(p)


# ---- data ---------------------------------------------------------------------------------------
def network_input(pair):
    """[S, S, S, 2] FP32: moving and fixed intensities, each scaled to [0, 1] by its maximum"""
    mv = pair.moving.astype(np.float32)
    fx = pair.fixed.astype(np.float32)
    mv = mv / max(float(mv.max()), 1e-6)
    fx = np.clip(fx, 0.0, None) / max(float(fx.max()), 1e-6)
    return np.stack([mv, fx], -1)


def coarse_target(displacement, f=COARSE):
    """block means of a [S, S, S, 3] displacement over f^3 blocks: the [S/f]^3 x 3 target"""
    S = displacement.shape[0]
    c = S // f
    return displacement.reshape(c, f, c, f, c, f, 3).mean(axis=(1, 3, 5)).astype(np.float32)


def upsample_displacement(coarse, shape):
    """the coarse displacement on the full grid (order-1 resize on the GPU, the resampling
    FastRegistration.py:562-564 applies between resolutions)"""
    from . import _core
    return _core.resize_linear(np.asarray(coarse, np.float64), shape)


def make_pair(seed, size=SIZE):
    from . import phantoms
    return phantoms.make_pair((size,) * 3, seed, bins=BINS)


@functools.lru_cache(maxsize=8)
def grid_and_prior(shape):
    """the identity grid [*shape, 3] and the prior's DCT-domain field of a shape (FP32; callers
    do not modify them), computed once per shape: a batch of pairs of one size shares them"""
    from . import phantoms
    from .utils import initialize_fourier_domain_smoothing
    grid = phantoms.identity_positions(shape).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3).astype(np.float32)
    return grid, D


def registration(core, pair, init_displacement=None, precision=None):
    """a Registration of the pair from the identity grid, or from identity + init_displacement"""
    shape = tuple(int(s) for s in pair.u.shape)
    V = int(np.prod(shape))
    grid, D = grid_and_prior(shape)
    start = grid if init_displacement is None else \
        (grid + np.asarray(init_displacement, np.float32)).astype(np.float32)
    g = GAMMA_INIT * V
    reg = core.Registration(start, 1, grid, grid, *shape, *shape, 3,
                            float(np.count_nonzero(pair.u)))
    reg.setNonLinearTransformation(g, g, g, 1, 1, 1, 1, 1, 1, D)
    reg.setMILikelihood(ALPHA, np.full((BINS, BINS), 1.0 / BINS, np.float32), BINS, BINS, 1,
                        pair.v, pair.u)
    if precision is not None:
        reg.set_precision(precision)
    return reg


def refine(core, pair, init_displacement=None, precision=0, max_iter=MAX_EM, th=CONVERGENCE):
    """the plain method to convergence: (iterations, final displacement [S,S,S,3], final
    min-log-posterior per non-zero voxel, the Registration)"""
    from . import phantoms
    reg = registration(core, pair, init_displacement, precision)
    it = reg.EM(max_iter, th, 1, 0)
    fin = reg.get_final_locations_as_numpy_array().astype(np.float64)
    disp = fin - phantoms.identity_positions(pair.u.shape)
    mlp = float(reg.iteration_stats()[-1, 3] / np.count_nonzero(pair.u))
    return it, disp, mlp, reg


def negative_jacobians(core, reg, shape, correct=False):
    """negative Jacobian determinants of a registration's field; with correct=True after the
    topology correction the reference pipeline applies once EM is done (FastRegistration.py:
    527-546, its defaults e1 = 0.01, e2 = 100, 10 outer and 10 inner iterations), in place"""
    if correct:
        reg.correct_topology(0.01, 100.0, 10, 10, (1.0, 1.0, 1.0))
    pos = reg.get_final_locations_as_numpy_array().astype(np.float64)
    return int((core.compute_jacobian_determinant_3D(pos, *shape, 1, 1, 1) < 0).sum())


def _pair_job(args):
    """one phantom pair (module level, so a spawn pool can run it)"""
    return make_pair(*args)


def make_pairs(seeds, size=SIZE, workers=None):
    """phantom pairs for the seeds, generated on the host cores by a spawn pool"""
    import multiprocessing as mp
    import os
    jobs = [(int(sd), size) for sd in seeds]
    n = min(len(jobs), workers or os.cpu_count() or 1)
    if n <= 1:
        return [_pair_job(j) for j in jobs]
    with mp.get_context("spawn").Pool(n) as pool:
        return pool.map(_pair_job, jobs, chunksize=max(1, len(jobs) // (4 * n)))


EARLY_EM = 16  # EM iterations before the network, for the EM-seeded input


def early_em(core, pair, n=EARLY_EM):
    """the plain method's first n iterations from the identity: (Registration, displacement)"""
    from . import phantoms
    reg = registration(core, pair, None, 0)
    reg.EM(n, -1e300, 1, 0)
    fin = reg.get_final_locations_as_numpy_array().astype(np.float64)
    return reg, fin - phantoms.identity_positions(pair.u.shape)


def make_input(pair, early=None):
    """the network input of a pair: [S, S, S, 2] intensities, or [S, S, S, 5] with the early EM
    displacement appended (the EM-seeded form)"""
    x = network_input(pair)
    if early is None:
        return x
    return np.concatenate([x, np.asarray(early, np.float32)], -1)


def fill_input(out, pair, early):
    """make_input(pair, early) of the EM-seeded form written into out [S, S, S, 5] (a slot of a
    batch buffer), without the intermediate arrays"""
    mv = pair.moving
    fx = pair.fixed
    out[..., 0] = mv
    out[..., 0] /= max(float(mv.max()), 1e-6)
    np.clip(fx, 0.0, None, out=out[..., 1])
    out[..., 1] /= max(float(fx.max()), 1e-6)
    out[..., 2:] = early
    return out


def training_set(core, seeds, size=SIZE, seeded=False):
    """inputs and targets for the seeds' phantom pairs.  Plain form: input the two intensities,
    target the plain method's converged displacement (4^3 block means).  EM-seeded form: input
    also the displacement after EARLY_EM iterations, target the rest of the way (converged minus
    early)."""
    xs, ts = [], []
    for pair in make_pairs(seeds, size):
        if seeded:
            reg, early = early_em(core, pair)
            reg.EM(MAX_EM, CONVERGENCE, 1, 0)  # the same run, on to convergence
            from . import phantoms
            fin = reg.get_final_locations_as_numpy_array().astype(np.float64) - \
                phantoms.identity_positions(pair.u.shape)
            xs.append(make_input(pair, early))
            ts.append(coarse_target(fin - early))
        else:
            _, disp, _, _ = refine(core, pair)
            xs.append(make_input(pair))
            ts.append(coarse_target(disp))
    return np.stack(xs), np.stack(ts)


def predict_coarse(net, pair, early):
    """the network's coarse displacement [S/4, S/4, S/4, 3] for one pair (EM-seeded form)"""
    x = np.zeros((net.batch,) + tuple(pair.u.shape) + (net.in_channels,), np.float32)
    fill_input(x[0], pair, early)
    return net.predict(x)[0]


def learned_registration(core, net, pair, precision=3, max_iter=MAX_EM, th=CONVERGENCE):
    """registration seeded by the network: (total EM iterations, final displacement, final
    min-log-posterior per voxel, Registration).  EM-seeded networks (5 input channels): EARLY_EM
    plain iterations from the identity, the network's coarse prediction added to the positions
    of the same registration (add_displacement, order-1 resize), then EM to convergence with
    `precision` passes, theta carried on -- the run the training targets come from; the early
    iterations are counted."""
    if net.in_channels == 5:
        shape = tuple(int(s) for s in pair.u.shape)
        grid = grid_and_prior(shape)[0]
        reg = registration(core, pair, None, 0)
        reg.EM(EARLY_EM, -1e300, 1, 0)
        early = reg.get_final_locations_as_numpy_array() - grid
        reg.add_displacement(predict_coarse(net, pair, early))
        reg.set_precision(precision)
        it = reg.EM(max_iter, th, 1, 0)
        disp = reg.get_final_locations_as_numpy_array().astype(np.float64) - grid
        mlp = float(reg.iteration_stats()[-1, 3] / np.count_nonzero(pair.u))
        return EARLY_EM + it, disp, mlp, reg
    init = predict_displacement(net, pair)
    return refine(core, pair, init_displacement=init, precision=precision)


def train(net, xs, ts, steps, lr=1e-3, seed=0, log=None, warmup=200):
    """Adam on random mini-batches of the training set, the learning rate ramped up linearly over
    the first `warmup` steps and cosine-decayed after; returns the loss history"""
    rng = np.random.default_rng(seed)
    n = len(xs)
    hist = []
    for step in range(steps):
        idx = rng.choice(n, net.batch, replace=n < net.batch)
        # random flips of the three axes (the displacement component flips with its axis)
        x, t = xs[idx].copy(), ts[idx].copy()
        for a in range(3):
            if rng.random() < 0.5:
                x = np.flip(x, axis=1 + a)
                t = np.flip(t, axis=1 + a)
                t[..., a] = -t[..., a]
        cur = lr * (0.5 * (1 + np.cos(np.pi * step / max(1, steps))))  # cosine decay
        if step < warmup:
            cur *= (step + 1) / warmup
        hist.append(net.train_step(np.ascontiguousarray(x), np.ascontiguousarray(t), cur))
        if log and (step % 100 == 0 or step == steps - 1):
            log(f"step {step}: loss {hist[-1]:.5f}")
    return hist


def predict_displacement(net, pair, early=None):
    """the network's displacement for one pair, up-sampled to the full grid"""
    x1 = make_input(pair, early)
    x = np.zeros((net.batch,) + x1.shape, np.float32)
    x[0] = x1
    coarse = net.predict(x)[0]
    return upsample_displacement(coarse, pair.u.shape)


def main():
    from . import _core as core
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", required=True)
    ap.add_argument("--pairs", type=int, default=512)
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--seeded", action="store_true",
                    help="EM-seeded form: the input includes the displacement after EARLY_EM "
                         "iterations")
    ap.add_argument("--evaluate", type=int, default=0,
                    help="held-out pairs (seeds from 900000) to compare against zero "
                         "initialisation after training")
    a = ap.parse_args()
    t0 = time.time()
    xs, ts = training_set(core, range(a.seed, a.seed + a.pairs), seeded=a.seeded)
    print(f"{a.pairs} training pairs in {time.time() - t0:.1f} s", flush=True)
    net = InitNet(a.batch, SIZE, a.seed, in_channels=xs.shape[-1])
    t0 = time.time()
    hist = train(net, xs, ts, a.steps, a.lr, a.seed, log=lambda s: print(s, flush=True),
                 warmup=a.warmup)
    print(f"{a.steps} steps in {time.time() - t0:.1f} s; mean loss of the first / last 200 "
          f"steps {np.mean(hist[:200]):.5f} / {np.mean(hist[-200:]):.5f}", flush=True)
    net.save(a.out, bf16_weights=True)
    if a.evaluate:
        ev = InitNet(1, SIZE, 0, in_channels=xs.shape[-1])
        ev.load(a.out)
        rows = []
        for pair in make_pairs(range(900000, 900000 + a.evaluate)):
            it0, _, mlp0, _ = refine(core, pair, precision=0)
            it1, _, mlp1, _ = learned_registration(core, ev, pair)
            rows.append((it0, it1, mlp0, mlp1))
        r = np.array(rows)
        print("held-out: EM iterations %.1f (zero initialisation, FP32 passes) -> %.1f (learned, "
              "BF16 passes); final min-log-posterior per voxel %.5f -> %.5f" % tuple(r.mean(0)),
              flush=True)
        print("per pair (zero, learned):", r[:, :2].astype(int).tolist(), flush=True)


if __name__ == "__main__":
    main()
