"""Stage runner for profilers: one stage of the EM iteration of a registration of a seeded
phantom pair, run a few times after a warm-up, with the device time per run printed.

    python -m binder_b200.stageprof --stage estep --n 3
    python -m binder_b200.stageprof --stage mstep --precision 3 --n 2

The pair is the benchmark's 3D MI workload by default (160x192x160, 64 bins, seed 20260001, a
3-voxel-RMS prior-sampled warp; ``binder_b200/phantoms.py``); a profiler such as ncu captures the
stage's kernels of one run (``-k`` with the kernel's name, ``-s`` past the warm-up).  Stages:
``estep`` (the E-step kernel), ``mstep`` (the DCT M-step's passes), ``em`` (whole EM iterations,
captured as CUDA graphs), ``sampler`` (Gibbs sweeps of a batch of chains, every sampling switch on,
after 10 EM iterations; ``--chains``).  No counterpart in the reference.
"""
from __future__ import annotations

import argparse

import numpy as np

GAMMA_INIT = 1e-6  # run_BINDER's default gamma, per voxel of a 1 mm grid
ALPHA = 2.0


def make_registration(core, shape, bins, seed):
    from . import phantoms
    from .utils import initialize_fourier_domain_smoothing
    pair = phantoms.make_pair(shape, seed, bins=bins)
    V = int(np.prod(shape))
    grid = phantoms.identity_positions(shape).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3).astype(np.float32)
    g = GAMMA_INIT * V
    reg = core.Registration(grid, 1, grid, grid, *shape, *shape, 3,
                            float(np.count_nonzero(pair.u)))
    reg.setNonLinearTransformation(g, g, g, 1, 1, 1, 1, 1, 1, D)
    reg.setMILikelihood(ALPHA, np.full((bins, bins), 1.0 / bins, np.float32), bins, bins, 1,
                        pair.v, pair.u)
    return reg


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--stage", choices=["estep", "mstep", "em", "sampler"], default="estep")
    ap.add_argument("--chains", type=int, default=32, help="chains of the sampler stage")
    ap.add_argument("--shape", type=int, nargs=3, default=[160, 192, 160])
    ap.add_argument("--bins", type=int, default=64)
    ap.add_argument("--seed", type=int, default=20260001)
    ap.add_argument("--precision", type=int, default=None,
                    help="DCT pass format (0 FP32, 1 3xTF32, 2 TF32, 3 BF16 split, 4 BF16)")
    ap.add_argument("--hist-precision", type=int, default=0,
                    help="E-step bin columns (0 FP32, 1 FP16)")
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--n", type=int, default=3, help="timed runs of the stage")
    a = ap.parse_args(argv)
    from . import _core as core
    reg = make_registration(core, tuple(a.shape), a.bins, a.seed)
    if a.precision is not None:
        reg.set_precision(a.precision)
    reg.set_histogram_precision(a.hist_precision)
    if a.stage == "sampler":
        reg.EM(10, -1e300, 1, 0)
        reg.sampler_chains(1, a.chains, 1, 1, 1, 1, 1, 1, 1, per_chain=False)  # warm-up
        for _ in range(a.n):
            reg.sampler_chains(7, a.chains, 4, 16, 1, 1, 1, 1, 1, per_chain=False)
            ms = reg.last_elapsed_ms()
            print(f"sampler: {ms / 20:.4f} ms per sweep of {a.chains} chains", flush=True)
        return
    if a.stage == "em":
        reg.EM(a.warmup, -1e300, 1, 0)
        for _ in range(a.n):
            reg.reset()
            reg.EM(8, -1e300, 1, 0)
            print(f"em: {reg.last_elapsed_ms() / 8:.4f} ms per iteration", flush=True)
        return
    stage = 0 if a.stage == "estep" else 1
    reg.profile_stage(stage, a.warmup)
    for _ in range(a.n):
        print(f"{a.stage}: {reg.profile_stage(stage, 1):.4f} ms", flush=True)


if __name__ == "__main__":
    main()
