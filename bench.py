#!/usr/bin/env python
"""Throughput of BINDER's registration hot path on B200.

Workload (one "step" = one registration of one image pair): the 160x192x160 synthetic 3D MI
pair (40 random ellipsoids, blur 1, noise 0.02; moving = prior-sampled warp with 3-voxel RMS and
5-voxel correlation + monotone 8-knot LUT; 64 robust bins), registered at full resolution by 50
EM iterations (E-step, theta update, DCT-prior M-step; convergence test disabled so every step
does the same work) followed by topology correction (e1 = 0.01, e2 = 100, 10/10 iterations).
Inputs are seeded synthetic volumes standing in for the reference's unpublished data.

  value : registrations/s with inputs resident in HBM (device-timed with CUDA events on the
          engine's stream; each step restores the initial positions device-to-device)
  e2e   : the same through the public API with host buffers: create the Registration from host
          arrays, set likelihood/prior, EM, topology correction, read the final field back.

`--impl reference` times the reference's own CPU implementation (BINDER/src/cpu's EM driver and
classes, compiled in oracle/_ref with FFT-based DCTs in place of FFTW; OpenMP over all host cores)
on a bounded sample of the same workload, or the FP64 oracle port where that library is absent.  Under torchrun every rank
registers its own pair (replicas; no data-path collective) and rank 0 reports the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SHAPE = (160, 192, 160)
BINS = 64
SEED = 20260001
EM_ITERS = 50
TOPO = dict(e1=0.01, e2=100.0, max_outer=10, max_inner=10)
GAMMA_INIT = 1e-6  # run_BINDER default (cli/run_BINDER.py), scaled as FastRegistration.py:412-417
ALPHA = 2.0
# compulsory HBM bytes per voxel of one E-step launch with this layout: positions in (12), fixed
# bin (1), dream displacement out (12), padded moving-bin volume read once (~1.1)
ESTEP_BYTES_PER_VOXEL = 26.0


GIBBS_SHAPE = (96, 96, 96)
GIBBS_CHAINS = 32
GIBBS_BURN, GIBBS_SAMPLES = 20, 80  # sweeps per chain in the timed window
GIBBS_SEED = 1000
# compulsory HBM bytes per voxel of one post-burn-in sweep: E-step (positions 12, bins ~2, dream
# 12), M-step (dream 12, positions 12), FP64 Welford (positions 12, mean 24 x 2, M2 48 x 2) ~ 210
GIBBS_BYTES_PER_VOXEL = 210.0


def run_gibbs(core, rank, chains, dist):
    """Gibbs sweeps/s: `chains` chains of GIBBS_BURN + GIBBS_SAMPLES sweeps on a 96^3 MI pair (64
    bins) after 10 EM iterations, all chains in one batch (sampler_chains: every kernel of a sweep
    launched once for all chains; Philox chain index = chain number).  value: device time of the
    batch call (CUDA events on the engine stream); e2e: the call through the public API with the
    chains' pooled FP64 mean / covariance read back.  For comparison the same chains run one
    sampler call after another (the reference's one-chain-per-object shape)."""
    from binder_b200 import phantoms
    from binder_b200.replicas import unit_seed
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape = GIBBS_SHAPE
    V = int(np.prod(shape))
    pair = phantoms.make_pair(shape, unit_seed(GIBBS_SEED, rank), bins=BINS)
    grid = phantoms.identity_positions(shape).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3).astype(np.float32)
    g = GAMMA_INIT * V
    reg = core.Registration(grid, 1, grid, grid, *shape, *shape, 3, float(np.count_nonzero(pair.u)))
    reg.setNonLinearTransformation(g, g, g, 1, 1, 1, 1, 1, 1, D)
    reg.setMILikelihood(ALPHA, np.full((BINS, BINS), 1.0 / BINS, np.float32), BINS, BINS, 1,
                        pair.v, pair.u)
    reg.EM(10, -1e300, 1, 0)
    start = reg.get_final_locations_as_numpy_array().astype(np.float64)
    theta = reg.get_likelihood_parameters()[: BINS * BINS].astype(np.float64)
    sweeps_per_chain = GIBBS_BURN + GIBBS_SAMPLES
    seed = unit_seed(GIBBS_SEED, rank)
    reg.sampler_chains(seed, chains, 2, 3, 1, 1, 1, 1, 1, per_chain=False)  # warm-up
    barrier(dist)
    reg.sampler_chains(seed, chains, GIBBS_BURN, GIBBS_SAMPLES, 1, 1, 1, 1, 1, per_chain=False,
                       pooled=False)
    dev_ms = max_over_ranks(reg.last_elapsed_ms(), dist)
    t0 = time.perf_counter()
    reg.sampler_chains(seed, chains, GIBBS_BURN, GIBBS_SAMPLES, 1, 1, 1, 1, 1, per_chain=False)
    wall = max_over_ranks(time.perf_counter() - t0, dist)
    # the same chains one call after another
    seq_ms = 0.0
    n_seq = min(chains, 4)
    for c in range(n_seq):
        reg.set_chain(c)
        reg.sampler(seed, GIBBS_BURN, GIBBS_SAMPLES, 1, 1, 1, 1, 1)
        seq_ms += reg.last_elapsed_ms()
        reg.reset()
    world = dist.get_world_size() if dist is not None else 1
    sweeps = world * chains * sweeps_per_chain
    hbm = hbm_peak()[0]
    achieved = GIBBS_BYTES_PER_VOXEL * V * chains * sweeps_per_chain / (dev_ms * 1e-3) / 1e9
    cpu = cpu_gibbs(pair, start, theta, D, g) if rank == 0 else None
    return {"metric": f"Gibbs sweeps/s (96x96x96 MI pair, 64 bins, {chains} chains x "
                      f"{sweeps_per_chain} sweeps in one batch, all sampling switches on)",
            "value": sweeps / (dev_ms / 1e3), "unit": "sweeps/s", "higher_is_better": True,
            "ms_per_sweep": dev_ms / (chains * sweeps_per_chain),
            "ms_per_batch_sweep": dev_ms / sweeps_per_chain,
            "sequential_chains_sweeps_per_s": n_seq * sweeps_per_chain / (seq_ms / 1e3),
            "e2e": {"value": sweeps / wall, "unit": "sweeps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(V * 12 * 8)},
            "roofline": {"bound": "hbm", "bytes_per_voxel_sweep": GIBBS_BYTES_PER_VOXEL,
                         "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm},
            "sample_moments": "FP64 Welford per chain, pooled mean [V,3] + covariance [V,3,3]",
            "cpu_baseline": cpu}


REF_NOTE = ("the reference's own CPU sources (BINDER/src/cpu: Registration.cpp and the classes it "
            "drives) compiled in oracle/_ref, with FFT-based DCTs in place of FFTW")


def ref_lib():
    """The reference's CPU sources compiled in oracle/_ref, or None where that library is absent
    (the CPU legs then time the FP64 oracle port instead)."""
    from oracle import pyoracle
    try:
        return pyoracle.ref_lib()
    except OSError:
        return None


class stdout_to_stderr:
    """The reference prints progress on stdout; this script's stdout carries one JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def cpu_gibbs(pair, start, theta, D, g, sweeps=3):
    """Sweeps/s of the reference's own sampler (Registration::sampler, all host cores) on the same
    96^3 pair from the same state as the GPU chains (the positions and theta after the 10 EM
    iterations), or of the FP64 oracle sampler where the reference library is absent."""
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    shape = GIBBS_SHAPE
    x = phantoms_grid(shape)
    R = ref_lib()
    if R is not None:
        with stdout_to_stderr():
            _, _, t = pyoracle.ref_sampler(R, start, x, D.astype(np.float64), (g, g, g), shape,
                                           pair.v, pair.u, ALPHA, theta.reshape(BINS, BINS),
                                           GIBBS_SEED, 0, sweeps, threads=threads)
        return {"value": sweeps / t, "unit": "sweeps/s", "cores": threads, "kind": "reference",
                "sample": f"{sweeps} sweeps (every switch on) of the 96^3 pair from the GPU chains' "
                          f"start state ({t:.2f} s) by {REF_NOTE}"}
    pyoracle.set_threads(threads)
    t0 = time.perf_counter()
    pyoracle.sampler(start, start, x, pair.u, pair.v, theta, ALPHA, D.astype(np.float64),
                     (g, g, g), math.sqrt(9.0 / (8.0 * math.pi)), (1.0, 1.0, 1.0),
                     (1.0, 1.0, 1.0), shape, shape, BINS, BINS, GIBBS_SEED, 0, sweeps, 1, 1, 1,
                     1, 1)
    t = time.perf_counter() - t0
    return {"value": sweeps / t, "unit": "sweeps/s", "cores": threads, "kind": "port",
            "sample": f"{sweeps} sweeps of the 96^3 pair from the GPU chains' start state "
                      f"({t:.2f} s)"}


def phantoms_grid(shape):
    from binder_b200 import phantoms
    return phantoms.identity_positions(shape).astype(np.float64)


C4_PAIRS = 64
C4_SIDES = (48, 160)
C4_SEED = 4242


def _c4_pair(args):
    """one pair of the batch (a module-level function, so a spawn pool can run it)"""
    shape, seed = args
    from binder_b200 import phantoms
    return phantoms.make_pair(tuple(int(x) for x in shape), int(seed), bins=BINS)


def c4_shapes():
    rng = np.random.default_rng(C4_SEED)
    return [tuple(int(v) for v in rng.integers(C4_SIDES[0], C4_SIDES[1] + 1, 3))
            for _ in range(C4_PAIRS)]


def run_batch(core, rank, em_iters, dist):
    """Batched serving-style workload: 64 phantom pairs of uneven sizes (sides uniform in
    48..160, seed 4242), each registered by em_iters EM iterations, all pairs in one batch
    (RegistrationBatch: one graph per EM chunk, every pair on a branch of its own; launch shapes
    per size class from the autotuner).  value: pairs/s by device time; compared with the same
    registrations one after another (each pair's own EM calls)."""
    import multiprocessing as mp
    import tempfile

    from binder_b200 import autotune
    from binder_b200.initnet import registration
    shapes = c4_shapes()
    work = [(s, C4_SEED + i + 1000 * rank) for i, s in enumerate(shapes)]
    with mp.get_context("spawn").Pool(min(len(work), os.cpu_count() or 1)) as pool:
        pairs = pool.map(_c4_pair, work)
    regs = [registration(core, p) for p in pairs]
    # one by one
    seq_ms = 0.0
    for r in regs:
        r.EM(em_iters, -1e300, 1, 0)
        r.reset()
        r.EM(em_iters, -1e300, 1, 0)
        seq_ms += r.last_elapsed_ms()
        r.reset()
    cache = os.path.join(tempfile.gettempdir(), "binder_b200_autotune.json")
    table = autotune.tune(core, regs, shapes, cache=cache, retune=True)
    batch = core.RegistrationBatch(regs)
    batch.EM(em_iters, -1e300, 1)  # warm-up
    for r in regs:
        r.reset()
    barrier(dist)
    its = batch.EM(em_iters, -1e300, 1)
    ms = max_over_ranks(batch.last_ms, dist)
    world = dist.get_world_size() if dist is not None else 1
    voxels = int(sum(np.prod(s) for s in shapes))
    return {"metric": f"batched registrations/s ({C4_PAIRS} MI pairs, sides 48..160, 64 bins, "
                      f"{em_iters} EM iterations each, one batch)",
            "value": world * C4_PAIRS / (ms / 1e3), "unit": "pairs/s", "higher_is_better": True,
            "ms_per_batch": ms, "one_by_one_pairs_per_s": C4_PAIRS / (seq_ms / 1e3),
            "speedup_vs_one_by_one": seq_ms / ms, "total_voxels": voxels,
            "iterations": sorted(set(int(i) for i in its)), "autotune": table}


INITNET_CKPT = os.path.join(ROOT, "binder_b200", "data", "initnet_seeded_64.npz")
LEARNED_PAIRS = 8


def run_learned(core, rank, dist):
    """The metric's comparison with the learned initialiser (64^3 held-out pairs, seeds
    900000.., the reference CLI's convergence rule): the plain FP32 method from the identity
    against the committed EM-seeded network + BF16-split passes (16 plain iterations, the
    network, then EM to convergence).  Device time of every EM call (CUDA events) plus the
    network's inference (CUDA events around it); the two arms' iterations, final
    min-log-posterior per voxel and negative Jacobians."""
    import torch
    from binder_b200 import initnet as I
    if not os.path.exists(INITNET_CKPT):
        return None
    net = I.InitNet(1, I.SIZE, 0, in_channels=5)
    net.load(INITNET_CKPT)
    pairs = I.make_pairs(range(900000 + 1000 * rank, 900000 + 1000 * rank + LEARNED_PAIRS))
    # warm-up of both paths
    I.refine(core, pairs[0], precision=0, max_iter=8)
    I.learned_registration(core, net, pairs[0])
    plain_ms = learned_ms = 0.0
    its0, its1, mlp0, mlp1, neg0, neg1 = [], [], [], [], [], []
    for pair in pairs:
        shape = tuple(int(x) for x in pair.u.shape)
        it, d, mlp, reg = I.refine(core, pair, precision=0)
        plain_ms += reg.last_elapsed_ms()
        its0.append(it), mlp0.append(mlp)
        neg0.append((I.negative_jacobians(core, reg, shape),
                     I.negative_jacobians(core, reg, shape, correct=True)))
        # learned: early EM, the network's prediction added on the device, EM to convergence on
        # the same registration; the EM calls device-timed, the network step by CUDA events
        reg = I.registration(core, pair, None, 0)
        reg.EM(I.EARLY_EM, -1e300, 1, 0)
        ms = reg.last_elapsed_ms()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        early = reg.get_final_locations_as_numpy_array() - I.grid_and_prior(shape)[0]
        reg.add_displacement(I.predict_coarse(net, pair, early))
        e1.record()
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
        reg.set_precision(3)
        it = reg.EM(I.MAX_EM, I.CONVERGENCE, 1, 0)
        ms += reg.last_elapsed_ms()
        mlp = float(reg.iteration_stats()[-1, 3] / np.count_nonzero(pair.u))
        learned_ms += ms
        its1.append(I.EARLY_EM + it), mlp1.append(mlp)
        neg1.append((I.negative_jacobians(core, reg, shape),
                     I.negative_jacobians(core, reg, shape, correct=True)))
    plain_ms = max_over_ranks(plain_ms, dist)
    learned_ms = max_over_ranks(learned_ms, dist)
    n = len(pairs)
    return {"metric": "64^3 registrations/s to convergence (held-out pairs): learned init + BF16 "
                      "against plain FP32 from the identity",
            "plain_fp32": {"registrations_per_s": n / (plain_ms / 1e3),
                           "mean_iterations": float(np.mean(its0)),
                           "mean_final_mlp_per_voxel": float(np.mean(mlp0)),
                           "negative_jacobians_after_em": int(sum(c[0] for c in neg0)),
                           "negative_jacobians_after_topology_correction":
                               int(sum(c[1] for c in neg0))},
            "learned_bf16": {"registrations_per_s": n / (learned_ms / 1e3),
                             "mean_iterations": float(np.mean(its1)),
                             "mean_final_mlp_per_voxel": float(np.mean(mlp1)),
                             "negative_jacobians_after_em": int(sum(c[0] for c in neg1)),
                             "negative_jacobians_after_topology_correction":
                                 int(sum(c[1] for c in neg1))},
            "speedup": plain_ms / learned_ms, "pairs": n,
            "note": "inference time of the network included in the learned arm; the network "
                    "input includes the displacement after 16 plain EM iterations; negative "
                    "Jacobians counted after EM and after the topology correction the "
                    "reference pipeline applies next (e1 0.01, e2 100, 10/10 iterations, not "
                    "timed)"}


TARGET_PAIRS = 32
TARGET_SEED0 = 900100  # held-out: the network never saw these seeds


def run_target(core, rank, dist):
    """The metric's comparison as a whole, on held-out 64^3 pairs: the plain FP32 GPU path (one
    registration after another, zero initialisation, FP32 CUDA-core passes) against the
    learned-init + mixed-precision + batched path (16 early EM iterations for all pairs as one
    batch, the network's prediction in batches of 8 added to each registration's positions on
    the device, then every pair's EM to convergence in the same batch with BF16-split passes and
    autotuned launch shapes).  Both arms timed end to end with
    CUDA events around the whole set (registration set-up from host arrays, EM, read-back, and for
    the learned arm the network's input building and inference), the reference CLI's convergence
    rule; final min-log-posterior and negative Jacobians (after EM, and after the topology
    correction the reference pipeline applies next) per arm."""
    import tempfile

    import torch
    from binder_b200 import autotune
    from binder_b200 import initnet as I
    if not os.path.exists(INITNET_CKPT):
        return None
    seeds = range(TARGET_SEED0 + 1000 * rank, TARGET_SEED0 + 1000 * rank + TARGET_PAIRS)
    pairs = I.make_pairs(seeds)
    shape = tuple(int(x) for x in pairs[0].u.shape)
    nb = 8
    net = I.InitNet(nb, I.SIZE, 0, in_channels=5)
    net.load(INITNET_CKPT)
    cache = os.path.join(tempfile.gettempdir(), "binder_b200_autotune_64.json")

    def plain():
        out = []
        for p in pairs:
            r = I.registration(core, p, None, 0)
            it = r.EM(I.MAX_EM, I.CONVERGENCE, 1, 0)
            out.append((it, r))
        return out

    grid32 = I.grid_and_prior(shape)[0]  # the identity grid, shared by both arms
    xs = np.zeros((nb,) + shape + (5,), np.float32)

    tuned = {}

    def learned(retune=False):
        regs = [I.registration(core, p, None, 3) for p in pairs]
        tuned.update(autotune.tune(core, regs, [shape] * len(regs), cache=cache,
                                   retune=retune))
        batch = core.RegistrationBatch(regs)
        batch.EM(I.EARLY_EM, -1e300, 1)
        for b in range(0, len(pairs), nb):
            for j, (p, r) in enumerate(zip(pairs[b:b + nb], regs[b:b + nb])):
                I.fill_input(xs[j], p, r.get_final_locations_as_numpy_array() - grid32)
            pred = net.predict(xs)
            for j, r in enumerate(regs[b:b + nb]):
                r.add_displacement(pred[j])
        its = batch.EM(I.MAX_EM, I.CONVERGENCE, 1)
        return [(I.EARLY_EM + int(i), r) for i, r in zip(its, regs)]

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        barrier(dist)
        e0.record()
        res = fn()
        for _, r in res:
            r.get_final_locations_as_numpy_array()
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), dist), res

    learned(retune=True)  # warm-up (graph capture, the autotuner's timing, first launches)
    plain_ms, res0 = timed(plain)
    learned_ms, res1 = timed(learned)

    def summary(ms, res):
        n = len(res)
        mlp = [float(r.iteration_stats()[-1, 3] / np.count_nonzero(p.u))
               for (_, r), p in zip(res, pairs)]
        neg = [I.negative_jacobians(core, r, shape) for _, r in res]
        negc = [I.negative_jacobians(core, r, shape, correct=True) for _, r in res]
        world = dist.get_world_size() if dist is not None else 1
        return {"registrations_per_s": world * n / (ms / 1e3), "ms": ms,
                "mean_iterations": float(np.mean([i for i, _ in res])),
                "mean_final_mlp_per_voxel": float(np.mean(mlp)),
                "negative_jacobians_after_em": int(sum(neg)),
                "negative_jacobians_after_topology_correction": int(sum(negc))}

    a, b = summary(plain_ms, res0), summary(learned_ms, res1)
    return {"metric": f"64^3 registrations/s to convergence, {TARGET_PAIRS} held-out MI pairs: "
                      "learned init + BF16 split + batched against the plain FP32 GPU path",
            "plain_fp32_one_by_one": a, "learned_bf16_batched": b,
            "speedup": plain_ms / learned_ms,
            "mlp_rel_diff": (b["mean_final_mlp_per_voxel"] - a["mean_final_mlp_per_voxel"]) /
                            a["mean_final_mlp_per_voxel"],
            "autotune": tuned,
            "note": "end to end per arm: set-up from host arrays, EM to the convergence rule "
                    "(th 2.5e-5, at most 400 iterations), read-back; the learned arm adds its 16 "
                    "early iterations (counted in its iterations), the network input and "
                    "inference; the topology correction after EM is not timed"}


C1_SHAPE = (128, 128)
C1_BINS = 32
C1_SEED = 12345
C1_REPS = 20  # registrations per timed window


def run_2d(core, rank, em_iters, dist):
    """2D registrations/s on the 128x128 MI pair (12 ellipses, blur 1.5, moving = prior-sampled
    2-pixel-RMS warp + monotone LUT, 32 robust bins): em_iters EM iterations + 2D topology
    correction per registration, C1_REPS registrations per window.  Device-timed on the engine
    stream (positions restored device-to-device); e2e creates every registration from pinned
    host buffers and reads the field back."""
    import torch
    from binder_b200 import phantoms
    from binder_b200.replicas import unit_seed
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape = C1_SHAPE
    V = int(np.prod(shape))
    pair = phantoms.make_pair(shape, unit_seed(C1_SEED, rank), bins=C1_BINS, rms=2.0, spacing=8.0)
    grid = np.ascontiguousarray(phantoms.identity_positions(shape).astype(np.float32))
    D = initialize_fourier_domain_smoothing(shape, True, 2, 2).astype(np.float32)
    g = GAMMA_INIT * V
    theta = np.full((C1_BINS, C1_BINS), 1.0 / C1_BINS, np.float32)
    nzv = float(np.count_nonzero(pair.u))

    def make():
        r = core.Registration(grid, 1, grid, grid, *shape, 1, *shape, 1, 3, nzv)
        r.setNonLinearTransformation(g, g, g, 1, 1, 1, 1, 1, 1, D)
        r.setMILikelihood(ALPHA, theta, C1_BINS, C1_BINS, 1, pair.v, pair.u)
        return r

    reg = make()
    stream = torch.cuda.ExternalStream(reg.stream())

    def one():
        reg.reset()
        reg.EM(em_iters, -1e300, 1, 0)
        reg.correct_topology(TOPO["e1"], TOPO["e2"], TOPO["max_outer"], TOPO["max_inner"],
                             [1.0, 1.0])

    for _ in range(3):
        one()
    torch.cuda.synchronize()
    barrier(dist)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(C1_REPS):
        one()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    del reg

    def e2e_one():
        r = make()
        r.EM(em_iters, -1e300, 1, 0)
        r.correct_topology(TOPO["e1"], TOPO["e2"], TOPO["max_outer"], TOPO["max_inner"],
                           [1.0, 1.0])
        return r.get_final_locations_as_numpy_array()

    e2e_one()
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(C1_REPS):
        e2e_one()
    wall = max_over_ranks(time.perf_counter() - t0, dist)
    world = dist.get_world_size() if dist is not None else 1
    cpu = None
    if rank == 0:
        from oracle import pyoracle
        threads = os.cpu_count() or 1
        vshape = shape + (1,)
        it = em_iters
        R = ref_lib()
        if R is not None:
            tm = []
            with stdout_to_stderr():
                pyoracle.ref_em(R, grid, grid, D, (g, g, g), vshape, vshape, pair.v, pair.u, it,
                                mi=(ALPHA, theta.reshape(C1_BINS, C1_BINS)), non_zero_voxels=nzv,
                                threads=threads, timing=tm)
            t, kind, who = tm[0], "reference", f" by {REF_NOTE}"
        else:
            pyoracle.set_threads(threads)
            t0 = time.perf_counter()
            pyoracle.em(grid, grid, pair.u, pair.v, theta, ALPHA, D, (g, g, g),
                        math.sqrt(9.0 / (8.0 * math.pi)), vshape, vshape, C1_BINS, C1_BINS, nzv,
                        it, -1e300)
            t, kind, who = time.perf_counter() - t0, "port", ""
        cpu = {"value": 1.0 / t, "unit": "registrations/s", "cores": threads,
               "kind": kind, "sample": f"{it} EM iterations of the 128x128 pair ({t:.2f} s)"
                                       f"{who}, topology excluded"}
    h2d = grid.nbytes + D.nbytes + theta.nbytes + pair.u.nbytes + pair.v.nbytes
    return {"metric": f"2D registrations/s (128x128 MI pair, 32 bins, {em_iters} EM iterations + "
                      "topology correction)",
            "value": world * C1_REPS / (ms / 1e3), "unit": "registrations/s",
            "higher_is_better": True, "ms_per_registration": ms / C1_REPS,
            "e2e": {"value": world * C1_REPS / wall, "unit": "registrations/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(V * 2 * 4)},
            "cpu_baseline": cpu}


def metric(em_iters):
    return (f"3D registrations/s (160x192x160 MI pair, 64 bins, {em_iters} EM iterations + "
            "topology correction)")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["b200", "reference"], default="b200")
    p.add_argument("--em-iters", type=int, default=EM_ITERS)
    p.add_argument("--gibbs-chains", type=int, default=GIBBS_CHAINS)
    return p.parse_args()


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    elif n_gpus > 1:
        print("note: --gpus > 1 needs torchrun; running one replica", file=sys.stderr)
    return rank, world, local, dist


def max_over_ranks(x, dist):
    from binder_b200.replicas import max_over_ranks as mor
    return mor(x, dist)


def barrier(dist):
    if dist is not None:
        dist.barrier()


class Clocks(threading.Thread):
    """nvidia-smi sampler (200 ms) for the timed region: SM clock and throttle reasons."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        super().__init__(daemon=True)
        self.index, self.rows, self.stop_ev, self.proc = index, [], threading.Event(), None

    def run(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            for line in self.proc.stdout:
                self.rows.append([c.strip() for c in line.split(",")])
                if self.stop_ev.is_set():
                    break
        except (OSError, ValueError):
            pass

    def stop(self):
        self.stop_ev.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.join(timeout=5)
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8
                          for i, v in enumerate(r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def make_inputs(rank):
    from binder_b200 import phantoms
    from binder_b200.replicas import unit_seed
    from binder_b200.utils import initialize_fourier_domain_smoothing
    pair = phantoms.make_pair(SHAPE, unit_seed(SEED, rank), bins=BINS)  # one pair per rank
    V = int(np.prod(SHAPE))
    grid = phantoms.identity_positions(SHAPE).astype(np.float32)
    D = initialize_fourier_domain_smoothing(SHAPE, True, 2, 3).astype(np.float32)
    g = GAMMA_INIT * 1.0 * V * 1.0  # voxel sizes 1 mm
    theta = np.full((BINS, BINS), 1.0 / BINS, np.float32)
    return dict(pair=pair, grid=grid, D=D, gamma=(g, g, g), theta=theta,
                nzv=float(np.count_nonzero(pair.u)), V=V)


def setup_registration(core, inp):
    reg = core.Registration(inp["grid"], 1, inp["grid"], inp["grid"], *SHAPE, *SHAPE, 3,
                            inp["nzv"])
    reg.setNonLinearTransformation(*inp["gamma"], 1, 1, 1, 1, 1, 1, inp["D"])
    reg.setMILikelihood(ALPHA, inp["theta"], BINS, BINS, 1, inp["pair"].v, inp["pair"].u)
    return reg


def hbm_peak():
    """(GB/s, source) of the roofline denominator: the measured copy bandwidth in
    MEASURED_PEAKS.json, else the pool's earlier measurement."""
    try:
        hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs")
    except (OSError, ValueError):
        hbm = None
    return (float(hbm), "measured") if hbm else (6650.0, "fallback")


# the violating 160x192x160 field of the timed topology correction: identity plus a smooth random
# displacement (seed 777, 0.8-voxel RMS, 3-voxel correlation) with 3,549 voxels below e1 = 0.01
TOPO_FIELD = dict(seed=777, rms=0.8, spacing=3.0)


def topology_field():
    from binder_b200 import phantoms
    rng = np.random.default_rng(TOPO_FIELD["seed"])
    return (phantoms.identity_positions(SHAPE).astype(np.float64) +
            phantoms.smooth_random_field(SHAPE, TOPO_FIELD["rms"], TOPO_FIELD["spacing"], rng)
            .astype(np.float64))


def time_registration(core, inp, args, precision, steps, warmup):
    """(ms per registration, final min-log-posterior per non-zero voxel, topology stats) of the
    C2 step -- reset, EM, topology correction -- at a DCT precision, device-timed on the engine
    stream"""
    import torch
    reg = setup_registration(core, inp)
    reg.set_precision(precision)
    stream = torch.cuda.ExternalStream(reg.stream())
    topo = {}

    def step():
        reg.reset()
        reg.EM(args.em_iters, -1e300, 1, 0)
        topo.update(reg.correct_topology(TOPO["e1"], TOPO["e2"], TOPO["max_outer"],
                                         TOPO["max_inner"], [1.0, 1.0, 1.0]))

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    mlp = float(reg.iteration_stats()[-1, 3] / inp["nzv"])
    del reg
    return e0.elapsed_time(e1) / steps, mlp, dict(topo)


def run_topology(core, rank, dist):
    """Topology correction of the violating 160x192x160 field (3,549 voxels with J < 0.01):
    device-timed on the engine stream (positions restored device-to-device each repeat), and
    through the public C-ABI entry point with the FP64 field from host memory and back."""
    import torch
    f0 = topology_field()
    grid = f0.astype(np.float32)
    reg = core.Registration(grid, 1, grid, grid, *SHAPE, *SHAPE, 3, float(np.prod(SHAPE)))
    stream = torch.cuda.ExternalStream(reg.stream())
    stats = {}
    for _ in range(2):
        reg.reset()
        stats = reg.correct_topology(TOPO["e1"], TOPO["e2"], TOPO["max_outer"],
                                     TOPO["max_inner"], [1.0, 1.0, 1.0])
    reps = 3
    torch.cuda.synchronize()
    ms = 0.0
    for _ in range(reps):
        reg.reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        reg.correct_topology(TOPO["e1"], TOPO["e2"], TOPO["max_outer"], TOPO["max_inner"],
                             [1.0, 1.0, 1.0])
        e1.record(stream)
        torch.cuda.synchronize()
        ms += e0.elapsed_time(e1)
    ms = max_over_ranks(ms / reps, dist)
    del reg
    tc = core.topology_correction_3D()
    tc.correct_topology(f0, TOPO["e1"], TOPO["e2"], TOPO["max_outer"], TOPO["max_inner"], 1,
                        [1.0, 1.0, 1.0], *SHAPE)
    t0 = time.perf_counter()
    tc.correct_topology(f0, TOPO["e1"], TOPO["e2"], TOPO["max_outer"], TOPO["max_inner"], 1,
                        [1.0, 1.0, 1.0], *SHAPE)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
    out = {"metric": "topology corrections/s (160x192x160 field violating [0.01, 100] in 3,549 "
                     "voxels, 10/10 iterations)",
           "value": 1e3 / ms, "unit": "corrections/s", "ms_per_correction": ms,
           "iterations": [stats.get("outer_iterations"), stats.get("inner_iterations")],
           "e2e": {"value": 1.0 / e2e_s, "unit": "corrections/s",
                   "h2d_bytes_per_step": int(f0.nbytes), "d2h_bytes_per_step": int(f0.nbytes)}}
    if rank == 0:
        out["cpu_baseline"] = cpu_topology(f0)
    return out


def run_b200(args, rank, world, local, dist):
    import torch
    from binder_b200 import build
    build.build()
    from binder_b200 import _core as core
    torch.cuda.set_device(local)
    inp = make_inputs(rank)
    reg = setup_registration(core, inp)
    stream = torch.cuda.ExternalStream(reg.stream())
    topo_stats = {}

    def step():
        reg.reset()
        reg.EM(args.em_iters, -1e300, 1, 0)
        topo_stats.update(reg.correct_topology(TOPO["e1"], TOPO["e2"], TOPO["max_outer"],
                                               TOPO["max_inner"], [1.0, 1.0, 1.0]))

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    barrier(dist)
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = core.kernel_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_local = e0.elapsed_time(e1)
    launches = core.kernel_launch_count() - launches0
    clk = clocks.stop()
    barrier(dist)
    ms = max_over_ranks(ms_local, dist)
    value = world * args.steps / (ms / 1e3)
    mlp_fast = float(reg.iteration_stats()[-1, 3] / inp["nzv"])

    # per-stage device times (CUDA events, eager launches) and the E-step roofline
    est_ms = reg.profile_stage(0, 10)
    mstep_ms = reg.profile_stage(1, 5)
    theta_ms = reg.profile_stage(2, 10)
    reg.reset()
    reg.EM(args.em_iters, -1e300, 1, 0)
    em_ms = reg.last_elapsed_ms()
    reg.reset()

    # e2e: public API from host buffers, H2D of the inputs and D2H of the result every step
    pinned = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for k, a in
              dict(grid=inp["grid"], D=inp["D"], theta=inp["theta"], u=inp["pair"].u,
                   v=inp["pair"].v).items()}
    V = inp["V"]
    # the starting positions and the voxel grid are the same host array, which the library
    # copies to the device once
    h2d = (pinned["grid"].nbytes + pinned["D"].nbytes + pinned["theta"].nbytes +
           pinned["u"].nbytes + pinned["v"].nbytes)
    d2h = V * 3 * 4

    def e2e_step():
        r = core.Registration(pinned["grid"], 1, pinned["grid"], pinned["grid"], *SHAPE, *SHAPE,
                              3, inp["nzv"])
        r.setNonLinearTransformation(*inp["gamma"], 1, 1, 1, 1, 1, 1, pinned["D"])
        r.setMILikelihood(ALPHA, pinned["theta"], BINS, BINS, 1, pinned["v"], pinned["u"])
        r.EM(args.em_iters, -1e300, 1, 0)
        r.correct_topology(TOPO["e1"], TOPO["e2"], TOPO["max_outer"], TOPO["max_inner"],
                           [1.0, 1.0, 1.0])
        out = r.get_final_locations_as_numpy_array()
        del r
        return out

    e2e_step()
    torch.cuda.synchronize()
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
    e2e_value = world * args.steps / e2e_s
    del reg

    # the metric's comparison: the same registration with the plain FP32 DCT (CUDA cores) against
    # the tensor-core path timed above
    plain_ms, mlp_plain, topo_plain = time_registration(core, inp, args, 0, max(2, args.steps // 4),
                                                        2)
    plain_ms = max_over_ranks(plain_ms, dist)
    arms = {"plain_fp32": {"ms_per_registration": plain_ms, "registrations_per_s": 1e3 / plain_ms,
                           "final_mlp_per_voxel": mlp_plain,
                           "J_below_e1": topo_plain.get("below_e1_before")},
            "tensor_bf16x3": {"ms_per_registration": ms / args.steps,
                              "registrations_per_s": 1e3 * args.steps / ms,
                              "final_mlp_per_voxel": mlp_fast,
                              "J_below_e1": topo_stats.get("below_e1_before")},
            "speedup_vs_plain_fp32": plain_ms / (ms / args.steps)}

    topology = run_topology(core, rank, dist)
    learned = run_learned(core, rank, dist)
    # learned init + BF16 split + batched against the plain FP32 path, 32 held-out 64^3 pairs
    target = run_target(core, rank, dist)
    # Gibbs sampling throughput on the 96^3 pair (every rank runs its own chains)
    gibbs = run_gibbs(core, rank, args.gibbs_chains, dist)
    # 64 pairs of uneven sizes in one batch
    batched = run_batch(core, rank, args.em_iters, dist)
    # 2D registrations on the 128x128 pair
    reg2d = run_2d(core, rank, args.em_iters, dist)

    if rank != 0:
        return None
    hbm, peak_src = hbm_peak()
    achieved = ESTEP_BYTES_PER_VOXEL * V / (est_ms * 1e-3) / 1e9
    traffic = read_profile_traffic()
    line = {
        "metric": metric(args.em_iters), "value": value, "unit": "registrations/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded phantom pair per rank)",
        "config": config_dict(args, world),
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": "registrations/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "estep_em_fast_kernel (E-step)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm, "peak_source": peak_src, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "algorithmic_bytes_per_launch": ESTEP_BYTES_PER_VOXEL * V},
        "stage_ms": {"estep": est_ms, "mstep_dct": mstep_ms, "theta": theta_ms,
                     "em_iteration": (em_ms / args.em_iters) if em_ms else None,
                     "topology_stats": topo_stats},
        "em_iterations_per_s": world * args.em_iters / ((em_ms or 1) / 1e3),
        "precision_arms": arms,
        "learned_init": learned,
        "learned_bf16_batched_vs_plain": target,
        "topology_c2": topology,
        "gibbs": gibbs,
        "batch_c4": batched,
        "registration_2d": reg2d,
        "cpu_baseline": cpu_baseline(inp, args.em_iters),
    }
    return line


def config_dict(args, world):
    """the workload, shared by both arms' lines"""
    return {"workload": "C2 3D MI registration 160x192x160, 64 bins", "em_iterations":
            args.em_iters, "topology": TOPO, "gamma": GAMMA_INIT, "alpha": ALPHA,
            "parallelism": f"replicas x{world}",
            "l2": "working set ~330 MB > 126 MB L2 (no flush needed)"}


def read_profile_traffic():
    """dram read+write bytes per E-step launch from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "estep_c2_ncu.md")
    try:
        for ln in open(path):
            if ln.startswith("traffic_bytes_per_launch:"):
                return float(ln.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


class captured_stdout:
    """The reference prints its per-phase times on stdout: collect them in a file (this
    script's stdout carries one JSON line)."""

    def __enter__(self):
        import tempfile
        sys.stdout.flush()
        self.f = tempfile.TemporaryFile(mode="w+")
        self.saved = os.dup(1)
        os.dup2(self.f.fileno(), 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        self.f.seek(0)
        self.text = self.f.read()
        self.f.close()
        sys.stderr.write(self.text[-4000:])


def cpu_em_phases(inp, threads, iters):
    """The reference's own EM driver on the C2 pair for `iters` iterations (all host cores): the
    EM call's wall seconds and the per-iteration E-step ("Time updating theta and dream
    locations") and M-step ("Time constraining transformation") seconds it prints
    (BINDER/src/cpu/Registration.cpp:150-193); (None, ...) where the reference library is
    absent, with the FP64 oracle port timed instead."""
    import re
    from oracle import pyoracle
    pair = inp["pair"]
    grid = inp["grid"].astype(np.float64)
    R = ref_lib()
    if R is not None:
        tm = []
        with captured_stdout() as log:
            final, _ = pyoracle.ref_em(R, grid, grid, inp["D"], inp["gamma"], SHAPE, SHAPE,
                                       pair.v, pair.u, iters,
                                       mi=(ALPHA, inp["theta"].astype(np.float64).reshape(BINS,
                                                                                          BINS)),
                                       non_zero_voxels=inp["nzv"], threads=threads, timing=tm)
        num = r"([-0-9.eE+]+)"
        est = [float(x) for x in re.findall("Time updating theta and dream locations: " + num,
                                            log.text)]
        mst = [float(x) for x in re.findall("Time constraining transformation: " + num,
                                            log.text)]
        return "reference", tm[0], est, mst, final
    pyoracle.set_threads(threads)
    t0 = time.perf_counter()
    _, final, _, _ = pyoracle.em(grid, grid, pair.u, pair.v, inp["theta"].astype(np.float64),
                                 ALPHA, inp["D"], inp["gamma"], math.sqrt(9.0 / (8.0 * math.pi)),
                                 SHAPE, SHAPE, BINS, BINS, inp["nzv"], iters, -1e300)
    t = time.perf_counter() - t0
    return "port", t, [], [], final


def cpu_topology_seconds(field, threads):
    """wall seconds of the reference's topology_correction_3D::correct_topology (all host cores
    for its FFTs) on `field` with the benchmark's e1, e2 and iteration limits, or None"""
    from oracle import pyoracle
    R = ref_lib()
    if R is None:
        return None
    out = np.zeros(field.size)
    sec = pyoracle.C.c_double(0.0)
    with captured_stdout():
        R.ref_topology3d_mt(np.ascontiguousarray(field, np.float64).ravel(), TOPO["e1"],
                            TOPO["e2"], TOPO["max_outer"], TOPO["max_inner"], np.ones(3), *SHAPE,
                            out, threads, pyoracle.C.byref(sec))
    return sec.value


def cpu_topology(field):
    threads = os.cpu_count() or 1
    t = cpu_topology_seconds(field, threads)
    if t is None:
        return None
    return {"value": 1.0 / t, "unit": "corrections/s", "cores": threads, "kind": "reference",
            "sample": f"one correction of the violating 160x192x160 field ({t:.2f} s) by "
                      "BINDER/src/cpu/topology_correction_3D.cpp compiled in oracle/_ref "
                      "(FFTW replaced by an FFT-based stand-in; its FFTs threaded over lines)"}


CPU_EM_ITERS = 4  # the first iteration is dropped from the per-iteration means


def cpu_registration(inp, em_iters, iters=CPU_EM_ITERS):
    """The reference's CPU registration time of the C2 step, assembled from a bounded sample: the
    mean E-step and M-step seconds of EM iterations 2..iters, times em_iters, plus its topology
    correction of the sample's final field (which, like the GPU's, finds no violation)."""
    threads = os.cpu_count() or 1
    kind, wall, est, mst, final = cpu_em_phases(inp, threads, iters)
    if est and mst and len(est) >= 2:
        e, m = float(np.mean(est[1:])), float(np.mean(mst[1:]))
        rest = max(0.0, wall - sum(est) - sum(mst)) / iters
        t_iter = e + m + rest
    else:
        e = m = rest = None
        t_iter = wall / iters
    t_topo = cpu_topology_seconds(final, threads) or 0.0
    t = em_iters * t_iter + t_topo
    who = f"by {REF_NOTE}" if kind == "reference" else "by the FP64 oracle port"
    return {"value": 1.0 / t, "unit": "registrations/s", "cores": threads, "kind": kind,
            "seconds_per_registration": t,
            "estep_s": e, "mstep_s": m, "other_s_per_iteration": rest, "topology_s": t_topo,
            "sample": f"{iters} EM iterations of the 160x192x160 pair {who} on {threads} threads "
                      f"(EM call {wall:.2f} s); per-iteration E-step {e} s and M-step {m} s "
                      f"(means of iterations 2..{iters}; the M-step's DCTs run on the FFT-based "
                      f"FFTW stand-in), x {em_iters} iterations, + topology correction of the "
                      f"final field {t_topo:.2f} s"}


def cpu_baseline(inp, em_iters):
    return cpu_registration(inp, em_iters)


def run_reference(args, rank, world):
    """The reference's own CPU implementation on the host cores (rank 0 only): `steps` EM
    iterations of the C2 pair in one EM call (the per-iteration E-step and M-step times the
    reference prints), extrapolated to a registration of em_iters iterations plus its topology
    correction; the Gibbs and full-size topology figures alongside."""
    if rank != 0:
        return None
    inp = make_inputs(0)
    iters = max(CPU_EM_ITERS, args.steps)
    cpu = cpu_registration(inp, args.em_iters, iters)
    value = cpu["value"]
    return {"metric": metric(args.em_iters), "value": value, "unit": "registrations/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": cpu["seconds_per_registration"] * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded phantom pair per rank)", "impl": "reference",
            "config": config_dict(args, world),
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "registrations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "topology_c2": cpu_topology(topology_field()),
            "gibbs": reference_gibbs()}


def reference_gibbs():
    """Gibbs sweeps/s of the reference's sampler on the 96^3 pair from the identity grid (the
    --impl reference line has no GPU EM to start from)."""
    from binder_b200 import phantoms
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape = GIBBS_SHAPE
    pair = phantoms.make_pair(shape, GIBBS_SEED, bins=BINS)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3).astype(np.float32)
    cpu = cpu_gibbs(pair, phantoms_grid(shape), np.full(BINS * BINS, 1.0 / BINS), D,
                    GAMMA_INIT * float(np.prod(shape)))
    return {"metric": "Gibbs sweeps/s (96x96x96 MI pair, 64 bins)", "value": cpu["value"],
            "unit": "sweeps/s", "cpu_baseline": cpu}


def main():
    args = parse()
    rank, world, local, dist = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            line = run_reference(args, rank, world)
        else:
            line = run_b200(args, rank, world, local, dist)
        if line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
