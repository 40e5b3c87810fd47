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


def run_gibbs(core, rank, chains, dist):
    """Gibbs sweeps/s: `chains` chains of GIBBS_BURN + GIBBS_SAMPLES sweeps on a 96^3 MI pair
    (64 bins) after 10 EM iterations, one Registration, Philox chain index = chain number.  The
    device time of each sampler call (CUDA events on the engine stream) is summed; e2e adds the
    FP64 mean / covariance read-back of every call."""
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
    reg.sampler(GIBBS_SEED, 2, 3, 1, 1, 1, 1, 1)  # warm-up
    barrier(dist)
    dev_ms = 0.0
    t0 = time.perf_counter()
    for c in range(chains):
        reg.set_chain(c)
        reg.sampler(unit_seed(GIBBS_SEED, c), GIBBS_BURN, GIBBS_SAMPLES, 1, 1, 1, 1, 1)
        dev_ms += reg.last_elapsed_ms()
    wall = time.perf_counter() - t0
    dev_ms = max_over_ranks(dev_ms, dist)
    wall = max_over_ranks(wall, dist)
    world = dist.get_world_size() if dist is not None else 1
    sweeps = world * chains * (GIBBS_BURN + GIBBS_SAMPLES)
    cpu = cpu_gibbs(pair, grid, D, g) if rank == 0 else None
    return {"metric": f"Gibbs sweeps/s (96x96x96 MI pair, 64 bins, {chains} chains x "
                      f"{GIBBS_BURN + GIBBS_SAMPLES} sweeps, all sampling switches on)",
            "value": sweeps / (dev_ms / 1e3), "unit": "sweeps/s", "higher_is_better": True,
            "ms_per_sweep": dev_ms / (chains * (GIBBS_BURN + GIBBS_SAMPLES)),
            "e2e": {"value": sweeps / wall, "unit": "sweeps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(chains * V * 12 * 8)},
            "sample_moments": "FP64 Welford, mean [V,3] + covariance [V,3,3] per chain",
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


def cpu_gibbs(pair, grid, D, g, sweeps=2):
    """Sweeps/s of the reference's own sampler (Registration::sampler, all host cores) on the same
    96^3 pair, or of the FP64 oracle sampler where the reference library is absent."""
    from oracle import pyoracle
    threads = os.cpu_count() or 1
    shape = GIBBS_SHAPE
    x = grid.astype(np.float64)
    R = ref_lib()
    if R is not None:
        theta = np.full(BINS * BINS, 1.0 / BINS)
        with stdout_to_stderr():
            t = R.ref_sampler_seconds(np.ascontiguousarray(x).ravel(),
                                      np.ascontiguousarray(x).ravel(), *shape,
                                      np.array([g, g, g], np.float64),
                                      np.ascontiguousarray(D, np.float64).ravel(), ALPHA, theta,
                                      BINS, BINS, np.ascontiguousarray(pair.v, np.int32).ravel(),
                                      np.ascontiguousarray(pair.u, np.int32).ravel(), GIBBS_SEED,
                                      0, sweeps, 1, 1, 1, 1, 1, threads)
        return {"value": sweeps / t, "unit": "sweeps/s", "cores": threads, "kind": "reference",
                "sample": f"{sweeps} sweeps of the 96^3 pair from the identity grid ({t:.2f} s) "
                          f"by {REF_NOTE}"}
    pyoracle.set_threads(threads)
    t0 = time.perf_counter()
    pyoracle.sampler(x, x, x, pair.u, pair.v, np.full(BINS * BINS, 1.0 / BINS), ALPHA,
                     D.astype(np.float64), (g, g, g), math.sqrt(9.0 / (8.0 * math.pi)),
                     (1.0, 1.0, 1.0), (1.0, 1.0, 1.0), shape, shape, BINS, BINS, GIBBS_SEED, 0,
                     sweeps, 1, 1, 1, 1, 1)
    t = time.perf_counter() - t0
    return {"value": sweeps / t, "unit": "sweeps/s", "cores": threads, "kind": "port",
            "sample": f"{sweeps} sweeps of the 96^3 pair from the identity grid ({t:.2f} s)"}


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

    # per-stage device times (CUDA events, eager launches) and the E-step roofline
    est_ms = reg.profile_stage(0, 10)
    mstep_ms = reg.profile_stage(1, 5)
    theta_ms = reg.profile_stage(2, 10)
    reg.reset()
    em_ms = None
    reg.EM(args.em_iters, -1e300, 1, 0)
    em_ms = reg.last_elapsed_ms()
    reg.reset()

    # e2e: public API from host buffers, H2D of the inputs and D2H of the result every step
    pinned = {k: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for k, a in
              dict(grid=inp["grid"], D=inp["D"], theta=inp["theta"], u=inp["pair"].u,
                   v=inp["pair"].v).items()}
    V = inp["V"]
    h2d = (pinned["grid"].nbytes * 2 + pinned["D"].nbytes + pinned["theta"].nbytes +
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

    # Gibbs sampling throughput on the 96^3 pair (every rank runs its own chains)
    del reg
    gibbs = run_gibbs(core, rank, args.gibbs_chains, dist)
    # 2D registrations on the 128x128 pair
    reg2d = run_2d(core, rank, args.em_iters, dist)

    if rank != 0:
        return None
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm else "fallback"
    hbm = hbm or 6650.0
    achieved = ESTEP_BYTES_PER_VOXEL * V / (est_ms * 1e-3) / 1e9
    traffic = read_profile_traffic()
    line = {
        "metric": metric(args.em_iters), "value": value, "unit": "registrations/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded phantom pair per rank)",
        "config": {"workload": "C2 3D MI registration 160x192x160, 64 bins", "em_iterations":
                   args.em_iters, "topology": TOPO, "gamma": GAMMA_INIT, "alpha": ALPHA,
                   "parallelism": f"replicas x{world}",
                   "l2": "working set ~330 MB > 126 MB L2 (no flush needed)"},
        "clocks": clk,
        "e2e": {"value": e2e_value, "unit": "registrations/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "estep_kernel<EM>", "bound": "hbm", "achieved": achieved,
                     "peak": hbm, "peak_source": peak_src, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic,
                     "algorithmic_bytes_per_launch": ESTEP_BYTES_PER_VOXEL * V},
        "stage_ms": {"estep": est_ms, "mstep_dct": mstep_ms, "theta": theta_ms,
                     "em_iteration": (em_ms / args.em_iters) if em_ms else None,
                     "topology_stats": topo_stats},
        "em_iterations_per_s": world * args.em_iters / ((em_ms or 1) / 1e3),
        "gibbs": gibbs,
        "registration_2d": reg2d,
        "cpu_baseline": cpu_baseline(inp, args.em_iters),
    }
    return line


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


def cpu_time_em_iteration(inp, threads):
    """(seconds, kind) of one EM iteration (E-step + theta update + DCT M-step) by the
    reference's own EM driver (the EM call alone), or by the FP64 oracle port where the reference
    library is absent."""
    from oracle import pyoracle
    pair = inp["pair"]
    grid = inp["grid"].astype(np.float64)
    R = ref_lib()
    if R is not None:
        tm = []
        with stdout_to_stderr():
            pyoracle.ref_em(R, grid, grid, inp["D"], inp["gamma"], SHAPE, SHAPE, pair.v, pair.u,
                            1, mi=(ALPHA, inp["theta"].astype(np.float64).reshape(BINS, BINS)),
                            non_zero_voxels=inp["nzv"], threads=threads, timing=tm)
        return tm[0], "reference"
    pyoracle.set_threads(threads)
    t0 = time.perf_counter()
    pyoracle.em(grid, grid, pair.u, pair.v, inp["theta"].astype(np.float64), ALPHA, inp["D"],
                inp["gamma"], math.sqrt(9.0 / (8.0 * math.pi)), SHAPE, SHAPE, BINS, BINS,
                inp["nzv"], 1, -1e300)
    return time.perf_counter() - t0, "port"


def cpu_sample_text(kind, threads, t, em_iters, tail=""):
    who = f" by {REF_NOTE}" if kind == "reference" else " by the FP64 oracle port"
    return (f"1 EM iteration of the 160x192x160 pair{who} on {threads} threads ({t:.2f} s{tail}), "
            f"extrapolated to {em_iters} iterations; topology correction excluded (it would only "
            "lower the CPU figure)")


def cpu_baseline(inp, em_iters):
    threads = os.cpu_count() or 1
    t, kind = cpu_time_em_iteration(inp, threads)
    return {"value": 1.0 / (em_iters * t), "unit": "registrations/s", "cores": threads,
            "kind": kind, "sample": cpu_sample_text(kind, threads, t, em_iters)}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    inp = make_inputs(0)
    threads = os.cpu_count() or 1
    for _ in range(max(0, min(args.warmup, 1))):
        pass  # the oracle has no warm-up state; a warm-up would only repeat the bounded sample
    runs = [cpu_time_em_iteration(inp, threads) for _ in range(max(1, min(args.steps, 2)))]
    times, kind = [r[0] for r in runs], runs[0][1]
    t = statistics.median(times)
    value = 1.0 / (args.em_iters * t)
    sample = cpu_sample_text(kind, threads, t, args.em_iters, f" median of {len(times)} steps")
    return {"metric": metric(args.em_iters), "value": value, "unit": "registrations/s", "n_gpus": world,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded phantom pair)", "impl": "reference",
            "config": {"workload": "C2 3D MI registration 160x192x160, 64 bins",
                       "em_iterations": args.em_iters, "parallelism": "host cores"},
            "cpu_baseline": {"value": value, "unit": "registrations/s", "cores": threads,
                             "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "registrations/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "gibbs": reference_gibbs()}


def reference_gibbs():
    """Gibbs sweeps/s of the oracle sampler on the 96^3 pair (the --impl reference line)."""
    from binder_b200 import phantoms
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape = GIBBS_SHAPE
    pair = phantoms.make_pair(shape, GIBBS_SEED, bins=BINS)
    grid = phantoms.identity_positions(shape).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3).astype(np.float32)
    cpu = cpu_gibbs(pair, grid, D, GAMMA_INIT * float(np.prod(shape)))
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
