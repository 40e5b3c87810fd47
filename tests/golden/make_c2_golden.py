"""Fixture for parity at the full 160x192x160 size against the reference's own CPU code (compiled
unmodified in oracle/_ref), so the FP32 histogram accumulation over 4.9 M voxels, the fixed-point
CTA histograms and the full-size DCT passes are checked, not only toy shapes.

EM: the 160x192x160 MI pair of the benchmark (40 ellipsoids, 64 bins, seed 20260001) registered
from the identity grid by EM_ITERS iterations of the reference's Registration::EM
(BINDER/src/cpu/Registration.cpp:122-217).  Stored: the final positions at SAMPLE random voxels,
theta, the min-log-posterior per non-zero voxel of every iteration (the reference's own print),
the FP64 mutual information of the final field (soft joint histogram with the final theta, by the
oracle's E-step), and the Jacobian statistics of the final field.

Topology: a 160x192x160 field that violates [e1, e2] = [0.01, 100] in 3,549 voxels (identity plus
a smooth random displacement, seed 777, 0.8-voxel RMS, 3-voxel correlation), corrected by the
reference's topology_correction_3D::correct_topology (topology_correction_3D.cpp:17-143), 10/10
iterations.  Stored: the corrected positions at SAMPLE random voxels and at every initially
violating voxel, the iteration counts from the reference's log, and the Jacobian statistics
before and after.

The inputs are regenerated by the tests from the same seeds; checksums of them are stored so a
test can tell that it rebuilt the same inputs.  Run from the repository root (about two minutes):
    python tests/golden/make_c2_golden.py
"""
from __future__ import annotations

import os
import re
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
from binder_b200 import phantoms  # noqa: E402
from oracle import pyoracle  # noqa: E402

EM_ITERS = 5
SAMPLE = 20000
TOPO_SEED, TOPO_RMS, TOPO_SPACING = 777, 0.8, 3.0
E1, E2, OUTER, INNER = 0.01, 100.0, 10, 10


def topology_field():
    """the violating 160x192x160 field of the topology check (grid units, AoS, FP64)"""
    rng = np.random.default_rng(TOPO_SEED)
    return (phantoms.identity_positions(bench.SHAPE).astype(np.float64) +
            phantoms.smooth_random_field(bench.SHAPE, TOPO_RMS, TOPO_SPACING, rng)
            .astype(np.float64))


def checksum(a):
    """order-sensitive FP64 checksum of an array (sum and index-weighted sum)"""
    x = np.asarray(a, np.float64).ravel()
    w = (np.arange(x.size, dtype=np.float64) % 9973.0) + 1.0
    return np.array([x.sum(), (x * w).sum()])


def jac_stats(R, field, shape):
    J = np.zeros(int(np.prod(shape)))
    R.ref_jacobian3d(np.ascontiguousarray(field, np.float64).ravel(), *shape, 1.0, 1.0, 1.0, J)
    return J, np.array([J.min(), J.max(), (J < 0).sum(), (J < E1).sum(), (J > E2).sum()])


class captured_stdout:
    """the reference prints its progress on stdout: collect it in a file"""

    def __enter__(self):
        self.f = tempfile.TemporaryFile(mode="w+")
        os.sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(self.f.fileno(), 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self.saved, 1)
        os.close(self.saved)
        self.f.seek(0)
        self.text = self.f.read()
        self.f.close()


def main():
    R = pyoracle.ref_lib()
    assert R is not None, "oracle/_ref/libbinder_ref.so is needed (make -C oracle)"
    threads = os.cpu_count() or 1
    inp = bench.make_inputs(0)
    shape, V = bench.SHAPE, inp["V"]
    pair = inp["pair"]
    rng = np.random.default_rng(4242)
    idx = np.sort(rng.choice(V, SAMPLE, replace=False))
    grid = inp["grid"].astype(np.float64)
    theta0 = inp["theta"].astype(np.float64).reshape(bench.BINS, bench.BINS)
    with captured_stdout() as log:
        final, theta = pyoracle.ref_em(R, grid, grid, inp["D"], inp["gamma"], shape, shape,
                                       pair.v, pair.u, EM_ITERS, mi=(bench.ALPHA, theta0),
                                       non_zero_voxels=inp["nzv"], threads=threads)
    mlp = [float(x) for x in re.findall(r"Min Log-Posterior per nonzero voxel: ([-0-9.eE+]+)",
                                        log.text)]
    assert len(mlp) == EM_ITERS, log.text[-2000:]
    pyoracle.set_threads(threads)
    _, _, hist, _ = pyoracle.estep(final, pair.u, pair.v, theta, shape, shape, bench.BINS,
                                   bench.BINS)
    mi = pyoracle.mutual_information(hist, bench.BINS, bench.BINS)
    _, em_jac = jac_stats(R, final, shape)

    f0 = topology_field()
    J0, topo_before = jac_stats(R, f0, shape)
    viol = np.flatnonzero((J0 < E1) | (J0 > E2))
    out = np.zeros(V * 3)
    sec = pyoracle.C.c_double(0.0)
    with captured_stdout() as log:
        R.ref_topology3d_mt(np.ascontiguousarray(f0).ravel(), E1, E2, OUTER, INNER, np.ones(3),
                            *shape, out, threads, pyoracle.C.byref(sec))
    outer = len(re.findall(r"^Outer iteration", log.text, re.M))
    inner = len(re.findall(r"^Inner iteration", log.text, re.M))
    _, topo_after = jac_stats(R, out, shape)
    out3 = out.reshape(V, 3)
    np.savez_compressed(
        os.path.join(HERE, "c2_ref.npz"),
        em_iters=EM_ITERS, idx=idx, u_sum=checksum(pair.u), v_sum=checksum(pair.v),
        em_final=final.reshape(V, 3)[idx], em_theta=theta.reshape(bench.BINS, bench.BINS),
        em_mlp_per_voxel=np.array(mlp), em_mi=mi, em_jac=em_jac,
        topo_field_sum=checksum(f0), topo_e=np.array([E1, E2, OUTER, INNER]),
        topo_iters=np.array([outer, inner]), topo_before=topo_before, topo_after=topo_after,
        topo_viol_idx=viol, topo_out_at_idx=out3[idx], topo_out_at_viol=out3[viol],
        topo_seconds=sec.value, topo_threads=threads)
    print(f"c2_ref.npz: EM {EM_ITERS} its, MI {mi:.6f}, mlp/voxel {mlp[-1]:.8f}; topology "
          f"{outer}/{inner} its, {len(viol)} violating voxels, {sec.value:.1f} s")


if __name__ == "__main__":
    main()
