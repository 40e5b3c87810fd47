"""Multi-resolution registration with the resolution changes on the device.

``FastRegistration.run`` (BINDER/FastRegistration.py:428-548) registers coarse to fine: for each
resolution it calls ``move_resolution`` (:550-650) on host arrays -- strided bins and voxel
positions, an order-1 ``skimage`` resize (or the spectral ``up_sample``) of the deformation, the
prior eigenvalues D and the gammas -- and builds a new ``_core.Registration`` from them.
``Pyramid`` keeps the full-resolution data on the GPU and does the same step there
(``binder_pyramid_level``); ``run`` is the loop of ``FastRegistration.run`` for the MI metric on
top of it, with the topology correction between levels done on the device as well.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _core
from ._lib import check, lib

INFO_KEYS = ("voxels_shape", "nodes_shape", "gamma", "voxels_voxel_size", "nodes_voxel_size")


class Pyramid:
    """Full-resolution bins and voxel positions on the device, and the options of
    FastRegistration that ``move_resolution`` reads."""

    def __init__(self, binned_voxels, binned_nodes, voxels_voxel_size=(1.0, 1.0, 1.0),
                 nodes_voxel_size=(1.0, 1.0, 1.0), gamma=5e-7, finite_difference_order=2,
                 increase_gamma_at_DS_resolution=False, upsample_in_frequency_domain=False,
                 spline_order=3, voxel_pos=None):
        bv = np.ascontiguousarray(binned_voxels, dtype=np.int32)
        bn = np.ascontiguousarray(binned_nodes, dtype=np.int32)
        if bv.ndim == 2:
            bv = bv[:, :, None]
        if bn.ndim == 2:
            bn = bn[:, :, None]
        self.voxels_shape = tuple(int(s) for s in bv.shape)
        self.nodes_shape = tuple(int(s) for s in bn.shape)
        self.N = 2 if self.voxels_shape[2] == 1 else 3
        pos = None
        if voxel_pos is not None:
            pos = np.ascontiguousarray(voxel_pos, dtype=np.float64)
            if pos.size != bv.size * self.N:
                raise ValueError(f"voxel_pos has {pos.size} elements, expected {bv.size * self.N}")
        self._pos = pos
        self.spline_order = int(spline_order)
        self._h = C.c_void_p()
        check(lib().binder_pyramid_create(
            C.byref(self._h), bv.ravel(), bn.ravel(),
            None if pos is None else pos.ctypes.data, *self.voxels_shape, *self.nodes_shape,
            np.asarray(voxels_voxel_size, np.float64)[:3].copy(),
            np.asarray(nodes_voxel_size, np.float64)[:3].copy(), float(gamma),
            int(finite_difference_order), int(bool(increase_gamma_at_DS_resolution)),
            int(bool(upsample_in_frequency_domain)), self.spline_order))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and callable(lib):  # module globals may be gone at interpreter shutdown
            lib().binder_pyramid_destroy(h)
            self._h = C.c_void_p()

    def level(self, resolution, prev=None, prev_resolution=1, alpha=2.0, theta=None, K=None,
              L=None):
        """``move_resolution(resolution)`` plus the level's ``Registration`` (with
        setNonLinearTransformation and setMILikelihood applied).  Returns (registration, info)
        where info holds the FastRegistration attributes move_resolution sets."""
        if theta is not None:
            th = np.ascontiguousarray(theta, dtype=np.float32)
            K = th.shape[0] if K is None else K
            L = th.shape[1] if (L is None and th.ndim == 2) else L
            if th.size != int(K) * int(L):
                raise ValueError("theta must have K * L entries")
            th_ptr = th.ctypes.data
        else:
            if prev is None:
                raise ValueError("theta is needed for the first level")
            K = prev._K if K is None else K
            L = prev._L if L is None else L
            th, th_ptr = None, None
        out = C.c_void_p()
        info = np.zeros(16, np.float64)
        check(lib().binder_pyramid_level(self._h, int(resolution),
                                         prev._h if prev is not None else None,
                                         int(prev_resolution), float(alpha), th_ptr, int(K),
                                         int(L), C.byref(out), info.ctypes.data))
        d = {k: info[3 * i:3 * i + 3].copy() for i, k in enumerate(INFO_KEYS)}
        d["voxels_shape"] = tuple(int(v) for v in d["voxels_shape"])
        d["nodes_shape"] = tuple(int(v) for v in d["nodes_shape"])
        d["non_zero_voxels"] = float(info[15])
        reg = _core.Registration._adopt(out, d["voxels_shape"], d["nodes_shape"], K, L)
        return reg, d


def run(pyramid, resolutions, max_number_of_iterations, theta, alpha=2.0, convergence_th=5e-5,
        update_likelihood_parameters=1, topology_correction=True, e1=0.01, e2=100.0,
        max_outer_it=10, max_inner_it=10):
    """The loop of FastRegistration.run (MI metric): per resolution, the device-side
    move_resolution, EM with max_number_of_iterations * resolution iterations, and the topology
    correction of the level's positions.  Returns the last level's registration and info."""
    prev, prev_res, info = None, 1, None
    for r in resolutions:
        reg, info = pyramid.level(r, prev, prev_res, alpha, theta if prev is None else None)
        reg.EM(max_number_of_iterations * r, convergence_th, update_likelihood_parameters, 0)
        if topology_correction:
            reg.correct_topology(e1, e2, max_outer_it, max_inner_it, info["voxels_voxel_size"])
        prev, prev_res = reg, r
    return prev, info
