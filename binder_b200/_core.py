"""Drop-in mirror of the reference's ``BINDER._core`` extension module on the B200 engine.

Same classes, method names, keyword names and argument meaning as the pybind11 bindings of the
reference (ste93ste/BINDER, BINDER/src/gpu/bindings.cpp:14-289, plus the CPU-only
``compute_jacobian_determinant_3D`` of BINDER/src/cpu/bindings.cpp:564-593), so the reference's
``FastRegistration`` and CLI can import this module in place of ``BINDER._core``.  Inputs of any
float dtype are accepted (the CUDA backend force-casts to float32, the CPU backend to float64);
positions and theta are computed in FP32, Welford moments, Jacobians and topology correction in
FP64.  Errors raise ``BinderError`` (a RuntimeError), as the reference's std::runtime_error does.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from ._lib import BinderError, check, lib

backend = "b200"
has_topology_correction = True

__all__ = ["backend", "has_topology_correction", "Registration", "NonLinearTransformation",
           "topology_correction_3D", "topology_correction_2D", "compute_jacobian_determinant_3D",
           "compute_jacobian_determinant_2D", "BinderError"]


def _f32(a, n=None, name="array"):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1))
    if n is not None and a.size != n:
        raise ValueError(f"{name} has {a.size} elements, expected {n}")
    return a


def _f64(a, n=None, name="array"):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    if n is not None and a.size != n:
        raise ValueError(f"{name} has {a.size} elements, expected {n}")
    return a


_PINNED_MIN_BYTES = 1 << 20


def _out(n, dtype):
    """A fresh 1-D output array of n elements.  From 1 MiB up it lives in page-locked memory from
    the library's cache, so the device-to-host copy into it runs at link speed; the buffer goes
    back to the cache when the array (and every view of it) is gone."""
    dt = np.dtype(dtype)
    nbytes = int(n) * dt.itemsize
    if nbytes < _PINNED_MIN_BYTES:
        return np.empty(int(n), dt)
    p = C.c_void_p()
    check(lib().binder_pinned_alloc(nbytes, C.byref(p)))
    buf = (C.c_char * nbytes).from_address(p.value)
    weakref.finalize(buf, lib().binder_pinned_free, p.value, nbytes)
    return np.frombuffer(buf, dtype=dt, count=int(n))


def _i32(a, n=None, name="array"):
    a = np.asarray(a)
    if a.dtype.kind == "f":
        a = a.astype(np.int32)  # pybind11 forcecast truncates float bins the same way
    a = np.ascontiguousarray(a.astype(np.int32, copy=False).reshape(-1))
    if n is not None and a.size != n:
        raise ValueError(f"{name} has {a.size} elements, expected {n}")
    return a


class Registration:
    """``_core.Registration`` (gpu/bindings.cpp:17-157)."""

    def __init__(self, final_locations, threads, voxel_pos, node_pos, Nx_v, Ny_v, Nz_v, Nx_n,
                 Ny_n, Nz_n, spline_order, non_zero_voxels):
        self._h = C.c_void_p()
        self._shape = (int(Nx_v), int(Ny_v), int(Nz_v))
        self._nshape = (int(Nx_n), int(Ny_n), int(Nz_n))
        V = int(Nx_v) * int(Ny_v) * int(Nz_v)
        N = 2 if int(Nz_v) == 1 else 3
        fl = _f32(final_locations, V * N, "final_locations")
        vp = _f32(voxel_pos, V * N, "voxel_pos")
        check(lib().binder_registration_create(C.byref(self._h), fl, int(threads), vp, None,
                                               int(Nx_v), int(Ny_v), int(Nz_v), int(Nx_n),
                                               int(Ny_n), int(Nz_n), int(spline_order),
                                               float(non_zero_voxels)))
        self._V = V
        self._N = N
        self._K = self._L = None

    @classmethod
    def _adopt(cls, handle, shape, nshape, K, L):
        """Wrap a registration the library created (binder_pyramid_level); takes ownership."""
        self = cls.__new__(cls)
        self._h = handle
        self._shape = tuple(int(s) for s in shape)
        self._nshape = tuple(int(s) for s in nshape)
        self._V = int(np.prod(self._shape))
        self._N = 2 if self._shape[2] == 1 else 3
        self._K, self._L = int(K), int(L)
        return self

    def __del__(self):
        h = getattr(self, "_h", None)
        # at interpreter shutdown the module's globals may already be gone; the process exit then
        # releases the device memory
        if h and callable(lib):
            lib().binder_registration_destroy(h)
            self._h = C.c_void_p()

    # -- set-up ------------------------------------------------------------------------------
    def setMILikelihood(self, alpha, theta, K, L, threads, binned_nodes, binned_voxels):
        K, L = int(K), int(L)
        Vn = int(np.prod(self._nshape))
        check(lib().binder_registration_set_mi_likelihood(
            self._h, float(alpha), _f32(theta, K * L, "theta"), K, L, int(threads),
            _i32(binned_nodes, Vn, "binned_nodes"), _i32(binned_voxels, self._V, "binned_voxels")))
        self._K, self._L, self._M = K, L, 1
        self._ssd = False
        self._ssdf = (0, 0)

    def setMILikelihoodFilter(self, alpha, theta, threads, binned_nodes, binned_voxels, K, L, M):
        """``setMILikelihoodFilter`` of the CPU module (cpu/bindings.cpp:90-115): M channels,
        theta [M][K][L]; channel m of voxel (node) i is read at [i + m] as MILikelihoodFilter.cpp
        reads it, so the bin arrays need at least V + M - 1 (Vn + M - 1) entries (the usual
        [..., M] arrays have more).  EM and the sampler (M * K * L up to about 22000 there)."""
        K, L, M = int(K), int(L), int(M)
        Vn = int(np.prod(self._nshape))
        nodes = _i32(binned_nodes)
        voxels = _i32(binned_voxels)
        if nodes.size < Vn + M - 1 or voxels.size < self._V + M - 1:
            raise ValueError(f"binned_nodes / binned_voxels need at least {Vn + M - 1} / "
                             f"{self._V + M - 1} bins for M = {M}")
        check(lib().binder_registration_set_mi_likelihood_filter(
            self._h, float(alpha), _f32(theta, M * K * L, "theta"), int(threads), nodes, voxels,
            K, L, M))
        self._K, self._L, self._M = K, L, M
        self._ssd = False
        self._ssdf = (0, 0)

    def setSSDLikelihoodFilter(self, coeff, threads, sigma, features_nodes, features_voxels,
                               reg_across_features, alpha_0, beta_0, M, F):
        """``setSSDLikelihoodFilter`` of the CPU module (cpu/bindings.cpp:154-189): M fixed-image
        channels ([V][M] features), F moving-image features ([Vn][F], or [Vn][M] with
        reg_across_features), coeff [M][F], sigma [M].  EM and the sampler."""
        M, F = int(M), int(F)
        Fn = M if reg_across_features else F
        Vn = int(np.prod(self._nshape))
        check(lib().binder_registration_set_ssd_likelihood_filter(
            self._h, _f64(coeff, M * F, "coeff"), int(threads), _f64(sigma, M, "sigma"),
            _f64(features_nodes, Vn * Fn, "features_nodes"),
            _f64(features_voxels, self._V * M, "features_voxels"), int(reg_across_features),
            float(alpha_0), float(beta_0), M, F))
        self._K, self._L, self._M = F, M, 1
        self._ssd, self._ssdf = False, (M, F)

    def ssd_filter_parameters(self):
        """(coeff [M][F], sigma [M]) of the SSD filter likelihood."""
        M, F = getattr(self, "_ssdf", (0, 0))
        if not M:
            raise BinderError(4, "setSSDLikelihoodFilter has not been called")
        c, s = np.zeros(M * F), np.zeros(M)
        check(lib().binder_registration_get_ssd_filter_parameters(self._h, c, s))
        return c.reshape(M, F), s

    def setSSDLikelihood(self, bins, threads, sigma_sq, scale_shift, scale, shift, binned_nodes,
                         binned_voxels, alpha_0, beta_0):
        """``setSSDLikelihood`` of the CPU module (cpu/bindings.cpp:120-152); EM and the
        sampler."""
        bins = int(bins)
        Vn = int(np.prod(self._nshape))
        check(lib().binder_registration_set_ssd_likelihood(
            self._h, bins, int(threads), float(sigma_sq), int(scale_shift), float(scale),
            float(shift), _i32(binned_nodes, Vn, "binned_nodes"),
            _i32(binned_voxels, self._V, "binned_voxels"), float(alpha_0), float(beta_0)))
        self._K = self._L = bins
        self._M = 1
        self._ssd = True
        self._ssdf = (0, 0)

    def ssd_parameters(self):
        """(sigma^2, shift, scale) of the SSD likelihood (no reference counterpart)."""
        out = np.zeros(3, np.float64)
        check(lib().binder_registration_get_ssd_parameters(self._h, out))
        return {"sigma_sq": float(out[0]), "shift": float(out[1]), "scale": float(out[2])}

    def setNonLinearTransformation(self, gamma_x, gamma_y, gamma_z, voxels_size_x, voxels_size_y,
                                   voxels_size_z, nodes_size_x, nodes_size_y, nodes_size_z, D):
        check(lib().binder_registration_set_nonlinear_transformation(
            self._h, float(gamma_x), float(gamma_y), float(gamma_z), float(voxels_size_x),
            float(voxels_size_y), float(voxels_size_z), float(nodes_size_x), float(nodes_size_y),
            float(nodes_size_z), _f32(D, self._V, "D")))

    # -- hot path ----------------------------------------------------------------------------
    def EM(self, max_EM_iterations, convergence_th, update_likelihood_parameters, debug):
        it = C.c_int(0)
        check(lib().binder_registration_em(self._h, int(max_EM_iterations), float(convergence_th),
                                           int(update_likelihood_parameters), int(debug),
                                           C.byref(it)))
        return it.value

    def sampler(self, seed, N_b, N_s, sample_gamma, sample_gamma_every, sample_posteriors,
                sample_likelihood_parameters, sample_transformation_parameters):
        N = self._N
        mean = _out(self._V * N, np.float64)
        cov = _out(self._V * N * N, np.float64)
        check(lib().binder_registration_sampler(
            self._h, int(seed) & 0xFFFFFFFFFFFFFFFF, int(N_b), int(N_s), int(sample_gamma),
            int(sample_gamma_every), int(sample_posteriors), int(sample_likelihood_parameters),
            int(sample_transformation_parameters), mean, cov))
        return mean.reshape(*self._shape, N), cov.reshape(*self._shape, N, N)

    def sampler_chains(self, seed, chains, N_b, N_s, sample_gamma, sample_gamma_every,
                       sample_posteriors, sample_likelihood_parameters,
                       sample_transformation_parameters, per_chain=True, pooled=True):
        """`chains` independent chains in one batch (no counterpart in the reference, which runs
        one chain per object).  Returns (means [chains, *shape, N], covs [chains, *shape, N, N])
        when per_chain, and (pooled mean [*shape, N], pooled cov [*shape, N, N]) when pooled, in
        that order; chain c equals sampler() after set_chain(chain index + c), draw for draw."""
        N, V, C = self._N, self._V, int(chains)
        mean = _out(C * V * N, np.float64) if per_chain else None
        cov = _out(C * V * N * N, np.float64) if per_chain else None
        pm = _out(V * N, np.float64) if pooled else None
        pc = _out(V * N * N, np.float64) if pooled else None

        def ptr(a):
            return None if a is None else a.ctypes.data

        check(lib().binder_registration_sampler_chains(
            self._h, int(seed) & 0xFFFFFFFFFFFFFFFF, C, int(N_b), int(N_s), int(sample_gamma),
            int(sample_gamma_every), int(sample_posteriors), int(sample_likelihood_parameters),
            int(sample_transformation_parameters), ptr(mean), ptr(cov), ptr(pm), ptr(pc)))
        out = []
        if per_chain:
            out += [mean.reshape(C, *self._shape, N), cov.reshape(C, *self._shape, N, N)]
        if pooled:
            out += [pm.reshape(*self._shape, N), pc.reshape(*self._shape, N, N)]
        return tuple(out)

    # -- getters / setters -------------------------------------------------------------------
    def get_final_locations_as_numpy_array(self):
        out = _out(self._V * self._N, np.float32)
        check(lib().binder_registration_get_final_locations(self._h, out))
        return out.reshape(*self._shape, self._N)

    def get_final_locations(self):
        return self.get_final_locations_as_numpy_array().reshape(-1)

    def get_dream_locations(self):
        out = _out(self._V * self._N, np.float32)
        check(lib().binder_registration_get_dream_locations(self._h, out))
        return out

    def set_dream_locations(self, dream_locations):
        check(lib().binder_registration_set_dream_locations(
            self._h, _f32(dream_locations, self._V * self._N, "dream_locations")))

    def add_displacement(self, field, shape=None):
        """Positions += the order-1 resize of a displacement field [fx, fy, fz, N] (numpy, FP32)
        to the voxel grid (no counterpart in the reference); a device buffer can be given as an
        integer address with its `shape` (fx, fy, fz).  Theta and the other state are kept."""
        if isinstance(field, int):
            fx, fy, fz = (int(v) for v in shape)
            ptr = C.c_void_p(field)
        else:
            f = np.ascontiguousarray(field, np.float32)
            if f.ndim == 3 and self._N == 2:
                f = f[:, :, None, :]
            if f.ndim != 4 or f.shape[-1] != self._N:
                raise ValueError(f"field must be [fx, fy, fz, {self._N}]")
            fx, fy, fz = f.shape[:3]
            ptr = f.ctypes.data_as(C.c_void_p)
        check(lib().binder_registration_add_displacement(self._h, ptr, int(fx), int(fy), int(fz)))

    def get_likelihood_parameters(self):
        if self._K is None:
            raise BinderError(4, "setMILikelihood has not been called")
        M = getattr(self, "_M", 1)
        n = 2 if getattr(self, "_ssd", False) else M * self._K * self._L  # SSD: (scale, shift)
        out = np.zeros(max(n, self._K * self._L), np.float32)
        check(lib().binder_registration_get_likelihood_parameters(self._h, out))
        return out[:n]

    def get_shape(self):
        out = np.zeros(4, np.int32)
        check(lib().binder_registration_get_shape(self._h, out))
        return [int(v) for v in out]

    # -- additions (no reference counterpart) ------------------------------------------------
    def iteration_stats(self, max_n=1 << 20):
        """[n, 4] FP64 (mll, Dirichlet prior, deformation prior, min-log-posterior) per EM step."""
        cap = max(1, int(max_n))
        buf = np.zeros(cap * 4, np.float64)
        n = C.c_int(0)
        check(lib().binder_registration_get_iteration_stats(self._h, buf, cap, C.byref(n)))
        return buf[: n.value * 4].reshape(n.value, 4)

    def state(self):
        g = np.zeros(3, np.float64)
        nu = C.c_double(0)
        deg = C.c_ulonglong(0)
        fl = C.c_uint(0)
        check(lib().binder_registration_get_state(self._h, g, C.byref(nu), C.byref(deg),
                                                  C.byref(fl)))
        return {"gamma": g, "nu": nu.value, "degenerate": deg.value, "flags": fl.value}

    def last_elapsed_ms(self):
        ms = C.c_double(0)
        check(lib().binder_registration_last_elapsed_ms(self._h, C.byref(ms)))
        return ms.value

    def set_chain(self, chain):
        check(lib().binder_registration_set_chain(self._h, int(chain)))

    def set_precision(self, precision):
        """DCT pass arithmetic: 0 FP32 CUDA cores, 1 tensor-core 3xTF32, 2 tensor-core TF32,
        3 tensor-core BF16 split (three products), 4 tensor-core BF16."""
        check(lib().binder_registration_set_precision(self._h, int(precision)))

    def set_histogram_precision(self, precision):
        """E-step bin columns of the MI likelihood: 0 FP32 (the default), 1 FP16 (each voxel's
        per-bin posterior mass rounded to FP16; three CTAs per SM instead of two)."""
        check(lib().binder_registration_set_histogram_precision(self._h, int(precision)))

    def set_estep_grid(self, ctas):
        """CTAs of the EM E-step launch (0: the default, every SM times its occupancy)."""
        check(lib().binder_registration_set_estep_grid(self._h, int(ctas)))

    def stream(self):
        """The object's cudaStream_t as an integer (e.g. for torch.cuda.ExternalStream)."""
        p = C.c_void_p()
        check(lib().binder_registration_get_stream(self._h, C.byref(p)))
        return int(p.value or 0)

    def profile_stage(self, stage, n=10):
        """Average ms of one launch of stage 0 (E-step), 1 (M-step) or 2 (theta update), timed
        with CUDA events; leaves positions unspecified (call reset() afterwards)."""
        ms = C.c_double(0)
        check(lib().binder_registration_profile_stage(self._h, int(stage), int(n), C.byref(ms)))
        return ms.value

    def reset(self):
        """Restore creation-time positions and theta on the device (no host transfer)."""
        check(lib().binder_registration_reset(self._h))

    def correct_topology(self, e1, e2, max_outer_it, max_it, voxel_sizes):
        """Topology correction of this object's positions on the device, in place (replaces the
        host round trip of FastRegistration.py:527-546).  Returns the iteration / count stats."""
        stats = np.zeros(6, np.int64)
        vs = np.ones(3, np.float64)
        v = np.asarray(voxel_sizes, np.float64).ravel()
        if v.size not in (self._N, 3):
            raise ValueError(f"voxel_sizes has {v.size} elements, expected {self._N}")
        vs[:v.size] = v
        check(lib().binder_registration_correct_topology(
            self._h, float(e1), float(e2), int(max_outer_it), int(max_it), vs,
            stats.ctypes.data))
        return dict(zip(["outer_iterations", "inner_iterations", "below_e1_before",
                         "below_e1_after", "above_e2_before", "above_e2_after"], stats.tolist()))


class RegistrationBatch:
    """Many Registration objects (pairs of any sizes) run as one: each chunk of EM iterations is
    one CUDA graph with every pair's kernels on a branch of its own (no counterpart in the
    reference, which runs one pair per object).  Keeps references to its registrations."""

    def __init__(self, registrations):
        self._regs = list(registrations)
        arr = (C.c_void_p * len(self._regs))(*[r._h.value for r in self._regs])
        self._h = C.c_void_p()
        check(lib().binder_batch_create(arr, len(self._regs), C.byref(self._h)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                lib().binder_batch_destroy(h)
            except Exception:  # interpreter shutdown
                pass
            self._h = C.c_void_p()

    def EM(self, max_EM_iterations, convergence_th, update_likelihood_parameters):
        """EM of every pair; returns the iteration counts and sets last_ms (device time)"""
        its = np.zeros(len(self._regs), np.int32)
        ms = C.c_double(0)
        check(lib().binder_batch_em(self._h, int(max_EM_iterations), float(convergence_th),
                                    int(update_likelihood_parameters), its, C.byref(ms)))
        self.last_ms = ms.value
        return its


class NonLinearTransformation:
    """``_core.NonLinearTransformation`` (gpu/bindings.cpp:160-255)."""

    def __init__(self, gamma_x, gamma_y, gamma_z, voxels_size_x, voxels_size_y, voxels_size_z,
                 nodes_size_x, nodes_size_y, nodes_size_z, D, Nx_v, Ny_v, Nz_v, threads,
                 sigma_spline, spline_offset):
        self._h = C.c_void_p()
        self._shape = (int(Nx_v), int(Ny_v), int(Nz_v))
        self._V = int(np.prod(self._shape))
        self._N = 2 if int(Nz_v) == 1 else 3
        check(lib().binder_transform_create(
            C.byref(self._h), float(gamma_x), float(gamma_y), float(gamma_z),
            float(voxels_size_x), float(voxels_size_y), float(voxels_size_z), float(nodes_size_x),
            float(nodes_size_y), float(nodes_size_z), _f32(D, self._V, "D"), int(Nx_v), int(Ny_v),
            int(Nz_v), int(threads), float(sigma_spline), float(spline_offset)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and callable(lib):  # see Registration.__del__
            lib().binder_transform_destroy(h)
            self._h = C.c_void_p()

    def get_shape(self):
        out = np.zeros(4, np.int32)
        check(lib().binder_transform_get_shape(self._h, out))
        return [int(v) for v in out]

    def set_precision(self, precision):
        """DCT pass arithmetic: 0 FP32 CUDA cores, 1 tensor-core 3xTF32, 2 tensor-core TF32,
        3 tensor-core BF16 split (three products), 4 tensor-core BF16."""
        check(lib().binder_transform_set_precision(self._h, int(precision)))

    def smooth_deformation(self, deformation):
        N = self._N
        out = _out(self._V * N, np.float32)
        cost = C.c_double(0)
        check(lib().binder_transform_smooth_deformation(
            self._h, _f32(deformation, self._V * N, "deformation"), out, C.byref(cost)))
        return cost.value, out.reshape(*self._shape, N)

    def sampleDeformationField(self, deformationField, number_of_samples):
        n = int(number_of_samples)
        N = self._N
        out = _out(max(n, 0) * self._V * N, np.float32)
        check(lib().binder_transform_sample_deformation_field(
            self._h, _f32(deformationField, self._V * N, "deformationField"), n, out))
        return out.reshape(n, *self._shape, N)

    @staticmethod
    def up_sample(deformation_field, N_x, N_y, N_z, N_x_o, N_y_o, N_z_o, threads):
        """``NonLinearTransformation.up_sample`` (cpu/bindings.cpp:408-434), FP64 on the GPU."""
        N = 2 if int(N_z_o) == 1 else 3
        Vi = int(N_x) * int(N_y) * int(N_z)
        out = _out(int(N_x_o) * int(N_y_o) * int(N_z_o) * N, np.float64)
        check(lib().binder_transform_up_sample(
            _f64(deformation_field, Vi * N, "deformation_field"), int(N_x), int(N_y), int(N_z),
            int(N_x_o), int(N_y_o), int(N_z_o), int(threads), out))
        return out.reshape(int(N_x_o), int(N_y_o), int(N_z_o), N)


class topology_correction_3D:
    """``_core.topology_correction_3D`` (gpu/bindings.cpp:259-287); FP64 throughout."""

    def __init__(self):
        self.last_stats = None

    def correct_topology(self, h_init, e1, e2, max_outer_it, max_it, threads, voxel_sizes, Nx_v,
                         Ny_v, Nz_v):
        V = int(Nx_v) * int(Ny_v) * int(Nz_v)
        field = _f64(h_init, V * 3, "h_init")
        out = _out(V * 3, np.float64)
        stats = np.zeros(6, np.int64)
        check(lib().binder_topology_correct_3d(
            field, float(e1), float(e2), int(max_outer_it), int(max_it), int(threads),
            _f64(voxel_sizes, 3, "voxel_sizes"), int(Nx_v), int(Ny_v), int(Nz_v), out,
            stats.ctypes.data))
        self.last_stats = dict(zip(["outer_iterations", "inner_iterations", "below_e1_before",
                                    "below_e1_after", "above_e2_before", "above_e2_after"],
                                   stats.tolist()))
        return out.reshape(int(Nx_v), int(Ny_v), int(Nz_v), 3)


class topology_correction_2D:
    """``_core.topology_correction_2D`` (cpu/bindings.cpp:447-480); FP64 throughout."""

    def __init__(self):
        self.last_stats = None

    def correct_topology(self, h_init, e1, e2, max_outer_it, max_it, threads, voxel_sizes, Nx_v,
                         Ny_v):
        V = int(Nx_v) * int(Ny_v)
        field = _f64(h_init, V * 2, "h_init")
        out = _out(V * 2, np.float64)
        stats = np.zeros(6, np.int64)
        check(lib().binder_topology_correct_2d(
            field, float(e1), float(e2), int(max_outer_it), int(max_it), int(threads),
            _f64(voxel_sizes, 2, "voxel_sizes"), int(Nx_v), int(Ny_v), out, stats.ctypes.data))
        self.last_stats = dict(zip(["outer_iterations", "inner_iterations", "below_e1_before",
                                    "below_e1_after", "above_e2_before", "above_e2_after"],
                                   stats.tolist()))
        return out.reshape(int(Nx_v), int(Ny_v), 2)


def kernel_launch_count():
    """Kernels launched by the library in this process (graph replays count every node)."""
    return int(lib().binder_kernel_launch_count())


def compute_jacobian_determinant_3D(field, Nx, Ny, Nz, voxel_size_x, voxel_size_y, voxel_size_z):
    """``_core.compute_jacobian_determinant_3D`` (cpu/bindings.cpp:564-593), FP64 on the GPU."""
    V = int(Nx) * int(Ny) * int(Nz)
    J = _out(V, np.float64)
    check(lib().binder_jacobian_determinant_3d(_f64(field, V * 3, "field"), int(Nx), int(Ny),
                                               int(Nz), float(voxel_size_x), float(voxel_size_y),
                                               float(voxel_size_z), J))
    return J.reshape(int(Nx), int(Ny), int(Nz))


def resize_linear(field, output_shape, scale=1.0):
    """skimage.transform.resize(field, output_shape, order=1) * scale on the GPU (FP64), for the
    deformation fields FastRegistration.py:562-564 resamples between resolutions.  field is
    [*shape, N] with a 2- or 3-D spatial shape; output_shape gives the new spatial shape."""
    f = np.asarray(field, np.float64)
    sp = tuple(int(s) for s in output_shape)
    nd = len(sp)
    if nd not in (2, 3) or f.ndim != nd + 1:
        raise ValueError("field must be [*shape, N] with a 2-D or 3-D spatial shape")
    ish = f.shape[:nd] + (1,) * (3 - nd)
    osh = sp + (1,) * (3 - nd)
    N = f.shape[-1]
    out = _out(int(np.prod(osh)) * N, np.float64)
    check(lib().binder_resize_linear(_f64(f, f.size, "field"), *ish, int(N), *osh, float(scale),
                                     out))
    return out.reshape(*sp, N)


def compute_jacobian_determinant_2D(field, Nx, Ny, voxel_size_x, voxel_size_y):
    """``_core.compute_jacobian_determinant_2D`` (cpu/bindings.cpp:535-560), FP64 on the GPU."""
    V = int(Nx) * int(Ny)
    J = _out(V, np.float64)
    check(lib().binder_jacobian_determinant_2d(_f64(field, V * 2, "field"), int(Nx), int(Ny),
                                               float(voxel_size_x), float(voxel_size_y), J))
    return J.reshape(int(Nx), int(Ny))
