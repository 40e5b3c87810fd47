"""ctypes front end of the CPU checkers (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/liboracle.so`` (the FP64 restatement in binder_oracle.c) and, when present,
``oracle/_ref/libbinder_ref.so`` (the reference's own CPU sources built by oracle/Makefile).
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may import this module; the
product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbinder_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build() -> None:
    """Build the checkers in place (the reference build only where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


class _IterStats(C.Structure):
    _fields_ = [("mll", C.c_double), ("log_prior_likelihood", C.c_double),
                ("log_prior_transformation", C.c_double), ("mlp", C.c_double)]


def _load_oracle():
    if not os.path.exists(ORACLE_SO):
        build()
    lib = C.CDLL(ORACLE_SO)
    i, d, ll, u64, u32 = C.c_int, C.c_double, C.c_longlong, C.c_uint64, C.c_uint32
    lib.orc_philox4x32_10.argtypes = [_u32p, _u32p, _u32p]
    lib.orc_spline3.argtypes = [d, _dp]
    lib.orc_set_spline_order.argtypes = [i]
    lib.orc_ssd_estep.argtypes = [_dp, _ip, _ip, C.c_void_p] + [i] * 8 + [_dp, _dp]
    lib.orc_ssd_estep.restype = d
    lib.orc_ssd_update.argtypes = [_dp, i, i, C.c_void_p, i]
    lib.orc_ssd_update.restype = d
    lib.orc_ssd_sample.argtypes = [_dp, i, i, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32]
    lib.orc_ssd_sample.restype = i
    lib.orc_ssd_em.argtypes = [_dp, _dp, _ip, _ip, C.c_void_p, _dp, _dp, d] + [i] * 8 + \
        [d, i, d, i, C.c_void_p]
    lib.orc_ssd_em.restype = i
    lib.orc_spline.argtypes = [i, d, _dp]
    lib.orc_get_spline_order.restype = i
    lib.orc_estep.argtypes = [_dp, _ip, _ip, _dp] + [i] * 8 + [_dp, _dp, C.POINTER(ll)]
    lib.orc_estep.restype = d
    lib.orc_mi_filter_likelihood.argtypes = [_dp, _ip, _ip] + [i] * 6 + [C.c_long, i, i, i]
    lib.orc_mi_filter_likelihood.restype = d
    lib.orc_estep_filter.argtypes = [_dp, _ip, _ip, _dp] + [i] * 9 + [_dp, _dp, C.POINTER(ll)]
    lib.orc_estep_filter.restype = d
    lib.orc_ssdf_loglik.argtypes = [C.c_void_p, _dp, _dp, i, i, i, C.c_long, i, i, i]
    lib.orc_ssdf_loglik.restype = d
    lib.orc_ssdf_estep.argtypes = [_dp, _dp, _dp, C.c_void_p] + [i] * 6 + [_dp] * 5
    lib.orc_ssdf_estep.restype = d
    lib.orc_ssdf_update.argtypes = [C.c_void_p, _dp, i, i, i, _dp, _dp, _dp, _dp, i]
    lib.orc_ssdf_update.restype = d
    lib.orc_ssdf_sample.argtypes = [C.c_void_p, _dp, i, i, i, _dp, _dp, _dp, _dp, u64, u32, u32]
    lib.orc_ssdf_sample.restype = i
    lib.orc_estep_sample.argtypes = [_dp, _ip, _ip, _dp] + [i] * 8 + [u64, u32, u32, _dp, _dp]
    lib.orc_estep_sample.restype = d
    lib.orc_theta_map.argtypes = [_dp, i, i, d]
    lib.orc_dirichlet_cost.argtypes = [_dp, i, i, d]
    lib.orc_dirichlet_cost.restype = d
    lib.orc_dirichlet_sample.argtypes = [_dp, i, i, d, u64, u32, u32]
    lib.orc_dirichlet_sample.restype = i
    lib.orc_gamma_sample.argtypes = [d, u64, u32, u32, u32, u32, C.POINTER(i)]
    lib.orc_gamma_sample.restype = d
    lib.orc_dct3.argtypes = [_dp, _dp, i, i, i, i]
    lib.orc_up_sample.argtypes = [_dp, i, i, i, i, i, i, _dp]
    lib.orc_smooth.argtypes = [_dp, _dp, _dp, _dp, d, i, i, i, _dp, i, u64, u32, u32,
                               C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_smooth.restype = d
    lib.orc_sample_field.argtypes = [_dp, _dp, _dp, d, i, i, i, i, u64, u32, _dp]
    lib.orc_em.argtypes = [_dp, _dp, _ip, _ip, _dp, d, _dp, _dp, d] + [i] * 8 + \
        [d, i, d, i, C.c_void_p]
    lib.orc_em.restype = i
    lib.orc_sampler.argtypes = [_dp, _dp, _dp, _ip, _ip, _dp, d, _dp, _dp, d, _dp, _dp] + \
        [i] * 8 + [u64, u32, i, i, i, i, i, i, i, _dp, _dp]
    lib.orc_sampler.restype = i
    lib.orc_jacobian3d.argtypes = [_dp, i, i, i, d, d, d, _dp]
    lib.orc_jacobian2d.argtypes = [_dp, i, i, d, d, _dp]
    lib.orc_corner_jacobians3d.argtypes = [_dp, i, i, i, _dp, d, d, _dp, C.POINTER(i),
                                           C.POINTER(i)]
    lib.orc_gradients3d.argtypes = [_dp, i, i, i, _dp, _dp]
    lib.orc_limit_gradients3d.argtypes = [_dp, _dp, i, i, i, d, d]
    lib.orc_limit_gradients3d.restype = i
    lib.orc_integrate3d.argtypes = [_dp, _dp, i, i, i, _dp, _dp]
    lib.orc_topology3d.argtypes = [_dp, d, d, i, i, _dp, i, i, i]
    lib.orc_topology3d.restype = i
    lib.orc_corner_jacobians2d.argtypes = [_dp, i, i, _dp, d, d, _dp, C.POINTER(i), C.POINTER(i)]
    lib.orc_topology2d.argtypes = [_dp, d, d, i, i, _dp, i, i]
    lib.orc_topology2d.restype = i
    lib.orc_mutual_information.argtypes = [_dp, i, i]
    lib.orc_mutual_information.restype = d
    lib.orc_set_threads.argtypes = [i]
    lib.orc_get_threads.restype = i
    return lib


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        _LIB = _load_oracle()
    return _LIB


def ref_lib():
    """The reference's own CPU sources (None when the prebuilt library is absent)."""
    if not os.path.exists(REF_SO):
        return None
    r = C.CDLL(REF_SO)
    i, d = C.c_int, C.c_double
    r.ref_spline.argtypes = [i, d, _dp]
    r.ref_jacobian3d.argtypes = [_dp, i, i, i, d, d, d, _dp]
    r.ref_jacobian2d.argtypes = [_dp, i, i, d, d, _dp]
    r.ref_topology3d.argtypes = [_dp, d, d, i, i, _dp, i, i, i, _dp]
    r.ref_topology2d.argtypes = [_dp, d, d, i, i, _dp, i, i, _dp]
    r.ref_topology3d_mt.argtypes = [_dp, d, d, i, i, _dp, i, i, i, _dp, i, C.POINTER(d)]
    r.ref_up_sample.argtypes = [_dp, i, i, i, i, i, i, _dp]
    r.ref_smooth_deformation.argtypes = [_dp, _dp, _dp, _dp, i, i, i, d, d, _dp, _dp]
    r.ref_smooth_deformation.restype = d
    r.ref_mi_update.argtypes = [d, _dp, _dp, i, i, _dp]
    r.ref_mi_update.restype = d
    r.ref_dirichlet_cost.argtypes = [d, _dp, i, i]
    r.ref_dirichlet_cost.restype = d
    r.ref_mi_filter_likelihood.argtypes = [_dp, _ip, _ip] + [i] * 9 + [i, i, i, i]
    r.ref_mi_filter_likelihood.restype = d
    r.ref_mi_filter_update.argtypes = [d, _dp, _ip, _ip] + [i] * 9 + [i, _ip, _dp, _dp]
    r.ref_mi_filter_update.restype = d
    r.ref_ssdf_loglik.argtypes = [_dp, _dp, _dp, _dp, i, d, d, i, i] + [i] * 6 + [i, i, i, i]
    r.ref_ssdf_loglik.restype = d
    r.ref_ssdf_update.argtypes = [_dp, _dp, _dp, _dp, i, d, d, i, i] + [i] * 6 + \
        [i, _ip, _dp, _dp, _dp]
    r.ref_ssdf_update.restype = d
    r.ref_em.argtypes = [_dp, _dp, _dp] + [i] * 7 + [d, _dp, _dp, _dp, _dp, i, d, _dp, i, i, _dp,
                                                      _ip, _ip, i, d, i, _dp, _dp, i,
                                                      C.POINTER(d)]
    r.ref_sampler_seconds.argtypes = [_dp, _dp, i, i, i, _dp, _dp, d, _dp, i, i, _ip, _ip] + \
        [i] * 9
    r.ref_sampler_seconds.restype = d
    r.ref_sampler.argtypes = [_dp, _dp, i, i, i, _dp, _dp, d, _dp, i, i, _ip, _ip] + \
        [i] * 9 + [_dp, _dp]
    r.ref_sampler.restype = d
    r.ref_sampler_ssd.argtypes = [_dp, _dp, i, i, i, _dp, _dp, i, _dp, _ip, _ip] + \
        [i] * 9 + [_dp, _dp, _dp]
    r.ref_sampler_ssd.restype = d
    r.ref_sampler_filter.argtypes = [_dp, _dp, i, i, i, _dp, _dp, i, d, _dp, i, i, i, _ip, _ip,
                                     _dp, _dp, _dp, _dp, i, d, d, i] + [i] * 8 + \
        [_dp, _dp, _dp]
    r.ref_em_filter.argtypes = [_dp, _dp] + [i] * 7 + [d, _dp, _dp, i, d, _dp, i, i, i, _ip, _ip,
                                                       _dp, _dp, _dp, _dp, i, d, d, i, i, d, i,
                                                       _dp, _dp]
    return r


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c32i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def philox(ctr, key):
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32_10(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
    return out


def spline(order: int, d: float):
    w = np.zeros(4)
    lib().orc_spline(int(order), float(d), w)
    return w


def set_spline_order(order: int) -> None:
    """Spline order (1, 2 or 3) of the E-step, EM and sampler calls that follow."""
    lib().orc_set_spline_order(int(order))


def spline3(d: float):
    w = np.zeros(4)
    lib().orc_spline3(float(d), w)
    return w


def estep(d, u, v, theta, vshape, nshape, K, L):
    """EM E-step. Returns (mll, dream[V*N], hist[K*L], degenerate)."""
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    dream = np.zeros(nx * ny * nz * N)
    hist = np.zeros(K * L)
    deg = C.c_longlong(0)
    mll = lib().orc_estep(_c64(d).ravel(), _c32i(u).ravel(), _c32i(v).ravel(),
                          _c64(theta).ravel(), nx, ny, nz, *nshape, K, L, dream, hist,
                          C.byref(deg))
    return mll, dream, hist, deg.value


def estep_filter(d, u, v, theta, vshape, nshape, K, L, M):
    """EM E-step with the MI filter likelihood (M channels; u and v hold at least V + M - 1 and
    Vn + M - 1 bins, read at [index + m]).  Returns (mll, dream[V*N], hist[M*K*L], degenerate)."""
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    dream = np.zeros(nx * ny * nz * N)
    hist = np.zeros(M * K * L)
    deg = C.c_longlong(0)
    mll = lib().orc_estep_filter(_c64(d).ravel(), _c32i(u).ravel(), _c32i(v).ravel(),
                                 _c64(theta).ravel(), nx, ny, nz, *nshape, K, L, M, dream, hist,
                                 C.byref(deg))
    return mll, dream, hist, deg.value


def mi_filter_likelihood(theta, u, v, K, L, M, nshape, voxel, node):
    return lib().orc_mi_filter_likelihood(_c64(theta).ravel(), _c32i(u).ravel(), _c32i(v).ravel(),
                                          K, L, M, *nshape, int(voxel), *[int(t) for t in node])


def estep_sample(d, u, v, theta, vshape, nshape, K, L, seed, sweep, chain=0):
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    dream = np.zeros(nx * ny * nz * N)
    hist = np.zeros(K * L)
    mll = lib().orc_estep_sample(_c64(d).ravel(), _c32i(u).ravel(), _c32i(v).ravel(),
                                 _c64(theta).ravel(), nx, ny, nz, *nshape, K, L, seed, sweep,
                                 chain, dream, hist)
    return mll, dream, hist


def theta_map(hist, K, L, alpha):
    th = _c64(hist).ravel().copy()
    lib().orc_theta_map(th, K, L, float(alpha))
    return th


def dirichlet_cost(theta, K, L, alpha):
    return lib().orc_dirichlet_cost(_c64(theta).ravel(), K, L, float(alpha))


def dirichlet_sample(hist, K, L, alpha, seed, sweep, chain=0):
    th = _c64(hist).ravel().copy()
    capped = lib().orc_dirichlet_sample(th, K, L, float(alpha), seed, sweep, chain)
    return th, capped


def gamma_sample(shape, seed, index, sweep, tag, chain=0):
    c = C.c_int(0)
    g = lib().orc_gamma_sample(float(shape), seed, index, sweep, tag, chain, C.byref(c))
    return g, c.value


def dct3(x, inverse=False):
    x = _c64(x)
    out = np.zeros_like(x)
    nx, ny, nz = x.shape
    lib().orc_dct3(x.reshape(-1), out.reshape(-1), nx, ny, nz, int(inverse))
    return out


def smooth(dream, voxel_pos, D, gamma, sigma, shape, noise=None, rho=None, eta=None,
           want_raw=False):
    """DCT-prior M-step. noise = (seed, sweep, chain) adds the sampling noise.
    Returns (cost, final[V*N]) or (cost, final, raw_reg) when want_raw."""
    nx, ny, nz = shape
    N = 2 if nz == 1 else 3
    out = np.zeros(nx * ny * nz * N)
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    raw = C.c_double(0.0)
    rho_a = _c64(rho if rho is not None else [1, 1, 1])
    eta_a = _c64(eta if eta is not None else [1, 1, 1])
    seed, sweep, chain = noise if noise is not None else (0, 0, 0)
    cost = lib().orc_smooth(_c64(dream).ravel(), _c64(voxel_pos).ravel(), _c64(D).ravel(), g,
                            float(sigma), nx, ny, nz, out, int(noise is not None), seed, sweep,
                            chain, rho_a.ctypes.data, eta_a.ctypes.data,
                            C.addressof(raw) if want_raw else None)
    if want_raw:
        return cost, out, raw.value
    return cost, out


def up_sample(field, shape, oshape):
    """NonLinearTransformation.up_sample on an AoS field: shape -> oshape (nz == 1: 2D)."""
    N = 2 if oshape[2] == 1 else 3
    out = np.zeros(int(np.prod(oshape)) * N)
    lib().orc_up_sample(_c64(field).ravel(), *shape, *oshape, out)
    return out.reshape(*oshape, N)


def resize_linear(field, oshape, scale=1.0):
    """skimage.transform.resize(field, oshape, order=1) * scale, the call at
    BINDER/FastRegistration.py:562-564, restated from scikit-image's published resize (0.19 and
    later; the package is not installed here): with the default mode 'reflect' and anti-aliasing
    on when any axis shrinks, it Gaussian-filters with sigma = max(0, (n/m - 1)/2) per axis
    (scipy.ndimage 'mirror' boundary), zooms with scipy.ndimage.zoom(order=1, grid_mode=True,
    mode='mirror') and clips to the input's value range.  field is [*shape, N]; oshape the new
    spatial shape (the component axis keeps its length)."""
    from scipy import ndimage as ndi
    f = np.asarray(field, np.float64)
    ishape = f.shape
    out_shape = tuple(int(s) for s in oshape) + ishape[len(oshape):]
    factors = np.divide(ishape, out_shape)
    g = f
    if any(o < i for o, i in zip(out_shape, ishape)):
        sig = np.maximum(0, (factors - 1) / 2)
        g = ndi.gaussian_filter(f, sig, mode="mirror")
    z = ndi.zoom(g, [1 / x for x in factors], order=1, mode="mirror", grid_mode=True)
    z = np.clip(z, f.min(), f.max())
    return z * scale


def warp_image(image, positions, order=1):
    """The resampling of BINDER/utils.py:222-227 (skimage.transform.warp with mode 'constant',
    cval 0, clip, preserve_range), restated from scikit-image's published warp (not installed
    here): scipy.ndimage.map_coordinates(order, mode='grid-constant', prefilter only above order
    1), then the output clipped to the input's range, widened to 0 when 0 lies outside the input's
    range but inside the output's."""
    from scipy import ndimage as ndi
    im = np.asarray(image, np.float64)
    pos = np.asarray(positions, np.float64)
    coords = np.moveaxis(pos, -1, 0)
    out = ndi.map_coordinates(im, coords, order=order, mode="grid-constant", cval=0.0,
                              prefilter=order > 1)
    lo, hi = im.min(), im.max()
    if not (lo <= 0.0 <= hi) and out.min() <= 0.0 <= out.max():
        lo, hi = min(lo, 0.0), max(hi, 0.0)
    return np.clip(out, lo, hi)


def sample_field(field, D, gamma, sigma, shape, n, seed=1234, sweep0=0):
    nx, ny, nz = shape
    N = 2 if nz == 1 else 3
    out = np.zeros(n * nx * ny * nz * N)
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    lib().orc_sample_field(_c64(field).ravel(), _c64(D).ravel(), g, float(sigma), nx, ny, nz,
                           int(n), seed, sweep0, out)
    return out.reshape(n, nx, ny, nz, N)


def em(final_locations, voxel_pos, u, v, theta, alpha, D, gamma, sigma, vshape, nshape, K, L,
       non_zero_voxels, max_iter, convergence_th, update_theta=True):
    """Full EM. Returns (iterations, final[V*N], theta[K*L], stats[iters, 4])."""
    fl = _c64(final_locations).ravel().copy()
    th = _c64(theta).ravel().copy()
    stats = (_IterStats * max(1, max_iter))()
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    it = lib().orc_em(fl, _c64(voxel_pos).ravel(), _c32i(u).ravel(), _c32i(v).ravel(), th,
                      float(alpha), _c64(D).ravel(), g, float(sigma), *vshape, *nshape, K, L,
                      float(non_zero_voxels), int(max_iter), float(convergence_th),
                      int(update_theta), C.addressof(stats))
    st = np.array([[s.mll, s.log_prior_likelihood, s.log_prior_transformation, s.mlp]
                   for s in stats[:it]])
    return it, fl, th, st


def sampler(final_locations, dream, voxel_pos, u, v, theta, alpha, D, gamma, sigma, rho, eta,
            vshape, nshape, K, L, seed, N_b, N_s, sample_gamma=0, sample_gamma_every=1,
            sample_posteriors=1, sample_likelihood_parameters=1,
            sample_transformation_parameters=1, chain=0):
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    V = nx * ny * nz
    fl = _c64(final_locations).ravel().copy()
    dr = _c64(dream).ravel().copy()
    th = _c64(theta).ravel().copy()
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    mean = np.zeros(V * N)
    cov = np.zeros(V * N * N)
    capped = lib().orc_sampler(fl, dr, _c64(voxel_pos).ravel(), _c32i(u).ravel(),
                               _c32i(v).ravel(), th, float(alpha), _c64(D).ravel(), g,
                               float(sigma), _c64(rho), _c64(eta), nx, ny, nz, *nshape, K, L,
                               seed, chain, N_b, N_s, sample_gamma, sample_gamma_every,
                               sample_posteriors, sample_likelihood_parameters,
                               sample_transformation_parameters, mean, cov)
    return mean, cov, fl, th, g, capped


class SSDParams(C.Structure):
    """orc_ssd: the SSD likelihood's state (BINDER/src/cpu/SSDLikelihood.cpp)."""
    _fields_ = [("shift_scale", C.c_int), ("sigma2", C.c_double), ("shift", C.c_double),
                ("scale", C.c_double), ("alpha0", C.c_double), ("beta0", C.c_double)]


def ssd_estep(d, u, v, params, vshape, nshape, K, L):
    """Log-space E-step with the SSD likelihood. Returns (mll, dream[V*N], hist[K*L])."""
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    dream = np.zeros(nx * ny * nz * N)
    hist = np.zeros(K * L)
    mll = lib().orc_ssd_estep(_c64(d).ravel(), _c32i(u).ravel(), _c32i(v).ravel(),
                              C.addressof(params), nx, ny, nz, *nshape, K, L, dream, hist)
    return mll, dream, hist


def ssd_update(hist, K, L, params, update=True):
    return lib().orc_ssd_update(_c64(hist).ravel(), K, L, C.addressof(params), int(update))


def ssd_sample(hist, K, L, params, seed, sweep, chain=0):
    """the sampler's parameter draw from the sweep's counts (params updated in place); returns
    1 if the gamma draw hit its attempt cap"""
    return lib().orc_ssd_sample(_c64(hist).ravel(), K, L, C.addressof(params), int(seed),
                                int(sweep), int(chain))


def ssd_em(final_locations, voxel_pos, u, v, params, D, gamma, sigma, vshape, nshape, K, L,
           non_zero_voxels, max_iter, convergence_th, update=True):
    """Full EM with the SSD likelihood. Returns (iterations, final[V*N], stats[iters, 4]);
    params is updated in place."""
    fl = _c64(final_locations).ravel().copy()
    stats = (_IterStats * max(1, max_iter))()
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    it = lib().orc_ssd_em(fl, _c64(voxel_pos).ravel(), _c32i(u).ravel(), _c32i(v).ravel(),
                          C.addressof(params), _c64(D).ravel(), g, float(sigma), *vshape,
                          *nshape, K, L, float(non_zero_voxels), int(max_iter),
                          float(convergence_th), int(update), C.addressof(stats))
    st = np.array([[s.mll, s.log_prior_likelihood, s.log_prior_transformation, s.mlp]
                   for s in stats[:it]])
    return it, fl, st


def jacobian3d(field, shape, vs=(1.0, 1.0, 1.0)):
    nx, ny, nz = shape
    J = np.zeros(nx * ny * nz)
    lib().orc_jacobian3d(_c64(field).ravel(), nx, ny, nz, *map(float, vs), J)
    return J


def jacobian2d(field, shape, vs=(1.0, 1.0)):
    nx, ny = shape
    J = np.zeros(nx * ny)
    lib().orc_jacobian2d(_c64(field).ravel(), nx, ny, *map(float, vs), J)
    return J


def corner_jacobians3d(pos, shape, vs, e1, e2):
    nx, ny, nz = shape
    Jc = np.zeros(max(1, (nx - 1) * (ny - 1) * (nz - 1)) * 8)
    nb, na = C.c_int(0), C.c_int(0)
    lib().orc_corner_jacobians3d(_c64(pos).ravel(), nx, ny, nz, _c64(vs), float(e1), float(e2),
                                 Jc, C.byref(nb), C.byref(na))
    return Jc, nb.value, na.value


def topology3d(field, e1, e2, max_outer, max_inner, vs, shape):
    f = _c64(field).ravel().copy()
    outer = lib().orc_topology3d(f, float(e1), float(e2), int(max_outer), int(max_inner),
                                 _c64(vs), *shape)
    return f, outer


def corner_jacobians2d(pos, shape, vs, e1, e2):
    nx, ny = shape
    Jc = np.zeros(max(1, (nx - 1) * (ny - 1)) * 4)
    nb, na = C.c_int(0), C.c_int(0)
    lib().orc_corner_jacobians2d(_c64(pos).ravel(), nx, ny, _c64(vs), float(e1), float(e2), Jc,
                                 C.byref(nb), C.byref(na))
    return Jc, nb.value, na.value


def topology2d(field, e1, e2, max_outer, max_inner, vs, shape):
    f = _c64(field).ravel().copy()
    outer = lib().orc_topology2d(f, float(e1), float(e2), int(max_outer), int(max_inner),
                                 _c64(vs), *shape)
    return f, outer


def mutual_information(hist, K, L):
    return lib().orc_mutual_information(_c64(hist).ravel(), K, L)


class SSDFParams(C.Structure):
    """orc_ssdf: the SSD filter likelihood's state (BINDER/src/cpu/SSDLikelihoodFilter.cpp)."""
    _fields_ = [("M", C.c_int), ("F", C.c_int), ("rfa", C.c_int), ("alpha0", C.c_double),
                ("beta0", C.c_double), ("coeff", C.c_double * 64), ("sigma", C.c_double * 8)]


def ssdf_params(coeff, sigma, rfa, alpha0, beta0):
    coeff = np.asarray(coeff, np.float64)
    M, F = coeff.shape
    p = SSDFParams(M=M, F=F, rfa=int(rfa), alpha0=float(alpha0), beta0=float(beta0))
    for q, v in enumerate(coeff.ravel()):
        p.coeff[q] = v
    for m, v in enumerate(np.asarray(sigma, np.float64).ravel()):
        p.sigma[m] = v
    return p


def ssdf_loglik(params, nodes, voxels, nshape, voxel, node):
    return lib().orc_ssdf_loglik(C.addressof(params), _c64(nodes).ravel(), _c64(voxels).ravel(),
                                 *nshape, int(voxel), *[int(t) for t in node])


def ssdf_estep(d, nodes, voxels, params, vshape, nshape):
    """Log-space E-step with the SSD filter likelihood.  Returns (mll, dream[V*N], acc) with acc
    the accumulate_info sums (gamma [Vn], s1 [M*Vn], s2 [M*Vn], outside [1 + 2M])."""
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    Vn, M = int(np.prod(nshape)), params.M
    dream = np.zeros(nx * ny * nz * N)
    acc = (np.zeros(Vn), np.zeros(M * Vn), np.zeros(M * Vn), np.zeros(1 + 2 * M))
    mll = lib().orc_ssdf_estep(_c64(d).ravel(), _c64(nodes).ravel(), _c64(voxels).ravel(),
                               C.addressof(params), nx, ny, nz, *nshape, dream, *acc)
    return mll, dream, acc


def ssdf_update(params, nodes, nshape, acc, update=True):
    """update_parameters (when update) and compute_cost; params is updated in place."""
    return lib().orc_ssdf_update(C.addressof(params), _c64(nodes).ravel(), *nshape, *acc,
                                 int(update))


def ssdf_sample(params, nodes, nshape, acc, seed, sweep, chain=0):
    """sample_parameters from the accumulators acc = (gamma, s1, s2, outside); params is
    updated in place; returns 1 if a gamma draw hit its attempt cap"""
    return lib().orc_ssdf_sample(C.addressof(params), _c64(nodes).ravel(), *nshape, *acc,
                                 int(seed), int(sweep), int(chain))


def ref_em(R, final_locations, voxel_pos, D, gamma, vshape, nshape, nodes, voxels, max_iter,
           mi=None, ssd=None, spline_order=3, non_zero_voxels=None, th=-1e30, update=True,
           threads=1, timing=None):
    """The reference's own Registration::EM (compiled in oracle/_ref; R = ref_lib()).  mi =
    (alpha, theta[K][L]) or ssd = (bins, sigmaSq, shiftScale, scale, shift, alpha_0, beta_0).
    Returns (final [V*N], likelihood parameters); timing (a list) receives the EM call's seconds."""
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    V = nx * ny * nz
    fl = _c64(final_locations).ravel()
    vp = _c64(voxel_pos).ravel()
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    out = np.zeros(V * N)
    if mi is not None:
        alpha, theta = mi
        K, L = np.asarray(theta).shape
        lk, th_arr, ssd_arr, npar = 0, _c64(theta).ravel(), np.zeros(6), K * L
    else:
        K = L = int(ssd[0])
        lk, alpha, th_arr, ssd_arr, npar = 1, 0.0, np.zeros(1), _c64(ssd[1:]), 2
    params = np.zeros(max(npar, 2))
    nzv = float(V if non_zero_voxels is None else non_zero_voxels)
    sec = C.c_double(0.0)
    R.ref_em(fl, vp, vp, nx, ny, nz, *nshape, int(spline_order), nzv, g, np.ones(3), np.ones(3),
             _c64(D).ravel(), lk, float(alpha), th_arr, K, L, ssd_arr, _c32i(nodes).ravel(),
             _c32i(voxels).ravel(), int(max_iter), float(th), int(update), out, params,
             int(threads), C.byref(sec))
    if timing is not None:
        timing.append(sec.value)
    return out, params[:npar]


def ref_sampler(R, final_locations, voxel_pos, D, gamma, shape, nodes, voxels, alpha, theta,
                seed, N_b, N_s, sample_gamma=1, every=1, posteriors=1, lik=1, transf=1,
                threads=1):
    """The reference's own Registration::sampler (compiled in oracle/_ref; R = ref_lib()) with the
    MI likelihood from the given positions and theta [K][L].  Returns (mean [V*3], cov [V*9],
    seconds of the sampler call)."""
    nx, ny, nz = shape
    V = nx * ny * nz
    K, L = np.asarray(theta).shape
    mean, cov = np.zeros(V * 3), np.zeros(V * 9)
    sec = R.ref_sampler(_c64(final_locations).ravel(), _c64(voxel_pos).ravel(), nx, ny, nz,
                        _c64(np.asarray(gamma, np.float64)), _c64(D).ravel(), float(alpha),
                        _c64(theta).ravel(), K, L, _c32i(nodes).ravel(), _c32i(voxels).ravel(),
                        int(seed), int(N_b), int(N_s), int(sample_gamma), int(every),
                        int(posteriors), int(lik), int(transf), int(threads), mean, cov)
    return mean, cov, sec


def ref_sampler_ssd(R, final_locations, voxel_pos, D, gamma, shape, nodes, voxels, bins, ssd,
                    seed, N_b, N_s, sample_gamma=1, every=1, posteriors=1, lik=1, transf=1,
                    threads=1):
    """The reference's Registration::sampler with the SSD likelihood, ssd = (sigmaSq, shiftScale,
    scale, shift, alpha_0, beta_0).  Returns (mean [V*3], cov [V*9], (scale, shift), seconds)."""
    nx, ny, nz = shape
    V = nx * ny * nz
    mean, cov, par = np.zeros(V * 3), np.zeros(V * 9), np.zeros(2)
    sec = R.ref_sampler_ssd(_c64(final_locations).ravel(), _c64(voxel_pos).ravel(), nx, ny, nz,
                            _c64(np.asarray(gamma, np.float64)), _c64(D).ravel(), int(bins),
                            _c64(np.asarray(ssd, np.float64)), _c32i(nodes).ravel(),
                            _c32i(voxels).ravel(), int(seed), int(N_b), int(N_s),
                            int(sample_gamma), int(every), int(posteriors), int(lik), int(transf),
                            int(threads), mean, cov, par)
    return mean, cov, (par[0], par[1]), sec


def ref_sampler_filter(R, final_locations, voxel_pos, D, gamma, shape, seed, N_b, N_s, mi=None,
                       ssd=None, sample_gamma=1, every=1, posteriors=1, lik=1, transf=1):
    """The reference's Registration::sampler with setMILikelihoodFilter (mi = (alpha,
    theta[M][K][L], nodes, voxels)) or setSSDLikelihoodFilter (ssd = (coeff[M][F], sigma[M],
    fnodes, fvoxels, rfa, alpha_0, beta_0)).  Returns (mean [V*3], cov [V*9], parameters)."""
    nx, ny, nz = shape
    V = nx * ny * nz
    mean, cov = np.zeros(V * 3), np.zeros(V * 9)
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    z, zi = np.zeros(1), np.zeros(1, np.int32)
    if mi is not None:
        alpha, theta, nodes, voxels = mi
        M, K, L = np.asarray(theta).shape
        params = np.zeros(M * K * L)
        R.ref_sampler_filter(_c64(final_locations).ravel(), _c64(voxel_pos).ravel(), nx, ny, nz,
                             g, _c64(D).ravel(), 2, float(alpha), _c64(theta).ravel(), K, L, M,
                             _c32i(nodes).ravel(), _c32i(voxels).ravel(), z, z, z, z, 0, 1.0,
                             1.0, 1, int(seed), int(N_b), int(N_s), int(sample_gamma),
                             int(every), int(posteriors), int(lik), int(transf), mean, cov, params)
    else:
        coeff, sigma, fnodes, fvoxels, rfa, a0, b0 = ssd
        M, F = np.asarray(coeff).shape
        params = np.zeros(M * F)
        R.ref_sampler_filter(_c64(final_locations).ravel(), _c64(voxel_pos).ravel(), nx, ny, nz,
                             g, _c64(D).ravel(), 3, 0.0, z, 1, 1, M, zi, zi,
                             _c64(coeff).ravel(), _c64(sigma).ravel(), _c64(fnodes).ravel(),
                             _c64(fvoxels).ravel(), int(rfa), float(a0), float(b0), F, int(seed),
                             int(N_b), int(N_s), int(sample_gamma), int(every), int(posteriors),
                             int(lik), int(transf), mean, cov, params)
    return mean, cov, params


def ref_em_filter(R, final_locations, voxel_pos, D, gamma, vshape, max_iter, mi=None, ssd=None,
                  th=-1e30, update=True):
    """The reference's Registration::EM with setMILikelihoodFilter (mi = (alpha, theta[M][K][L],
    nodes, voxels)) or setSSDLikelihoodFilter (ssd = (coeff[M][F], sigma[M], fnodes, fvoxels, rfa,
    alpha_0, beta_0)).  Returns (final [V*N], theta or coeff)."""
    nx, ny, nz = vshape
    N = 2 if nz == 1 else 3
    out = np.zeros(nx * ny * nz * N)
    g = np.zeros(3)
    g[:len(gamma)] = gamma
    z, zi = np.zeros(1), np.zeros(1, np.int32)
    if mi is not None:
        alpha, theta, nodes, voxels = mi
        M, K, L = np.asarray(theta).shape
        params = np.zeros(M * K * L)
        R.ref_em_filter(_c64(final_locations).ravel(), _c64(voxel_pos).ravel(), nx, ny, nz, nx,
                        ny, nz, 3, float(nx * ny * nz), g, _c64(D).ravel(), 2, float(alpha),
                        _c64(theta).ravel(), K, L, M, _c32i(nodes).ravel(), _c32i(voxels).ravel(),
                        z, z, z, z, 0, 1.0, 1.0, 1, int(max_iter), float(th), int(update), out,
                        params)
    else:
        coeff, sigma, fnodes, fvoxels, rfa, a0, b0 = ssd
        M, F = np.asarray(coeff).shape
        params = np.zeros(M * F)
        R.ref_em_filter(_c64(final_locations).ravel(), _c64(voxel_pos).ravel(), nx, ny, nz, nx,
                        ny, nz, 3, float(nx * ny * nz), g, _c64(D).ravel(), 3, 2.0, z, 1, 1, M, zi,
                        zi, _c64(coeff).ravel(), _c64(sigma).ravel(), _c64(fnodes).ravel(),
                        _c64(fvoxels).ravel(), int(rfa), float(a0), float(b0), F, int(max_iter),
                        float(th), int(update), out, params)
    return out, params

