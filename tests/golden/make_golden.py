"""Generate the golden fixtures in this directory from the reference's own CPU sources.

The reference's Spline.cpp, MILikelihood.cpp, MILikelihoodFilter.cpp, SSDLikelihood.cpp,
SSDLikelihoodFilter.cpp, Registration.cpp, utils.cpp, DCT.cpp, FFT.cpp,
NonLinearTransformation.cpp, topology_correction_3D.cpp and topology_correction_2D.cpp are compiled
unmodified by oracle/Makefile into oracle/_ref/libbinder_ref.so (FFTW and Eigen replaced by the
project-written subsets in oracle/ref_shim, the affine / rigid transformations by stand-ins).  This script feeds them seeded inputs and stores inputs and outputs as small
.npz files, so the parity tests are pinned to the reference even where its sources are absent.

Run from the repository root:  python tests/golden/make_golden.py [--reference <checkout>]
(default: $BINDER_REFERENCE_ROOT).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle  # noqa: E402

# the reference checkout: BINDER_REFERENCE_ROOT, or --reference <dir> on the command line
REF_ROOT = os.environ.get("BINDER_REFERENCE_ROOT", "/root/reference")
if "--reference" in sys.argv:
    REF_ROOT = sys.argv[sys.argv.index("--reference") + 1]


def grid(shape):
    return np.stack(np.indices(shape), -1).astype(np.float64)


def reference_functions(names):
    """Module-level functions of the reference's BINDER/utils.py, compiled from its source with
    numpy as their only global (their other imports are not needed by these functions)."""
    import ast
    src = open(os.path.join(REF_ROOT, "BINDER", "utils.py")).read()
    tree = ast.parse(src)
    ns = {"np": np}
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name in names:
            exec(compile(ast.Module(body=[node], type_ignores=[]), "BINDER/utils.py", "exec"), ns)
    return {n: ns[n] for n in names}


def main():
    R = pyoracle.ref_lib()
    if R is None:
        pyoracle.build()
        R = pyoracle.ref_lib()
    assert R is not None, "oracle/_ref/libbinder_ref.so could not be built"
    rng = np.random.default_rng(20260101)

    # spline weights, orders 1-3 (Spline.cpp:44-109)
    ds = np.concatenate([[0.0, 0.5, 1.0 - 1e-12], rng.random(13)])
    W = np.zeros((3, ds.size, 4))
    for o in (1, 2, 3):
        for i, d in enumerate(ds):
            w = np.zeros(4)
            R.ref_spline(o, float(d), w)
            W[o - 1, i] = w
    np.savez(os.path.join(HERE, "spline_ref.npz"), d=ds, weights=W)

    # Jacobian determinant (utils.cpp:100-345): smooth field with folds, anisotropic voxels
    shape = (9, 11, 10)
    f = grid(shape) + rng.normal(0, 0.45, shape + (3,))
    vs = np.array([1.1, 0.9, 1.3])
    J = np.zeros(np.prod(shape))
    R.ref_jacobian3d(f.ravel(), *shape, *vs, J)
    np.savez(os.path.join(HERE, "jacobian_ref.npz"), field=f, shape=shape, vs=vs, J=J)

    # topology correction (topology_correction_3D.cpp:17-143)
    cases = {}
    for k, (shape, sig, vs) in enumerate([((8, 9, 10), 0.45, (1.0, 1.2, 0.9)),
                                         ((12, 10, 11), 0.55, (1.0, 1.0, 1.0))]):
        f = grid(shape) + rng.normal(0, sig, shape + (3,))
        out = np.zeros(f.size)
        R.ref_topology3d(f.ravel(), 0.01, 100.0, 10, 10, np.asarray(vs, float), *shape, out)
        cases[f"field{k}"] = f
        cases[f"shape{k}"] = np.array(shape)
        cases[f"vs{k}"] = np.array(vs, float)
        cases[f"out{k}"] = out.reshape(f.shape)
    np.savez(os.path.join(HERE, "topology_ref.npz"), e1=0.01, e2=100.0, max_outer=10,
             max_inner=10, **cases)

    # DCT smoothing + prior cost (NonLinearTransformation.cpp:226-278)
    shape = (11, 20, 7)
    field = rng.standard_normal(shape + (3,))
    from binder_b200.utils import initialize_fourier_domain_smoothing
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3).ravel()
    gamma = np.array([5.0, 3.0, 7.0])
    one = np.ones(3)
    out = np.zeros(field.size)
    cost = R.ref_smooth_deformation(gamma, one, one, D, *shape, 1.0, 0.0, field.ravel(), out)
    np.savez(os.path.join(HERE, "smoothing_ref.npz"), field=field, D=D, gamma=gamma, sigma=1.0,
             out=out.reshape(field.shape), cost=cost)

    # MI parameter update and Dirichlet cost (MILikelihood.cpp:33-124)
    K, L = 16, 12
    hist = rng.random((K, L)) * 50.0
    th0 = np.full((K, L), 1.0 / L)
    th = np.zeros(K * L)
    cost = R.ref_mi_update(2.0, th0.ravel(), hist.ravel(), K, L, th)
    np.savez(os.path.join(HERE, "mi_ref.npz"), hist=hist, alpha=2.0, theta=th.reshape(K, L),
             cost=cost)

    # 2D Jacobian determinant (utils.cpp:10-98): folds, anisotropic pixels
    shape2 = (13, 17)
    f2 = np.stack(np.indices(shape2), -1).astype(np.float64) + rng.normal(0, 0.45, shape2 + (2,))
    vs2 = np.array([1.2, 0.8])
    J2 = np.zeros(np.prod(shape2))
    R.ref_jacobian2d(f2.ravel(), *shape2, *vs2, J2)
    np.savez(os.path.join(HERE, "jacobian2d_ref.npz"), field=f2, shape=shape2, vs=vs2, J=J2)

    # 2D DCT smoothing + prior cost (NonLinearTransformation.cpp with Nz = 1)
    shape = (14, 23, 1)
    field = rng.standard_normal(shape[:2] + (2,))
    D = initialize_fourier_domain_smoothing(shape, True, 2, 2).ravel()
    gamma = np.array([4.0, 6.0, 0.0])
    out = np.zeros(field.size)
    cost = R.ref_smooth_deformation(gamma, one, one, D, *shape, 1.0, 0.0, field.ravel(), out)
    np.savez(os.path.join(HERE, "smoothing2d_ref.npz"), field=field, D=D, gamma=gamma, sigma=1.0,
             out=out.reshape(field.shape), cost=cost)
    # 2D topology correction (topology_correction_2D.cpp:17-163)
    cases = {}
    # (shape, noise, voxel sizes, e1, e2): folds only; folds with anisotropic pixels; a tight band
    # that also caps expansions
    for k, (shape, sig, vs, e1, e2) in enumerate([((14, 12), 0.45, (1.0, 1.2), 0.01, 100.0),
                                                 ((20, 17), 0.5, (1.0, 1.0), 0.01, 100.0),
                                                 ((16, 15), 0.35, (0.9, 1.1), 0.5, 1.6)]):
        f = np.stack(np.indices(shape), -1).astype(np.float64) + rng.normal(0, sig, shape + (2,))
        out = np.zeros(f.size)
        R.ref_topology2d(f.ravel(), e1, e2, 10, 10, np.asarray(vs, float), *shape, out)
        cases[f"field{k}"] = f
        cases[f"shape{k}"] = np.array(shape)
        cases[f"vs{k}"] = np.array(vs, float)
        cases[f"e{k}"] = np.array([e1, e2])
        cases[f"out{k}"] = out.reshape(f.shape)
    np.savez(os.path.join(HERE, "topology2d_ref.npz"), ncases=3, max_outer=10, max_inner=10,
             **cases)
    # spectral up-sampling of a displacement field (NonLinearTransformation.cpp:366-430): a
    # resolution-2 -> 1 step in 3D and 2D, odd and even sizes
    ups = {}
    for k, (shape, oshape) in enumerate([((6, 7, 5), (12, 13, 10)), ((9, 8, 1), (17, 16, 1))]):
        N = 2 if oshape[2] == 1 else 3
        f = rng.standard_normal(shape + (N,))
        out = np.zeros(int(np.prod(oshape)) * N)
        R.ref_up_sample(f.ravel(), *shape, *oshape, out)
        ups[f"field{k}"] = f
        ups[f"oshape{k}"] = np.array(oshape)
        ups[f"out{k}"] = out.reshape(oshape + (N,))
    np.savez(os.path.join(HERE, "upsample_ref.npz"), ncases=2, **ups)
    # intensity binning (BINDER/utils.py:12-82): the reference's own functions, taken from its
    # source (the module itself imports packages absent here) and run under numpy
    fns = reference_functions(["bin_signal", "bin_signal_robust"])
    from binder_b200 import phantoms
    prep = {}
    img = phantoms.ellipsoid_phantom((40, 36, 30), 12, (3.0, 15.0), 1.0, 0.02, rng).astype(np.float64)
    mask = (rng.random(img.shape) > 0.1).astype(np.float64)
    img32 = (img * 3.7 + 0.2).astype(np.float32)
    # 62 % of the mass at the minimum: the lower percentile needs the reference's raising loop
    spiky = np.concatenate([np.zeros(5000), np.abs(rng.normal(0, 1, 3000)), [40.0]])
    cases = [("f64", img * mask, 64), ("f32", img32, 32), ("spiky", spiky, 16)]
    for name, sig, nb in cases:
        b, e = fns["bin_signal_robust"](sig, nb)
        prep[f"{name}_signal"] = sig
        prep[f"{name}_bins"] = np.int32(nb)
        prep[f"{name}_robust"] = b
        prep[f"{name}_edges"] = e
        prep[f"{name}_plain"] = fns["bin_signal"](sig, nb)
    np.savez(os.path.join(HERE, "preprocess_ref.npz"), names=np.array([c[0] for c in cases]),
             **prep)

    # MI filter likelihood (MILikelihoodFilter.cpp:38-124): M channels, bins read at [index + m],
    # nodes outside the grid included; then accumulate_info / update_parameters / compute_cost
    M, K, L = 3, 5, 4
    nshape, vshape = (4, 3, 5), (6, 5, 4)
    Vn, V = int(np.prod(nshape)), int(np.prod(vshape))
    theta = rng.random((M, K, L)) + 0.05
    theta /= theta.sum(-1, keepdims=True)
    nodes = rng.integers(0, K, Vn + M - 1).astype(np.int32)
    voxels = rng.integers(0, L, V + M - 1).astype(np.int32)
    npairs = 200
    pv = rng.integers(0, V, npairs)
    pn = np.stack([rng.integers(-2, n + 2, npairs) for n in nshape], -1)
    like = np.array([R.ref_mi_filter_likelihood(theta.ravel(), voxels, nodes, K, L, M, *nshape,
                                                *vshape, int(v), *[int(t) for t in xyz])
                     for v, xyz in zip(pv, pn)])
    vxyz = np.ascontiguousarray(np.concatenate([pv[:, None], pn], 1).astype(np.int32))
    post = rng.random(npairs) * 3.0
    th_out = np.zeros(M * K * L)
    fcost = R.ref_mi_filter_update(2.0, theta.ravel(), voxels, nodes, K, L, M, *nshape, *vshape,
                                   npairs, vxyz.ravel(), post, th_out)
    np.savez(os.path.join(HERE, "mi_filter_ref.npz"), M=M, K=K, L=L, nshape=nshape,
             vshape=vshape, theta=theta, nodes=nodes, voxels=voxels, pairs=vxyz, likelihood=like,
             posterior=post, alpha=2.0, theta_out=th_out.reshape(M, K, L), cost=fcost)

    # SSD filter likelihood (SSDLikelihoodFilter.cpp:72-389): compute_log_likelihood at (voxel,
    # node) pairs, then accumulate_info / update_parameters / compute_cost, for both layouts
    # (reg_across_features 0: nodes [Vn][F] and a coefficient fit; 1: nodes [Vn][M])
    ssdf = {}
    for rfa, M, F in ((0, 2, 3), (1, 3, 3)):
        Fn = M if rfa else F
        nodes_f = rng.normal(0.0, 2.0, (Vn, Fn)) + 1.0
        voxels_f = rng.normal(0.0, 2.0, (V, M))
        coeff = rng.normal(0.0, 1.0, (M, F))
        sig = rng.random(M) * 2.0 + 0.5
        like = np.array([R.ref_ssdf_loglik(coeff.ravel(), sig, nodes_f.ravel(), voxels_f.ravel(),
                                           rfa, 3.0, 0.7, M, F, *nshape, *vshape, int(v),
                                           *[int(t) for t in xyz])
                         for v, xyz in zip(pv, pn)])
        c_out, s_out = np.zeros(M * F), np.zeros(M)
        scost = R.ref_ssdf_update(coeff.ravel(), sig, nodes_f.ravel(), voxels_f.ravel(), rfa, 3.0,
                                  0.7, M, F, *nshape, *vshape, npairs, vxyz.ravel(), post,
                                  c_out, s_out)
        key = f"rfa{rfa}_"
        ssdf.update({key + "M": M, key + "F": F, key + "nodes": nodes_f, key + "voxels": voxels_f,
                     key + "coeff": coeff, key + "sigma": sig, key + "loglik": like,
                     key + "coeff_out": c_out.reshape(M, F), key + "sigma_out": s_out,
                     key + "cost": scost})
    np.savez(os.path.join(HERE, "ssd_filter_ref.npz"), nshape=nshape, vshape=vshape, pairs=vxyz,
             posterior=post, alpha0=3.0, beta0=0.7, **ssdf)

    # whole EM runs through the reference's own driver (Registration.cpp:122-217, one thread):
    # MI in 3D and 2D, spline orders 1 and 2, SSD with both fits
    from binder_b200.utils import bin_signal_robust, initialize_fourier_domain_smoothing
    em = {}

    def em_case(name, shape, K, L, seed, iters, ssd=None, order=3):
        rs = np.random.default_rng(seed)
        pair = phantoms.make_pair(shape, seed, bins=L, n_objects=10, axes=(2.0, 6.0), rms=1.0,
                                  spacing=3.0)
        v, _ = bin_signal_robust(pair.moving, K)
        g = phantoms.identity_positions(shape).astype(np.float64)
        d0 = g + phantoms.smooth_random_field(shape, 0.6, 3.0, rs)
        th = rs.random((K, L)) + 0.05
        th /= th.sum(1, keepdims=True)
        D = initialize_fourier_domain_smoothing(shape, True, 2, len(shape))
        gamma = (0.8, 0.6, 1.1)
        vs = shape if len(shape) == 3 else shape + (1,)
        out, par = pyoracle.ref_em(R, d0, g, D, gamma, vs, vs, v.astype(np.int32),
                                   pair.u.astype(np.int32), iters,
                                   mi=None if ssd else (2.0, th), ssd=ssd, spline_order=order)
        em.update({f"{name}_shape": np.array(vs), f"{name}_K": K, f"{name}_L": L,
                   f"{name}_iters": iters, f"{name}_order": order, f"{name}_d0": d0,
                   f"{name}_grid": g, f"{name}_D": D, f"{name}_gamma": np.array(gamma),
                   f"{name}_v": v.astype(np.int32), f"{name}_u": pair.u.astype(np.int32),
                   f"{name}_theta": th, f"{name}_final": out, f"{name}_params": par,
                   f"{name}_ssd": np.array(ssd if ssd else [0.0] * 7)})

    em_case("mi3d", (12, 10, 9), 8, 6, 101, 6)
    em_case("mi2d", (24, 20), 8, 6, 102, 6)
    em_case("order1", (10, 9, 8), 8, 6, 103, 4, order=1)
    em_case("order2", (10, 9, 8), 8, 6, 104, 4, order=2)
    em_case("ssd0", (10, 9, 8), 16, 16, 105, 4, ssd=(16, 4.0, 0, 0.9, 0.5, 1.0, 1.0))
    em_case("ssd1", (10, 9, 8), 16, 16, 106, 4, ssd=(16, 4.0, 1, 0.9, 0.5, 1.0, 1.0))
    np.savez(os.path.join(HERE, "em_ref.npz"),
             names=np.array(["mi3d", "mi2d", "order1", "order2", "ssd0", "ssd1"]), **em)

    # EM runs with the filter likelihoods through the reference's driver (3 iterations each)
    from scipy import ndimage as ndi
    rs = np.random.default_rng(107)
    shape = (10, 9, 8)
    V = int(np.prod(shape))
    g = phantoms.identity_positions(shape).astype(np.float64)
    d0 = g + phantoms.smooth_random_field(shape, 0.6, 3.0, rs)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 3)
    gamma = np.array([0.8, 0.6, 1.1])
    M, K, L = 2, 6, 5
    smooth = np.stack([ndi.gaussian_filter(rs.normal(0, 1, shape), 1.5) for _ in range(2)], -1)
    bins_n = np.clip(((smooth - smooth.min()) / np.ptp(smooth) * K).astype(np.int32), 0, K - 1)
    bins_v = np.clip((np.roll(smooth, 1, 0) - smooth.min()) / np.ptp(smooth) * L, 0,
                     L - 1).astype(np.int32)
    th = rs.random((M, K, L)) + 0.05
    th /= th.sum(-1, keepdims=True)
    mif_out, mif_par = pyoracle.ref_em_filter(R, d0, g, D, gamma, shape, 3,
                                              mi=(2.0, th, bins_n.ravel(), bins_v.ravel()))
    Mf, F = 2, 3
    fn = np.stack([ndi.gaussian_filter(rs.normal(0, 1, shape), 1.5) * 6.0 + f for f in range(F)], -1)
    fv = fn[..., :Mf] @ rs.normal(0, 1, (Mf, Mf)).T + rs.normal(0, 0.3, shape + (Mf,))
    coeff = rs.normal(0.0, 1.0, (Mf, F))
    sig = rs.random(Mf) * 1.5 + 0.5
    ssdf_out, ssdf_par = pyoracle.ref_em_filter(R, d0, g, D, gamma, shape, 3,
                                                ssd=(coeff, sig, fn.reshape(-1, F),
                                                     fv.reshape(-1, Mf), 0, 2.0, 0.5))
    np.savez(os.path.join(HERE, "em_filter_ref.npz"), shape=np.array(shape), d0=d0, grid=g, D=D,
             gamma=gamma, iters=3, mif_theta=th, mif_nodes=bins_n.ravel(),
             mif_voxels=bins_v.ravel(), mif_final=mif_out, mif_params=mif_par, ssdf_coeff=coeff,
             ssdf_sigma=sig, ssdf_nodes=fn.reshape(-1, F), ssdf_voxels=fv.reshape(-1, Mf),
             ssdf_alpha0=2.0, ssdf_beta0=0.5, ssdf_final=ssdf_out, ssdf_params=ssdf_par)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
