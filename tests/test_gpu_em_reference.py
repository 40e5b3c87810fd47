"""Whole EM runs on the GPU against the reference's own EM driver (Registration.cpp:122-217,
compiled from the reference's CPU sources into oracle/_ref; fixtures in tests/golden/em_ref.npz):
MI in 3D and 2D, spline orders 1 and 2, and the SSD likelihood with both fits.  Tolerances as in
the multi-iteration oracle tests (FP32 positions and histograms, a few iterations)."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["mi3d", "mi2d", "order1", "order2", "ssd0", "ssd1"])
def test_em_matches_reference_driver(core, name):
    g = golden("em_ref.npz")
    vs = tuple(int(t) for t in g[f"{name}_shape"])
    K, L, it = int(g[f"{name}_K"]), int(g[f"{name}_L"]), int(g[f"{name}_iters"])
    order = int(g[f"{name}_order"])
    N = 2 if vs[2] == 1 else 3
    d0 = g[f"{name}_d0"].astype(np.float32).reshape(-1, N)
    grid = g[f"{name}_grid"].astype(np.float32).reshape(-1, N)
    reg = core.Registration(d0, 1, grid, grid, *vs, *vs, order, float(np.prod(vs)))
    reg.setNonLinearTransformation(*g[f"{name}_gamma"], 1, 1, 1, 1, 1, 1,
                                   g[f"{name}_D"].astype(np.float32))
    if name.startswith("ssd"):
        s = g[f"{name}_ssd"]
        reg.setSSDLikelihood(K, 1, float(s[1]), int(s[2]), float(s[3]), float(s[4]),
                             g[f"{name}_v"], g[f"{name}_u"], float(s[5]), float(s[6]))
    else:
        reg.setMILikelihood(2.0, g[f"{name}_theta"].astype(np.float32), K, L, 1, g[f"{name}_v"],
                            g[f"{name}_u"])
    assert reg.EM(it, -1e30, 1, 0) == it
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(),
                               g[f"{name}_final"], rtol=0, atol=2e-3)
    params = reg.get_likelihood_parameters()
    if name.startswith("ssd"):   # (scale, shift) as the reference reports them
        np.testing.assert_allclose(params, g[f"{name}_params"], rtol=1e-3, atol=1e-4)
    else:
        np.testing.assert_allclose(params, g[f"{name}_params"], rtol=2e-3, atol=1e-5)


@pytest.mark.parametrize("lk", ["mif", "ssdf"])
def test_filter_em_matches_reference_driver(core, lk):
    g = golden("em_filter_ref.npz")
    shape = tuple(int(t) for t in g["shape"])
    it = int(g["iters"])
    reg = core.Registration(g["d0"].astype(np.float32).reshape(-1, 3), 1,
                            g["grid"].astype(np.float32).reshape(-1, 3),
                            g["grid"].astype(np.float32).reshape(-1, 3), *shape, *shape, 3,
                            float(np.prod(shape)))
    reg.setNonLinearTransformation(*g["gamma"], 1, 1, 1, 1, 1, 1, g["D"].astype(np.float32))
    if lk == "mif":
        M, K, L = g["mif_theta"].shape
        reg.setMILikelihoodFilter(2.0, g["mif_theta"].astype(np.float32), 1, g["mif_nodes"],
                                  g["mif_voxels"], K, L, M)
    else:
        M, F = g["ssdf_coeff"].shape
        reg.setSSDLikelihoodFilter(g["ssdf_coeff"], 1, g["ssdf_sigma"], g["ssdf_nodes"],
                                   g["ssdf_voxels"], 0, float(g["ssdf_alpha0"]),
                                   float(g["ssdf_beta0"]), M, F)
    assert reg.EM(it, -1e30, 1, 0) == it
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), g[f"{lk}_final"],
                               rtol=0, atol=1e-3)
    np.testing.assert_allclose(reg.get_likelihood_parameters(), g[f"{lk}_params"], rtol=1e-3,
                               atol=1e-5)
