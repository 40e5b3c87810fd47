"""2D registration (Nz = 1, two position components, 16-neighbour E-step, 2D DCT prior) through the
C ABI / _core mirror against the FP64 oracle and the reference's 2D golden outputs.  Tolerances
as in the 3D parity tests: positions and theta FP32 on the GPU, Welford and Jacobians FP64."""
import math

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

SIGMA_CUBIC = math.sqrt(9.0 / (8.0 * math.pi))


def make_case2d(shape=(40, 36), K=16, L=12, seed=0, disp=0.6):
    from binder_b200 import phantoms
    from binder_b200.utils import bin_signal_robust, initialize_fourier_domain_smoothing
    rng = np.random.default_rng(seed)
    pair = phantoms.make_pair(shape, seed, bins=L, n_objects=8, axes=(3.0, 10.0), rms=1.0,
                              spacing=3.0)
    v, _ = bin_signal_robust(pair.moving, K)
    grid = phantoms.identity_positions(shape)
    d0 = (grid + phantoms.smooth_random_field(shape, disp, 3.0, rng)).astype(np.float32)
    theta = rng.random((K, L)) + 0.05
    theta = (theta / theta.sum(1, keepdims=True)).astype(np.float32)
    D = initialize_fourier_domain_smoothing(shape, True, 2, 2).astype(np.float32)
    return dict(shape=shape, vshape=shape + (1,), K=K, L=L, u=pair.u, v=v.astype(np.int32),
                grid=grid, d0=d0, theta=theta, D=D, gamma=(0.8, 0.6, 1.0))


def new_reg2d(core, c):
    nx, ny = c["shape"]
    reg = core.Registration(c["d0"], 1, c["grid"], c["grid"], nx, ny, 1, nx, ny, 1, 3,
                            float(nx * ny))
    reg.setNonLinearTransformation(*c["gamma"], 1, 1, 1, 1, 1, 1, c["D"])
    reg.setMILikelihood(2.0, c["theta"], c["K"], c["L"], 1, c["v"], c["u"])
    return reg


def test_shapes_follow_the_reference(core):
    c = make_case2d()
    nx, ny = c["shape"]
    reg = new_reg2d(core, c)
    assert reg.get_shape() == [nx, ny, 1, 2]
    assert reg.get_final_locations_as_numpy_array().shape == (nx, ny, 1, 2)
    assert reg.get_dream_locations().size == nx * ny * 2


def test_one_em_iteration_matches_oracle(core, oracle):
    c = make_case2d()
    vshape, K, L = c["vshape"], c["K"], c["L"]
    reg = new_reg2d(core, c)
    assert reg.EM(1, -1e30, 1, 0) == 1
    dream_g = reg.get_dream_locations()
    theta_g = reg.get_likelihood_parameters()
    final_g = reg.get_final_locations_as_numpy_array().ravel()
    st = reg.iteration_stats()[0]

    d0 = c["d0"].astype(np.float64)
    mll, dream, hist, deg = oracle.estep(d0, c["u"], c["v"], c["theta"].astype(np.float64),
                                         vshape, vshape, K, L)
    theta = oracle.theta_map(hist, K, L, 2.0)
    lpt, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA_CUBIC, vshape)
    assert deg == 0
    np.testing.assert_allclose(dream_g, dream, rtol=0, atol=5e-5)       # FP32 E-step
    np.testing.assert_allclose(theta_g, theta, rtol=1e-4, atol=1e-7)    # FP32 histogram
    assert st[0] == pytest.approx(mll, rel=1e-6)
    assert st[1] == pytest.approx(oracle.dirichlet_cost(theta, K, L, 2.0), rel=1e-6)
    assert st[2] == pytest.approx(lpt, rel=2e-4)                        # FP32 DCT prior cost
    np.testing.assert_allclose(final_g, final, rtol=0, atol=2e-4)      # FP32 DCT M-step


def test_em_run_matches_oracle_and_mi(core, oracle):
    c = make_case2d(shape=(48, 44), seed=1)
    vshape, K, L = c["vshape"], c["K"], c["L"]
    reg = new_reg2d(core, c)
    assert reg.EM(12, -1e30, 1, 0) == 12
    final_g = reg.get_final_locations_as_numpy_array().astype(np.float64).ravel()
    theta_g = reg.get_likelihood_parameters()
    stats = reg.iteration_stats()
    it, final_o, theta_o, stats_o = oracle.em(c["d0"], c["grid"], c["u"], c["v"], c["theta"], 2.0,
                                             c["D"], c["gamma"], SIGMA_CUBIC, vshape, vshape, K, L,
                                             float(np.prod(vshape)), 12, -1e30)
    assert it == 12
    np.testing.assert_allclose(final_g, final_o, rtol=0, atol=2e-3)
    np.testing.assert_allclose(theta_g, theta_o, rtol=2e-3, atol=1e-5)
    np.testing.assert_allclose(stats[:, 3], stats_o[:, 3], rtol=1e-5)
    _, _, h_g, _ = oracle.estep(final_g, c["u"], c["v"], theta_o, vshape, vshape, K, L)
    _, _, h_o, _ = oracle.estep(final_o, c["u"], c["v"], theta_o, vshape, vshape, K, L)
    mi_g, mi_o = oracle.mutual_information(h_g, K, L), oracle.mutual_information(h_o, K, L)
    assert abs(mi_g - mi_o) <= 1e-3 * abs(mi_o)


def test_em_convergence_rule(core, oracle):
    c = make_case2d(seed=2)
    reg = new_reg2d(core, c)
    n = reg.EM(200, 1e-3, 1, 0)
    it, *_ = oracle.em(c["d0"], c["grid"], c["u"], c["v"], c["theta"], 2.0, c["D"], c["gamma"],
                       SIGMA_CUBIC, c["vshape"], c["vshape"], c["K"], c["L"],
                       float(np.prod(c["vshape"])), 200, 1e-3)
    assert 1 <= n < 200 and abs(n - it) <= 1


def test_smoothing_matches_reference_golden(core):
    g = golden("smoothing2d_ref.npz")
    nx, ny = g["field"].shape[:2]
    t = core.NonLinearTransformation(*g["gamma"], 1, 1, 1, 1, 1, 1, g["D"], nx, ny, 1, 1,
                                     float(g["sigma"]), 0.0)
    assert t.get_shape() == [nx, ny, 1, 2]
    cost, out = t.smooth_deformation(g["field"])
    np.testing.assert_allclose(out.reshape(g["out"].shape), g["out"], rtol=0, atol=2e-6)
    assert cost == pytest.approx(float(g["cost"]), rel=1e-5)


@pytest.mark.parametrize("order", [1, 2])
def test_prior_sampling_covariance(core, order):
    """The 3D covariance test of the prior sampler (tests/gpu/test_sampling_DCT_3D.py) restated on
    a 2D grid: the Neumann finite-difference covariance with Nz = 1 (1e5 samples)."""
    from test_oracle import _prior_covariance
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape, gamma, sigma = (4, 5), 5.0, 0.34
    cov = _prior_covariance(shape + (1,), gamma, sigma, order)
    D = initialize_fourier_domain_smoothing(shape, True, order, 2)
    t = core.NonLinearTransformation(gamma, gamma, gamma, 1, 1, 1, 1, 1, 1, D, *shape, 1, 1, sigma,
                                     0.0)
    s = t.sampleDeformationField(np.zeros(shape + (2,)), 100000)
    for n in range(2):
        x = s[..., n].astype(np.float64).reshape(-1, np.prod(shape), order="F")
        np.testing.assert_allclose(x.T @ x / x.shape[0], cov, rtol=1e-3, atol=1e-3)


def test_sampler_matches_oracle_draw_for_draw(core, oracle):
    c = make_case2d(seed=3)
    vshape, K, L = c["vshape"], c["K"], c["L"]
    reg = new_reg2d(core, c)
    mean_g, cov_g = reg.sampler(777, 1, 4, 1, 2, 1, 1, 1)
    assert mean_g.shape == vshape + (2,) and cov_g.shape == vshape + (2, 2)
    gam_g = reg.state()["gamma"]
    mean_o, cov_o, _, _, gam_o, capped = oracle.sampler(
        c["d0"], np.zeros_like(c["d0"]), c["grid"], c["u"], c["v"], c["theta"], 2.0, c["D"],
        c["gamma"], SIGMA_CUBIC, [1, 1, 1], [1, 1, 1], vshape, vshape, K, L, 777, 1, 4,
        sample_gamma=1, sample_gamma_every=2)
    assert capped == 0
    dm = np.abs(mean_g.ravel() - mean_o)
    assert np.quantile(dm, 0.99) < 1e-3
    assert np.median(np.abs(cov_g.ravel() - cov_o)) < 1e-4
    np.testing.assert_allclose(gam_g[:2], gam_o[:2], rtol=1e-3)


def test_jacobian2d_bit_exact_vs_reference(core):
    g = golden("jacobian2d_ref.npz")
    nx, ny = (int(s) for s in g["shape"])
    J = core.compute_jacobian_determinant_2D(g["field"], nx, ny, *g["vs"])
    assert J.shape == (nx, ny)
    assert np.array_equal(J.ravel(), g["J"])


def test_jacobian2d_large_bit_exact_vs_oracle(core, oracle):
    from binder_b200 import phantoms
    shape = (1024, 768)
    rng = np.random.default_rng(9)
    f = phantoms.identity_positions(shape) + \
        phantoms.smooth_random_field(shape, 3.0, 2.0, rng).astype(np.float64)
    J = core.compute_jacobian_determinant_2D(f, *shape, 0.8, 1.3).ravel()
    assert np.array_equal(J, oracle.jacobian2d(f, shape, (0.8, 1.3)))
    assert (J < 0).sum() > 0


def test_topology2d_matches_reference_golden(core, oracle):
    g = golden("topology2d_ref.npz")
    tc = core.topology_correction_2D()
    for k in range(int(g["ncases"])):
        shape = tuple(int(s) for s in g[f"shape{k}"])
        e1, e2 = (float(v) for v in g[f"e{k}"])
        out = tc.correct_topology(g[f"field{k}"], e1, e2, 10, 10, 1, g[f"vs{k}"], *shape)
        assert out.shape == shape + (2,)
        ref = g[f"out{k}"]
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-9)   # FP64 Hartley vs FFT Poisson
        vs = tuple(g[f"vs{k}"])
        Jg, Jr = oracle.jacobian2d(out, shape, vs), oracle.jacobian2d(ref, shape, vs)
        assert np.array_equal((Jg < e1) | (Jg > e2), (Jr < e1) | (Jr > e2))
        assert tc.last_stats["below_e1_before"] > 0
        assert tc.last_stats["below_e1_after"] == 0 and tc.last_stats["above_e2_after"] == 0


def test_topology2d_larger_field_matches_oracle(core, oracle):
    from binder_b200 import phantoms
    shape = (96, 80)
    rng = np.random.default_rng(11)
    f = phantoms.identity_positions(shape) + \
        phantoms.smooth_random_field(shape, 2.5, 1.5, rng).astype(np.float64)
    assert (oracle.jacobian2d(f, shape) < 0.01).sum() > 0
    tc = core.topology_correction_2D()
    out = tc.correct_topology(f, 0.01, 100.0, 10, 10, 1, [1.0, 1.0], *shape)
    ref, _ = oracle.topology2d(f, 0.01, 100.0, 10, 10, [1.0, 1.0], shape)
    np.testing.assert_allclose(out.ravel(), ref, rtol=0, atol=1e-8)
    assert tc.last_stats["below_e1_after"] == 0


def first_walk_size(f, shape, e1, e2):
    """Flagged cells of the limiter's first walk and the nodes their flagged corners read (corner
    (vx, vy) of cell (x, y): the cell's x edge on row y + vy and y edge on column x + vx)."""
    P = f.reshape(shape + (2,))
    nx, ny = shape
    flag = np.zeros((nx - 1, ny - 1), bool)
    nodes = set()
    for vx in (0, 1):
        for vy in (0, 1):
            ex = P[1:, vy:ny - 1 + vy] - P[:-1, vy:ny - 1 + vy]
            ey = P[vx:nx - 1 + vx, 1:] - P[vx:nx - 1 + vx, :-1]
            det = ex[..., 0] * ey[..., 1] - ey[..., 0] * ex[..., 1]
            out = (det < e1) | (det > e2)
            flag |= out
            for x, y in zip(*np.nonzero(out)):
                nodes.update({(x, y + vy), (x + vx, y)})
    return int(flag.sum()), len(nodes)


# the limiter walks shared-memory copies of up to 4096 cells and 6016 nodes, else global memory
@pytest.mark.parametrize("shape,amp,sigma,seed,regime", [
    ((200, 200), 0.35, 0.5, 4, "staged"),
    ((200, 200), 0.404, 0.5, 4, "too many nodes"),
    ((200, 180), 3.0, 1.0, 1, "too many cells"),
])
def test_topology2d_limiter_walks_match_oracle(core, oracle, shape, amp, sigma, seed, regime):
    from binder_b200 import phantoms
    rng = np.random.default_rng(seed)
    f = phantoms.identity_positions(shape) + \
        phantoms.smooth_random_field(shape, amp, sigma, rng).astype(np.float64)
    cells, nodes = first_walk_size(f, shape, 0.01, 100.0)
    assert {"staged": cells <= 4096 and nodes <= 6016,
            "too many nodes": cells <= 4096 and nodes > 6016,
            "too many cells": cells > 4096}[regime], (cells, nodes)
    tc = core.topology_correction_2D()
    out = tc.correct_topology(f, 0.01, 100.0, 10, 10, 1, [1.0, 1.0], *shape)
    ref, _ = oracle.topology2d(f, 0.01, 100.0, 10, 10, [1.0, 1.0], shape)
    np.testing.assert_allclose(out.ravel(), ref, rtol=0, atol=1e-8)
    assert tc.last_stats["below_e1_after"] == (oracle.jacobian2d(ref, shape) < 0.01).sum()


def test_registration_topology2d_on_device(core):
    """The device-side correction of a 2D registration's positions equals the host entry point
    applied to the same (FP32) positions."""
    c = make_case2d(seed=5, disp=2.0)
    nx, ny = c["shape"]
    reg = new_reg2d(core, c)
    before = reg.get_final_locations_as_numpy_array().reshape(nx, ny, 2).astype(np.float64)
    st = reg.correct_topology(0.01, 100.0, 10, 10, [1.0, 1.0])
    after = reg.get_final_locations_as_numpy_array().reshape(nx, ny, 2)
    host = core.topology_correction_2D().correct_topology(before, 0.01, 100.0, 10, 10, 1,
                                                          [1.0, 1.0], nx, ny)
    assert st["below_e1_before"] > 0 and st["below_e1_after"] == 0
    np.testing.assert_allclose(after, host.astype(np.float32), rtol=0, atol=1e-5)


@pytest.mark.parametrize("fused", ["1", "0"])
def test_small_image_m_step_kinds_match_oracle(core, oracle, fused, monkeypatch):
    """Images up to 128 x 128 run the whole M-step as one cluster launch (mstep2d.cu);
    BINDER_B200_FUSED2D=0 keeps the separate tensor-core passes.  Both give the oracle's
    iteration, on a ragged shape whose rows and columns do not split evenly over the cluster."""
    monkeypatch.setenv("BINDER_B200_FUSED2D", fused)
    c = make_case2d(shape=(45, 38), seed=8)
    vshape, K, L = c["vshape"], c["K"], c["L"]
    reg = new_reg2d(core, c)
    assert reg.EM(1, -1e30, 1, 0) == 1
    mll, dream, hist, _ = oracle.estep(c["d0"].astype(np.float64), c["u"], c["v"],
                                       c["theta"].astype(np.float64), vshape, vshape, K, L)
    lpt, final = oracle.smooth(dream, c["grid"], c["D"], c["gamma"], SIGMA_CUBIC, vshape)
    st = reg.iteration_stats()[0]
    assert st[2] == pytest.approx(lpt, rel=2e-4)
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array().ravel(), final, rtol=0,
                               atol=2e-4)
