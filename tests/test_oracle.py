"""The FP64 oracle against the reference's own outputs (golden fixtures from its compiled CPU
sources), published known-answer vectors, and the analytic checks of the reference's tests."""
import os

import numpy as np
import pytest
from scipy import fft as sfft

from conftest import golden


# Random123 known-answer vectors for philox4x32-10 (Salmon et al., SC'11 distribution)
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
    ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
    ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
     [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(oracle, ctr, key, want):
    assert list(oracle.philox(ctr, key)) == want


def test_spline_matches_reference(oracle):
    g = golden("spline_ref.npz")
    for d, w in zip(g["d"], g["weights"][2]):
        np.testing.assert_allclose(oracle.spline3(d), w, rtol=0, atol=1e-15)
    for order in (1, 2, 3):   # Spline.cpp:44-123, every order
        for d, w in zip(g["d"], g["weights"][order - 1]):
            np.testing.assert_allclose(oracle.spline(order, d), w, rtol=0, atol=1e-15)
    # partition of unity (tests/cpu/test_check_spline.py)
    for d in np.linspace(0, 1, 17, endpoint=False):
        assert abs(oracle.spline3(d).sum() - 1.0) < 1e-14


def test_jacobian_bit_exact_vs_reference(oracle):
    g = golden("jacobian_ref.npz")
    J = oracle.jacobian3d(g["field"], tuple(g["shape"]), g["vs"])
    assert np.array_equal(J, g["J"])
    assert (J < 0).sum() > 0  # the fixture has folds


def test_topology_matches_reference(oracle):
    g = golden("topology_ref.npz")
    for k in range(2):
        shape = tuple(int(s) for s in g[f"shape{k}"])
        out, outer = oracle.topology3d(g[f"field{k}"], g["e1"], g["e2"], 10, 10, g[f"vs{k}"], shape)
        ref = g[f"out{k}"].ravel()
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-9)
        Jo = oracle.jacobian3d(out, shape)
        Jr = oracle.jacobian3d(ref, shape)
        assert np.array_equal(Jo < 0.01, Jr < 0.01)
        assert (oracle.jacobian3d(g[f"field{k}"], shape) < 0).sum() > 0


def test_topology2d_matches_reference(oracle):
    g = golden("topology2d_ref.npz")
    for k in range(int(g["ncases"])):
        shape = tuple(int(s) for s in g[f"shape{k}"])
        e1, e2 = (float(v) for v in g[f"e{k}"])
        out, outer = oracle.topology2d(g[f"field{k}"], e1, e2, 10, 10, g[f"vs{k}"], shape)
        np.testing.assert_allclose(out, g[f"out{k}"].ravel(), rtol=0, atol=1e-12)
        J0 = oracle.jacobian2d(g[f"field{k}"], shape, tuple(g[f"vs{k}"]))
        J1 = oracle.jacobian2d(out, shape, tuple(g[f"vs{k}"]))
        assert ((J0 < e1) | (J0 > e2)).sum() > 0 and not ((J1 < e1) | (J1 > e2)).any()


def test_smoothing_matches_reference(oracle):
    g = golden("smoothing_ref.npz")
    shape = g["field"].shape[:3]
    zeros = np.zeros_like(g["field"])
    cost, out = oracle.smooth(g["field"], zeros, g["D"], g["gamma"], float(g["sigma"]), shape)
    np.testing.assert_allclose(out.reshape(g["out"].shape), g["out"], rtol=0, atol=1e-12)
    assert cost == pytest.approx(float(g["cost"]), rel=1e-12)


def test_jacobian2d_bit_exact_vs_reference(oracle):
    g = golden("jacobian2d_ref.npz")
    J = oracle.jacobian2d(g["field"], tuple(int(s) for s in g["shape"]), tuple(g["vs"]))
    assert np.array_equal(J, g["J"])
    assert (J < 0).sum() > 0


def test_smoothing2d_matches_reference(oracle):
    g = golden("smoothing2d_ref.npz")
    shape = g["field"].shape[:2] + (1,)
    zeros = np.zeros_like(g["field"])
    cost, out = oracle.smooth(g["field"], zeros, g["D"], g["gamma"], float(g["sigma"]), shape)
    np.testing.assert_allclose(out.reshape(g["out"].shape), g["out"], rtol=0, atol=1e-12)
    assert cost == pytest.approx(float(g["cost"]), rel=1e-12)


def test_dct_is_scipy_ortho(oracle):
    rng = np.random.default_rng(3)
    x = rng.standard_normal((5, 8, 7))
    np.testing.assert_allclose(oracle.dct3(x), sfft.dctn(x, norm="ortho"), atol=1e-12)
    np.testing.assert_allclose(oracle.dct3(oracle.dct3(x), inverse=True), x, atol=1e-12)


def test_smoothing_equals_mirrored_dft(oracle):
    """tests/gpu/test_smoothing_and_log_cost.py: DCT smoothing equals a DFT of the mirrored
    signal with the full eigenvalue matrix, and the prior cost agrees (restated)."""
    from binder_b200.utils import initialize_fourier_domain_smoothing
    rng = np.random.default_rng(7)
    shape = (11, 20, 7)
    gamma = 5.0
    field = rng.standard_normal(shape + (3,))
    D, Dfull = initialize_fourier_domain_smoothing(shape, True, 2, 3, return_full_matrix=True)
    cost, out = oracle.smooth(field, np.zeros_like(field), D, [gamma] * 3, 1.0, shape)
    out = out.reshape(field.shape)
    cost_fft = 0.0
    for n in range(3):
        m = field[..., n]
        for ax in range(3):
            m = np.concatenate([m, np.flip(m, axis=ax)], axis=ax)
        C = np.fft.fftn(m) / m.size / (1 + gamma * Dfull)
        cost_fft += 0.5 * gamma * m.size * np.sum(Dfull * np.abs(C) ** 2) / 8
        t = np.fft.ifftn(C).real * m.size
        np.testing.assert_allclose(t[:shape[0], :shape[1], :shape[2]], out[..., n], atol=1e-10)
    assert cost == pytest.approx(cost_fft, rel=1e-9)


def test_mi_update_matches_reference(oracle):
    g = golden("mi_ref.npz")
    K, L = g["hist"].shape
    th = oracle.theta_map(g["hist"], K, L, float(g["alpha"]))
    np.testing.assert_allclose(th.reshape(K, L), g["theta"], rtol=1e-15, atol=0)
    assert oracle.dirichlet_cost(th, K, L, float(g["alpha"])) == pytest.approx(float(g["cost"]),
                                                                               rel=1e-13)


def test_mi_filter_matches_reference(oracle):
    """MILikelihoodFilter (compute_likelihood, accumulate_info, update_parameters, compute_cost)
    against the reference's compiled class: bins of channel m read at [index + m]."""
    g = golden("mi_filter_ref.npz")
    M, K, L = int(g["M"]), int(g["K"]), int(g["L"])
    nshape = tuple(int(t) for t in g["nshape"])
    theta, nodes, voxels = g["theta"], g["nodes"], g["voxels"]
    for (v, x, y, z), want in zip(g["pairs"], g["likelihood"]):
        got = oracle.mi_filter_likelihood(theta, voxels, nodes, K, L, M, nshape, v, (x, y, z))
        assert got == want                                                  # bit-exact
    # the histogram of the same (voxel, node, posterior) triples, indexed as the likelihood reads
    hist = np.zeros((M, K, L))
    for (v, x, y, z), p in zip(g["pairs"], g["posterior"]):
        inside = 0 <= x < nshape[0] and 0 <= y < nshape[1] and 0 <= z < nshape[2]
        node = (x * nshape[1] + y) * nshape[2] + z
        for m in range(M):
            hist[m, nodes[node + m] if inside else 0, voxels[v + m]] += p
    th = oracle.theta_map(hist, M * K, L, float(g["alpha"]))
    np.testing.assert_allclose(th.reshape(M, K, L), g["theta_out"], rtol=1e-15, atol=0)
    assert oracle.dirichlet_cost(th, M * K, L, float(g["alpha"])) == \
        pytest.approx(float(g["cost"]), rel=1e-13)


def test_mi_filter_estep_reduces_to_mi(oracle):
    """One channel is the MI likelihood exactly; a second channel with a flat theta scales every
    weight by 1/L, so posteriors and channel 0's histogram are unchanged and mll grows by V log L."""
    rng = np.random.default_rng(11)
    vshape, nshape, K, L = (7, 6, 5), (7, 6, 5), 6, 5
    V = int(np.prod(vshape))
    d = np.stack(np.indices(vshape), -1).reshape(-1, 3) + rng.normal(0, 0.7, (V, 3))
    u = rng.integers(0, L, V + 1).astype(np.int32)
    v = rng.integers(0, K, V + 1).astype(np.int32)
    th = rng.random((K, L)) + 0.05
    th /= th.sum(1, keepdims=True)
    mll, dream, hist, deg = oracle.estep(d, u[:V], v[:V], th, vshape, nshape, K, L)
    mll1, dream1, hist1, deg1 = oracle.estep_filter(d, u[:V], v[:V], th, vshape, nshape, K, L, 1)
    assert mll1 == pytest.approx(mll, rel=1e-13) and deg1 == deg  # OpenMP reduction order
    np.testing.assert_array_equal(dream1, dream)
    np.testing.assert_array_equal(hist1, hist)
    th2 = np.stack([th, np.full((K, L), 1.0 / L)])
    mll2, dream2, hist2, _ = oracle.estep_filter(d, u, v, th2, vshape, nshape, K, L, 2)
    assert mll2 == pytest.approx(mll + V * np.log(L), rel=1e-12)
    np.testing.assert_allclose(dream2, dream, rtol=0, atol=1e-12)
    np.testing.assert_allclose(hist2[:K * L], hist, rtol=1e-12, atol=1e-12)
    assert hist2[K * L:].sum() == pytest.approx(hist.sum(), rel=1e-12)


def _prior_covariance(shape, gamma, sigma, order):
    """sigma^2 (I + gamma sigma^2 Gamma)^-1 with Neumann finite differences
    (tests/gpu/test_sampling_DCT_3D.py), in Fortran voxel order."""
    Nx, Ny, Nz = shape

    def d1(n):
        G = np.diag(np.ones(n)) - np.diag(np.ones(n - 1), -1)
        return G[1:, :]

    gp = gamma * sigma ** 2
    N = Nx * Ny * Nz
    if order == 1:
        Gr = np.kron(np.eye(Nz), np.kron(np.eye(Ny), d1(Nx)))
        Gc = np.kron(np.eye(Nz), np.kron(d1(Ny), np.eye(Nx)))
        Gd = np.kron(d1(Nz), np.kron(np.eye(Nx), np.eye(Ny)))
        A = np.eye(N) + gp * (Gr.T @ Gr + Gc.T @ Gc + Gd.T @ Gd)
    else:
        G2 = [d1(n).T @ d1(n) for n in (Nx, Ny, Nz)]
        G = np.kron(np.eye(Nz), np.kron(np.eye(Ny), G2[0])) + \
            np.kron(np.eye(Nz), np.kron(G2[1], np.eye(Nx))) + \
            np.kron(G2[2], np.kron(np.eye(Nx), np.eye(Ny)))
        A = np.eye(N) + gp * G.T @ G
    return sigma ** 2 * np.linalg.inv(A)


@pytest.mark.parametrize("order", [1, 2])
def test_prior_sampling_covariance(oracle, order):
    """tests/gpu/test_sampling_DCT_3D.py restated on the oracle's prior sampler (1e5 samples)."""
    from binder_b200.utils import initialize_fourier_domain_smoothing
    shape, gamma, sigma = (3, 5, 4), 5.0, 0.34
    cov = _prior_covariance(shape, gamma, sigma, order)
    D = initialize_fourier_domain_smoothing(shape, True, order, 3)
    s = oracle.sample_field(np.zeros(shape + (3,)), D, [gamma] * 3, sigma, shape, 100000, seed=99)
    x = s[..., 0].reshape(-1, np.prod(shape), order="F")
    emp = x.T @ x / x.shape[0]
    np.testing.assert_allclose(emp, cov, rtol=1e-3, atol=1e-3)


@pytest.mark.parametrize("rfa", [0, 1])
def test_ssd_filter_matches_reference(oracle, rfa):
    """SSDLikelihoodFilter (compute_log_likelihood, accumulate_info, update_parameters with the
    coefficient solve and the sigma update, compute_cost) against the reference's compiled class."""
    g = golden("ssd_filter_ref.npz")
    k = f"rfa{rfa}_"
    M, F = int(g[k + "M"]), int(g[k + "F"])
    nshape = tuple(int(t) for t in g["nshape"])
    nodes, voxels = g[k + "nodes"], g[k + "voxels"]
    p = oracle.ssdf_params(g[k + "coeff"], g[k + "sigma"], rfa, float(g["alpha0"]),
                           float(g["beta0"]))
    got = [oracle.ssdf_loglik(p, nodes, voxels, nshape, v, (x, y, z))
           for v, x, y, z in g["pairs"]]
    np.testing.assert_allclose(got, g[k + "loglik"], rtol=1e-14, atol=0)
    # the accumulators of the same (voxel, node, posterior) triples, as accumulate_info sums them
    Vn = int(np.prod(nshape))
    gam, s1, s2, out = np.zeros(Vn), np.zeros(M * Vn), np.zeros(M * Vn), np.zeros(1 + 2 * M)
    for (v, x, y, z), w in zip(g["pairs"], g["posterior"]):
        xv = voxels[v]
        if 0 <= x < nshape[0] and 0 <= y < nshape[1] and 0 <= z < nshape[2]:
            j = (x * nshape[1] + y) * nshape[2] + z
            gam[j] += w
            s1[np.arange(M) * Vn + j] += w * xv
            s2[np.arange(M) * Vn + j] += w * xv * xv
        else:
            out[0] += w
            out[1:1 + M] += w * xv
            out[1 + M:] += w * xv * xv
    cost = oracle.ssdf_update(p, nodes, nshape, (gam, s1, s2, out))
    np.testing.assert_allclose(np.array(p.coeff[:M * F]).reshape(M, F), g[k + "coeff_out"],
                               rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(np.array(p.sigma[:M]), g[k + "sigma_out"], rtol=1e-10)
    assert cost == pytest.approx(float(g[k + "cost"]), rel=1e-10)


def test_em_runs_match_reference_driver(oracle):
    """Whole EM runs (MI 3D and 2D, spline orders 1 and 2, SSD with both fits) of the oracle against
    the reference's own EM driver (Registration.cpp:122-217, compiled in oracle/_ref)."""
    import math
    g = golden("em_ref.npz")
    sig = {3: math.sqrt(9.0 / (8.0 * math.pi)), 2: math.sqrt(8.0 / (9.0 * math.pi)), 1: 0.4}
    for name in g["names"]:
        vs = tuple(int(t) for t in g[f"{name}_shape"])
        K, L, it = int(g[f"{name}_K"]), int(g[f"{name}_L"]), int(g[f"{name}_iters"])
        order = int(g[f"{name}_order"])
        oracle.set_spline_order(order)
        try:
            if name.startswith("ssd"):
                s = g[f"{name}_ssd"]
                p = oracle.SSDParams(int(s[2]), s[1], s[4], s[3], s[5], s[6])
                n, final, _ = oracle.ssd_em(g[f"{name}_d0"], g[f"{name}_grid"], g[f"{name}_u"],
                                            g[f"{name}_v"], p, g[f"{name}_D"],
                                            g[f"{name}_gamma"], sig[order], vs, vs, K, L,
                                            float(np.prod(vs)), it, -1e30)
                np.testing.assert_allclose([p.scale, p.shift], g[f"{name}_params"], rtol=1e-12,
                                           err_msg=name)
            else:
                n, final, theta, _ = oracle.em(g[f"{name}_d0"], g[f"{name}_grid"], g[f"{name}_u"],
                                               g[f"{name}_v"], g[f"{name}_theta"], 2.0,
                                               g[f"{name}_D"], g[f"{name}_gamma"], sig[order], vs,
                                               vs, K, L, float(np.prod(vs)), it, -1e30)
                np.testing.assert_allclose(theta, g[f"{name}_params"], rtol=0, atol=1e-13,
                                           err_msg=name)
        finally:
            oracle.set_spline_order(3)
        assert n == it
        np.testing.assert_allclose(final, g[f"{name}_final"], rtol=0, atol=1e-11, err_msg=name)


def test_filter_em_runs_match_reference_driver(oracle):
    """EM runs with the MI filter and SSD filter likelihoods: the oracle's E-steps and updates,
    iterated with its smoothing, against the reference's own EM driver."""
    import math
    g = golden("em_filter_ref.npz")
    shape = tuple(int(t) for t in g["shape"])
    sig = math.sqrt(9.0 / (8.0 * math.pi))
    M, K, L = g["mif_theta"].shape
    d, th = g["d0"], g["mif_theta"]
    for _ in range(int(g["iters"])):
        _, dream, hist, _ = oracle.estep_filter(d, g["mif_voxels"], g["mif_nodes"], th, shape,
                                                shape, K, L, M)
        th = oracle.theta_map(hist, M * K, L, 2.0)
        _, d = oracle.smooth(dream, g["grid"], g["D"], g["gamma"], sig, shape)
    np.testing.assert_allclose(d, g["mif_final"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(th, g["mif_params"], rtol=0, atol=1e-13)
    p = oracle.ssdf_params(g["ssdf_coeff"], g["ssdf_sigma"], 0, float(g["ssdf_alpha0"]),
                           float(g["ssdf_beta0"]))
    d = g["d0"]
    for _ in range(int(g["iters"])):
        _, dream, acc = oracle.ssdf_estep(d, g["ssdf_nodes"], g["ssdf_voxels"], p, shape, shape)
        oracle.ssdf_update(p, g["ssdf_nodes"], shape, acc, True)
        _, d = oracle.smooth(dream, g["grid"], g["D"], g["gamma"], sig, shape)
    np.testing.assert_allclose(d, g["ssdf_final"], rtol=0, atol=1e-11)
    Mf, F = g["ssdf_coeff"].shape
    np.testing.assert_allclose(np.array(p.coeff[:Mf * F]), g["ssdf_params"], rtol=1e-10, atol=1e-12)


def _oracle_chains(oracle, g, gamma, chains=32, seed0=5000):
    import math
    from sampler_stats import UPPER
    shape = tuple(int(s) for s in g["shape"])
    V = int(np.prod(shape))
    K, L = int(g["K"]), int(g["L"])
    grid = np.stack(np.indices(shape), -1).astype(np.float64)
    oracle.set_threads(os.cpu_count() or 1)
    means, covs = [], []
    for ch in range(chains):
        m, cv, *_ = oracle.sampler(g["d0"], np.zeros_like(g["d0"]), grid, g["u"], g["v"],
                                   g["theta"], float(g["alpha"]), g["D"], gamma,
                                   math.sqrt(9.0 / (8.0 * math.pi)), [1, 1, 1], [1, 1, 1], shape,
                                   shape, K, L, seed0 + ch, int(g["N_b"]), int(g["N_s"]),
                                   sample_gamma=1, sample_gamma_every=1, chain=ch)
        means.append(m.reshape(V, 3))
        covs.append(cv.reshape(V, 9)[:, UPPER])
    return means, covs


def test_oracle_sampler_matches_reference_in_distribution(oracle):
    """32 oracle chains against 32 chains of the reference's own Registration::sampler from the
    same start, every switch on (categorical draws, Dirichlet theta, DCT-domain noise, nu):
    chain means and covariances agree within Monte Carlo error."""
    from sampler_stats import agrees, fixture, summary, zscores
    g = fixture()
    zm, zc = zscores(g, *_oracle_chains(oracle, g, g["gamma"]))
    assert agrees(zm), summary(zm)
    assert agrees(zc), summary(zc)


def test_sampler_parity_check_has_power(oracle):
    """The same check rejects a sampler with a planted mistake: the oracle run with the prior's
    precisions gamma tripled (a wrong model) leaves Monte Carlo error far behind."""
    from sampler_stats import agrees, fixture, summary, zscores
    g = fixture()
    zm, zc = zscores(g, *_oracle_chains(oracle, g, 3.0 * g["gamma"], chains=8))
    assert not agrees(zm) or not agrees(zc), (summary(zm), summary(zc))


def _ssd_counts(K=16, L=16, seed=5):
    """a joint count histogram with a linear bin relation l ~ 0.9 k + 1 plus noise"""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, K, 4000)
    l = np.clip(np.rint(0.9 * k + 1 + rng.normal(0, 1.2, k.size)), 0, L - 1).astype(int)
    h = np.zeros((K, L))
    np.add.at(h, (k, l), 1.0)
    return h


@pytest.mark.parametrize("shift_scale", [0, 1])
def test_ssd_sample_distribution(oracle, shift_scale):
    """The SSD likelihood's parameter draw (SSDLikelihood.cpp:167-302 with sample = 1), restated
    with Philox: over 4000 sweeps, (shift, scale) has the mean A^-1 b and covariance A^-1 of the
    reference's bivariate normal, and 1 / sigmaSq the mean den^2 / num of its gamma draw
    (shape den / 2, scale 2 den / num, the reference's parameterisation); with shiftScale 1 the
    num of each draw depends on the drawn shift and scale, so there the gamma is checked through
    its shape: the coefficient of variation of g * num / den^2 is sqrt(2 / den)."""
    K = L = 16
    h = _ssd_counts(K, L)
    n = 4000
    draws = []
    for sweep in range(n):
        p = oracle.SSDParams(shift_scale, 4.0, 0.0, 1.0, 1.0, 1.0)
        assert oracle.ssd_sample(h, K, L, p, 77, sweep) == 0
        draws.append((p.shift, p.scale, p.sigma2))
    d = np.array(draws)
    kk = np.arange(K, dtype=float)
    ll = np.arange(L, dtype=float)
    G = h.sum(1)
    S1 = h @ ll
    S2 = h @ (ll * ll)
    den = G.sum() + 1.0
    if shift_scale == 0:
        num = (h * (ll[None, :] - kk[:, None]) ** 2).sum() + 1.0
        g = 1.0 / d[:, 2]
        want = den * den / num
        assert abs(g.mean() - want) < 4 * want * np.sqrt(2.0 / den) / np.sqrt(n)
        assert np.all(d[:, 0] == 0.0) and np.all(d[:, 1] == 1.0)
        return
    A = np.array([[G.sum(), G @ kk], [G @ kk, G @ (kk * kk)]])
    b = np.array([S1.sum(), S1 @ kk])
    x = np.linalg.solve(A, b)
    cov = np.linalg.inv(A)
    sd = np.sqrt(np.diag(cov))
    assert np.all(np.abs(d[:, :2].mean(0) - x) < 4 * sd / np.sqrt(n))
    emp = np.cov(d[:, :2].T)
    np.testing.assert_allclose(emp, cov, rtol=0.12)
    num = np.array([S2.sum() - 2 * (S1 @ (s + c * kk)) + G @ (s + c * kk) ** 2 + 1.0
                    for s, c, _ in d])
    ratio = (1.0 / d[:, 2]) * num / (den * den)
    assert abs(ratio.mean() - 1.0) < 4 * np.sqrt(2.0 / den) / np.sqrt(n)
    assert ratio.std() == pytest.approx(np.sqrt(2.0 / den), rel=0.1)
