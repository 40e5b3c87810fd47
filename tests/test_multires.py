"""The device-side multi-resolution step (binder_pyramid_*) against a host restatement of
FastRegistration.move_resolution (BINDER/FastRegistration.py:550-650) built from the oracle's
resamplers, and the device coarse-to-fine loop against the same loop run through host arrays."""
import math

import numpy as np
import pytest

SIGMA_CUBIC = math.sqrt(9.0 / (8.0 * math.pi))


def _pair(shape, K, seed):
    from binder_b200 import phantoms
    from binder_b200.utils import bin_signal_robust
    pair = phantoms.make_pair(shape, seed, bins=K, n_objects=10, rms=1.5, spacing=4.0)
    v, _ = bin_signal_robust(pair.moving, K)
    return pair.u.astype(np.int32), v.astype(np.int32)


def _D(shape, order, vs):
    """BINDER/utils.py:270-365 (DCT branch, cropped), restated in numpy."""
    nd = 2 if shape[2] == 1 else 3
    grids = np.meshgrid(*[np.arange(n) for n in shape[:nd]], indexing="ij")
    D = sum((2.0 - 2 * np.cos(np.pi * g / n)) / vs[a] ** 2
            for a, (g, n) in enumerate(zip(grids, shape[:nd])))
    return (D ** order).reshape(shape)


def host_move_resolution(oracle, full, cur, field, res, freq=False, increase_gamma=False):
    """FastRegistration.move_resolution for the MI metric without smoothing, on host arrays."""
    u, v, pos = full["u"], full["v"], full["pos"]
    vsz = np.asarray(full["voxel_size"], float) * res
    nsz = np.asarray(full["node_size"], float) * res
    vshape = tuple(int(np.ceil(x / res)) for x in u.shape)
    nshape = tuple(int(np.ceil(x / res)) for x in v.shape)
    vpos = pos[::res, ::res, ::res, :] / res
    if not freq or cur - res < 0:
        new = oracle.resize_linear(field, vshape, cur / res)
    elif res != cur:
        delta = field - pos[::cur, ::cur, ::cur, :] / cur
        new = oracle.up_sample(delta, field.shape[:3], vshape) * cur / res + vpos
    else:
        new = field
    bu = u[::res, ::res, ::res]
    bv = v[::res, ::res, ::res]
    D = _D(vshape, full["order"], vsz)
    cnt = np.prod(u.shape) if increase_gamma else np.prod(vshape)
    gamma = [full["gamma"] * np.prod(vsz) * cnt * nsz[a] ** 2 for a in range(3)]
    return dict(field=new, vpos=vpos, u=bu, v=bv, D=D, gamma=gamma, vsz=vsz, nsz=nsz,
                vshape=vshape, nshape=nshape, nonzero=np.count_nonzero(bu))


def _full(shape, K=16, seed=0, vs=(1.0, 1.0, 1.0), ns=(1.0, 1.0, 1.0)):
    from binder_b200 import phantoms
    u, v = _pair(shape, K, seed)
    if len(shape) == 2:
        u, v = u[:, :, None], v[:, :, None]
        pos = phantoms.identity_positions(shape)[:, :, None, :]
    else:
        pos = phantoms.identity_positions(shape)
    return dict(u=u, v=v, pos=pos, voxel_size=vs, node_size=ns, gamma=1e-6, order=2, K=K)


def _host_registration(core, h, field, theta, K, L):
    vx, vy, vz = h["vshape"]
    reg = core.Registration(field.astype(np.float32), 1, h["vpos"].astype(np.float32),
                            h["vpos"].astype(np.float32), vx, vy, vz, *h["nshape"], 3,
                            float(h["nonzero"]))
    reg.setNonLinearTransformation(*h["gamma"], *h["vsz"], *h["nsz"],
                                   h["D"].astype(np.float32))
    reg.setMILikelihood(2.0, theta, K, L, 1, h["v"], h["u"])
    return reg


def _pyramid(mr, full, freq=False):
    return mr.Pyramid(full["u"], full["v"], full["voxel_size"], full["node_size"], full["gamma"],
                      full["order"], upsample_in_frequency_domain=freq)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(30, 26, 22), (64, 52)])
def test_first_level_matches_move_resolution(core, oracle, shape):
    from binder_b200 import multires as mr
    full = _full(shape, vs=(1.0, 1.1, 0.9)[:3], ns=(1.2, 1.0, 1.0))
    K = full["K"]
    theta = np.full((K, K), 1.0 / K, np.float32)
    pyr = _pyramid(mr, full)
    reg, info = pyr.level(2, None, 1, 2.0, theta)
    h = host_move_resolution(oracle, full, 1, full["pos"], 2)
    assert info["voxels_shape"] == h["vshape"] and info["nodes_shape"] == h["nshape"]
    assert info["non_zero_voxels"] == h["nonzero"]
    np.testing.assert_allclose(info["gamma"], h["gamma"], rtol=1e-14)
    np.testing.assert_allclose(info["voxels_voxel_size"], h["vsz"], rtol=0)
    f = reg.get_final_locations_as_numpy_array()
    np.testing.assert_allclose(f, h["field"].astype(np.float32), rtol=0, atol=4e-6)
    # same D, bins and gammas: one EM iteration from the same start gives the same positions
    ref = _host_registration(core, h, h["field"], theta, K, K)
    assert reg.EM(1, -1e30, 1, 0) == 1 and ref.EM(1, -1e30, 1, 0) == 1
    np.testing.assert_allclose(reg.get_final_locations_as_numpy_array(),
                               ref.get_final_locations_as_numpy_array(), rtol=0, atol=1e-5)
    np.testing.assert_allclose(reg.state()["gamma"], ref.state()["gamma"], rtol=1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("freq", [False, True])
@pytest.mark.parametrize("shape", [(30, 26, 22), (64, 52)])
def test_next_level_matches_move_resolution(core, oracle, shape, freq):
    from binder_b200 import multires as mr
    full = _full(shape, seed=1)
    K = full["K"]
    theta = np.full((K, K), 1.0 / K, np.float32)
    pyr = _pyramid(mr, full, freq)
    coarse, _ = pyr.level(2, None, 1, 2.0, theta)
    coarse.EM(4, -1e30, 1, 0)
    fine, info = pyr.level(1, coarse, 2, 2.0, None)
    prev_field = coarse.get_final_locations_as_numpy_array().astype(np.float64)
    h = host_move_resolution(oracle, full, 2, prev_field, 1, freq=freq)
    assert info["voxels_shape"] == h["vshape"]
    np.testing.assert_allclose(fine.get_final_locations_as_numpy_array(),
                               h["field"].astype(np.float32), rtol=0, atol=1e-5)
    # theta carried over from the coarse level
    np.testing.assert_array_equal(fine.get_likelihood_parameters(),
                                  coarse.get_likelihood_parameters())


@pytest.mark.gpu
def test_device_loop_matches_host_loop(core, oracle, monkeypatch):
    """multires.run (device hand-offs) against FastRegistration.run's loop through host arrays
    and the _core mirror (positions after [4, 2, 1] with topology correction).  Both loops run
    their DCT passes in the TF32 split, so what is compared is the hand-off between levels (FP32
    on the device, FP64 through the host) and not the operand format: the EM trajectories
    amplify differences at the passes' rounding level, and the BF16 split's is larger."""
    from binder_b200 import multires as mr
    monkeypatch.setenv("BINDER_B200_PRECISION", "1")
    full = _full((48, 40, 36), seed=2)
    K = full["K"]
    theta = np.full((K, K), 1.0 / K, np.float32)
    pyr = _pyramid(mr, full)
    reg_d, info = mr.run(pyr, [4, 2, 1], 3, theta, convergence_th=-1e30)

    cur, field, th = 1, full["pos"], theta
    for r in [4, 2, 1]:
        h = host_move_resolution(oracle, full, cur, field, r)
        reg = _host_registration(core, h, h["field"], th, K, K)
        reg.EM(3 * r, -1e30, 1, 0)
        field = reg.get_final_locations_as_numpy_array().astype(np.float64)
        th = np.asarray(reg.get_likelihood_parameters(), np.float32).reshape(K, K)
        field = core.topology_correction_3D().correct_topology(
            field, 0.01, 100.0, 10, 10, 1, h["vsz"], *h["vshape"])
        cur = r
    out_d = reg_d.get_final_locations_as_numpy_array().astype(np.float64)
    assert np.quantile(np.abs(out_d - field), 0.99) < 1e-3
    assert np.abs(out_d - field).max() < 2e-2


@pytest.mark.gpu
def test_level_errors(core):
    from binder_b200 import multires as mr
    full = _full((20, 18, 16))
    pyr = _pyramid(mr, full)
    with pytest.raises(ValueError):
        pyr.level(2, None, 1, 2.0, None)
    bad = full["u"].copy()
    bad.flat[3] = 99
    pyr2 = mr.Pyramid(bad, full["v"], gamma=1e-6)
    with pytest.raises(core.BinderError):
        pyr2.level(1, None, 1, 2.0, np.full((16, 16), 1 / 16, np.float32))
