"""A batch of sampler chains in one pass per step (Registration.sampler_chains) against the
single-chain sampler: chain c of the batch is the single-chain run with chain index c from the
same state, draw for draw, and the pooled moments are the chains' moments combined."""
import numpy as np
import pytest

from test_gpu_parity import make_case, new_reg

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(12, 14, 10), (9, 7, 20)])
def test_batch_chain_equals_single_chain_draw_for_draw(core, shape):
    c = make_case(shape=shape, seed=5)
    reg = new_reg(core, c)
    C, seed, Nb, Ns = 4, 31337, 2, 5
    reg.set_chain(0)
    means, covs, pm, pc = reg.sampler_chains(seed, C, Nb, Ns, 1, 2, 1, 1, 1)
    for ch in range(C):
        reg.reset()
        reg.set_chain(ch)
        m1, c1 = reg.sampler(seed, Nb, Ns, 1, 2, 1, 1, 1)
        dm = np.abs(means[ch] - m1).ravel()
        dc = np.abs(covs[ch] - c1).ravel()
        # the same Philox draws and the same arithmetic per element; only the FP64 cost sums that
        # feed nu (atomics in launch order) may differ in their last bits
        assert np.quantile(dm, 0.999) < 1e-5 and dm.max() < 1e-2, (ch, dm.max())
        assert np.quantile(dc, 0.999) < 1e-5, (ch, dc.max())
    # chains are different chains
    assert np.abs(means[0] - means[1]).max() > 1e-3
    # pooled moments: the average of the chain means, and M2 combined over the chains
    np.testing.assert_allclose(pm, means.mean(0), rtol=0, atol=1e-9)
    dev = means - means.mean(0)
    m2 = (covs * (Ns - 1)).sum(0) + Ns * np.einsum("c...i,c...j->...ij", dev, dev)
    np.testing.assert_allclose(pc, m2 / (C * Ns - 1), rtol=1e-9, atol=1e-12)


def test_batch_leaves_object_state(core):
    c = make_case(seed=6)
    reg = new_reg(core, c)
    before = reg.get_final_locations_as_numpy_array().copy()
    theta = reg.get_likelihood_parameters().copy()
    reg.sampler_chains(5, 3, 1, 3, 1, 1, 1, 1, 1, per_chain=False)
    assert np.array_equal(reg.get_final_locations_as_numpy_array(), before)
    assert np.array_equal(reg.get_likelihood_parameters(), theta)
