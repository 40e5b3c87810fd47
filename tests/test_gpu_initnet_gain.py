"""What the trained initialiser gains over the method without it, on held-out pairs.

The committed checkpoint (binder_b200/data/initnet_seeded_64.npz, from the recipe in
binder_b200/initnet.py) is the EM-seeded network: it sees the moving and fixed images and the
displacement after 16 plain iterations, and predicts the rest of the way, which is added to the
same registration's positions before its EM continues.  On 8 held-out 64^3
pairs (seeds 900000..900007, never trained on) the registration seeded by it is compared with the
plain method from the identity, both run to the reference CLI's convergence rule: fewer EM
iterations in total (the 16 early ones included), a final mutual information (FP64, soft joint
histogram) no lower than 1e-3 relative below the plain method's, and no more negative Jacobians
in the pipeline's output, i.e. after the topology correction the reference's FastRegistration
applies once EM is done (its defaults).  Before that correction the learned arm's fields fold in
a few percent more voxels than the plain method's (a higher-MI optimum); the counts are
printed."""
import os

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

CKPT = os.path.join(ROOT, "binder_b200", "data", "initnet_seeded_64.npz")


def _mi(oracle, pair, reg, disp):
    from binder_b200.initnet import BINS
    from binder_b200 import phantoms
    shape = pair.u.shape
    pos = phantoms.identity_positions(shape) + disp
    theta = reg.get_likelihood_parameters()[: BINS * BINS].astype(np.float64)
    _, _, hist, _ = oracle.estep(pos, pair.u, pair.v, theta, shape, shape, BINS, BINS)
    return oracle.mutual_information(hist, BINS, BINS)


def test_learned_initialiser_gain_on_held_out_pairs(core, oracle):
    from binder_b200 import initnet as I
    net = I.InitNet(1, I.SIZE, 0, in_channels=5)
    net.load(CKPT)
    oracle.set_threads(os.cpu_count() or 1)
    rows = []
    for pair in I.make_pairs(range(900000, 900008)):
        shape = pair.u.shape
        it0, d0, mlp0, r0 = I.refine(core, pair, precision=0)
        it1, d1, mlp1, r1 = I.learned_registration(core, net, pair)
        mi = (_mi(oracle, pair, r0, d0), _mi(oracle, pair, r1, d1))
        raw = [I.negative_jacobians(core, r, shape) for r in (r0, r1)]
        neg = [I.negative_jacobians(core, r, shape, correct=True) for r in (r0, r1)]
        rows.append((it0, it1, *mi, *neg, mlp0, mlp1, *raw))
        print("pair: iterations %d -> %d, MI %.6f -> %.6f, negative J after correction %d -> %d, "
              "mlp %.6f -> %.6f, negative J before correction %d -> %d" % rows[-1])
    r = np.array(rows, np.float64)
    print("mean: iterations %.1f -> %.1f, MI %.6f -> %.6f; negative J (sum) before correction "
          "%d -> %d, after %d -> %d" % (r[:, 0].mean(), r[:, 1].mean(), r[:, 2].mean(),
                                        r[:, 3].mean(), r[:, 8].sum(), r[:, 9].sum(),
                                        r[:, 4].sum(), r[:, 5].sum()))
    assert r[:, 1].mean() < r[:, 0].mean()
    assert r[:, 3].mean() >= r[:, 2].mean() * (1 - 1e-3)
    assert r[:, 5].sum() <= r[:, 4].sum()
