"""Drop-in check: the reference's own, unmodified Python layer (BINDER/__init__.py,
FastRegistration.py, utils.py) and its GPU test tests/gpu/test_3D_MI_registration.py (EM on the
bundled 22x24x24 T1w pair, then the sampler, with the reference's own assertions) run with
`BINDER._core` bound to this library's `binder_b200._core`.  nibabel, skimage and matplotlib,
which are not installed, are replaced by the stand-ins in tests/dropin/.

The reference checkout is read from $BINDER_REFERENCE_ROOT (the directory holding BINDER/); the
test is skipped without it."""
import importlib
import importlib.util
import os
import sys

import pytest

from conftest import ROOT

REF = os.environ.get("BINDER_REFERENCE_ROOT", "")
HAVE_REF = bool(REF) and os.path.exists(os.path.join(REF, "BINDER", "FastRegistration.py"))

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not HAVE_REF, reason="BINDER_REFERENCE_ROOT not set")]


def _bind_reference_package():
    """import the reference's BINDER package with binder_b200._core as its extension"""
    stubs = os.path.join(ROOT, "tests", "dropin")
    if stubs not in sys.path:
        sys.path.insert(0, stubs)
    from binder_b200 import build
    build.build()
    from binder_b200 import _core
    for name in [m for m in sys.modules if m == "BINDER" or m.startswith("BINDER.")]:
        del sys.modules[name]
    sys.modules["BINDER._core"] = _core
    if REF not in sys.path:
        sys.path.insert(0, REF)
    binder = importlib.import_module("BINDER")
    assert binder._core is _core and binder.FastRegistration is not None
    return binder


def test_reference_3d_mi_registration_test_on_b200_core(tmp_path):
    binder = _bind_reference_package()
    import nibabel as nib
    spec = importlib.util.spec_from_file_location(
        "ref_test_3D_MI_registration",
        os.path.join(REF, "BINDER", "tests", "gpu", "test_3D_MI_registration.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    d = os.path.join(str(binder.BINDERDIR), "_internal_resources", "testing_files",
                     "3DTestImages")
    t1 = nib.load(os.path.join(d, "T1w_1_8mm.nii.gz"))
    t2 = nib.load(os.path.join(d, "T1w_2_8mm.nii.gz"))
    assert t1.get_fdata().shape == (22, 24, 24)
    # the reference's test body: EM, warped SSD below the starting SSD, then the sampler, whose
    # mean warp beats EM's
    mod.test_3D_MI_registration(t1, t2, str(tmp_path))
