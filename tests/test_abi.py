"""The C-ABI library loads and exports every entry point include/binder_b200.h declares; host-side
argument checks and error reporting work without a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import HAVE_GPU, ROOT

HEADER = os.path.join(ROOT, "include", "binder_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|long long|const char \*)\s*(binder_\w+)\s*\(",
                                 text, re.M)))


def test_header_lists_all_python_bindings():
    from binder_b200 import _lib
    assert declared_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(core):
    from binder_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_backend_and_capabilities(core):
    from binder_b200._lib import lib
    assert lib().binder_backend() == b"b200"
    assert lib().binder_has_topology_correction() == 1
    assert core.backend == "b200" and core.has_topology_correction


def test_null_arguments_are_rejected(core):
    from binder_b200._lib import lib
    h = ctypes.c_void_p()
    st = lib().binder_registration_em(None, 1, 0.0, 1, 0, None)
    assert st == 1 and b"NULL" in lib().binder_last_error()
    assert lib().binder_registration_destroy(None) == 0
    assert lib().binder_transform_destroy(None) == 0
    for fn in ("binder_registration_set_precision", "binder_registration_set_histogram_precision"):
        assert getattr(lib(), fn)(None, 0) == 1 and b"NULL" in lib().binder_last_error(), fn
    del h


def test_shape_mismatch_raises_before_any_device_work(core):
    with pytest.raises(ValueError):
        core.Registration(np.zeros(10), 1, np.zeros(12), np.zeros(12), 2, 2, 1, 2, 2, 1, 3, 4)


def test_topology_rejects_inadmissible_range(core):
    f = np.zeros((4, 4, 4, 3))
    with pytest.raises(core.BinderError) as e:
        core.topology_correction_3D().correct_topology(f, 1.5, 2.0, 1, 1, 1, [1, 1, 1], 4, 4, 4)
    assert e.value.status == 1


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device error path")
def test_no_device_reports_cuda_error(core):
    with pytest.raises(core.BinderError) as e:
        core.compute_jacobian_determinant_3D(np.zeros((3, 3, 3, 3)), 3, 3, 3, 1, 1, 1)
    assert e.value.status == 2
