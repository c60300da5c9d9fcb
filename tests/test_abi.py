"""C-ABI checks that need no GPU: libckd.so loads, exports every function declared
in include/ckd.h, the Python bindings cover them, and argument validation fails
cleanly before any device work."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ckd.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ckd_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from cosmokdtree_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        _lib.build_library()
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/ckd.h but not exported"


def test_bindings_cover_header():
    from cosmokdtree_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_version_and_validation_without_gpu(lib):
    from cosmokdtree_b200 import _lib
    assert lib.ckd_version() >= 100
    h = ctypes.c_void_p()
    # null points -> bad argument, reported before touching the device
    st = lib.ckd_build(None, 10, 3, 0, 16, None, 0, None, ctypes.byref(h))
    assert st == _lib.CKD_ERR_BAD_ARG
    assert "null" in _lib.last_error()
    buf = (ctypes.c_double * 30)()
    assert lib.ckd_build(buf, 10, 9, 0, 16, None, 0, None, ctypes.byref(h)) == _lib.CKD_ERR_BAD_DIM
    assert lib.ckd_build(buf, 10, 3, 0, 0, None, 0, None, ctypes.byref(h)) == _lib.CKD_ERR_BAD_ARG
    assert lib.ckd_tree_info(None, None, None, None, None, None, None, None, None) == \
        _lib.CKD_ERR_BAD_ARG
    assert lib.ckd_free(None) == 0


def test_python_validation_before_device():
    from cosmokdtree_b200 import kdtree, _lib
    import numpy as np
    P = np.zeros((4, 3))
    with pytest.raises(AssertionError):
        kdtree.build_kdtree(P, leaf=0)
    with pytest.raises(AssertionError):
        kdtree.build_kdtree(P, boxsize=[1.0, 1.0])
    with pytest.raises(_lib.CKDArgumentError):
        kdtree._check_k(2.0)
    with pytest.raises(AssertionError):
        kdtree._check_radius(0.0)


def test_forest_validation_without_gpu(lib):
    """Forest offsets are validated on the host before any device work."""
    from cosmokdtree_b200 import _lib
    import numpy as np
    P = np.zeros((100, 3))
    h = ctypes.c_void_p()
    pp = P.ctypes.data_as(ctypes.c_void_p)

    def build(off, nt):
        o = np.asarray(off, np.int64)
        return lib.ckd_forest_build(pp, o.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), nt, 3,
                                    0, 16, None, 0, None, ctypes.byref(h))

    assert build([0, 50, 50, 100], 3) == _lib.CKD_ERR_BAD_ARG  # empty tree
    assert "at least one point" in _lib.last_error()
    assert build([1, 50, 100], 2) == _lib.CKD_ERR_BAD_ARG      # must start at 0
    assert build([0, 100], 0) == _lib.CKD_ERR_BAD_ARG          # no trees
    assert lib.ckd_forest_build(pp, None, 2, 3, 0, 16, None, 0, None,
                                ctypes.byref(h)) == _lib.CKD_ERR_BAD_ARG
    n = ctypes.c_int64()
    assert lib.ckd_forest_info(None, ctypes.byref(n), None) == _lib.CKD_ERR_BAD_ARG
