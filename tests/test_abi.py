"""CPU: the C ABI library loads and exports every entry point include/b12g.h declares."""
import ctypes
import os
import re

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "b12g.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+char\s*\*|b12g_status)\s+(b12g_\w+)\s*\(", text, re.M)))


def test_header_declares_the_path():
    syms = declared_symbols()
    for s in ("b12g_tree_create", "b12g_subdivide", "b12g_set_flags_by_image", "b12g_remove",
              "b12g_transition_matrix", "b12g_invariant_measure", "b12g_insert_by_image",
              "b12g_subdivision_run", "b12g_continuation_run"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    from b12_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(_lib.DECLARED)


def test_library_is_sm100a_build():
    from b12_b200 import _lib
    assert b"sm_100a" in _lib.lib().b12g_version()


def test_no_device_is_reported_not_hidden():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import b12_b200 as B
    with pytest.raises(B.B12gError) as e:
        B.ImplicitBoxTree([0.0, 0.0], [1.0, 1.0])
    assert e.value.status == 7  # B12G_ERR_NO_DEVICE


def test_invalid_arguments_rejected_before_device_work():
    from b12_b200 import _lib
    L = _lib.lib()
    d = _lib.Domain()
    d.dim = 7
    h = ctypes.c_void_p()
    assert L.b12g_tree_create(ctypes.byref(d), ctypes.byref(h)) == _lib.ERR_INVALID
    assert L.b12g_tree_create(None, ctypes.byref(h)) == _lib.ERR_INVALID
    assert b"dim" in L.b12g_last_error() or b"NULL" in L.b12g_last_error()
