"""CPU checks of the C ABI: libchimex.so loads, exports every function that
include/chimex.h declares, and validates arguments before touching CUDA."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "chimex.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(chx_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for n in ("chx_plan_create", "chx_correlate", "chx_offset_accumulate", "chx_preseed",
              "chx_corr_compat", "chx_blocks_to_triangle", "chx_batch_create",
              "chx_stream_submit"):
        assert n in names


def test_library_exports_every_declared_symbol():
    import chimex
    lib = chimex.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_string():
    import chimex
    assert chimex.version().startswith("chimex-b200")


@pytest.mark.parametrize("args,code", [
    ((33, 1, 256, 256, 1, 0, 0), -1),     # E not a multiple of 32
    ((0, 1, 256, 256, 1, 0, 0), -1),
    ((256, 0, 256, 256, 1, 0, 0), -1),    # F < 1
    ((256, 1, 0, 256, 1, 0, 0), -1),      # T < 1
    ((256, 1, 1 << 24, 256, 1, 0, 0), -1),  # T beyond int32 exactness
    ((256, 1, 256, 256, 2, 0, 0), -1),    # bad convention
    ((256, 1, 256, 256, 1, 3, 0), -1),    # bad kernel family
])
def test_plan_validation_rejects_bad_shapes(args, code):
    import chimex
    h = ctypes.c_void_p()
    rc = chimex.lib().chx_plan_create(ctypes.byref(h), *args)
    assert rc == code
    assert chimex.lib().chx_last_error().decode()
    assert not h.value


def test_null_plan_is_rejected():
    import chimex
    assert chimex.lib().chx_correlate(None, None, None, None, 0) == chimex.E_INVALID
    assert chimex.lib().chx_plan_destroy(None) == chimex.OK
