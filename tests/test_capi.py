"""CPU: the C-ABI library loads, exports every entry point the header declares,
and reports argument errors as status codes (no GPU needed)."""
import ctypes as C
import re

import pytest

import qaxions_b200 as qx


def _declared():
    src = open(qx.HEADER_PATH).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qx_[A-Za-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    names = _declared()
    assert len(names) >= 35
    lib = C.CDLL(qx.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_null_handle():
    lib = qx.lib()
    assert lib.qx_version() >= 100
    assert lib.qx_kick(None, 0.1) == qx.QX_ERR_INVALID
    assert b"null" in lib.qx_last_error(None)
    assert lib.qx_destroy(None) == qx.QX_OK


@pytest.mark.parametrize("args,frag", [
    ((4, 64, 1.0, 1.0, 1.0, 0, 0, 1e-4), b"Dimension"),         # dim must be 2 or 3
    ((3, 100, 1.0, 1.0, 1.0, 0, 0, 1e-4), b"unsupported grid"),  # N not in the supported set
    ((3, 64, 1.0, 1.0, 1.0, 7, 0, 1e-4), b"dtype"),
    ((3, 64, 1.0, 1.0, 1.0, 0, 9, 1e-4), b"k0_policy"),
    ((3, 64, -1.0, 1.0, 1.0, 0, 0, 1e-4), b"box size"),
])
def test_create_rejects_bad_arguments(args, frag):
    h = C.c_void_p()
    st = qx.lib().qx_create(*args, C.byref(h))
    assert st == qx.QX_ERR_INVALID
    assert h.value is None
    assert frag in qx.lib().qx_last_error(None)


def test_python_field_validates_before_device():
    with pytest.raises(ValueError):
        qx.Field(3, 64, dtype="bf16")
    with pytest.raises(ValueError):
        qx.Field(3, 100)
