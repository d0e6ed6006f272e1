"""The C ABI library loads on a CPU-only host and exports every entry point
declared in include/aprl_gpu.h (no device call is made)."""
import ctypes as C
import os
import re

import pytest

from aprl_b200 import abi, native

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "aprl_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(aprl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    lib = native.load().lib
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if getattr(lib, n, None) is None]
    assert not missing, missing


def test_abi_version_and_struct_layout():
    b = native.load()
    assert b.fn["abi_version"]() == 3
    # Layout of the plain-data structs as the C compiler sees them.
    assert C.sizeof(abi.Magnet) == 8 + 3 * 8 + 10 * 8
    assert abi.RunConfig.magnets.offset % 8 == 0
    assert C.sizeof(abi.StepStats) % 8 == 0
    assert C.sizeof(abi.SelfFieldConfig) == 4 * 4 + 3 * 8 + 3 * 8 + 2 * 4
    assert abi.SelfFieldConfig.source_shape.offset == 64


def test_cowan_coefficients_need_no_device():
    b = native.load()
    out = (C.c_double * 12)()
    b("cowan_coefficients", 5e-6, 5e-6, 2e-6, out)
    assert abs(out[0] + 2 * out[4] + 2 * out[5] + 4 * out[7] - 1.0) < 1e-12


def test_kernel_names_are_listed():
    b = native.load()
    names = [b.fn["kernel_name"](i).decode() for i in range(15)]
    assert "push_deposit" in names and "cowan_magnetic" in names


def test_error_messages_cross_the_boundary():
    b = native.load()
    out = (C.c_double * 12)()
    status = b.fn["cowan_coefficients"](1e-6, 5e-6, 2e-6, out)
    assert status == abi.APRL_ERR_INVALID_ARGUMENT
    assert "smallest" in b.error()
    with pytest.raises(native.AprlError):
        b("cowan_coefficients", -1.0, 1.0, 1.0, out)
