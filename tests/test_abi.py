"""The C-ABI library loads and exports every entry point declared in
include/flowmol_b200.h; host-only calls work without a GPU."""
import ctypes as C
import os
import re

import pytest

from flowmol_b200 import api, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols():
    build.build()
    hdr = open(os.path.join(ROOT, "include", "flowmol_b200.h")).read()
    declared = set(re.findall(r"FM_API int (fm_\w+)\(", hdr))
    assert len(declared) >= 25
    exported = set(api.exported_symbols())
    assert declared == exported


def test_struct_layouts_match_header():
    # fm_params / fm_macro as ctypes must match the C layout the library uses
    assert C.sizeof(api.FmMacro) == 4 + 4 + 8 * 9
    p = api.make_params(10, [10.0, 10.0, 10.0], 2.5)
    assert p.np == 10 and p.tplot == 100


def test_errors_are_codes_not_aborts():
    L = api.lib()
    # null params -> FM_ERR_ARG, message available
    assert L.fm_create(None, None) == 1
    assert "null" in api.last_error()


def test_create_without_device_is_an_error_code():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    p = api.make_params(100, [20.0, 20.0, 20.0], 2.5)
    h = C.c_void_p()
    assert api.lib().fm_create(C.byref(p), C.byref(h)) == 9  # FM_ERR_NODEVICE
