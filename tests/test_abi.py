"""The C-ABI library loads and exports every symbol include/swcholesky_b200.h declares;
without a GPU, handle creation fails cleanly instead of computing anything."""
import os
import re

import pytest

import swcholesky_b200 as swc

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                   "swcholesky_b200.h")


def declared_functions():
    text = open(HDR).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sw_\w+|swc_\w+)\s*\(", text)))


def test_header_declares_exports_list():
    assert declared_functions() == sorted(swc.EXPORTS)


def test_library_exports_every_declared_symbol():
    L = swc.lib()
    for name in declared_functions():
        assert hasattr(L, name), name


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(swc.SWCError) as e:
        swc.Handle(0)
    assert e.value.code == swc.SWC_CUDA_ERROR


def test_null_handle_calls_fail_cleanly():
    """Every handle entry point rejects a NULL handle with SWC_INVALID_INPUT (this also
    checks that the Python argument lists match the C signatures)."""
    import ctypes
    L = swc.lib()
    info = ctypes.c_int(0)
    assert L.swc_analyze(None, 10, None, None, None, None, None, None, 1, None, None, 0,
                         None, None, None) == swc.SWC_INVALID_INPUT
    assert L.swc_factor(None, None, 0, 0, ctypes.byref(info)) == swc.SWC_INVALID_INPUT
    assert L.swc_get_L(None, None, 0) == swc.SWC_INVALID_INPUT
    assert L.swc_sizes(None, None) == swc.SWC_INVALID_INPUT
    assert L.swc_set_stream(None, None) == swc.SWC_INVALID_INPUT
    assert L.swc_profile(None, None, 0, 0, ctypes.byref(info), None, None, None, None) == \
        swc.SWC_INVALID_INPUT
    assert L.swc_get_stream(None) is None
    assert L.swc_device_L(None) is None
