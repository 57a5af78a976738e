"""CPU tests of the drop-in boundary: libtanb.so loads, exports every entry point
include/tanb.h declares, and fails loudly (no CPU fallback) without a GPU."""
import ctypes
import os
import re

import pytest

from tan_b200 import convolution as cv

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for hdr in os.listdir(os.path.join(ROOT, "include")):
        if hdr.endswith(".h"):
            text = open(os.path.join(ROOT, "include", hdr)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(tanb_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = cv.lib()
    declared = declared_symbols()
    assert len(declared) >= 19
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(cv.SIGNATURES), declared ^ set(cv.SIGNATURES)


def test_library_is_sm100a_only_and_has_no_host_fallback():
    data = open(cv.LIB_PATH, "rb").read()
    assert b"sm_100a" in data or b"sm_100" in data


def test_abi_constants_match_reference_values():
    # AMF_RESULT (amf/public/include/core/Result.h) and TAN enums (TrueAudioNext.h)
    assert (cv.AMF_OK, cv.AMF_INVALID_ARG, cv.AMF_NOT_SUPPORTED, cv.AMF_NOT_FOUND) == (0, 4, 10, 11)
    assert (cv.AMF_ALREADY_INITIALIZED, cv.AMF_NOT_INITIALIZED, cv.AMF_WRONG_STATE) == (12, 13, 15)
    assert cv.AMF_TAN_UNSUPPORTED_VERSION == 43
    assert cv.TAN_CONVOLUTION_METHOD_TIME_DOMAIN == 7
    assert cv.TAN_CONVOLUTION_METHOD_USE_PROCESS_FINALIZE == 0x8000
    hdr = open(os.path.join(ROOT, "include", "tanb.h")).read()
    for name, val in [("TANB_WRONG_STATE", 15), ("TANB_METHOD_TIME_DOMAIN", 7), ("TANB_NOT_FOUND", 11)]:
        assert re.search(rf"{name} = {val}\b", hdr), name


def test_version_check_and_no_device_errors():
    lib = cv.lib()
    h = ctypes.c_void_p()
    assert lib.tanb_create_context(2 << 48, 0, ctypes.byref(h)) == cv.AMF_TAN_UNSUPPORTED_VERSION
    rc = lib.tanb_create_context(cv.TAN_FULL_VERSION, 0, ctypes.byref(h))
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert rc == cv.AMF_NO_DEVICE
        with pytest.raises(cv.TANError):
            cv.TANContext(0)
    else:
        assert rc == cv.AMF_OK
        lib.tanb_context_release(h)


def test_null_handles_are_rejected():
    lib = cv.lib()
    assert lib.tanb_convolution_init(None, 1, 1024, 256, 2) == cv.AMF_INVALID_POINTER
    assert lib.tanb_convolution_process(None, None, None, 0, None, None) == cv.AMF_INVALID_POINTER
    assert lib.tanb_create_convolution(None, None) == cv.AMF_INVALID_POINTER


def test_no_alloc_entry_point_refuses_sizes_that_would_wrap():
    """Sizes whose scratch layout would overflow size_t are refused before any
    product is formed or any device call is made (so this runs without a GPU)."""
    lib = cv.lib()
    buf = (ctypes.c_float * 16)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    huge = (1 << 64) // 2
    for channels, ir_length, block in [(32, huge, 32), (1, huge + 32, 32), (1 << 31, 1024, 512),
                                       (64, 1 << 16, 512)]:
        rc = lib.tanb_convolve_no_alloc(p, p, p, channels, 4096, ir_length, block, None)
        assert rc == cv.AMF_INVALID_ARG, (channels, ir_length, block)
        assert "scratch" in cv.last_error()
