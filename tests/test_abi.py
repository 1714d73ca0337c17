"""The C-ABI libraries load and export every entry point include/velo_b200.h declares;
argument errors come back as codes (no GPU calls are made here)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT, cuda_available
from cuda_hlt_b200 import _lib, chain


def declared_functions():
    text = open(os.path.join(ROOT, "include", "velo_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(velo_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_expected_entry_points():
    names = declared_functions()
    assert set(_lib.HOST_SYMBOLS) | set(_lib.GPU_SYMBOLS) == set(names)


def test_libraries_export_every_declared_symbol():
    host = C.CDLL(_lib.HOST_LIB_PATH)
    gpu = C.CDLL(_lib.GPU_LIB_PATH)
    for name in declared_functions():
        lib = host if name in _lib.HOST_SYMBOLS else gpu
        assert hasattr(lib, name), name


def test_version_string():
    assert b"sm_100a" in _lib.gpu_lib().velo_version()


def test_argument_errors_without_launching():
    L = _lib.gpu_lib()
    geo = (C.c_uint8 * 19456)()
    cfg = _lib.VeloConfig(max_events=0, max_raw_bytes=1024)
    ctx = C.c_void_p()
    assert L.velo_create(C.byref(cfg), geo, 19456, C.byref(ctx)) == -1          # no events
    cfg.max_events = 4
    assert L.velo_create(C.byref(cfg), geo, 100, C.byref(ctx)) in (-5, -7)     # bad geometry (or no device)
    assert L.velo_create(None, geo, 19456, C.byref(ctx)) == -1
    assert L.velo_run(None, None, None, 0, None, None) == -1
    assert L.velo_sync(None, None, None, None) == -1
    assert L.velo_destroy(None) == -1
    assert L.velo_download(None, None, None, 0) == -1


@pytest.mark.skipif(cuda_available(), reason="checks the no-device path")
def test_no_device_is_reported():
    with pytest.raises(chain.VeloError, match="-7"):
        chain.VeloChain(4, 1 << 16)
