"""The C ABI library: it loads, exports every entry point include/ncpa_gpu.h
declares, and without a CUDA device refuses to run instead of falling back to
the CPU."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import PKG, ROOT

HEADER = os.path.join(ROOT, "include", "ncpa_gpu.h")


def _declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ncpa_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ncpa_gpu

    lib = ncpa_gpu.lib()
    names = _declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", ncpa_gpu.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (ncpa_[a-z0-9_]+)", out))
    assert set(names) <= exported
    assert set(ncpa_gpu.EXPORTED) <= exported


def test_status_strings():
    import ncpa_gpu

    lib = ncpa_gpu.lib()
    assert lib.ncpa_status_str(0) == b"ok"
    assert lib.ncpa_status_str(5) == b"too many modes"
    assert lib.ncpa_status_str(99) == b"unknown status"


def test_no_device_means_no_context():
    import torch

    import ncpa_gpu

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(ncpa_gpu.NcpaError) as e:
        ncpa_gpu.Context(0)
    assert e.value.status == 8  # NCPA_ENODEV: no CPU fallback


def test_null_arguments_rejected():
    import ncpa_gpu

    lib = ncpa_gpu.lib()
    assert lib.ncpa_ctx_create(None, None) == 1
    assert lib.ncpa_profile_destroy(None) == 1
    assert lib.ncpa_modes_destroy(None) == 1
