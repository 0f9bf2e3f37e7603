"""The C-ABI libraries load and export every entry point their headers declare
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "kssd3a-public_b200")


def _declared(header):
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kssd\w+)\s*\(", text)))


@pytest.mark.parametrize("header,lib", [
    (os.path.join(ROOT, "include", "kssdgpu.h"), os.path.join(PKG, "lib", "libkssdgpu.so")),
])
def test_library_exports_every_declared_symbol(header, lib):
    assert os.path.exists(lib), f"{lib} not built"
    so = ctypes.CDLL(lib)
    names = _declared(header)
    assert names, header
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_error_path_without_gpu_work():
    so = ctypes.CDLL(os.path.join(PKG, "lib", "libkssdgpu.so"))
    so.kssdgpu_last_error.restype = ctypes.c_char_p
    so.kssdgpu_index_info.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 4
    assert so.kssdgpu_index_info(None, None, None, None, None) == 1
    assert b"null" in so.kssdgpu_last_error()
