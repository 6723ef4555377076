"""The C-ABI library builds, loads and exports every declared symbol (CPU)."""
import glob
import os
import re
import subprocess

import pytest

from ftd_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names |= set(re.findall(r"FTDX_API\s+[\w\s\*]*?\b(ftdx_\w+)\s*\(", txt))
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert {"ftdx_create", "ftdx_destroy", "ftdx_herk", "ftdx_init_herk"} <= names


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for name in _declared():
        assert name in exported, name
        assert hasattr(L, name)


def test_python_prototypes_cover_header():
    assert _declared() <= set(_lib.PROTOTYPES)


def test_status_strings_and_version():
    L = _lib.load()
    assert L.ftdx_version() == (0 << 16) | 1
    for code in range(9):
        assert L.ftdx_status_string(code)
    assert L.ftdx_status_string(99) == b"unknown status"


def test_null_arguments_rejected_without_gpu():
    import ctypes
    L = _lib.load()
    assert L.ftdx_create(None, None) == 1
    assert L.ftdx_destroy(None) == 1
    assert L.ftdx_herk(None, None, None, 1, 1, 1, 1, 0, 1, 0, 1.0, 0.0, None, 0) == 1


def test_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ctypes
    h = ctypes.c_void_p()
    assert _lib.load().ftdx_create(ctypes.byref(h), None) == 4
