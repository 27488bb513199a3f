"""The C-ABI library loads and exports every symbol the header declares (no GPU)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fastpls_b200.h")


def _declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(fpls_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def built():
    from fastpls_b200.build import build_library
    return build_library()


def test_header_declares_entry_points():
    names = _declared()
    assert "fpls_pls_model1" in names and "fpls_pls_model2_fast" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol(built):
    out = subprocess.run(["nm", "-D", "--defined-only", built], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (fpls_[a-z0-9_]+)", out))
    missing = [s for s in _declared() if s not in exported]
    assert not missing, missing


def test_ctypes_binding_covers_header(built):
    from fastpls_b200 import _lib
    assert set(_declared()) <= set(_lib.exported_symbols())
    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name)


def test_library_has_no_torch_dependency(built):
    out = subprocess.run(["ldd", built], capture_output=True, text=True).stdout
    assert "torch" not in out and "c10" not in out


def test_version_string(built):
    from fastpls_b200 import _lib
    assert "sm_100a" in _lib.version()
