"""The C-ABI library: it loads without a GPU and exports every entry point
declared in include/gamdb200.h (no compute calls here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gamdb200.h")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gdb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from gamdpy_b200 import _lib
    return _lib.lib()


def test_header_declares_entry_points():
    names = declared()
    assert "gdb_sim_create" in names and "gdb_sim_run" in names and len(names) > 25


def test_every_declared_symbol_is_exported(lib):
    for name in declared():
        assert hasattr(lib, name), name


def test_bindings_cover_the_header():
    from gamdpy_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared()


def test_version_without_gpu(lib):
    assert lib.gdb_version() >= 100


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    """No silent fallback: a missing .so is an error at first use."""
    import importlib

    from gamdpy_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()
    importlib.reload(_lib)


def test_oracle_library_builds_and_loads(oracle):
    assert oracle.num_threads() >= 1
