"""The C-ABI library loads and exports every entry point the header declares
(CPU only: no entry point that needs a GPU is called)."""
import os
import re

import pytest

from ktplace_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(ktg_\w+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        from ktplace_b200 import build
        build.build()
    return _lib.load()


def test_header_declares_entry_points():
    assert len(declared_functions()) >= 15


def test_every_declared_symbol_is_exported(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_binding_covers_header():
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_version_string(lib):
    assert b"sm_100a" in lib.ktg_version()


def test_null_context_is_rejected(lib):
    assert lib.ktg_set_pointer_mode(None, 0) == _lib.KTG_ERR_ARG
    assert lib.ktg_build_b2b(None, None, None, 0.0, None, None, 1.0, 1.0) == _lib.KTG_ERR_ARG
    assert lib.ktg_solve(None, None, None, 1e-6, 10, None, None, None, 0) == _lib.KTG_ERR_ARG
    assert lib.ktg_last_error(None) == b"null context"
