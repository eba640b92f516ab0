"""The C-ABI library builds for sm_100a, loads, and exports every entry point
``include/cohsearch.h`` declares (no device calls: runs without a GPU)."""
import ctypes
import os
import re

import pytest

from tests.conftest import PKG, ROOT

HEADER = os.path.join(ROOT, "include", "cohsearch.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cs_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    import importlib.util
    spec = importlib.util.spec_from_file_location("cs_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build()


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("cs_create", "cs_destroy", "cs_set_spectrum", "cs_set_spectrum_device", "cs_search",
                 "cs_chunk_metrics", "cs_interp_chunk", "cs_last_error", "cs_search_stats"):
        assert must in names


def test_library_exports_every_declared_symbol(lib_path):
    lib = ctypes.CDLL(lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(lib_path):
    from cohsearch import _lib
    assert set(declared_functions()) == set(_lib.PROTOTYPES)
    lib = _lib.load()
    assert lib.cs_version().decode().startswith("cohsearch-b200")


def test_struct_layouts_match_header():
    from cohsearch import _lib
    assert ctypes.sizeof(_lib.cs_candidate) == 40
    assert ctypes.sizeof(_lib.cs_params) == 4 * 4 + 16 * 4 + 5 * 8 + 2 * 4


def test_invalid_params_rejected_before_device():
    from cohsearch import SearchParams
    with pytest.raises(ValueError):
        SearchParams(m=15).to_c()
    with pytest.raises(ValueError):
        SearchParams(precision="f16").to_c()
