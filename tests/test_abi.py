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


def test_every_struct_matches_the_c_layout():
    """Every struct of the ctypes binding against the header as a C compiler
    lays it out: sizeof and each field's offsetof, from a probe compiled with
    gcc against include/cohsearch.h (in the ignored _build folder)."""
    import shutil
    import subprocess
    from cohsearch import _lib
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    structs = {n: getattr(_lib, n) for n in ("cs_params", "cs_candidate", "cs_stats", "cs_spectrum",
                                              "cs_block_stats", "cs_mlp", "cs_mlp_grads", "cs_adam_param")}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "cohsearch.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'    printf("{name} sizeof %zu\\n", sizeof({name}));')
        for fname, *_ in cls._fields_:
            lines.append(f'    printf("{name} {fname} %zu\\n", offsetof({name}, {fname}));')
    lines += ["    return 0;", "}"]
    root = ROOT
    out = os.path.join(root, "_build", "abi_layout")
    os.makedirs(out, exist_ok=True)
    src, exe = os.path.join(out, "probe.c"), os.path.join(out, "probe")
    with open(src, "w") as f:
        f.write("\n".join(lines) + "\n")
    subprocess.run([gcc, "-std=c11", "-I", os.path.join(root, "include"), "-o", exe, src], check=True)
    got = {}
    for ln in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines():
        name, field, val = ln.split()
        got[(name, field)] = int(val)
    for name, cls in structs.items():
        assert got[(name, "sizeof")] == ctypes.sizeof(cls), name
        for fname, *_ in cls._fields_:
            assert got[(name, fname)] == getattr(cls, fname).offset, (name, fname)


def test_invalid_params_rejected_before_device():
    from cohsearch import SearchParams
    with pytest.raises(ValueError):
        SearchParams(m=15).to_c()
    with pytest.raises(ValueError):
        SearchParams(precision="f16").to_c()
