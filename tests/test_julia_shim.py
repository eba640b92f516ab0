"""The Julia binding (coherentsearch.jl_b200/julia/CohSearchB200.jl) against the
C ABI it binds: Julia is not installed where this library is built, so the
binding is checked statically -- every `ccall` names an entry point that
include/cohsearch.h declares, with as many argument types as the prototype has
parameters."""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "coherentsearch.jl_b200", "julia", "CohSearchB200.jl")
HDR = os.path.join(ROOT, "include", "cohsearch.h")


def _split_top(s, opens="({[", closes=")}]"):
    """Items of a comma-separated list, splitting only at nesting depth 0."""
    out, depth, cur = [], 0, []
    for ch in s:
        if ch in opens:
            depth += 1
        elif ch in closes:
            depth -= 1
        if ch == "," and depth == 0:
            out.append("".join(cur).strip())
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur).strip())
    return [x for x in out if x]


def _header_prototypes():
    text = re.sub(r"/\*.*?\*/", " ", open(HDR).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"^[A-Za-z_][\w \t\*]*?\b(cs_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text, re.M):
        params = _split_top(m.group(2))
        protos[m.group(1)] = 0 if params == ["void"] else len(params)
    return protos


def _julia_ccalls():
    text = open(JL).read()
    calls = []
    for m in re.finditer(r"ccall\(\(:(cs_[a-z0-9_]+),\s*LIB\),\s*[^,]+,\s*\(", text):
        # the argument-type tuple: from the opening parenthesis to its match
        i, depth = m.end() - 1, 0
        for j in range(i, len(text)):
            if text[j] == "(":
                depth += 1
            elif text[j] == ")":
                depth -= 1
                if depth == 0:
                    break
        calls.append((m.group(1), len(_split_top(text[i + 1:j]))))
    return calls


def test_every_julia_ccall_matches_a_header_prototype():
    protos = _header_prototypes()
    calls = _julia_ccalls()
    assert len(calls) >= 15
    for name, nargs in calls:
        assert name in protos, name
        assert nargs == protos[name], (name, nargs, protos[name])


def test_julia_binding_covers_the_reference_facing_calls():
    """The calls a CoherentSearch.jl user reaches for: the search and its
    block ranges, the batch over files, chunk and block metrics, the refold,
    and the metric statistics / normalisation."""
    names = {n for n, _ in _julia_ccalls()}
    want = {"cs_create", "cs_destroy", "cs_set_spectrum", "cs_search", "cs_search_range", "cs_search_batch",
            "cs_set_batch_graph", "cs_chunk_metrics", "cs_block_metrics", "cs_refold", "cs_set_metricstats",
            "cs_get_block_stats", "cs_get_metric_hists", "cs_set_metricnorm", "cs_last_error"}
    assert want <= names, sorted(want - names)


_JL_SIZES = {"Int32": (4, 4), "Int64": (8, 8), "Float32": (4, 4), "Float64": (8, 8), "UInt32": (4, 4)}


def _jl_field_layout(tname):
    """(size, align) of a Julia field type as Julia lays isbits structs out
    for C: natural alignment, NTuple{n,T} as an array, pointers 8 bytes."""
    if tname.startswith("Ptr{"):
        return 8, 8
    m = re.fullmatch(r"NTuple\{(\d+),\s*(\w+)\}", tname)
    if m:
        sz, al = _JL_SIZES[m.group(2)]
        return int(m.group(1)) * sz, al
    return _JL_SIZES[tname]


def _jl_structs():
    text = open(JL).read()
    out = {}
    for m in re.finditer(r"^struct (CS\w+)\n(.*?)^end", text, re.S | re.M):
        fields, off, align = [], 0, 1
        for ln in m.group(2).splitlines():
            fm = re.match(r"\s*(\w+)::(\S+)", ln)
            if not fm:
                continue
            sz, al = _jl_field_layout(fm.group(2))
            off = (off + al - 1) // al * al
            fields.append((fm.group(1), off))
            off += sz
            align = max(align, al)
        out[m.group(1)] = (fields, (off + align - 1) // align * align)
    return out


def test_julia_structs_match_the_c_layout():
    """CSParams, CSCandidate, CSSpectrum and CSBlockStats against the header
    as gcc lays it out: same field names, offsets and sizes."""
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    pairs = {"CSParams": "cs_params", "CSCandidate": "cs_candidate", "CSSpectrum": "cs_spectrum",
             "CSBlockStats": "cs_block_stats"}
    jl = _jl_structs()
    assert set(pairs) <= set(jl)
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "cohsearch.h"', "int main(void) {"]
    for js, cs in pairs.items():
        lines.append(f'    printf("{cs} sizeof %zu\\n", sizeof({cs}));')
        for fname, _ in jl[js][0]:
            lines.append(f'    printf("{cs} {fname} %zu\\n", offsetof({cs}, {fname}));')
    lines += ["    return 0;", "}"]
    out = os.path.join(ROOT, "_build", "julia_layout")
    os.makedirs(out, exist_ok=True)
    src, exe = os.path.join(out, "probe.c"), os.path.join(out, "probe")
    with open(src, "w") as f:
        f.write("\n".join(lines) + "\n")
    subprocess.run([gcc, "-std=c11", "-I", os.path.join(ROOT, "include"), "-o", exe, src], check=True)
    got = {}
    for ln in subprocess.run([exe], check=True, capture_output=True, text=True).stdout.splitlines():
        name, field, val = ln.split()
        got[(name, field)] = int(val)
    for js, cs in pairs.items():
        fields, size = jl[js]
        assert got[(cs, "sizeof")] == size, js
        for fname, off in fields:
            assert got[(cs, fname)] == off, (js, fname)
