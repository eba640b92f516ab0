"""Extract the reference's known-answer vectors into ``reference_kats.json``.

Reads CoherentSearch.jl's own test files as text (the Julia reference cannot
run here) and pulls out the literal golden values its tests assert, so the
oracle and the device path can be checked against exactly those numbers:

* ``finterp_coeffs(0.1, 10)`` golden coefficients (PRESTO ``gen_r_response``),
  test/test_fourierinterp.jl:5-22;
* ``nearby_fourier_bins`` 0->1-based index cases, test/test_fourierinterp.jl:24-33;
* ``next_pow_of_2`` / ``next_smooth`` cases, test/test_fourierinterp.jl:64-86;
* ``boxcar_widths`` and ``ladder_boxcar_widths`` banks, test/test_search.jl:23-77;
* the synthetic candidate lists of ``remove_duplicates`` / ``remove_harmonics``,
  test/test_search.jl:113-150.

Run once in a checkout that has the reference tree; the JSON it writes is the
committed fixture.  Usage: ``python make_reference_kats.py <reference_root>``,
the root of a CoherentSearch.jl checkout (the directory holding ``test/``).
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python make_reference_kats.py <reference_root>")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kats.json")


def _read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def _complex_list(text):
    """Parse a Julia ``ComplexF64[a + bim, ...]`` literal body."""
    out = []
    for a, sign, b in re.findall(r"(-?[0-9.eE+-]+)\s*([+-])\s*([0-9.eE+-]+)im", text):
        im = float(b) if sign == "+" else -float(b)
        out.append([float(a), im])
    return out


def _int_list(text):
    return [int(x) for x in re.findall(r"-?\d+", text)]


def main():
    fi = _read("test/test_fourierinterp.jl")
    se = _read("test/test_search.jl")
    kats = {"source": "CoherentSearch.jl test/test_fourierinterp.jl, test/test_search.jl"}

    # finterp_coeffs golden values.
    m = re.search(r"coeffs = finterp_coeffs\(([0-9.]+), (\d+)\)\s*expected = ComplexF64\[(.*?)\]", fi, re.S)
    kats["finterp_coeffs"] = {"dr": float(m.group(1)), "m": int(m.group(2)),
                              "expected": _complex_list(m.group(3))}
    m = re.search(r"coeffs ≈ expected rtol = ([0-9.e-]+) atol = ([0-9.e-]+)", fi)
    kats["finterp_coeffs"]["rtol"] = float(m.group(1))
    kats["finterp_coeffs"]["atol"] = float(m.group(2))

    # nearby_fourier_bins cases on ft = 0:9.
    cases = []
    for r, mm, vals in re.findall(
            r"collect\(nearby_fourier_bins\(([0-9.]+), ft, (\d+)\)\) == ComplexF64\[([0-9, ]+)\]", fi):
        cases.append({"r": float(r), "m": int(mm), "expected": _int_list(vals)})
    kats["nearby_fourier_bins"] = cases
    m = re.search(r"nearby_fourier_bin_range\(([0-9.]+), (\d+)\) == nearby_fourier_bin_range\(([0-9.]+), (\d+)\)", fi)
    kats["nearby_fourier_bin_range_same"] = [float(m.group(1)), float(m.group(3)), int(m.group(2))]

    # next_pow_of_2 / next_smooth.
    kats["next_pow_of_2"] = [[int(a), int(b)] for a, b in
                             re.findall(r"@test next_pow_of_2\((\d+)\) == (\d+)", fi)]
    kats["next_smooth"] = [[int(a), int(b)] for a, b in
                           re.findall(r"@test next_smooth\((\d+)\) == (\d+)", fi)]
    m = re.search(r"needs = \[([0-9, ]+)\]", fi)
    kats["smooth_needs"] = _int_list(m.group(1))

    # boxcar_widths banks.
    m = re.search(r"w = boxcar_widths\((\d+); fsp=([0-9.]+), maxfrac=([0-9.]+)\)\s*@test w == \[([0-9, ]+)\]", se)
    kats["boxcar_widths"] = [{"nbins": int(m.group(1)), "fsp": float(m.group(2)),
                              "maxfrac": float(m.group(3)), "expected": _int_list(m.group(4))}]
    m = re.search(r"@test boxcar_widths\((\d+)\) == \[([0-9, ]+)\]", se)
    kats["boxcar_widths"].append({"nbins": int(m.group(1)), "fsp": 1.5, "maxfrac": 0.3,
                                  "expected": _int_list(m.group(2))})
    ladder = {"nharms": int(re.search(r"nharms = (\d+)\s*# No ladder", se).group(1))}
    for k, vals in re.findall(r"@test banks\[(\d+)\] == \[([0-9, ]+)\]", se):
        ladder[k] = _int_list(vals)
    kats["ladder_banks"] = ladder

    # remove_duplicates / remove_harmonics synthetic lists.
    blk = re.search(r'@testset "remove_duplicates collapses clusters"(.*?)\nend', se, re.S).group(1)
    T = float(re.search(r"Candidate\(r / ([0-9.]+), s, r, (\d+)\)", blk).group(1))
    mk = [[float(a), float(b)] for a, b in re.findall(r"mk\(([0-9.]+), ([0-9.]+)\)", blk)]
    exp = [float(x) for x in re.search(r"metrics ≈ \[([0-9., ]+)\]", blk).group(1).split(",")]
    kats["remove_duplicates"] = {"T": T, "nharm": 32, "cands": mk, "dr_tol": 1.0,
                                 "expected_metrics": exp, "expected_len": int(
                                     re.search(r"@test length\(kept\) == (\d+)", blk).group(1))}
    blk = re.search(r'@testset "remove_harmonics collapses harmonic families"(.*?)\nend', se, re.S).group(1)
    fam = [[float(a), float(b)] for a, b in
           re.findall(r"mk\(([0-9.]+), ([0-9.]+)\)", re.search(r"fam = \[(.*?)\]\n", blk, re.S).group(1))]
    extra = [[float(a), float(b)] for a, b in
             re.findall(r"mk\(([0-9.]+), ([0-9.]+)\)", re.search(r"mixed = vcat\(fam, \[(.*?)\]\)", blk).group(1))]
    kats["remove_harmonics"] = {
        "T": float(re.search(r"Candidate\(r / ([0-9.]+), s, r, (\d+)\)", blk).group(1)),
        "fam": fam, "extra": extra,
        "fam_kept": [float(x) for x in re.search(r"kept\[1\]\.r == ([0-9.]+) && kept\[1\]\.metric == ([0-9.]+)",
                                                 blk).groups()],
        "mixed_kept_r": _int_list(re.search(r"Set\(\[([0-9, ]+)\]\)", blk).group(1)),
        "numharm1_len": int(re.search(r"remove_harmonics\(fam; numharm=1, tol=1.0\)\) == (\d+)", blk).group(1)),
    }

    with open(OUT, "w") as f:
        json.dump(kats, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
