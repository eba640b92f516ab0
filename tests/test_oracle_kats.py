"""Pin the CPU oracle to the reference's own known-answer tests.

Every assertion here restates one of CoherentSearch.jl's self-contained tests
(test/test_fourierinterp.jl, test/test_search.jl) with the literal values
extracted into ``tests/golden/reference_kats.json``.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle import cs_ref as o

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def test_finterp_coeffs_golden():
    """test/test_fourierinterp.jl:5-22 (PRESTO gen_r_response values)."""
    g = KATS["finterp_coeffs"]
    got = o.finterp_coeffs(g["dr"], g["m"])
    exp = np.array([complex(a, b) for a, b in g["expected"]])
    assert np.allclose(got, exp, rtol=g["rtol"], atol=g["atol"])
    assert np.allclose(o.finterp_coeffs(0.0, 6), [0, 0, 1, 0, 0, 0], atol=1e-12)
    with pytest.raises(ValueError):
        o.finterp_coeffs(0.1, 5)
    with pytest.raises(ValueError):
        o.finterp_coeffs(1.0, 6)


def test_nearby_fourier_bins_index_translation():
    """test/test_fourierinterp.jl:24-33."""
    ft = np.arange(10, dtype=np.complex128)
    for case in KATS["nearby_fourier_bins"]:
        assert list(o.nearby_fourier_bins(case["r"], ft, case["m"]).real.astype(int)) == case["expected"]
    r1, r2, m = KATS["nearby_fourier_bin_range_same"]
    lo, hi = o.nearby_fourier_bin_range(r1, m)
    assert hi - lo == m
    assert o.nearby_fourier_bin_range(r1, m) == o.nearby_fourier_bin_range(r2, m)


def _cosine_ft(r, N=32768, phs=math.pi / 4):
    n = np.arange(N)
    return np.fft.rfft(np.cos(2 * np.pi * r * n / N + phs))


@pytest.mark.parametrize("r,idx", [(12400.55, 11), (12400.0, 0)])
def test_fourier_interp_analytic_cosine(r, idx):
    """test/test_fourierinterp.jl:35-50."""
    N = 32768
    ft = _cosine_ft(r, N)
    iv = o.fourier_interp(r, ft, 60)
    exp = N / 2 / math.sqrt(2) * (1 + 1j)
    assert abs(iv - exp) <= 1e-3 + 1e-2 * abs(exp)
    rs = math.floor(r) + np.linspace(0.0, 1.0, 21)[:-1]
    iv2 = o.finterp_multi(rs, ft, 60)
    assert abs(iv2[idx] - iv) <= 1e-9


def test_finterp_multi_equals_finterp_fft():
    """test/test_fourierinterp.jl:52-62."""
    ft = _cosine_ft(12400.0)
    rs = 12400.0 + np.linspace(0.0, 1.0, 21)[:-1]
    v1 = o.finterp_multi(rs, ft, 16)
    v2 = o.finterp_fft(12400, 1, len(rs), ft, 16)
    assert np.allclose(v1, v2, rtol=1e-5, atol=1e-7)


def test_pow2_and_smooth():
    """test/test_fourierinterp.jl:64-86."""
    for a, b in KATS["next_pow_of_2"]:
        assert o.next_pow_of_2(a) == b
    with pytest.raises(ValueError):
        o.next_pow_of_2(0)
    assert o.is_smooth(1) and o.is_smooth(2) and o.is_smooth(2 * 3 * 5 * 7)
    assert not o.is_smooth(11) and not o.is_smooth(22) and not o.is_smooth(13)
    for a, b in KATS["next_smooth"]:
        assert o.next_smooth(a) == b
    assert o.is_smooth(o.next_smooth(12345)) and o.next_smooth(12345) >= 12345
    needs = KATS["smooth_needs"]
    assert all(o.next_smooth(n) / n < 1.02 for n in needs)
    assert max(o.next_pow_of_2(n) / n for n in needs) > 1.9


def test_finterp_fft_padding_independent():
    """test/test_fourierinterp.jl:88-105."""
    ft = _cosine_ft(12400.0)
    need = (4 + 16) * 8
    a = o.finterp_fft(12400, 4, 8, ft, 16, fftlen=o.next_pow_of_2(need))
    b = o.finterp_fft(12400, 4, 8, ft, 16, fftlen=o.next_smooth(need))
    assert o.next_smooth(need) != o.next_pow_of_2(need)
    assert np.max(np.abs(a - b)) / np.max(np.abs(a)) < 1e-13
    with pytest.raises(ValueError):
        o.finterp_fft(12400, 4, 8, ft, 16, fftlen=need - 1)


def test_finterp_direct_is_exact_kernel():
    """test/test_fourierinterp.jl:107-126."""
    ft = _cosine_ft(12400.0)
    for m in (8, 16, 32):
        got = o.finterp_direct(12395.137, 41, 0.25, ft, m)
        want = np.array([o.fourier_interp(12395.137 + k * 0.25, ft, m) for k in range(41)])
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < 1e-13
    ex = o.finterp_direct(12400.0, 1, 1.0, ft, 16)
    assert np.isfinite(ex[0].real) and np.isfinite(ex[0].imag)
    assert abs(ex[0] - o.fourier_interp(12400.0, ft, 16)) <= 1e-12 * abs(ex[0])
    with pytest.raises(ValueError):
        o.finterp_direct(12400.0, 4, 0.25, ft, 15)


def test_irfft_convention_ignores_dc_nyquist_imag():
    """test/test_fourierinterp.jl:128-143 (the brfft convention the oracle uses)."""
    rng = np.random.default_rng(8)
    nh = 8
    X = rng.standard_normal(nh + 1) + 1j * rng.standard_normal(nh + 1)
    prof = np.fft.irfft(X, 2 * nh)
    Xc = X.copy()
    Xc[0] = Xc[0].real
    Xc[-1] = Xc[-1].real
    full = np.concatenate([Xc, np.conj(Xc[1:-1][::-1])])
    ref = np.fft.ifft(full).real
    assert np.allclose(prof, ref, atol=1e-10)
    assert np.allclose(o.brfft(X[None, :], 2 * nh)[0], 2 * nh * ref, atol=1e-9)


def test_boxcar_widths_bank():
    """test/test_search.jl:23-31."""
    for c in KATS["boxcar_widths"]:
        w = o.boxcar_widths(c["nbins"], c["fsp"], c["maxfrac"])
        assert w == c["expected"]
    w = o.boxcar_widths(64)
    assert all(w[i + 1] == max(math.floor(1.5 * w[i]), w[i] + 1) for i in range(len(w) - 1))
    assert w[-1] <= math.floor(0.3 * 64)
    assert o.boxcar_widths(64, maxfrac=0.5)[-1] <= 32


def test_ladder_banks():
    """test/test_search.jl:33-77."""
    nh = KATS["ladder_banks"]["nharms"]
    solo = o.SearchParams(nharms=nh)
    assert o.ladder_boxcar_widths(2 * nh, 1, solo) == o.boxcar_widths(2 * nh)
    p = o.SearchParams(nharms=nh, decimations=o.decimation_set(nh, 6))
    assert p.decimations == [1, 2, 3, 4, 5, 6]
    banks = {k: o.ladder_boxcar_widths(2 * (nh // k), k, p) for k in p.decimations}
    assert banks[1] == KATS["ladder_banks"]["1"]
    assert banks[6] == KATS["ladder_banks"]["6"]
    for k in range(2, 7):
        assert 1 not in banks[k]
    for k in range(1, 6):
        assert max(banks[k]) <= 6
    assert max(banks[6]) == max(o.boxcar_widths(2 * (nh // 6)))
    for k in p.decimations:
        full = o.boxcar_widths(2 * (nh // k))
        assert banks[k] and set(banks[k]) <= set(full)
    sparse = o.SearchParams(nharms=nh, decimations=[1, 6])
    assert o.ladder_boxcar_widths(2 * nh, 1, sparse) == o.boxcar_widths(2 * nh)
    assert o.ladder_boxcar_widths(2 * (nh // 6), 6, sparse) == o.boxcar_widths(2 * (nh // 6))
    assert o.ladder_boxcar_widths(2 * nh, 1, o.SearchParams(nharms=nh, decimations=[1, 2, 4])) != \
        o.boxcar_widths(2 * nh)


def test_boxcar_metric_properties():
    """test/test_search.jl:79-111."""
    nb = 64
    ramp = np.arange(1.0, nb + 1)
    m1 = o.snr_metrics(ramp[None, :])[0]
    m2 = o.snr_metrics(7.0 * ramp[None, :])[0]
    assert abs(m1 - m2) <= 1e-12 * abs(m1) and m1 > 0
    assert o.snr_metrics(np.full((1, nb), 3.0))[0] == 0.0
    rng = np.random.default_rng(1234)
    noise = rng.standard_normal(nb)
    sn = o.snr_metrics(noise[None, :])[0]
    sig = noise.copy()
    sig[29] += 20.0
    ss = o.snr_metrics(sig[None, :])[0]
    assert ss > sn + 10 and 0 < sn < 8 and ss > 15
    small = np.random.default_rng(7).standard_normal((4, nb))
    assert np.array_equal(o.snr_metrics(small), o.snr_metrics(small, sigma_samples=o.BOXCAR_SIGMA_SAMPLES))


def _mk(T, nharm, lst):
    return [o.Candidate(r / T, s, r, nharm) for r, s in lst]


def test_remove_duplicates_kat():
    """test/test_search.jl:113-131."""
    g = KATS["remove_duplicates"]
    cands = _mk(g["T"], g["nharm"], g["cands"])
    kept = o.remove_duplicates(cands, g["dr_tol"])
    assert len(kept) == g["expected_len"]
    assert [c.freq for c in kept] == sorted(c.freq for c in kept)
    assert np.allclose(sorted(c.metric for c in kept), g["expected_metrics"])
    assert len(o.remove_duplicates(cands, 1e9)) == 1
    assert o.remove_duplicates([]) == []


def test_remove_harmonics_kat():
    """test/test_search.jl:133-150."""
    g = KATS["remove_harmonics"]
    fam = _mk(g["T"], 16, g["fam"])
    kept = o.remove_harmonics(fam, 16, 1.0)
    assert len(kept) == 1 and kept[0].r == g["fam_kept"][0] and kept[0].metric == g["fam_kept"][1]
    mixed = fam + _mk(g["T"], 16, g["extra"])
    kept2 = o.remove_harmonics(mixed, 16, 1.0)
    assert len(kept2) == 2
    assert {round(c.r) for c in kept2} == set(g["mixed_kept_r"])
    assert len(o.remove_harmonics(fam, 1, 1.0)) == g["numharm1_len"]
    assert o.remove_harmonics([]) == []


def _naive_best(prof, nb):
    s = np.sort(prof)
    med = s[(nb + 1) // 2 - 1] if nb % 2 else 0.5 * (s[nb // 2 - 1] + s[nb // 2])
    z = prof - med
    best, bw = -math.inf, 0
    for w in o.boxcar_widths(nb):
        for p in range(nb):
            v = sum(z[(p + i) % nb] for i in range(w)) / math.sqrt(w)
            if v > best:
                best, bw = v, w
    return bw


def test_boxcar_best_width():
    """test/test_search.jl:685-741."""
    nb = 64
    for w in o.boxcar_widths(nb):
        prof = np.zeros(nb)
        prof[9:9 + w] = 1.0
        bw, ducy = o.boxcar_best_width(prof)
        assert bw == w and abs(ducy - w / nb) < 1e-15
    prof = np.zeros(nb)
    prof[62:64] = 1.0
    prof[0:2] = 1.0
    assert o.boxcar_best_width(prof)[0] == 4
    prof = np.zeros(nb)
    prof[19:25] = 1.0
    w0 = o.boxcar_best_width(prof)[0]
    assert o.boxcar_best_width(1e6 * prof)[0] == w0
    assert o.boxcar_best_width(prof + 37.0)[0] == w0
    rng = np.random.default_rng(20260811)
    for w in (1, 3, 9, 13):
        for _ in range(5):
            prof = 0.05 * rng.standard_normal(nb)
            prof[29:29 + w] += 3.0
            assert o.boxcar_best_width(prof)[0] == _naive_best(prof, nb)
    for _ in range(20):
        prof = rng.standard_normal(nb)
        assert o.boxcar_best_width(prof)[0] == _naive_best(prof, nb)


def test_trial_grid_rational():
    """src/directinterp.jl:217-225 on the default and a few other grids."""
    assert o.trial_grid_rational(0.5 / 60) == (1, 120)
    assert o.trial_grid_rational(0.5 / 32) == (1, 64)
    assert o.trial_grid_rational(0.25 / 60) == (1, 240)
    assert o.trial_grid_rational(1.0 / 3.0) == (1, 3)
    assert o.trial_grid_rational(0.5 / 7) == (1, 14)
    assert o.trial_grid_rational(math.pi / 100) is None
    assert o.trial_grid_rational(0.0) is None
