"""Candidate refold on the device (candidate_profile / measure_ducy,
src/candidate.jl:37-99) against the numpy FP64 oracle: profiles within 1e-10
of the profile's RMS, duty cycles exact (the same width wins), and the
reference's edge rules -- the harmonic sum stops at Nyquist, nharm < 1 or
r <= 0 leave the duty cycle NaN."""
import math

import numpy as np
import pytest

from oracle import cs_ref as o
from tests.fixtures import PSR_F, pulsar_spectrum

pytestmark = pytest.mark.gpu


def test_refold_matches_oracle_and_edges():
    import cohsearch as cs
    amps, N, dt = pulsar_spectrum()
    T = N * dt
    params = cs.SearchParams(nharms=32)
    eng = cs.Engine(params)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    rng = np.random.default_rng(5)
    r = np.concatenate([[PSR_F * T, 2 * PSR_F * T, PSR_F * T + 0.37], rng.uniform(100.0, 2e5, 20),
                        [N / 2 - 40.0, N / 2 / 3.0 + 0.5]])
    nh = np.concatenate([[32, 16, 60], rng.integers(1, 61, 20), [8, 32]]).astype(np.int32)
    H, profs, ducy = eng.refold(r, nh, 64)
    for i in range(len(r)):
        want = o.candidate_profile(amps, N, float(r[i]), int(nh[i]), 64)
        assert len(profs[i]) == len(want)
        scale = max(float(np.sqrt(np.mean(want ** 2))), 1e-30)
        assert np.max(np.abs(profs[i] - want)) <= 1e-10 * scale
        wd = o.measure_ducy(amps, N, [float(r[i])], [int(nh[i])], o.SearchParams(nharms=32))[0]
        assert ducy[i] == wd
    assert H[-2] < 8 and H[-1] < 32                       # stopped at Nyquist
    assert H[0] == 32 and abs(ducy[0] - 0.03) < 0.05        # the pulsar's narrow pulse
    H2, _, d2 = eng.refold(np.array([0.0, 500.0]), np.array([5, 0], np.int32), 64)
    assert list(H2) == [-1, -1] and all(math.isnan(x) for x in d2)
    c = cs.Candidate(PSR_F, 40.0, PSR_F * T, 32)
    out = cs.measure_ducy(cs.FFTFile.from_array(amps, N, dt), [c], params)
    assert out[0].ducy == ducy[0] and out[0].r == c.r
    prof = cs.candidate_profile(cs.FFTFile.from_array(amps, N, dt), PSR_F * T, 32)
    assert np.array_equal(prof, profs[0])


def test_refold_reference_properties():
    """test/test_candidate.jl:24-56 and test/test_cli.jl:87-103 restated on the
    synthetic pulsar (the reference's example file is absent)."""
    import cohsearch as cs
    amps, N, dt = pulsar_spectrum()
    T = N * dt
    ft = cs.FFTFile.from_array(amps, N, dt)
    nh = 32
    params = cs.SearchParams(nharms=nh, m=32, numbetween=256)
    rbest = float(cs.search(ft, params, lofreq=9.9, hifreq=10.1, threshold=8.0)[0].r)
    ref = o.reference_profiles(amps, N, np.array([rbest]), o.SearchParams(nharms=nh, m=32, numbetween=256))[0]
    cand = cs.candidate_profile(ft, rbest, nh, m=32)
    assert len(cand) == 2 * nh
    assert np.max(np.abs(cand - ref)) / np.max(np.abs(ref)) < 1e-3
    wide = cs.candidate_profile(ft, rbest, nh)
    assert len(wide) == 2 * nh and int(np.argmax(cs.rotate_to_peak(wide))) == nh
    r_fast = 0.49 * N / 2 / 150.0 * 2.0           # ~150 harmonics fit below Nyquist
    capped = cs.candidate_profile(ft, r_fast, 200)
    H = len(capped) // 2
    assert len(capped) % 2 == 0 and H < 200
    assert r_fast * H < N // 2 and r_fast * (H + 2) > N // 2
    sp = cs.SearchParams(nharms=nh)
    cands = cs.search(ft, sp, lofreq=5.0, hifreq=25.0, threshold=8.0)
    assert cands and all(math.isnan(c.ducy) for c in cands)
    measured = cs.measure_ducy(ft, cands, sp)
    for a, c in zip(measured, cands):
        assert a.freq == c.freq and a.metric == c.metric and a.r == c.r and a.nharm == c.nharm
        assert 0 < a.ducy <= sp.boxcar_maxfrac
    best = measured[int(np.argmax([c.metric for c in measured]))]
    assert best.ducy < sp.boxcar_maxfrac
