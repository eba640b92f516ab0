"""Metric statistics and in-situ normalisation on the device (the reference's
--metricstats / --normalize, src/search.jl:1296-1643 and :2063-2094).

* The reference's own testsets (test/test_search.jl:584-684) read the absent
  example file `harmonics_hi.fft`; their properties are restated here on the
  synthetic stand-in (a 10.0123456789123 Hz pulsar, N = 2^20, dt = 1 ms).
* Exactness: the device's per-(block, k) statistics and histograms are checked
  against numpy over the device's own per-trial exact metrics -- n, min, max,
  median and every histogram count exactly; mean, std, sum and sumsq to 1e-12
  relative (FP64 sums in a different order).
* The normalised pass's candidates equal numpy's z = (M - loc)/scale > threshold
  over the same metrics and the MetricNorm built from the stats pass.
"""
import math

import numpy as np
import pytest

from tests.fixtures import pulsar_spectrum

pytestmark = pytest.mark.gpu

NH = 60
KW = dict(lofreq=8.0, hifreq=12.0, lobin=100, blocksize=1024)


def _cs():
    import cohsearch
    return cohsearch


def _engine(params, diag=1):
    cs = _cs()
    amps, N, dt = pulsar_spectrum()
    eng = cs.Engine(params)
    eng.set_diagnostics(diag)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    return eng, N, dt


def test_metricstats_reference_properties():
    """test/test_search.jl:584-653 restated on the synthetic spectrum."""
    cs = _cs()
    amps, N, dt = pulsar_spectrum()
    params = cs.SearchParams(nharms=NH, decimations=cs.decimation_set(NH, 3))
    ft = cs.FFTFile.from_array(amps, N, dt)
    ref = cs.search(ft, params, threshold=8.0, **KW)
    ms = cs.MetricStats(hist_hi=30000.0, hist_nb=6000)
    with_ = cs.search(ft, params, threshold=8.0, metricstats=ms, **KW)
    assert len(with_) == len(ref)
    assert all(a.freq == b.freq and a.metric == b.metric for a, b in zip(with_, ref))
    assert ms.blocks
    assert {s.k for s in ms.blocks} == {1, 2, 3}
    assert all(s.nbins == 2 * s.Hk and s.Hk == NH // s.k for s in ms.blocks)
    assert all(s.min <= s.median <= s.max and s.min <= s.mean <= s.max for s in ms.blocks)
    assert [h.k for h in ms.hists] == [1, 2, 3]
    for h in ms.hists:
        assert int(h.counts.sum()) + h.under + h.over == h.total
        assert h.total == sum(s.n for s in ms.blocks if s.k == h.k)
        assert h.vmin <= cs.hist_quantile(h, 0.5) <= h.vmax
        assert cs.hist_quantile(h, 0.1) <= cs.hist_quantile(h, 0.9)
    assert {h.k for h in ms.whists} == {1, 2, 3}
    for h in ms.whists:
        assert sum(1 for w in ms.whists if w.k == h.k) == ms.nwin
        assert h.flo < h.fhi
    for g in ms.hists:
        wk = sorted([h for h in ms.whists if h.k == g.k], key=lambda h: h.win)
        assert sum(h.total for h in wk) == g.total
        assert math.isclose(sum(h.sum for h in wk), g.sum, rel_tol=1e-12)
        assert np.array_equal(sum(h.counts for h in wk), g.counts)
        assert all(math.isclose(wk[i].fhi, wk[i + 1].flo, rel_tol=1e-12) for i in range(len(wk) - 1))
    summ = cs.metricstats_summary(ms, faps=(0.1, 0.01, 1e-3))
    assert [r["k"] for r in summ] == [1, 2, 3]
    for r, h in zip(summ, ms.hists):
        assert r["ntrials"] == h.total
        assert math.isclose(r["mean"], h.sum / h.total)
        assert r["max"] == h.vmax and len(r["fap"]) == 3
    assert summ[0]["mean"] > summ[1]["mean"] > summ[2]["mean"]
    assert summ[0]["fap"][0] > summ[2]["fap"][0]
    wrows = cs.metricstats_windows(ms, faps=(0.1, 0.01))
    assert wrows and all(r["ntrials"] > 0 for r in wrows)
    assert {r["k"] for r in wrows} <= {1, 2, 3}


def _numpy_stats(eng, N, dt, ms, params, lofreq, hifreq, blocksize):
    """Block stats and histograms recomputed in numpy from the device's exact
    per-trial metrics of the last search, with the reference's expressions."""
    cs = _cs()
    T = N * dt
    lodr = params.hidr / params.nharms
    r_lo = lofreq * T
    tm = eng.trial_metrics()
    sig, nv = eng.block_values()
    ks = [1] + [k for k in params.decimations if k > 1]
    nlev = len(ks)
    nblk = len(nv) // nlev
    tm = tm.reshape(nblk, nlev, blocksize)
    nv = nv.reshape(nblk, nlev)
    total = int(math.floor((hifreq * T - r_lo) / lodr)) + 1
    # window edges by the reference rule (_logedges, src/search.jl:1405-1411),
    # restated here; the device's histograms must carry the same edges
    r_hi = hifreq * T

    def logedges(a, b, nwin):
        a = max(float(a), np.finfo(np.float64).tiny)
        b = max(float(b), a * (1 + 1e-9))
        la, lb = math.log10(a), math.log10(b)
        return [10.0 ** (la + (lb - la) * i / nwin) for i in range(nwin + 1)]

    edges = {h.k: logedges(h.k * r_lo / T, h.k * r_hi / T, ms.nwin) for h in ms.hists}
    for h in ms.hists:
        dev = [w.flo for w in sorted([x for x in ms.whists if x.k == h.k], key=lambda x: x.win)] + [h.fhi]
        assert np.allclose(dev, edges[h.k], rtol=1e-13, atol=0.0)
    invw = ms.hist_nb / (ms.hist_hi - ms.hist_lo)
    blocks, hist = [], {}
    for c in range(nblk):
        i0 = c * blocksize
        n = min(blocksize, total - i0)
        rstart = r_lo + i0 * lodr
        rmean = rstart + (n - 1) * lodr / 2
        for l, k in enumerate(ks):
            v = tm[c, l, :nv[c, l]].astype(np.float64)
            if k > 1 and len(v) == 0:
                continue
            f = rmean / T if k == 1 else k * rmean / T
            from cohsearch.metricstats import window_index
            w = window_index(edges[k], f)
            blocks.append((c + 1, k, len(v), v.min(), float(np.median(v)), v.mean(),
                           v.std(ddof=1) if len(v) > 1 else 0.0, v.max()))
            hc = hist.setdefault((k, w), [np.zeros(ms.hist_nb, np.int64), 0, 0, 0, 0.0, 0.0])
            lo_m = v < ms.hist_lo
            hi_m = v >= ms.hist_hi
            mid = v[~lo_m & ~hi_m]
            b = np.minimum(np.floor((mid - ms.hist_lo) * invw).astype(np.int64), ms.hist_nb - 1)
            np.add.at(hc[0], b, 1)
            hc[1] += int(lo_m.sum())
            hc[2] += int(hi_m.sum())
            hc[3] += len(v)
            hc[4] += float(np.sum(v))
            hc[5] += float(np.sum(v * v))
    return blocks, hist


@pytest.mark.parametrize("synth", ["fp32", "fp16"])
def test_metricstats_exact_against_the_device_metrics(synth):
    cs = _cs()
    params = cs.SearchParams(nharms=NH, decimations=cs.decimation_set(NH, 3), synth=synth)
    eng, N, dt = _engine(params)
    ms = cs.MetricStats(hist_hi=30000.0, hist_nb=6000, nwin=8)
    eng.set_metricstats(ms)
    eng.search_raw(KW["lofreq"], KW["hifreq"], 100, KW["blocksize"], 8.0)
    eng.fetch_metricstats(ms)
    eng.set_metricstats(None)
    blocks, hist = _numpy_stats(eng, N, dt, ms, params, KW["lofreq"], KW["hifreq"], KW["blocksize"])
    assert len(blocks) == len(ms.blocks)
    for s, (blk, k, n, mn, med, mean, std, mx) in zip(ms.blocks, blocks):
        assert (s.block, s.k, s.n) == (blk, k, n)
        assert s.min == mn and s.max == mx and s.median == med
        assert math.isclose(s.mean, mean, rel_tol=1e-12) and math.isclose(s.std, std, rel_tol=1e-10)
    for h in ms.whists:
        ref = hist.get((h.k, h.win))
        if ref is None:
            assert h.total == 0 and int(h.counts.sum()) == 0
            continue
        assert np.array_equal(h.counts, ref[0])
        assert (h.under, h.over, h.total) == (ref[1], ref[2], ref[3])
        assert math.isclose(h.sum, ref[4], rel_tol=1e-12) and math.isclose(h.sumsq, ref[5], rel_tol=1e-12)


def test_normalize_two_pass_exact_and_reference_properties():
    """test/test_search.jl:655-684 restated, plus the exact candidate set."""
    cs = _cs()
    from cohsearch.metricstats import normalize
    params = cs.SearchParams(nharms=NH, decimations=cs.decimation_set(NH, 3))
    amps, N, dt = pulsar_spectrum()
    ft = cs.FFTFile.from_array(amps, N, dt)
    ms = cs.MetricStats(hist_hi=30000.0, hist_nb=6000, nwin=8)
    kw = dict(lofreq=9.5, hifreq=10.5, blocksize=1024)
    cands = cs.search(ft, params, threshold=5.0, metricstats=ms, normalize=True, remove=False,
                      harm_remove=False, **kw)
    assert ms.hists
    assert any(abs(c.freq - 10.0123) < 1e-2 for c in cands)
    norm = cs.build_metricnorm(ms)
    assert set(norm.loc) == {1, 2, 3}
    for g in ms.hists:
        assert len(norm.loc[g.k]) == ms.nwin
        assert all(x > 0 for x in norm.scale[g.k])
        assert all(g.vmin <= x <= g.vmax for x in norm.loc[g.k])
    assert normalize(norm, 1, 10.0123, 200.0) > normalize(norm, 1, 10.0123, 100.0)
    # exact: the detection pass's candidates are numpy's z > threshold over the
    # device's exact metrics (identical to the stats pass's)
    eng, N, dt = _engine(params)
    eng.set_metricnorm(norm)
    raw = eng.search_raw(kw["lofreq"], kw["hifreq"], 100, kw["blocksize"], 5.0)
    eng.set_metricnorm(None)
    T = N * dt
    lodr = params.hidr / params.nharms
    r_lo = kw["lofreq"] * T
    tm = eng.trial_metrics()
    sig, nv = eng.block_values()
    ks = [1] + [k for k in params.decimations if k > 1]
    nlev = len(ks)
    nblk = len(nv) // nlev
    tm = tm.reshape(nblk, nlev, kw["blocksize"])
    nv = nv.reshape(nblk, nlev)
    want = []
    for c in range(nblk):
        rstart = r_lo + (c * kw["blocksize"]) * lodr
        for l, k in enumerate(ks):
            for j in range(nv[c, l]):
                rf = rstart + j * lodr
                r = rf if k == 1 else k * rf
                z = normalize(norm, k, r / T, float(tm[c, l, j]))
                if z > 5.0:
                    want.append((c * kw["blocksize"] + j, k, z))
    got = sorted((int(c["trial"]), int(c["k"]), float(c["metric"])) for c in raw)
    assert got == sorted(want)
