"""Host side of the metric statistics (no GPU): hist_quantile, the merged and
summarised histograms and build_metricnorm follow the reference's formulas
(src/search.jl:1419-1473, :1518-1559, :1603-1643) on hand-built histograms."""
import math

import numpy as np
import pytest

from cohsearch.metricstats import (MIN_WIN_TRIALS, MetricHistogram, MetricStats, build_metricnorm,
                                   hist_quantile, merge_hists, metricstats_summary, normalize, window_index)


def _hist(k, win, counts, lo=0.0, hi=10.0, under=0, over=0, flo=1.0, fhi=2.0, values=None):
    counts = np.asarray(counts, np.int64)
    nb = len(counts)
    h = MetricHistogram(k, 60 // k, 2 * (60 // k), win, flo, fhi, lo, hi, nb / (hi - lo), counts.copy(),
                        under, over)
    h.total = int(counts.sum()) + under + over
    if values is not None:
        h.sum = float(np.sum(values))
        h.sumsq = float(np.sum(np.square(values)))
        h.vmin, h.vmax = float(np.min(values)), float(np.max(values))
    return h


def test_hist_quantile_formula():
    h = _hist(1, 1, [10, 0, 30, 60], lo=0.0, hi=4.0)      # bins of width 1
    assert hist_quantile(h, 0.05) == pytest.approx(0.5)    # inside bin 1
    assert hist_quantile(h, 0.10) == pytest.approx(1.0)    # exactly at bin 1's end
    assert hist_quantile(h, 0.25) == pytest.approx(2.5)    # empty bin skipped, halfway into bin 3
    assert hist_quantile(h, 1.0) == pytest.approx(4.0)
    u = _hist(1, 1, [0, 5], under=5)
    assert hist_quantile(u, 0.5) == u.lo                    # the underflow holds the quantile
    o = _hist(1, 1, [5, 0], over=5)
    assert hist_quantile(o, 0.9) == o.hi                    # in the overflow: the range's end
    assert math.isnan(hist_quantile(_hist(1, 1, [0, 0]), 0.5))


def test_merge_and_summary():
    rng = np.random.default_rng(1)
    vals = [rng.uniform(0, 10, 500), rng.uniform(0, 10, 300)]
    hs = []
    for w, v in enumerate(vals, start=1):
        c, _ = np.histogram(v, bins=20, range=(0, 10))
        hs.append(_hist(2, w, c, values=v, flo=w, fhi=w + 1))
    g = merge_hists(hs, 0, 1.0, 3.0)
    assert g.total == 800 and np.array_equal(g.counts, hs[0].counts + hs[1].counts)
    assert g.vmin == min(h.vmin for h in hs) and g.vmax == max(h.vmax for h in hs)
    ms = MetricStats(hist_lo=0.0, hist_hi=10.0, hist_nb=20, nwin=2, hists=[g], whists=hs)
    r = metricstats_summary(ms, faps=(0.1,))[0]
    allv = np.concatenate(vals)
    assert r["mean"] == pytest.approx(allv.mean()) and r["std"] == pytest.approx(allv.std(ddof=1))
    assert r["fap"][0] == pytest.approx(hist_quantile(g, 0.9))


def test_build_metricnorm_fallbacks_and_windows():
    rng = np.random.default_rng(2)
    dense = rng.normal(5.0, 1.0, 5000)
    sparse = rng.normal(5.0, 1.0, MIN_WIN_TRIALS - 1)
    edges = [1.0, 2.0, 4.0]
    ws = []
    for w, v in enumerate([dense, sparse], start=1):
        c, _ = np.histogram(v, bins=200, range=(0, 10))
        ws.append(_hist(1, w, c, values=v, flo=edges[w - 1], fhi=edges[w]))
    g = merge_hists(ws, 0, 1.0, 4.0)
    ms = MetricStats(hist_lo=0.0, hist_hi=10.0, hist_nb=200, nwin=2, hists=[g], whists=ws)
    norm = build_metricnorm(ms)
    assert norm.edges[1] == edges
    assert norm.loc[1][0] == pytest.approx(hist_quantile(ws[0], 0.5))
    assert norm.scale[1][0] == pytest.approx(hist_quantile(ws[0], 0.8413) - hist_quantile(ws[0], 0.5))
    # the sparse window falls back to the band-wide estimate
    assert norm.loc[1][1] == pytest.approx(hist_quantile(g, 0.5))
    assert window_index(edges, 0.5) == 1 and window_index(edges, 3.0) == 2 and window_index(edges, 9.0) == 2
    z1 = normalize(norm, 1, 1.5, 7.0)
    assert z1 == pytest.approx((7.0 - norm.loc[1][0]) / norm.scale[1][0])
    assert normalize(norm, 5, 1.5, 7.0) == 7.0                  # no model for k: unchanged


def test_rotate_to_peak():
    """test/test_candidate.jl:14-21: the maximum moves to bin n//2 (0-based)."""
    from cohsearch import rotate_to_peak
    for n in (8, 9, 64, 65):
        prof = np.arange(1.0, n + 1)
        rp = rotate_to_peak(prof)
        assert len(rp) == n and int(np.argmax(rp)) == n // 2 and sorted(rp) == sorted(prof)
    assert rotate_to_peak(np.zeros(0)).size == 0
