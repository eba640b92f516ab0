"""Metric statistics and in-situ normalisation: the host side of the
reference's ``--metricstats`` / ``--normalize`` (src/search.jl:1296-1643).

The device collects, in one exact pass over every trial, the per-(block, k)
moments (``BlockMetricStats``) and the per-(k, searched-frequency window)
histograms (``MetricHistogram``); this module holds those records with the
reference's names and fields, reads quantiles off the histograms, and builds
the per-(k, window) normalisation (``MetricNorm``) that a second pass applies.
"""
import math
from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np

MIN_WIN_TRIALS = 200   # _MIN_WIN_TRIALS (src/search.jl:1566): below this a window uses the per-k estimate


@dataclass
class BlockMetricStats:
    """One processed (block, k): exact min/median/mean/std/max of its trials'
    raw metric (src/search.jl:1321-1335)."""
    block: int
    k: int
    Hk: int
    nbins: int
    ngoodbins: float
    flo: float
    fhi: float
    n: int
    min: float
    median: float
    mean: float
    std: float
    max: float


@dataclass
class MetricHistogram:
    """Fixed-range histogram of the metric for one k within one searched-
    frequency window [flo, fhi) Hz (win = 0: merged over the band), with exact
    total/sum/sumsq/vmin/vmax (src/search.jl:1362-1402)."""
    k: int
    Hk: int
    nbins: int
    win: int
    flo: float
    fhi: float
    lo: float
    hi: float
    invw: float
    counts: np.ndarray
    under: int = 0
    over: int = 0
    total: int = 0
    sum: float = 0.0
    sumsq: float = 0.0
    vmin: float = math.inf
    vmax: float = -math.inf


@dataclass
class MetricStats:
    """The opt-in sink passed to ``search`` (src/search.jl:1481-1515)."""
    hist_lo: float = 0.0
    hist_hi: float = 64.0
    hist_nb: int = 3200
    nwin: int = 16
    blocks: List[BlockMetricStats] = field(default_factory=list)
    hists: List[MetricHistogram] = field(default_factory=list)
    whists: List[MetricHistogram] = field(default_factory=list)

    def __post_init__(self):
        self.nwin = max(1, int(self.nwin))
        if not self.hist_hi > self.hist_lo:
            raise ValueError(f"histogram hi ({self.hist_hi}) must exceed lo ({self.hist_lo})")
        if self.hist_nb < 1:
            raise ValueError("histogram bin count must be >= 1")


def merge_hists(hs, win, flo, fhi) -> MetricHistogram:
    """_merge_hists (src/search.jl:1419-1426): the windows of one k summed in order."""
    h1 = hs[0]
    g = MetricHistogram(h1.k, h1.Hk, h1.nbins, win, flo, fhi, h1.lo, h1.hi, h1.invw,
                        np.zeros_like(h1.counts))
    for h in hs:
        g.counts += h.counts
        g.under += h.under
        g.over += h.over
        g.total += h.total
        g.sum += h.sum
        g.sumsq += h.sumsq
        g.vmin = min(g.vmin, h.vmin)
        g.vmax = max(g.vmax, h.vmax)
    return g


def hist_quantile(h: MetricHistogram, q: float) -> float:
    """q-th quantile, linear within the containing bin (src/search.jl:1456-1473)."""
    if h.total == 0:
        return math.nan
    target = q * h.total
    cum = h.under
    if cum >= target:
        return h.lo
    w = 1 / h.invw
    for i, c in enumerate(h.counts):
        c = int(c)
        if cum + c >= target:
            edge = h.lo + i * w
            return edge if c == 0 else edge + (target - cum) / c * w
        cum += c
    return h.hi


def _hist_row(h: MetricHistogram, faps):
    N = h.total
    mean = h.sum / N if N > 0 else math.nan
    std = math.sqrt(max(0.0, (h.sumsq - N * mean ** 2) / (N - 1))) if N > 1 else 0.0
    return dict(k=h.k, Hk=h.Hk, nbins=h.nbins, win=h.win, flo=h.flo, fhi=h.fhi, ntrials=N,
                min=h.vmin if N > 0 else math.nan, median=hist_quantile(h, 0.5), mean=mean, std=std,
                max=h.vmax if N > 0 else math.nan, fap=tuple(hist_quantile(h, 1 - p) for p in faps),
                overflow=h.over / N if N > 0 else 0.0)


def metricstats_summary(ms: MetricStats, faps=(0.1, 0.01, 1e-3, 1e-4)):
    """One row per k over the whole band (src/search.jl:1518-1546)."""
    return [dict(_hist_row(h, faps), nblocks=sum(1 for s in ms.blocks if s.k == h.k and s.n > 0))
            for h in ms.hists]


def metricstats_windows(ms: MetricStats, faps=(0.1, 0.01, 1e-3, 1e-4)):
    """One row per non-empty (k, window) (src/search.jl:1548-1559)."""
    return [_hist_row(h, faps) for h in ms.whists if h.total > 0]


@dataclass
class MetricNorm:
    """Per-(k, window) location and scale of the metric (src/search.jl:1596-1600)."""
    edges: Dict[int, List[float]]
    loc: Dict[int, List[float]]
    scale: Dict[int, List[float]]


def _loc_scale(h: MetricHistogram):
    loc = hist_quantile(h, 0.5)
    scale = hist_quantile(h, 0.8413) - loc
    return loc, (scale if scale > 0 else math.nan)


def build_metricnorm(ms: MetricStats) -> MetricNorm:
    """build_metricnorm (src/search.jl:1603-1634): per (k, window) the noise
    median and upper 1-sigma spread, with the per-k band-wide estimate for
    sparse or degenerate windows."""
    edges, locs, scales = {}, {}, {}
    for g in ms.hists:
        k = g.k
        gloc, gscale = _loc_scale(g)
        if math.isnan(gscale):
            gscale = 1.0
        wins = sorted([h for h in ms.whists if h.k == k], key=lambda h: h.win)
        if not wins:
            continue
        edges[k] = [h.flo for h in wins] + [wins[-1].fhi]
        locv, sclv = [], []
        for h in wins:
            wloc, wscale = _loc_scale(h)
            if h.total < MIN_WIN_TRIALS or math.isnan(wscale):
                locv.append(gloc)
                sclv.append(gscale)
            else:
                locv.append(wloc)
                sclv.append(wscale)
        locs[k], scales[k] = locv, sclv
    return MetricNorm(edges, locs, scales)


def window_index(edges, f: float) -> int:
    """_window_index (src/search.jl:1415-1416), 1-based."""
    c = sum(1 for e in edges if e <= f)
    return min(max(c, 1), len(edges) - 1)


def normalize(norm: MetricNorm, k: int, f: float, M: float) -> float:
    """_normalize (src/search.jl:1638-1643)."""
    e = norm.edges.get(k)
    if e is None:
        return M
    w = window_index(e, f) - 1
    return (M - norm.loc[k][w]) / norm.scale[k][w]
