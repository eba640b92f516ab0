"""Host mirror of CoherentSearch.jl's search API over the B200 engine.

Same names, argument meaning and error behaviour as the Julia API
(src/CoherentSearch.jl:17-51): ``SearchParams``, ``decimation_set``,
``search``, ``SearchCache``, ``chunk_metrics``, ``Candidate``,
``remove_duplicates``, ``remove_harmonics``, ``write_candidates``, and the
command line's per-file loop with its ``.cohout`` naming (``search_files``,
``output_path``).  The hot
loop runs in ``libcohsearch_cuda.so`` through the C ABI; only the
post-processing of the few hundred raw detections (duplicate and harmonic
collapse, src/search.jl:2148-2214) runs here, as it runs in Julia in the
reference.  Invalid arguments raise ``ValueError`` (Julia ``ArgumentError``).
"""
import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib

# ---------------------------------------------------------------------------
# Parameters (src/search.jl:131-167, 387-459)
# ---------------------------------------------------------------------------


@dataclass(eq=False)
class SearchParams:
    """Tunable search parameters, defaults as src/search.jl:131-144.

    ``synth`` selects the device profile-synthesis arithmetic: ``"fp32"`` (the
    plain FP32 GPU form), ``"bf16"`` or ``"fp16"`` (tensor-core forms), or
    ``"bf16_split"`` / ``"fp16_split"`` (each amplitude split hi + lo into two
    16-bit operands: a closer gate for twice the A-tile bytes).
    Equality is identity, as ``SearchCache`` keys on the object.
    """
    nharms: int = 32
    m: int = 16
    numbetween: int = 16
    hidr: float = 0.5
    threshold: float = 8.0
    boxcar_fsp: float = 1.5
    boxcar_maxfrac: float = 0.3
    boxcar_medmargin: float = 2.0
    decimations: List[int] = field(default_factory=lambda: [1])
    precision: str = "f64"
    synth: str = "fp32"

    def to_c(self):
        if self.m % 2:
            raise ValueError("m must be even")
        if self.precision not in ("f64", "f32"):
            raise ValueError(f"precision must be :f64 or :f32, got {self.precision}")
        if self.synth not in _lib.CS_SYNTH:
            raise ValueError(f"synth must be one of {sorted(_lib.CS_SYNTH)}")
        if len(self.decimations) > _lib.CS_MAX_DECIM:
            raise ValueError("at most 16 decimation factors")
        p = _lib.cs_params()
        p.nharms = int(self.nharms)
        p.m = int(self.m)
        p.numbetween = int(self.numbetween)
        p.ndecim = len(self.decimations)
        for i, k in enumerate(self.decimations):
            p.decimations[i] = int(k)
        p.hidr = float(self.hidr)
        p.threshold = float(self.threshold)
        p.boxcar_fsp = float(self.boxcar_fsp)
        p.boxcar_maxfrac = float(self.boxcar_maxfrac)
        p.boxcar_medmargin = float(self.boxcar_medmargin)
        p.precision = 0 if self.precision == "f64" else 1
        p.synth = _lib.CS_SYNTH[self.synth]
        return p


def proftype(params: SearchParams):
    """src/search.jl:152-156."""
    if params.precision == "f64":
        return np.float64
    if params.precision == "f32":
        return np.float32
    raise ValueError(f"precision must be :f64 or :f32, got {params.precision}")


def decimation_set(nharms: int, maxdecim: int) -> List[int]:
    """src/search.jl:166-167."""
    return [k for k in range(1, max(1, maxdecim) + 1) if nharms // k >= 2]


def boxcar_widths(nbins: int, fsp: float = 1.5, maxfrac: float = 0.3) -> List[int]:
    """src/search.jl:387-396."""
    wmax = max(1, math.floor(maxfrac * nbins))
    ws, w = [], 1
    while w <= wmax:
        ws.append(w)
        w = max(math.floor(fsp * w), w + 1)
    return ws


def ladder_boxcar_widths(nbins: int, k: int, params: SearchParams) -> List[int]:
    """src/search.jl:443-459."""
    ws = boxcar_widths(nbins, params.boxcar_fsp, params.boxcar_maxfrac)
    ks = sorted(params.decimations)
    if len(ks) <= 1 or not all(ks[i + 1] <= 3 * ks[i] for i in range(len(ks) - 1)):
        return ws
    kmin, kmax = ks[0], ks[-1]
    pruned = [w for w in ws if (w >= 2 or k == kmin) and (w <= 6 or k == kmax)]
    return pruned or ws


# ---------------------------------------------------------------------------
# Candidates and post-processing (src/search.jl:179-191, 2148-2214)
# ---------------------------------------------------------------------------


@dataclass
class Candidate:
    """src/search.jl:179-191, plus the decimation factor and global trial."""
    freq: float
    metric: float
    r: float
    nharm: int
    ducy: float = math.nan
    k: int = 1
    trial: int = -1


def remove_duplicates(cands: Sequence[Candidate], dr_tol: float = 1.0) -> List[Candidate]:
    """Collapse runs of near-identical ``r`` to their strongest member."""
    if not cands:
        return []
    order = sorted(range(len(cands)), key=lambda i: cands[i].r)
    kept = []
    best = cands[order[0]]
    prev = best.r
    for i in order[1:]:
        c = cands[i]
        if c.r - prev <= dr_tol:
            if c.metric > best.metric:
                best = c
        else:
            kept.append(best)
            best = c
        prev = c.r
    kept.append(best)
    return sorted(kept, key=lambda c: c.freq)


def _harmonically_related(r1: float, r2: float, numharm: int, tol: float) -> bool:
    lo, hi = min(r1, r2), max(r1, r2)
    if not lo > 0:
        return False
    for m in range(1, numharm + 1):
        n = int(round(m * hi / lo))
        if 1 <= n <= numharm and abs(m * hi - n * lo) <= tol * m:
            return True
    return False


def remove_harmonics(cands: Sequence[Candidate], numharm: int = 16, tol: float = 1.0) -> List[Candidate]:
    """Keep the strongest member of each harmonically related family."""
    if not cands:
        return []
    order = sorted(range(len(cands)), key=lambda i: -cands[i].metric)
    kept: List[Candidate] = []
    for i in order:
        c = cands[i]
        if not any(_harmonically_related(c.r, k.r, numharm, tol) for k in kept):
            kept.append(c)
    return sorted(kept, key=lambda c: c.freq)


def write_candidates(cands: Sequence[Candidate], outfile: str, threshold) -> None:
    """The ``.cohout`` table of src/cli.jl:317-340 ('' writes to stdout)."""
    lines = ["#       'S/N'      Frequency (Hz)        Period (ms)    #Harm  Ducy(%)"]
    for i, c in enumerate(cands, 1):
        ducy = "-" if math.isnan(c.ducy) else f"{100 * c.ducy:.2f}"
        lines.append(f"{i:<4d}  {c.metric:8.2f}  {c.freq:18.12f}  {1000.0 / c.freq:18.12f}   "
                     f"{c.nharm:3d}   {ducy:>6s}")
    if not outfile:
        print("\n".join(lines))
        import sys
        print(f"# {len(cands)} candidates above threshold {threshold}", file=sys.stderr)
    else:
        with open(outfile, "w") as f:
            f.write("\n".join(lines) + "\n")


# ---------------------------------------------------------------------------
# Device engine
# ---------------------------------------------------------------------------


class Engine:
    """One ``cs_handle``: the device plans, buffers and stream for one
    ``SearchParams`` (the SearchCache's workspaces, src/search.jl:1914-1961)."""

    def __init__(self, params: SearchParams, device: int = 0):
        self.lib = _lib.load()
        self.params = params
        self.device = device
        self._h = ctypes.c_void_p()
        cp = params.to_c()
        st = self.lib.cs_create(ctypes.byref(self._h), ctypes.byref(cp), int(device))
        if st == _lib.CS_ERR_INVALID_ARGUMENT:
            raise ValueError("invalid SearchParams")
        _lib.check(st, None, "cs_create")
        self._spec_key = None
        self._spec_keep = None

    def close(self):
        if self._h:
            self.lib.cs_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        """Issue the engine's work on a caller's cudaStream_t (int pointer; 0 = own)."""
        _lib.check(self.lib.cs_set_stream(self._h, ctypes.c_void_p(int(stream_ptr) or None)), self._h)

    # -- spectrum ---------------------------------------------------------
    def set_spectrum(self, ft, force=False):
        """Copy `ft`'s spectrum to the device, unless this very FFTFile (and
        its amps array) was the last one attached.  The engine keeps both
        objects referenced, so their identities cannot be reused by new ones;
        after changing ft.amps in place, pass force=True."""
        if not force and self._spec_key == ("file",) and self._spec_keep is not None and \
                self._spec_keep[0] is ft and self._spec_keep[1] is ft.amps:
            return
        amps = np.ascontiguousarray(ft.amps, dtype=np.complex64)
        st = self.lib.cs_set_spectrum(self._h, amps.ctypes.data, len(amps), int(ft.N), float(ft.inf.dt))
        _lib.check(st, self._h, "cs_set_spectrum")
        self._spec_key = ("file",)
        self._spec_keep = (ft, ft.amps)

    def set_spectrum_host(self, ptr: int, namps: int, N: int, dt: float):
        """Copy a spectrum from host memory at ``ptr`` (cs_set_spectrum).  From
        pinned memory the copy overlaps the next search, so the buffer must stay
        unchanged until that search has returned."""
        st = self.lib.cs_set_spectrum(self._h, ctypes.c_void_p(ptr), int(namps), int(N), float(dt))
        _lib.check(st, self._h, "cs_set_spectrum")
        self._spec_key = ("host", ptr, namps, N)

    def set_spectrum_device(self, ptr: int, namps: int, N: int, dt: float, keep=None):
        """Attach a spectrum already resident on the device (no copy)."""
        st = self.lib.cs_set_spectrum_device(self._h, ctypes.c_void_p(ptr), int(namps), int(N), float(dt))
        _lib.check(st, self._h, "cs_set_spectrum_device")
        self._spec_key = ("device", ptr, namps, N)
        self._spec_keep = keep

    # -- calls ------------------------------------------------------------
    def search_raw(self, lofreq=0.1, hifreq=100.0, lobin=100, blocksize=2048, threshold=None,
                   exact_all=False, cap=1 << 16, blocks=None) -> np.ndarray:
        """Raw detections of the band (cs_search), or of the block range
        `blocks = (begin, end)` of the band's grid (cs_search_range)."""
        thr = self.params.threshold if threshold is None else threshold
        while True:
            # one reusable output array per engine: no per-call zero fill
            if getattr(self, "_cand_buf", None) is None or len(self._cand_buf) < cap:
                self._cand_buf = np.empty(cap, dtype=_lib.CAND_DTYPE)
            out = self._cand_buf
            n = ctypes.c_int64()
            if blocks is None:
                st = self.lib.cs_search(self._h, float(lofreq), float(hifreq), int(lobin), int(blocksize),
                                        float(thr), int(bool(exact_all)), out.ctypes.data, cap,
                                        ctypes.byref(n))
            else:
                st = self.lib.cs_search_range(self._h, float(lofreq), float(hifreq), int(lobin), int(blocksize),
                                              float(thr), int(bool(exact_all)), int(blocks[0]), int(blocks[1]),
                                              out.ctypes.data, cap, ctypes.byref(n))
            if st == _lib.CS_ERR_CAPACITY and n.value > cap:
                cap = int(n.value)
                continue
            _lib.check(st, self._h, "cs_search")
            return out[:n.value].copy()

    def set_batch_graph(self, enable: bool = True):
        """Replay a captured CUDA graph for repeated batches of device spectra
        (cs_set_batch_graph); the engine's stream must not be the legacy
        default stream."""
        _lib.check(self.lib.cs_set_batch_graph(self._h, int(bool(enable))), self._h, "cs_set_batch_graph")

    def search_blocks_raw(self, block_list, lofreq=0.1, hifreq=100.0, lobin=100, blocksize=2048, threshold=None,
                          cap=1 << 16) -> np.ndarray:
        """Raw detections of the listed blocks of the band's grid only
        (cs_search_blocks): each block exactly as in the whole search."""
        thr = self.params.threshold if threshold is None else threshold
        bl = np.ascontiguousarray(np.unique(np.asarray(block_list, np.int64)))
        while True:
            out = np.empty(cap, dtype=_lib.CAND_DTYPE)
            n = ctypes.c_int64()
            st = self.lib.cs_search_blocks(self._h, float(lofreq), float(hifreq), int(lobin), int(blocksize),
                                           float(thr), bl.ctypes.data, len(bl), out.ctypes.data, cap,
                                           ctypes.byref(n))
            if st == _lib.CS_ERR_CAPACITY and n.value > cap:
                cap = int(n.value)
                continue
            _lib.check(st, self._h, "cs_search_blocks")
            return out[:n.value].copy()

    def block_features(self, lofreq=0.1, hifreq=100.0, lobin=100, blocksize=2048):
        """Incoherent power-sum features of every block of the band
        (cs_block_features): a float32 CUDA tensor [nblocks, sum of Hk]."""
        import torch
        n, nf = ctypes.c_int64(), ctypes.c_int32()
        self.lib.cs_block_features(self._h, float(lofreq), float(hifreq), int(lobin), int(blocksize), None, 0,
                                   ctypes.byref(n), ctypes.byref(nf))
        out = torch.empty((max(1, n.value), nf.value), dtype=torch.float32, device=f"cuda:{self.device}")
        _lib.check(self.lib.cs_block_features(self._h, float(lofreq), float(hifreq), int(lobin), int(blocksize),
                                              out.data_ptr(), n.value, ctypes.byref(n), ctypes.byref(nf)), self._h,
                   "cs_block_features")
        return out[:n.value]

    def search_batch_raw(self, spectra, lofreq=0.1, hifreq=100.0, lobin=100, blocksize=2048, threshold=None,
                         on_device=False, cap=1 << 18):
        """cs_search_batch over `spectra`, a list of (amps, N, dt): amps a
        complex64 host array (pinned for full copy/compute overlap) or, with
        on_device, an integer device address.  Returns (candidates, file index)."""
        thr = self.params.threshold if threshold is None else threshold
        self._spec_key = None   # the batch replaces the handle's attached spectrum
        arr = (_lib.cs_spectrum * max(1, len(spectra)))()
        keep = []
        for i, (a, N, dt) in enumerate(spectra):
            if on_device:
                ptr, namps = int(a[0]), int(a[1])
            else:
                a = np.ascontiguousarray(a, dtype=np.complex64)
                keep.append(a)
                ptr, namps = a.ctypes.data, a.size
            arr[i] = _lib.cs_spectrum(ptr, namps, int(N), float(dt))
        while True:
            out = np.empty(cap, dtype=_lib.CAND_DTYPE)
            owner = np.empty(cap, dtype=np.int32)
            n = ctypes.c_int64()
            st = self.lib.cs_search_batch(self._h, arr, len(spectra), int(bool(on_device)), float(lofreq),
                                          float(hifreq), int(lobin), int(blocksize), float(thr), out.ctypes.data,
                                          owner.ctypes.data, cap, ctypes.byref(n))
            if st == _lib.CS_ERR_CAPACITY and n.value > cap:
                cap = int(n.value)
                continue
            _lib.check(st, self._h, "cs_search_batch")
            return out[:n.value].copy(), owner[:n.value].copy()

    def stats(self) -> dict:
        s = _lib.cs_stats()
        _lib.check(self.lib.cs_search_stats(self._h, ctypes.byref(s)), self._h, "cs_search_stats")
        return {n: getattr(s, n) for n, _ in s._fields_}

    def block_values(self):
        n = ctypes.c_int64()
        self.lib.cs_search_block_values(self._h, None, None, 0, ctypes.byref(n))
        sig = np.zeros(n.value, np.float32)
        nv = np.zeros(n.value, np.int32)
        _lib.check(self.lib.cs_search_block_values(self._h, sig.ctypes.data, nv.ctypes.data, n.value,
                                                   ctypes.byref(n)), self._h)
        return sig, nv

    def autotune(self, lofreq=0.1, hifreq=100.0, lobin=100, blocksize=2048, nsample=256) -> dict:
        """Time the launch-shape candidates on `nsample` blocks from the middle
        of the band (cs_autotune) and keep the fastest: the interpolation
        kernel, and in the tensor modes the epilogue segment size per profile
        bin count and the base level's TMEM double buffer.  Returns what was
        chosen and measured."""
        r = _lib.cs_tune_report()
        _lib.check(self.lib.cs_autotune(self._h, float(lofreq), float(hifreq), int(lobin), int(blocksize),
                                        int(nsample), ctypes.byref(r)), self._h, "cs_autotune")
        n = r.nlev
        return {"interp_kernel": "persistent" if r.interp_kernel else "per-item",
                "sigma_kernel": "256 threads, twiddles via L1" if r.sigma_kernel else "384 threads, twiddles in smem",
                "ms_sigma": list(r.ms_sigma),
                "tc_double_buffer": int(r.tc_double_buffer), "tc_div": list(r.tc_div),
                "units_per_level": {int(r.nbins[i]): int(r.units[i]) for i in range(n)},
                "ms_interp": {"per-item": r.ms_interp[0], "persistent": r.ms_interp[1]},
                "ms_synth_model": r.ms_synth_model, "ms_synth_tuned": r.ms_synth_tuned,
                "sample_blocks": int(r.sample_blocks)}

    def set_launch_shapes(self, interp_kernel=0, sigma_kernel=0, tc_double_buffer=1, tc_div=(0, 0)):
        """Pin the launch shapes (cs_set_launch_shapes): interpolation kernel 0
        (one CTA per item) or 1 (persistent), block-sigma kernel 0 (384 threads)
        or 1 (256), the base level's TMEM double buffer, and the epilogue
        segment divisor per phase (0: cost model)."""
        r = _lib.cs_tune_report()
        r.interp_kernel, r.sigma_kernel, r.tc_double_buffer = int(interp_kernel), int(sigma_kernel), int(tc_double_buffer)
        r.tc_div[0], r.tc_div[1] = int(tc_div[0]), int(tc_div[1])
        _lib.check(self.lib.cs_set_launch_shapes(self._h, ctypes.byref(r)), self._h, "cs_set_launch_shapes")

    def set_memory_limit(self, nbytes: int):
        """Cap the device memory the engine holds (0: no cap); searches split
        into waves under it, or raise CohSearchError(CS_ERR_OUT_OF_MEMORY)."""
        _lib.check(self.lib.cs_set_memory_limit(self._h, int(nbytes)), self._h, "cs_set_memory_limit")

    def set_wait_test(self, wait_ns: int):
        """Test hook of the bounded device waits (cs_set_wait_test): with
        wait_ns > 0 the next searches end in CS_ERR_TIMEOUT after a device wait
        of that length that nothing completes; 0 turns it off."""
        _lib.check(self.lib.cs_set_wait_test(self._h, int(wait_ns)), self._h, "cs_set_wait_test")

    def set_diagnostics(self, level: int):
        _lib.check(self.lib.cs_set_diagnostics(self._h, int(level)), self._h, "cs_set_diagnostics")

    def gate_values(self):
        n = ctypes.c_int64()
        self.lib.cs_search_gate_values(self._h, None, 0, ctypes.byref(n))
        out = np.zeros(n.value, np.float32)
        _lib.check(self.lib.cs_search_gate_values(self._h, out.ctypes.data, n.value, ctypes.byref(n)), self._h)
        return out

    def trial_metrics(self):
        n = ctypes.c_int64()
        self.lib.cs_search_trial_metrics(self._h, None, 0, ctypes.byref(n))
        out = np.zeros(n.value, np.float32)
        _lib.check(self.lib.cs_search_trial_metrics(self._h, out.ctypes.data, n.value, ctypes.byref(n)),
                   self._h)
        return out

    # -- metric statistics and normalisation (src/search.jl:1296-1643) --------------

    def set_metricstats(self, ms):
        """Collect `ms` (a MetricStats) in the following searches, or stop (None)."""
        if ms is None:
            st = self.lib.cs_set_metricstats(self._h, 0, 0.0, 1.0, 1, 1)
        else:
            st = self.lib.cs_set_metricstats(self._h, 1, float(ms.hist_lo), float(ms.hist_hi), int(ms.hist_nb),
                                             int(ms.nwin))
        _lib.check(st, self._h, "cs_set_metricstats")

    def fetch_metricstats(self, ms):
        """Append the last search's statistics to `ms`, as _search_region! does
        (src/search.jl:1870-1889): blocks by (block, k), per-(k, window)
        histograms and their per-k merges, sorted by k."""
        from .metricstats import BlockMetricStats, MetricHistogram, merge_hists
        n = ctypes.c_int64()
        self.lib.cs_get_block_stats(self._h, None, 0, ctypes.byref(n))
        recs = (_lib.cs_block_stats * max(1, n.value))()
        _lib.check(self.lib.cs_get_block_stats(self._h, recs, n.value, ctypes.byref(n)), self._h,
                   "cs_get_block_stats")
        for r in recs[:n.value]:
            ms.blocks.append(BlockMetricStats(int(r.block), int(r.k), int(r.Hk), int(r.nbins), r.ngoodbins, r.flo,
                                              r.fhi, int(r.n), r.min, r.median, r.mean, r.std, r.max))
        L, W, B = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        _lib.check(self.lib.cs_get_metric_hists(self._h, ctypes.byref(L), ctypes.byref(W), ctypes.byref(B), None,
                                                None, None, None), self._h, "cs_get_metric_hists")
        L, W, B = L.value, W.value, B.value
        if L == 0:
            return ms
        ks = np.zeros(L, np.int32)
        edges = np.zeros((L, W + 1))
        counts = np.zeros((L, W, B), np.int64)
        mom = np.zeros((L, W, 7))
        _lib.check(self.lib.cs_get_metric_hists(self._h, ctypes.byref(ctypes.c_int32(L)),
                                                ctypes.byref(ctypes.c_int32(W)), ctypes.byref(ctypes.c_int32(B)),
                                                ks.ctypes.data, edges.ctypes.data, counts.ctypes.data,
                                                mom.ctypes.data), self._h, "cs_get_metric_hists")
        for i in range(L):
            k = int(ks[i])
            Hk = self.params.nharms // k
            wins = []
            for w in range(W):
                m = mom[i, w]
                wins.append(MetricHistogram(k, Hk, 2 * Hk, w + 1, float(edges[i, w]), float(edges[i, w + 1]),
                                            float(ms.hist_lo), float(ms.hist_hi),
                                            ms.hist_nb / (ms.hist_hi - ms.hist_lo), counts[i, w].copy(),
                                            int(m[0]), int(m[1]), int(m[2]), float(m[3]), float(m[4]),
                                            float(m[5]), float(m[6])))
            ms.whists.extend(wins)
            ms.hists.append(merge_hists(wins, 0, float(edges[i, 0]), float(edges[i, W])))
        ms.hists.sort(key=lambda h: h.k)
        ms.whists.sort(key=lambda h: (h.k, h.win))
        return ms

    def set_metricnorm(self, norm):
        """Normalise the following searches' candidate test with `norm` (a
        MetricNorm), or stop (None)."""
        if norm is None:
            _lib.check(self.lib.cs_set_metricnorm(self._h, 0, 0, None, None, None, None), self._h,
                       "cs_set_metricnorm")
            return
        ks = sorted(norm.edges)
        W = len(norm.edges[ks[0]]) - 1
        kk = np.array(ks, np.int32)
        e = np.array([norm.edges[k] for k in ks], np.float64)
        lc = np.array([norm.loc[k] for k in ks], np.float64)
        sc = np.array([norm.scale[k] for k in ks], np.float64)
        _lib.check(self.lib.cs_set_metricnorm(self._h, len(ks), W, kk.ctypes.data, e.ctypes.data, lc.ctypes.data,
                                              sc.ctypes.data), self._h, "cs_set_metricnorm")

    def block_metrics(self, rfund, kernel: str = "fft", widths=None) -> np.ndarray:
        """block_metrics (src/search.jl:1061-1079) on the device, FP64."""
        if kernel not in ("fft", "direct"):
            raise ValueError(f"kernel must be :fft or :direct, got :{kernel}")
        r = np.ascontiguousarray(rfund, dtype=np.float64)
        if r.size == 0:
            return np.zeros(0)
        out = np.zeros(r.size, np.float64)
        w = None if widths is None else np.ascontiguousarray(widths, dtype=np.int32)
        _lib.check(self.lib.cs_block_metrics(self._h, r.ctypes.data, r.size, 0 if kernel == "fft" else 1,
                                             None if w is None else w.ctypes.data, 0 if w is None else w.size,
                                             out.ctypes.data), self._h, "cs_block_metrics")
        return out

    def refold(self, r, nharm, m: int = 64):
        """cs_refold: (H, profiles as a list of arrays, ducy) for candidates at
        fundamentals r with nharm requested harmonics each."""
        r = np.ascontiguousarray(r, dtype=np.float64)
        nh = np.ascontiguousarray(np.broadcast_to(nharm, r.shape), dtype=np.int32)
        n = r.size
        H = np.zeros(n, np.int32)
        prof = np.zeros((max(n, 1), 1024), np.float64)
        ducy = np.zeros(n, np.float64)
        if n:
            _lib.check(self.lib.cs_refold(self._h, r.ctypes.data, nh.ctypes.data, n, int(m), H.ctypes.data,
                                          prof.ctypes.data, ducy.ctypes.data), self._h, "cs_refold")
        profs = [prof[i, :2 * H[i]].copy() if H[i] >= 1 else np.zeros(2) for i in range(n)]
        return H, profs, ducy

    def chunk_metrics(self, rstart: float, n: int) -> np.ndarray:
        out = np.zeros(int(n), np.float64)
        _lib.check(self.lib.cs_chunk_metrics(self._h, float(rstart), int(n), out.ctypes.data), self._h,
                   "cs_chunk_metrics")
        return out

    def interp_chunk(self, r_lo: float, t0: int, n: int) -> np.ndarray:
        out = np.zeros((self.params.nharms, int(n)), np.complex64)
        _lib.check(self.lib.cs_interp_chunk(self._h, float(r_lo), int(t0), int(n), out.ctypes.data),
                   self._h, "cs_interp_chunk")
        return out


class SearchCache:
    """Reusable per-``SearchParams`` device engine (src/search.jl:1914-1961).

    Reuse is keyed on the ``params`` object identity, as in the reference.
    """

    def __init__(self):
        self.params = None
        self.engine: Optional[Engine] = None

    def engine_for(self, params: SearchParams, device: int = 0) -> Engine:
        if self.engine is None or self.params is not params or self.engine.device != device:
            if self.engine is not None:
                self.engine.close()
            self.engine = Engine(params, device)
            self.params = params
        return self.engine


def _to_candidates(raw: np.ndarray) -> List[Candidate]:
    return [Candidate(float(c["freq"]), float(c["metric"]), float(c["r"]), int(c["nharm"]),
                      math.nan, int(c["k"]), int(c["trial"])) for c in raw]


def search(ft, params: SearchParams = None, lofreq=0.1, hifreq=100.0, lobin=100, blocksize=2048,
           threshold=None, remove=True, dr_tol=1.0, harm_remove=True, numharm=16, harm_tol=1.0,
           progress="none", metricstats=None, normalize=False, verbose=False, wisdom=True,
           wisdom_file=None, cache: Optional[SearchCache] = None, device: int = 0) -> List[Candidate]:
    """Coherent harmonic-summing search over ``[lofreq, hifreq]`` Hz
    (src/search.jl:2002-2111) on the device.

    ``wisdom``/``wisdom_file`` are accepted for compatibility; no FFTW plans
    exist on the device path.  ``metricstats`` (a MetricStats) is filled from
    the search's exact pass; ``normalize`` runs the reference's two passes
    (src/search.jl:2063-2094): measure the per-(k, window) noise, build the
    MetricNorm, then detect on the normalised metric.
    """
    from .metricstats import MetricStats, build_metricnorm
    params = SearchParams() if params is None else params
    if progress not in ("none", "text", "bar"):
        raise ValueError(f"progress must be :none, :text or :bar, got :{progress}")
    thr = params.threshold if threshold is None else threshold
    eng = cache.engine_for(params, device) if cache is not None else Engine(params, device)
    eng.set_spectrum(ft)
    try:
        if normalize:
            normstats = MetricStats() if metricstats is None else metricstats
            eng.set_metricstats(normstats)
            eng.search_raw(lofreq, hifreq, lobin, blocksize, math.inf)
            eng.fetch_metricstats(normstats)
            eng.set_metricstats(None)
            eng.set_metricnorm(build_metricnorm(normstats))
            raw = eng.search_raw(lofreq, hifreq, lobin, blocksize, thr)
        elif metricstats is not None:
            eng.set_metricstats(metricstats)
            raw = eng.search_raw(lofreq, hifreq, lobin, blocksize, thr)
            eng.fetch_metricstats(metricstats)
        else:
            raw = eng.search_raw(lofreq, hifreq, lobin, blocksize, thr)
    finally:
        eng.set_metricstats(None)
        eng.set_metricnorm(None)
    cands = _to_candidates(raw)
    if remove:
        cands = remove_duplicates(cands, dr_tol)
    else:
        cands = sorted(cands, key=lambda c: c.freq)
    if harm_remove:
        cands = remove_harmonics(cands, numharm, harm_tol)
    return cands


def output_path(fftfile: str, outputfilenm: str = "", outdir: str = "", nfiles: int = 1) -> str:
    """Where one file's candidates go (output_path, src/cli.jl:263-270): a lone
    file with neither an output name nor an output directory writes to stdout
    (''); otherwise ``<fftfile without .fft>.cohout``, beside the input or in
    ``outdir``."""
    import os
    if nfiles == 1 and not outdir:
        return outputfilenm
    stem = os.path.splitext(fftfile)[0]
    if outdir:
        stem = os.path.join(outdir, os.path.basename(stem))
    return stem + ".cohout"


def search_files(fftfiles: Sequence[str], params: SearchParams = None, lofreq=0.1, hifreq=100.0, lobin=100,
                 blocksize=2048, threshold=None, ncands=100, outputfilenm: str = "", outdir: str = "",
                 remove=True, dr_tol=1.0, harm_remove=True, numharm=16, harm_tol=1.0, measure=True,
                 device: int = 0) -> List[List[Candidate]]:
    """The per-file loop of the reference's command line (src/cli.jl:237-246
    with search_one, :279-306): each ``.fft`` opened (FFTFile), searched with
    one shared SearchCache, its strongest ``ncands`` candidates (best metric
    first) refolded for their duty cycle and written to ``output_path``.  An
    output name with several files raises ValueError, as the reference's
    ArgumentError.  Returns each file's reported candidates."""
    import os
    from .fileio import FFTFile
    nfiles = len(fftfiles)
    if nfiles > 1 and outputfilenm:
        raise ValueError(f"an output file name names one output but {nfiles} FFT files were given; omit it "
                         "(each file gets its own .cohout) or give an output directory")
    if outdir:
        os.makedirs(outdir, exist_ok=True)
    params = SearchParams() if params is None else params
    thr = params.threshold if threshold is None else threshold
    cache = SearchCache()
    out = []
    for path in fftfiles:
        ft = FFTFile(path)
        cands = search(ft, params, lofreq=lofreq, hifreq=hifreq, lobin=lobin, blocksize=blocksize, threshold=thr,
                       remove=remove, dr_tol=dr_tol, harm_remove=harm_remove, numharm=numharm,
                       harm_tol=harm_tol, cache=cache, device=device)
        cands = sorted(cands, key=lambda c: -c.metric)[:ncands]
        if cands and measure:
            cands = measure_ducy(ft, cands, params, cache=cache, device=device)
        write_candidates(cands, output_path(path, outputfilenm, outdir, nfiles), thr)
        out.append(cands)
    return out


def search_batch(fts, params: SearchParams = None, lofreq=0.1, hifreq=100.0, lobin=100, blocksize=2048,
                 threshold=None, remove=True, dr_tol=1.0, harm_remove=True, numharm=16, harm_tol=1.0,
                 cache: Optional[SearchCache] = None, device: int = 0) -> List[List[Candidate]]:
    """`search` over many spectra (a DM sweep) with one device engine: each
    file's candidates, post-processed as `search` does, in file order."""
    params = SearchParams() if params is None else params
    thr = params.threshold if threshold is None else threshold
    eng = cache.engine_for(params, device) if cache is not None else Engine(params, device)
    raw, owner = eng.search_batch_raw([(ft.amps, ft.N, ft.dt) for ft in fts], lofreq, hifreq, lobin,
                                      blocksize, thr)
    res = []
    for i in range(len(fts)):
        cands = _to_candidates(raw[owner == i])
        cands = remove_duplicates(cands, dr_tol) if remove else sorted(cands, key=lambda c: c.freq)
        if harm_remove:
            cands = remove_harmonics(cands, numharm, harm_tol)
        res.append(cands)
    return res


def candidate_profile(ft, r: float, nharm: int, m: int = 64, params: SearchParams = None,
                      cache=None, device: int = 0) -> np.ndarray:
    """candidate_profile (src/candidate.jl:37-61) on the device: the 2H-bin
    coherent-fold profile of fundamental `r`, not rotated."""
    if nharm < 1:
        raise ValueError("nharm must be >= 1")
    if m % 2:
        raise ValueError("m must be even")
    params = SearchParams() if params is None else params
    eng = cache.engine_for(params, device) if cache is not None else Engine(params, device)
    eng.set_spectrum(ft)
    H, profs, _ = eng.refold([r], [nharm], m)
    return profs[0]


def measure_ducy(ft, cands: Sequence[Candidate], params: SearchParams, m: int = 64, cache=None,
                 device: int = 0) -> List[Candidate]:
    """measure_ducy (src/candidate.jl:63-99): each candidate refolded at its own
    r with its own nharm on the device; ducy = best boxcar width / bins."""
    eng = cache.engine_for(params, device) if cache is not None else Engine(params, device)
    eng.set_spectrum(ft)
    if not cands:
        return []
    _, _, ducy = eng.refold([c.r for c in cands], [c.nharm for c in cands], m)
    return [Candidate(c.freq, c.metric, c.r, c.nharm, float(d), c.k, c.trial) for c, d in zip(cands, ducy)]


def rotate_to_peak(prof) -> np.ndarray:
    """rotate_to_peak (src/candidate.jl:101-110): the maximum bin moved to phase 0.5."""
    prof = np.asarray(prof, dtype=np.float64)
    n = len(prof)
    if n == 0:
        return prof
    return np.roll(prof, n // 2 - int(np.argmax(prof)))


def block_metrics(ft, rfund, params: SearchParams, kernel="fft", widths=None, cache=None,
                  device: int = 0) -> np.ndarray:
    """Coherent-fold S/N of every trial fundamental in `rfund` through the
    reference path (src/search.jl:1061-1079), on the device."""
    eng = cache.engine_for(params, device) if cache is not None else Engine(params, device)
    eng.set_spectrum(ft)
    return eng.block_metrics(rfund, kernel, widths)


def search_block(ft, rfund, params: SearchParams, threshold=None, cache=None, device: int = 0) -> List[Candidate]:
    """search_block (src/search.jl:1087-1097): trials of `rfund` above threshold."""
    thr = params.threshold if threshold is None else threshold
    met = block_metrics(ft, rfund, params, cache=cache, device=device)
    return [Candidate(float(rfund[j]) / ft.T, float(met[j]), float(rfund[j]), params.nharms)
            for j in range(len(rfund)) if met[j] > thr]


def chunk_metrics(ft, params: SearchParams, rstart: float, n: int, lodr=None, cache=None,
                  device: int = 0) -> np.ndarray:
    """Equivalence bridge (src/search.jl:1740-1755) on the device."""
    if lodr is not None and lodr != params.hidr / params.nharms:
        raise ValueError("lodr must equal hidr/nharms")
    eng = cache.engine_for(params, device) if cache is not None else Engine(params, device)
    eng.set_spectrum(ft)
    return eng.chunk_metrics(rstart, n)
