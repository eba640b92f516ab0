"""Device parity: libcohsearch_cuda.so (through the C ABI) against the oracles.

Tolerances (stated once, used throughout):
  * amplitudes of the rational trial grid: bit-exact against the C oracle
    (same FP32 weights, same FMA chain, unfused complex product);
  * bin ranges, zeroed rows, valid decimated trials, candidate trial indices
    and decimation factors: exact;
  * block sigma: |d sigma| / sigma <= 1e-3 (FP32 profiles vs the FP64 oracle
    can move the median between adjacent order statistics);
  * S/N: |dS/N| <= 1e-3 * S/N (the plain FP32 path's stated tolerance);
  * candidate sets: equal outside the exclusion band |S/N - thr| < 1e-3 * thr.
"""
import math

import numpy as np
import pytest

from oracle import cs_cpu, cs_ref as o
from tests.fixtures import PSR_F, multi_spectrum, noise_spectrum, pulsar_spectrum

pytestmark = pytest.mark.gpu

SNR_RTOL = 1e-3
SIGMA_RTOL = 1e-3
# Tensor-core synthesis feeds only the gate and the sigma samples; its
# operands carry 8 (BF16) or 11 (FP16) significant bits.
TC_SIGMA_RTOL = {"bf16": 1e-2, "fp16": 2e-3}
TC_GATE_TOL = {"bf16": (2e-2, 0.05), "fp16": (4e-3, 0.01)}   # (relative, absolute) on the gate S/N


def _cs():
    import cohsearch
    return cohsearch


def _engine(params, amps, N, dt, diag=1):
    cs = _cs()
    eng = cs.Engine(params)
    eng.set_diagnostics(diag)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    return eng


@pytest.mark.parametrize("nharms,m,r_lo,t0,n", [
    (32, 16, 10010.0, 0, 2048),
    (60, 32, 5000.0, 0, 256),
    (60, 16, 4321.7, 777, 1000),        # fractional r_lo, misaligned chunk
    (32, 16, 123.456, 1_000_003, 37),   # large global trial index
    (60, 16, 3.0, 0, 512),              # low harmonics fall off the bottom of the file
    (32, 8, 524288 / 32 - 20.0, 0, 4096),  # top harmonics run past Nyquist
    (7, 18, 777.77, 12, 300),           # odd nharms, runtime-m kernel
])
def test_interp_bitexact_vs_c_oracle(nharms, m, r_lo, t0, n):
    amps, N, dt = pulsar_spectrum()
    cs = _cs()
    eng = _engine(cs.SearchParams(nharms=nharms, m=m), amps, N, dt)
    got = eng.interp_chunk(r_lo, t0, n)
    want = cs_cpu.interp_chunk(amps, N, nharms, m, 0.5, r_lo, t0, n)
    assert got.shape == want.shape
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_interp_nonrational_grid_fp64_path():
    """A trial step that is no small rational takes the per-trial FP64 path
    (src/directinterp.jl:623-661)."""
    amps, N, dt = pulsar_spectrum()
    cs = _cs()
    hidr = 0.5 * math.pi / 3.0
    eng = _engine(cs.SearchParams(nharms=16, m=16, hidr=hidr), amps, N, dt)
    got = eng.interp_chunk(2000.25, 5, 700)
    want = cs_cpu.interp_chunk(amps, N, 16, 16, hidr, 2000.25, 5, 700)
    scale = np.abs(want).max(axis=1, keepdims=True)
    assert np.array_equal(np.abs(got) == 0, np.abs(want) == 0)
    assert np.max(np.abs(got - want) / scale) < 1e-6


def test_interp_chunk_invariance_on_device():
    """test/test_search.jl:234-276 on the device: identical bits for any chunking."""
    amps, N, dt = pulsar_spectrum()
    cs = _cs()
    eng = _engine(cs.SearchParams(nharms=32, m=32), amps, N, dt)
    big = eng.interp_chunk(10010.0, 0, 384)
    for nsm in (128, 100, 37, 51):
        t0 = 0
        while t0 + nsm <= 384:
            assert np.array_equal(eng.interp_chunk(10010.0, t0, nsm), big[:, t0:t0 + nsm])
            t0 += nsm


@pytest.mark.parametrize("nharms,m,rstart,n", [(32, 32, 10010.0, 256), (60, 16, 5000.0, 2048),
                                               (60, 32, 9950.0 * 1.0, 500)])
def test_chunk_metrics_vs_oracle(nharms, m, rstart, n):
    """chunk_metrics (src/search.jl:1740-1755): device vs the FP64-profile oracle."""
    amps, N, dt = pulsar_spectrum()
    cs = _cs()
    p = cs.SearchParams(nharms=nharms, m=m)
    got = _engine(p, amps, N, dt).chunk_metrics(rstart, n)
    want = o.chunk_metrics(amps, N, o.SearchParams(nharms=nharms, m=m), rstart, n, weights=np.float32)
    assert np.all(np.abs(got - want) <= SNR_RTOL * np.maximum(np.abs(want), 1.0))


def _oracle_run(amps, N, dt, op, band, thr, medcut, blocksize=2048):
    T, lodr, r_lo, r_hi, total, Nprof = o.search_setup(N, dt, op, band[0], band[1], 100, blocksize)
    return o.search_region(amps, N, T, op, r_lo, r_hi, total, Nprof, thr, medcut, keep_blocks=True)


@pytest.mark.parametrize("synth", ["fp32", "bf16", "fp16"])
@pytest.mark.parametrize("maxdecim,band,blocksize", [(4, (1.0, 60.0), 2048), (6, (20.0, 900.0), 1000)])
def test_search_vs_oracle(maxdecim, band, blocksize, synth):
    """The hot loop end to end (src/search.jl:1768-1894): nvalid exact, sigma
    and S/N within tolerance, candidate (trial, k) sets equal outside the band,
    for the plain FP32 and both tensor-core synthesis forms."""
    amps, N, dt = multi_spectrum()
    cs = _cs()
    nh = 32
    thr = 7.0
    dec = cs.decimation_set(nh, maxdecim)
    eng = _engine(cs.SearchParams(nharms=nh, m=16, decimations=dec, threshold=thr, synth=synth), amps, N, dt)
    dev = eng.search_raw(band[0], band[1], 100, blocksize, thr)
    sig, nv = eng.block_values()
    op = o.SearchParams(nharms=nh, m=16, decimations=dec, threshold=thr)
    ref, blocks = _oracle_run(amps, N, dt, op, band, thr, thr - op.boxcar_medmargin, blocksize)
    nlev = len(dec)
    levk = [1] + [k for k in dec if k > 1]
    ref_nv = np.zeros(len(blocks), np.int32)
    ref_sig = np.zeros(len(blocks))
    for b in blocks:
        ref_nv[b.block * nlev + levk.index(b.k)] = b.nvalid
        ref_sig[b.block * nlev + levk.index(b.k)] = b.sigma
    assert np.array_equal(nv, ref_nv)
    ok = ref_sig > 0
    srtol = SIGMA_RTOL if synth == "fp32" else TC_SIGMA_RTOL[synth]
    assert np.all(np.abs(sig[ok] - ref_sig[ok]) <= srtol * ref_sig[ok])
    assert np.all(sig[~ok] == 0)
    dmap = {(int(c["trial"]), int(c["k"])): c for c in dev}
    rmap = {(blk * blocksize + j, k): c for (blk, k, j, c) in ref}
    band_hi = thr * (1 + 1e-3)
    for key, c in rmap.items():
        if key in dmap:
            d = dmap[key]
            assert abs(d["metric"] - c.metric) <= SNR_RTOL * c.metric
            assert d["r"] == c.r and d["freq"] == c.freq and d["nharm"] == c.nharm
        else:
            assert c.metric < band_hi, (key, c.metric)
    for key, d in dmap.items():
        if key not in rmap:
            assert thr < d["metric"] < band_hi, (key, float(d["metric"]))
    # the device list comes back in the single-task reference order
    order = [(int(c["trial"]) // blocksize, levk.index(int(c["k"])), int(c["trial"]) % blocksize) for c in dev]
    assert order == sorted(order)
    assert len(rmap) > 0


def test_exact_all_metrics_vs_oracle():
    """medcut = -Inf scores every trial exactly (metricstats/normalize mode)."""
    amps, N, dt = multi_spectrum()
    cs = _cs()
    nh = 16
    dec = cs.decimation_set(nh, 3)
    eng = _engine(cs.SearchParams(nharms=nh, m=16, decimations=dec), amps, N, dt)
    band = (2.0, 9.0)
    eng.search_raw(band[0], band[1], 100, 2048, 1e9, exact_all=True)
    tm = eng.trial_metrics()
    sig, nv = eng.block_values()
    op = o.SearchParams(nharms=nh, m=16, decimations=dec)
    ref, blocks = _oracle_run(amps, N, dt, op, band, 1e9, -math.inf)
    nlev = len(dec)
    levk = [1] + [k for k in dec if k > 1]
    tm = tm.reshape(-1, nlev, 2048)
    for b in blocks:
        got = tm[b.block, levk.index(b.k), :b.nvalid]
        want = b.metrics[:b.nvalid]
        assert np.all(np.abs(got - want) <= SNR_RTOL * np.maximum(np.abs(want), 1.0))


def test_public_search_detects_the_pulsar():
    """test/test_search.jl:378-385 through the public host API."""
    amps, N, dt = pulsar_spectrum()
    cs = _cs()
    ft = cs.FFTFile.from_array(amps, N, dt)
    p = cs.SearchParams(nharms=32, m=32)
    cands = cs.search(ft, p, lofreq=9.5, hifreq=10.5, threshold=8.0)
    assert cands
    best = max(cands, key=lambda c: c.metric)
    assert abs(best.freq - PSR_F) < 1e-2
    raw = cs.search(ft, p, lofreq=9.5, hifreq=10.5, threshold=8.0, remove=False, harm_remove=False)
    assert len(cands) < len(raw)


def test_device_gate_does_not_change_candidates():
    """test/test_search.jl:287-309 on the device."""
    amps, N, dt = pulsar_spectrum()
    cs = _cs()
    ft = cs.FFTFile.from_array(amps, N, dt)
    kw = dict(lofreq=9.5, hifreq=10.5, threshold=6.0, blocksize=512)
    g = cs.search(ft, cs.SearchParams(nharms=60, m=32, decimations=cs.decimation_set(60, 4)), **kw)
    e = cs.search(ft, cs.SearchParams(nharms=60, m=32, decimations=cs.decimation_set(60, 4),
                                      boxcar_medmargin=math.inf), **kw)
    assert len(g) == len(e) and g
    assert all(a.freq == b.freq and a.nharm == b.nharm and a.metric == b.metric for a, b in zip(g, e))


def test_pure_noise_has_no_candidates_above_8():
    amps, N, dt = noise_spectrum()
    cs = _cs()
    ft = cs.FFTFile.from_array(amps, N, dt)
    c = cs.search(ft, cs.SearchParams(nharms=32, decimations=cs.decimation_set(32, 4)), lofreq=1.0,
                  hifreq=200.0, threshold=8.0)
    assert c == []


def test_error_behaviour():
    cs = _cs()
    with pytest.raises(ValueError):
        cs.Engine(cs.SearchParams(m=15))
    eng = cs.Engine(cs.SearchParams(nharms=8))
    with pytest.raises(cs.CohSearchError) as ei:
        eng.search_raw(1.0, 2.0)
    assert ei.value.status == 2
    amps, N, dt = noise_spectrum()
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    assert len(eng.search_raw(5.0, 4.0)) == 0          # empty band: no trials
    with pytest.raises(ValueError):
        eng.chunk_metrics(100.0, 0)


@pytest.mark.parametrize("synth", ["bf16", "fp16"])
def test_tensor_gate_tracks_fp32_gate(synth):
    """The tcgen05 product reproduces the FP32 synthesis' gate values to its
    operand precision, for every level of a full decimation ladder."""
    amps, N, dt = multi_spectrum()
    cs = _cs()
    dec = cs.decimation_set(60, 6)
    band = (0.5, 40.0)
    res = {}
    for mode in ("fp32", synth):
        eng = _engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth=mode), amps, N, dt, diag=2)
        eng.search_raw(band[0], band[1], 100, 2048, 8.0)
        res[mode] = (eng.gate_values(), eng.block_values())
    g32, gtc = res["fp32"][0], res[synth][0]
    rel, ab = TC_GATE_TOL[synth]
    assert g32.shape == gtc.shape and np.any(g32 != 0)
    assert np.all(np.abs(gtc - g32) <= rel * np.abs(g32) + ab)


@pytest.mark.parametrize("synth", ["bf16", "fp16", "bf16_split", "fp16_split"])
def test_tensor_candidates_identical_to_plain(synth):
    """Every trial near the threshold is rescored by the same exact FP32 path,
    so the mixed form reports exactly the plain form's candidates."""
    amps, N, dt = multi_spectrum()
    cs = _cs()
    dec = cs.decimation_set(60, 6)
    out = {}
    for mode in ("fp32", synth):
        eng = _engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth=mode), amps, N, dt, diag=0)
        out[mode] = eng.search_raw(0.2, 180.0, 100, 2048, 8.0)
    a, b = out["fp32"], out[synth]
    assert len(a) > 0
    assert np.array_equal(a, b)


@pytest.mark.parametrize("synth,ladder", [("fp16", True), ("bf16_split", True), ("fp16", False)])
def test_tensor_gate_skip_keeps_the_flagged_set(synth, ladder):
    """The tensor epilogue skips a warp's full gate scan when a window-energy
    bound puts every trial of the warp below the medcut test.  With the exact
    gate values requested (diagnostics level 2) nothing is skipped; the
    rescanned trial count and the candidates must be the same either way, on
    the decimation ladder's widths and on the plain geometric width bank."""
    amps, N, dt = multi_spectrum()
    cs = _cs()
    dec = cs.decimation_set(60, 6) if ladder else [1]
    out = {}
    for diag in (2, 0):
        eng = _engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth=synth), amps, N, dt, diag=diag)
        c = eng.search_raw(0.2, 180.0, 100, 2048, 8.0)
        out[diag] = (c, eng.stats()["rescued"])
    assert out[2][1] > 0 and len(out[2][0]) > 0
    assert out[0][1] == out[2][1]
    assert np.array_equal(out[0][0], out[2][0])


@pytest.mark.parametrize("synth", ["bf16", "fp16", "fp16_split"])
@pytest.mark.parametrize("e", [17, -36])
def test_tensor_bright_spectrum_scale_invariant(synth, e):
    """A spectrum scaled by 2^17 (noise amplitudes ~1e5, past FP16's 65504) or
    by 2^-36 (every component below FP16's smallest subnormal, 2^-24) reports
    exactly the unscaled spectrum's candidates: a power of two scales every
    FP32 value exactly, and the FP16 A tiles carry a power-of-two range scale,
    up or down, taken from the largest component of the spectrum chunks their
    block reads and undone in the gate.  The FP16 gate values themselves scale
    exactly: the tiles of both spectra hold the same 16-bit values."""
    amps, N, dt = multi_spectrum()
    scaled = (amps * np.float32(2.0 ** e)).astype(np.complex64)
    if e > 0:
        assert np.abs(scaled.real).max() > 65504.0
    else:
        assert np.abs(scaled.view(np.float32)).max() < 2.0 ** -24
    cs = _cs()
    dec = cs.decimation_set(60, 6)
    plain = _engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth="fp32"), amps, N, dt, diag=0)
    want = plain.search_raw(0.2, 180.0, 100, 2048, 8.0)
    eng = _engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth=synth), scaled, N, dt, diag=2)
    got = eng.search_raw(0.2, 180.0, 100, 2048, 8.0)
    assert len(want) > 0
    assert np.array_equal(got, want)
    if synth != "bf16":
        ref = _engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth=synth), amps, N, dt, diag=2)
        ref.search_raw(0.2, 180.0, 100, 2048, 8.0)
        g = eng.gate_values() * np.float32(2.0 ** -e)
        assert np.array_equal(g, ref.gate_values(), equal_nan=True)


@pytest.mark.parametrize("synth", ["fp32", "fp16"])
def test_block_ranges_reproduce_the_search(synth):
    """cs_search_range over contiguous block ranges (the multi-GPU shard unit)
    concatenates to exactly the whole search: same records, bit for bit."""
    from cohsearch import parallel
    amps, N, dt = multi_spectrum()
    cs = _cs()
    dec = cs.decimation_set(32, 4)
    eng = _engine(cs.SearchParams(nharms=32, m=16, decimations=dec, threshold=7.0, synth=synth), amps, N, dt)
    whole = eng.search_raw(1.0, 60.0, 100, 2048, 7.0)
    nb = parallel.band_blocks(N, dt, 0.5, 32, 1.0, 60.0, 100, 2048)
    for world in (2, 3):
        parts = [eng.search_raw(1.0, 60.0, 100, 2048, 7.0, blocks=parallel.block_shard(nb, r, world))
                 for r in range(world)]
        assert np.array_equal(np.concatenate(parts), whole)
    assert len(eng.search_raw(1.0, 60.0, 100, 2048, 7.0, blocks=(nb, nb + 5))) == 0


def test_batch_equals_file_by_file_searches():
    """cs_search_batch over spectra of several lengths (host memory, copies
    overlapped with the searches) returns, file by file, exactly the
    candidates of separate cs_search calls."""
    cs = _cs()
    from cohsearch import synth
    files = []
    for i, nsamp in enumerate([1 << 18, 1 << 19, 1 << 18, 1 << 20]):
        dt = 64e-6
        amps = synth.make_spectrum(nsamp, dt, [synth.Pulsar(11.0 + 3.0 * i, 0.05, 40.0, 0.3)], 100 + i)
        files.append((amps, nsamp, dt))
    dec = cs.decimation_set(32, 4)
    params = cs.SearchParams(nharms=32, m=16, decimations=dec, threshold=7.0, synth="fp16")
    eng = cs.Engine(params)
    raw, owner = eng.search_batch_raw(files, 1.0, 60.0, 100, 2048, 7.0)
    st = eng.stats()
    assert st["trials"] > 0
    for i, (amps, N, dt) in enumerate(files):
        single = cs.Engine(params)
        single.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
        want = single.search_raw(1.0, 60.0, 100, 2048, 7.0)
        assert np.array_equal(raw[owner == i], want)
    assert any(len(raw[owner == i]) > 0 for i in range(len(files)))


def test_batch_graph_prefix_overflow_searches_again():
    """A replayed spectrum with more candidates than the captured 4096-record
    prefix is searched again the ordinary way: the records still equal the
    ordinary batch's, replay after replay."""
    import torch
    from cohsearch import synth
    cs = _cs()
    lens = [1 << 18, 1 << 12]
    arrs = [synth.make_spectrum_fd(n, 64e-6, [], 40 + i) for i, n in enumerate(lens)]
    dev = [torch.from_numpy(a.view(np.float32).copy()).cuda() for a in arrs]
    files = [((d.data_ptr(), len(a)), n, 64e-6) for d, a, n in zip(dev, arrs, lens)]
    # the first threshold (noise only) that puts the long spectrum past the prefix
    for thr in (3.0, 2.5, 2.0, 1.5):
        params = cs.SearchParams(nharms=32, m=16, decimations=cs.decimation_set(32, 4), threshold=thr,
                                 synth="fp16")
        ref = cs.Engine(params)
        want, wown = ref.search_batch_raw(files, 1.0, 60.0, 100, 2048, thr, on_device=True)
        if np.bincount(wown, minlength=len(lens))[0] > 4096:
            break
    assert np.bincount(wown, minlength=len(lens))[0] > 4096
    side = torch.cuda.Stream()
    eng = cs.Engine(params)
    eng.set_stream(side.cuda_stream)
    eng.set_batch_graph(True)
    for _ in range(3):
        got, own = eng.search_batch_raw(files, 1.0, 60.0, 100, 2048, thr, on_device=True)
        side.synchronize()
        assert np.array_equal(got, want) and np.array_equal(own, wown)


def test_batch_graph_replays_the_ordinary_batch():
    """cs_set_batch_graph: the batch of device spectra run once the ordinary
    way, captured into one graph and replayed -- the same records as the
    ordinary batch, also after the spectra are refilled in place, and again
    after an unrelated search drops the graph."""
    import torch
    from cohsearch import synth
    cs = _cs()
    rng = np.random.default_rng(12)
    lens = [1 << 20, 1 << 21, 1 << 20]
    def spectra(seed):
        out = []
        for i, n in enumerate(lens):
            ps = synth.random_pulsars(np.random.default_rng(seed + i), 6, 0.5, 200.0, 0.02, 0.2, 8.0, 20.0)
            out.append(synth.make_spectrum_fd(n, 64e-6, ps, seed + i))
        return out
    first = spectra(500)
    dev = [torch.from_numpy(a.view(np.float32).copy()).cuda() for a in first]
    files = [((d.data_ptr(), len(a)), n, 64e-6) for d, a, n in zip(dev, first, lens)]
    params = cs.SearchParams(nharms=32, m=16, decimations=cs.decimation_set(32, 4), synth="fp16")
    side = torch.cuda.Stream()
    ref = cs.Engine(params)
    want, wown = ref.search_batch_raw(files, 1.0, 60.0, 100, 2048, 8.0, on_device=True)
    assert len(want) > 0
    eng = cs.Engine(params)
    eng.set_stream(side.cuda_stream)
    eng.set_batch_graph(True)
    for _ in range(3):                       # capture, then replays
        got, own = eng.search_batch_raw(files, 1.0, 60.0, 100, 2048, 8.0, on_device=True)
        side.synchronize()
        assert np.array_equal(got, want) and np.array_equal(own, wown)
    # refill in place: the replay searches the new contents
    second = spectra(900)
    for d, a in zip(dev, second):
        d.copy_(torch.from_numpy(a.view(np.float32).copy()).cuda())
    torch.cuda.synchronize()
    want2, wown2 = ref.search_batch_raw(files, 1.0, 60.0, 100, 2048, 8.0, on_device=True)
    got2, own2 = eng.search_batch_raw(files, 1.0, 60.0, 100, 2048, 8.0, on_device=True)
    assert np.array_equal(got2, want2) and np.array_equal(own2, wown2)
    # an unrelated search drops the graph; the next batch rebuilds it
    eng.set_spectrum(cs.FFTFile.from_array(second[0], lens[0], 64e-6))
    eng.search_raw(1.0, 60.0, 100, 2048, 8.0)
    got3, own3 = eng.search_batch_raw(files, 1.0, 60.0, 100, 2048, 8.0, on_device=True)
    assert np.array_equal(got3, want2) and np.array_equal(own3, wown2)


def test_batch_graph_of_pinned_host_spectra():
    """cs_set_batch_graph with page-locked host spectra: each file's copy into
    the batch buffer of its parity is captured with the searches (the copy of
    file i+1 under file i's search) and replayed -- the same records as the
    ordinary batch of pageable copies, also after the pinned buffers are
    refilled in place, with every file's bytes counted as copied."""
    import torch
    from cohsearch import synth
    cs = _cs()
    lens = [1 << 20, 1 << 21, 1 << 20, 1 << 19]

    def spectra(seed):
        out = []
        for i, n in enumerate(lens):
            ps = synth.random_pulsars(np.random.default_rng(seed + i), 6, 0.5, 200.0, 0.02, 0.2, 8.0, 20.0)
            out.append(synth.make_spectrum_fd(n, 64e-6, ps, seed + i))
        return out
    first = spectra(700)
    pinned = [torch.from_numpy(a.view(np.float32).copy()).pin_memory() for a in first]
    files = [(p.numpy().view(np.complex64), n, 64e-6) for p, n in zip(pinned, lens)]
    params = cs.SearchParams(nharms=32, m=16, decimations=cs.decimation_set(32, 4), synth="fp16")
    ref = cs.Engine(params)
    want, wown = ref.search_batch_raw([(a, n, 64e-6) for a, n in zip(first, lens)], 1.0, 60.0, 100, 2048, 8.0)
    assert len(want) > 0
    side = torch.cuda.Stream()
    eng = cs.Engine(params)
    eng.set_stream(side.cuda_stream)
    eng.set_batch_graph(True)
    for it in range(3):                      # ordinary run and capture, then replays
        got, own = eng.search_batch_raw(files, 1.0, 60.0, 100, 2048, 8.0)
        side.synchronize()
        assert np.array_equal(got, want) and np.array_equal(own, wown)
        st = eng.stats()
        assert st["h2d_bytes"] >= sum(n // 2 * 8 for n in lens)
        # a replay times no stage (its kernels run inside one graph launch)
        assert (st["ms_interp"] == 0.0) == (it > 0), (it, st["ms_interp"])
    second = spectra(1100)
    for p, a in zip(pinned, second):
        p.copy_(torch.from_numpy(a.view(np.float32).copy()))
    want2, wown2 = ref.search_batch_raw([(a, n, 64e-6) for a, n in zip(second, lens)], 1.0, 60.0, 100, 2048, 8.0)
    got2, own2 = eng.search_batch_raw(files, 1.0, 60.0, 100, 2048, 8.0)
    side.synchronize()
    assert np.array_equal(got2, want2) and np.array_equal(own2, wown2)
