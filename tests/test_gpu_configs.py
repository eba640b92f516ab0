"""Parity at the full workloads the engine is measured on: every block of each
band searched on the device (through the C ABI) against the C port of the
reference search (oracle/cs_cpu.c: Float32-weight interpolation, FP64
profiles, block sigma, batched FP32 gate, exact rescan; all host threads).

  * small plain search: 2^21 samples, one 7.3 Hz pulsar, nharms 32, no
    decimation, 1-50 Hz;
  * survey: 2^23 samples, six pulsars, nharms 60, decimation_set(60, 6),
    0.1-125 Hz (the benchmarked step), plain FP32 and FP16 tensor synthesis;
  * DM sweep: one spectrum of each length 2^21 .. 2^24 through the batch entry
    point, from host memory and replayed from a captured CUDA graph;
  * learned proposal: a 2^24-sample spectrum with 200 injections, the blocks a
    trained network proposes, re-searched through cs_search_blocks.

Tolerances, as in test_gpu_parity: valid trial counts exact; block sigma
|d sigma| <= 1e-3 sigma; candidate (trial, k) sets equal outside the exclusion
band |S/N - thr| < 1e-3 thr; S/N |dS/N| <= 1e-3 S/N; every candidate's r and
frequency bit-equal to the reference's FP64 expressions
(src/search.jl:1812, :1833, :1696).
"""
import os

import numpy as np
import pytest

from oracle import cs_cpu, cs_ref as o

pytestmark = pytest.mark.gpu

SNR_RTOL = 1e-3
SIGMA_RTOL = 1e-3
THR = 8.0
BLOCK = 2048
NTHREADS = os.cpu_count() or 1


def _cs():
    import cohsearch
    return cohsearch


def _band(N, dt, nharms, lo, hi):
    op = o.SearchParams(nharms=nharms, m=16)
    T, lodr, r_lo, r_hi, total, _ = o.search_setup(N, dt, op, lo, hi, 100, BLOCK)
    return T, lodr, r_lo, total


def _port(amps, N, dt, nharms, dec, lo, hi, blocks=None):
    T, lodr, r_lo, total = _band(N, dt, nharms, lo, hi)
    return cs_cpu.search_blocks_ex(amps, N, dt, nharms, 16, 0.5, dec, r_lo, total, BLOCK, THR, NTHREADS,
                                   blocks=blocks)


def check_against_port(dev, dsig, dnv, port, N, dt, nharms, lo, hi, nlev):
    """Device records and per-(block, level) values against the port's; returns
    (matched candidates, largest relative S/N difference)."""
    T, lodr, r_lo, _ = _band(N, dt, nharms, lo, hi)
    assert np.array_equal(np.asarray(dnv).reshape(-1, nlev), port["nvalid"])
    psig = port["sigma"]
    dsig = np.asarray(dsig, np.float64).reshape(-1, nlev)
    ok = psig > 0
    assert np.all(np.abs(dsig[ok] - psig[ok]) <= SIGMA_RTOL * psig[ok])
    assert np.all(dsig[~ok] == 0)
    dmap = {(int(c["trial"]), int(c["k"])): c for c in dev}
    rmap = {(int(c["blk"]) * BLOCK + int(c["j"]), int(c["k"])): float(c["metric"]) for c in port["cands"]}
    band_hi = THR * (1 + 1e-3)
    worst, matched = 0.0, 0
    for key, m in rmap.items():
        if key not in dmap:
            assert m < band_hi, (key, m)
            continue
        d = dmap[key]
        worst = max(worst, abs(float(d["metric"]) - m) / m)
        assert abs(float(d["metric"]) - m) <= SNR_RTOL * m, (key, float(d["metric"]), m)
        t, k = key
        i0 = (t // BLOCK) * BLOCK
        rstart = r_lo + float(i0) * lodr
        rf = rstart + float(t - i0) * lodr
        r = rf if k == 1 else float(k) * rf
        assert float(d["r"]) == r and float(d["freq"]) == r / T, key
        assert int(d["nharm"]) == nharms // k
        matched += 1
    for key, d in dmap.items():
        if key not in rmap:
            assert THR < float(d["metric"]) < band_hi, (key, float(d["metric"]))
    return matched, worst


def _engine(params, amps, N, dt, diag=1):
    cs = _cs()
    eng = cs.Engine(params)
    eng.set_diagnostics(diag)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    return eng


def test_small_plain_search_whole_band():
    from cohsearch import synth
    cs = _cs()
    amps, N, dt = synth.small_config()
    eng = _engine(cs.SearchParams(nharms=32, m=16, decimations=[1], threshold=THR), amps, N, dt)
    dev = eng.search_raw(1.0, 50.0, 100, BLOCK, THR)
    sig, nv = eng.block_values()
    port = _port(amps, N, dt, 32, [1], 1.0, 50.0)
    matched, worst = check_against_port(dev, sig, nv, port, N, dt, 32, 1.0, 50.0, 1)
    print(f"\nsmall plain search: {len(dev)} device / {port['ncand']} port candidates, {matched} matched, "
          f"max |dS/N|/S/N {worst:.1e}")
    assert matched > 0
    assert np.any(np.abs(dev["freq"] - 7.3) < 0.01)


@pytest.mark.parametrize("synth_mode", ["fp32", "fp16"])
def test_survey_whole_band(synth_mode):
    """The benchmarked step, every one of its 3,930 blocks and six levels."""
    from cohsearch import synth
    cs = _cs()
    amps, N, dt = synth.survey_config(seed=2)
    dec = cs.decimation_set(60, 6)
    eng = _engine(cs.SearchParams(nharms=60, m=16, decimations=dec, threshold=THR, synth=synth_mode),
                  amps, N, dt)
    dev = eng.search_raw(0.1, 125.0, 100, BLOCK, THR)
    sig, nv = eng.block_values()
    assert len(nv) == 3930 * len(dec)
    port = _port(amps, N, dt, 60, dec, 0.1, 125.0)
    matched, worst = check_against_port(dev, sig, nv, port, N, dt, 60, 0.1, 125.0, len(dec))
    print(f"\nsurvey ({synth_mode}): {len(dev)} device / {port['ncand']} port candidates, {matched} matched, "
          f"max |dS/N|/S/N {worst:.1e}; port {port['seconds']:.1f} s on {NTHREADS} threads")
    assert matched > 100


def test_dmsweep_files_batch_and_graph_replay():
    """One spectrum of each length of the DM sweep, searched as one batch from
    host memory and as a replayed CUDA graph over device copies; each file's
    records against the port's search of that file."""
    import torch
    from cohsearch import synth
    cs = _cs()
    files = synth.dmsweep_config(seed=4, per_length=1)
    dec = cs.decimation_set(60, 6)
    params = cs.SearchParams(nharms=60, m=16, decimations=dec, threshold=THR, synth="fp16")
    eng = cs.Engine(params)
    raw, owner = eng.search_batch_raw(files, 0.1, 125.0, 100, BLOCK, THR)
    side = torch.cuda.Stream()
    geng = cs.Engine(params)
    geng.set_stream(side.cuda_stream)
    geng.set_batch_graph(True)
    dev = [torch.from_numpy(a.view(np.float32).copy()).cuda() for a, _, _ in files]
    on_dev = [((d.data_ptr(), len(a)), N, dt) for d, (a, N, dt) in zip(dev, files)]
    replays = []
    for _ in range(2):   # capture, then a replay
        g, gown = geng.search_batch_raw(on_dev, 0.1, 125.0, 100, BLOCK, THR, on_device=True)
        side.synchronize()
        replays.append((g, gown))
    for i, (amps, N, dt) in enumerate(files):
        one = _engine(params, amps, N, dt)
        single = one.search_raw(0.1, 125.0, 100, BLOCK, THR)
        sig, nv = one.block_values()
        port = _port(amps, N, dt, 60, dec, 0.1, 125.0)
        matched, worst = check_against_port(single, sig, nv, port, N, dt, 60, 0.1, 125.0, len(dec))
        mine = raw[owner == i]
        check_against_port(mine, sig, nv, port, N, dt, 60, 0.1, 125.0, len(dec))
        assert np.array_equal(mine, single)
        for g, gown in replays:
            assert np.array_equal(g[gown == i], single)
        print(f"\nDM-sweep file {N} samples: {len(single)} candidates, {matched} matched the port, "
              f"max |dS/N|/S/N {worst:.1e}")


def test_learned_proposal_blocks_vs_port():
    """The blocks a trained proposal network picks on a 2^24-sample spectrum
    with 200 injections, re-searched by cs_search_blocks, against the port's
    search of exactly those blocks."""
    import torch
    from cohsearch import FFTFile, learned, synth
    cs = _cs()
    nsamp, dt, band = 1 << 24, 64e-6, (0.1, 125.0)
    dec = cs.decimation_set(60, 6)
    eng = cs.Engine(cs.SearchParams(nharms=60, m=16, decimations=dec, threshold=THR, synth="fp16"))
    eng.set_diagnostics(1)

    def spectrum(seed):
        rng = np.random.default_rng(seed)
        ps = synth.random_pulsars(rng, 200, 0.1, 750.0, 0.01, 0.20, 6.0, 20.0)
        return synth.make_spectrum_fd(nsamp, dt, ps, seed)

    xs, ys = [], []
    for seed in range(10_000, 10_004):
        eng.set_spectrum(FFTFile.from_array(spectrum(seed), nsamp, dt))
        X = eng.block_features(band[0], band[1], 100, BLOCK)
        raw = eng.search_raw(band[0], band[1], 100, BLOCK, THR)
        xs.append(X)
        ys.append(torch.from_numpy(learned.block_labels(raw, X.shape[0], BLOCK, THR)))
    Xt, Yt = torch.cat(xs), torch.cat(ys)
    mlp = learned.ProposalMLP(Xt.shape[1], 256, seed=0)
    mlp.fit(Xt, Yt, epochs=6, batch=2048, lr=1e-3)
    tau = learned.choose_threshold(mlp.scores(Xt), Yt.numpy(), 0.995)
    amps = spectrum(30_000)
    eng.set_spectrum(FFTFile.from_array(amps, nsamp, dt))
    res = learned.learned_search(eng, mlp, tau, band[0], band[1], 100, BLOCK, THR)
    sig, nv = eng.block_values()
    assert 0 < len(res.blocks) < res.nblocks
    port = _port(amps, nsamp, dt, 60, dec, band[0], band[1], blocks=res.blocks)
    matched, worst = check_against_port(res.cands, sig, nv, port, nsamp, dt, 60, band[0], band[1], len(dec))
    print(f"\nlearned proposal: {len(res.blocks)} of {res.nblocks} blocks re-searched, {len(res.cands)} "
          f"candidates, {matched} matched the port, max |dS/N|/S/N {worst:.1e}")
    assert matched > 0
