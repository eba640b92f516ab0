"""The drop-in host surface over the device engine, as the reference tests it:
PRESTO files searched from disk, SearchCache reuse, the multi-file .cohout
output, and a truncated spectrum against the oracle.

  * SearchCache reuse (test/test_cli.jl:65-85): fresh, cached, reused and
    reopened-file runs give the same candidates bit for bit;
  * multi-file run (test/test_cli.jl:179-221): one .cohout per input, each with
    its own candidates and a measured duty cycle in every row;
  * a .fft holding fewer than N/2 amplitudes: the range guard uses the file's
    end (src/directinterp.jl:490-496), checked against the C port of the
    reference search (same tolerances as test_gpu_configs).
"""
import os

import numpy as np
import pytest

import cohsearch as cs
from oracle import cs_cpu
from tests.test_fileio_host import _synthetic

pytestmark = pytest.mark.gpu


def _write(tmp_path, name, bin0=210, N=1 << 15, dt=1.0e-4):
    return cs.write_fft(str(tmp_path / name), _synthetic(N, bin0), N, dt), N * dt


def test_search_cache_reuse_leaves_results_unchanged(tmp_path):
    path, T = _write(tmp_path, "synth")
    ft = cs.FFTFile(path)
    params = cs.SearchParams(nharms=8)
    kw = dict(lofreq=200 / T, hifreq=240 / T, blocksize=64, threshold=0.0)
    fresh = cs.search(ft, params, **kw)
    assert fresh
    cache = cs.SearchCache()
    first = cs.search(ft, params, cache=cache, **kw)
    eng = cache.engine
    second = cs.search(ft, params, cache=cache, **kw)      # the reuse path
    assert cache.engine is eng
    for got in (first, second):
        assert len(got) == len(fresh)
        assert all(c.r == f.r and c.metric == f.metric and c.nharm == f.nharm for c, f in zip(got, fresh))
    reopened = cs.search(cs.FFTFile(path), params, cache=cache, **kw)
    assert [c.metric for c in reopened] == [c.metric for c in fresh]
    # other params rebuild the engine (reuse is keyed on the params object)
    cs.search(ft, cs.SearchParams(nharms=8, hidr=0.25), cache=cache, **kw)
    assert cache.engine is not eng


def test_multi_file_run_writes_one_cohout_per_input(tmp_path):
    p1, T = _write(tmp_path, "obs_DM10.0")
    p2, _ = _write(tmp_path, "obs_DM20.0", bin0=214)
    res = cs.search_files([p1, p2], cs.SearchParams(nharms=8), lofreq=200 / T, hifreq=240 / T, blocksize=64,
                          threshold=0.0, ncands=3)
    o1, o2 = str(tmp_path / "obs_DM10.0.cohout"), str(tmp_path / "obs_DM20.0.cohout")
    assert os.path.isfile(o1) and os.path.isfile(o2)
    l1, l2 = open(o1).read().splitlines(), open(o2).read().splitlines()
    assert len(l1) > 1 and len(l2) > 1 and len(l1) <= 4
    assert l1[0].startswith("#") and "Ducy(%)" in l1[0]
    f1, f2 = float(l1[1].split()[2]), float(l2[1].split()[2])
    assert not np.isclose(f1, f2, rtol=1e-3)
    for line in l1[1:] + l2[1:]:
        f = line.split()
        assert len(f) == 6
        assert 0 < float(f[5]) <= 30.0
    # the rows are the returned candidates, strongest first
    assert [c.metric for c in res[0]] == sorted((c.metric for c in res[0]), reverse=True)
    # an output directory relocates them
    od = str(tmp_path / "sub" / "dir")
    cs.search_files([p1], cs.SearchParams(nharms=8), lofreq=200 / T, hifreq=240 / T, blocksize=64,
                    threshold=0.0, ncands=3, outdir=od)
    assert os.path.isfile(os.path.join(od, "obs_DM10.0.cohout"))


def test_truncated_spectrum_vs_port(tmp_path):
    """A spectrum cut at 60 % of N/2: harmonics whose window passes the file's
    end are guarded off, for the device and the port alike."""
    from cohsearch import synth
    from tests.test_gpu_configs import BLOCK, THR, check_against_port
    N, dt = 1 << 21, 64e-6
    full = synth.make_spectrum(N, dt, [synth.Pulsar(21.3, 0.05, 30.0, 0.4), synth.Pulsar(150.7, 0.1, 25.0, 0.1)], 77)
    namps = int(0.6 * (N // 2))
    path = cs.write_fft(str(tmp_path / "cut"), full[:namps], N, dt)
    ft = cs.FFTFile(path)
    assert len(ft.amps) == namps
    dec = cs.decimation_set(32, 4)
    eng = cs.Engine(cs.SearchParams(nharms=32, m=16, decimations=dec, threshold=THR))
    eng.set_diagnostics(1)
    eng.set_spectrum(ft)
    lo, hi = 5.0, 200.0
    dev = eng.search_raw(lo, hi, 100, BLOCK, THR)
    sig, nv = eng.block_values()
    from tests.test_gpu_configs import _band
    _, _, r_lo, total = _band(N, dt, 32, lo, hi)
    port = cs_cpu.search_blocks_ex(np.asarray(ft.amps), N, dt, 32, 16, 0.5, dec, r_lo, total, BLOCK, THR,
                                   os.cpu_count() or 1)
    matched, _ = check_against_port(dev, sig, nv, port, N, dt, 32, lo, hi, len(dec))
    assert matched > 0
    # the 150.7 Hz pulsar's upper harmonics lie past the cut: the row guard
    # zeroes them, yet the fundamental is still found
    assert np.any(np.abs(dev["freq"] - 150.7) < 0.05)


def test_batch_of_fft_files_from_disk(tmp_path):
    """Several PRESTO files of uneven length, opened as memory maps and
    searched as one batch (copies from the maps overlapped with the searches):
    each file's candidates equal its own search's."""
    from cohsearch import synth
    params = cs.SearchParams(nharms=32, m=16, decimations=cs.decimation_set(32, 4), threshold=7.0, synth="fp16")
    fts = []
    for i, nsamp in enumerate([1 << 19, 1 << 20, 1 << 18]):
        amps = synth.make_spectrum(nsamp, 64e-6, [synth.Pulsar(9.0 + 5.0 * i, 0.05, 30.0, 0.3)], 300 + i)
        fts.append(cs.FFTFile(cs.write_fft(str(tmp_path / f"dm{i}"), amps, nsamp, 64e-6)))
    assert all(isinstance(ft.amps, np.memmap) for ft in fts)
    batch = cs.search_batch(fts, params, lofreq=1.0, hifreq=60.0, threshold=7.0)
    for ft, got in zip(fts, batch):
        want = cs.search(ft, params, lofreq=1.0, hifreq=60.0, threshold=7.0)
        assert want and [(c.r, c.metric, c.nharm) for c in got] == [(c.r, c.metric, c.nharm) for c in want]


def test_each_new_spectrum_is_searched():
    """Spectra of one length attached one after another as temporaries (whose
    Python identities can be reused once freed): the engine must search each
    new one, never a previous one."""
    from oracle import cs_cpu as port
    eng = cs.Engine(cs.SearchParams(nharms=16, m=16))
    N, dt = 1 << 16, 1e-3
    for seed in range(24):
        amps = ((np.random.default_rng(seed).standard_normal(N // 2) +
                 1j * np.random.default_rng(seed + 1000).standard_normal(N // 2)) * 0.7).astype(np.complex64)
        eng.set_spectrum(cs.FFTFile.from_array(amps.copy(), N, dt))
        got = eng.interp_chunk(2000.0, 0, 64)
        want = port.interp_chunk(amps, N, 16, 16, 0.5, 2000.0, 0, 64)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), seed
