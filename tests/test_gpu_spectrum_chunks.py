"""A host spectrum arrives in chunks of doubling size (cs_set_spectrum): the
first search interpolates each run of blocks as soon as the chunks it reads
have landed, and each block's FP16 tile scale comes from the maxima of those
chunks only.

  * from page-locked memory (copy overlapped with the search) and from pageable
    memory: every record, block sigma and gate value equal to the same search
    of a device-resident copy, for FP16, BF16 and plain FP32 synthesis, on the
    first search (overlapped) and a second one (copy complete);
  * a bright bin in chunk 3: the blocks that read no bin of chunks 3 and up
    keep the gate values of the spectrum without it (their scale ignores those
    chunks), and the FP16 records still equal the plain FP32 form's;
  * the other calls that read the spectrum (block features) wait for the copy.
"""
import numpy as np
import pytest

import cohsearch as cs
from cohsearch import synth
from oracle import cs_ref as o

pytestmark = pytest.mark.gpu

THR = 8.0
BAND = (0.1, 125.0)


def _params(mode, nharms=60):
    return cs.SearchParams(nharms=nharms, m=16, decimations=cs.decimation_set(nharms, 6), synth=mode, threshold=THR)


def chunk_of(x, namps):
    """The chunk holding bin x: chunk 0 is [0, u), chunk c >= 1 is
    [u*2^(c-1), u*2^c), u = max(ceil(namps/32), 65536)."""
    u = max(-(-namps // 32), 1 << 16)
    c = 0
    while min(u << c, namps) <= x and (u << c) < namps:
        c += 1
    return c


def _search(eng):
    got = eng.search_raw(BAND[0], BAND[1], 100, 2048, THR)
    sig, nv = eng.block_values()
    return got, np.asarray(sig).copy(), np.asarray(nv).copy(), eng.gate_values().copy()


@pytest.mark.parametrize("mode", ["fp16", "bf16", "fp32"])
def test_chunked_host_copy_equals_device_resident(mode):
    import torch
    amps, N, dt = synth.survey_config(seed=5)        # 2^22 bins: 6 chunks
    namps = len(amps)
    d = torch.from_numpy(amps.view(np.float32).copy()).cuda()
    pinned = torch.from_numpy(amps.view(np.float32).copy()).pin_memory()
    dev = cs.Engine(_params(mode))
    dev.set_diagnostics(2)
    dev.set_spectrum_device(d.data_ptr(), namps, N, dt, keep=d)
    want = _search(dev)
    launches_dev = dev.stats()["launches"]
    assert len(want[0]) > 0

    eng = cs.Engine(_params(mode))
    eng.set_diagnostics(2)
    eng.set_spectrum_host(pinned.data_ptr(), namps, N, dt)
    first = _search(eng)                              # overlapped with the copy
    assert eng.stats()["launches"] > launches_dev     # interpolation ran run by run
    second = _search(eng)                             # copy complete: one launch
    pageable = cs.Engine(_params(mode))
    pageable.set_diagnostics(2)
    pageable.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    third = _search(pageable)
    for got in (first, second, third):
        assert np.array_equal(got[0], want[0])
        assert np.array_equal(got[1], want[1])
        assert np.array_equal(got[2], want[2])
        assert np.array_equal(got[3].view(np.uint32), want[3].view(np.uint32))


def test_bright_bin_scales_only_the_blocks_past_its_chunk():
    """2^21 samples (chunks [0, 64Ki), [64Ki, 128Ki), ..., [512Ki, 1Mi); the
    band's harmonics reach bin 537 Ki); one bin of chunk 3 set to 2^17 times
    the spectrum's largest component."""
    import torch
    N, dt = 1 << 21, 64e-6
    amps = synth.make_spectrum(N, dt, [synth.Pulsar(7.3, 0.05, 30.0, 0.4), synth.Pulsar(91.1, 0.1, 25.0, 0.1)], 21)
    namps = len(amps)
    assert namps == 1 << 20
    bright = 300_000
    assert chunk_of(bright, namps) == 3 and chunk_of(262_143, namps) == 2
    spike = amps.copy()
    spike[bright] = np.complex64(np.abs(amps.view(np.float32)).max() * 2.0 ** 17)
    res = {}
    for name, a in (("clean", amps), ("spike", spike)):
        for mode in ("fp16", "fp32"):
            eng = cs.Engine(_params(mode, nharms=32))
            eng.set_diagnostics(2)
            h = torch.from_numpy(a.view(np.float32).copy()).pin_memory()
            eng.set_spectrum_host(h.data_ptr(), namps, N, dt)
            res[name, mode] = _search(eng)
    # the FP16 records equal the plain form's, with and without the bright bin
    for name in ("clean", "spike"):
        assert np.array_equal(res[name, "fp16"][0], res[name, "fp32"][0])
    # blocks whose highest bin lies below chunk 3: same gates as without it
    op = o.SearchParams(nharms=32, m=16)
    T, lodr, r_lo, r_hi, total, _ = o.search_setup(N, dt, op, BAND[0], BAND[1], 100, 2048)
    nblk = (total + 2047) // 2048
    last_trial = np.minimum(np.arange(1, nblk + 1) * 2048, total) - 1
    top = np.floor(32 * (r_lo + last_trial * lodr)) + 8 + 4
    early = np.array([chunk_of(int(x), namps) < 3 for x in top])
    assert 0 < early.sum() < nblk
    nlev = len(cs.decimation_set(32, 6))
    g_clean = res["clean", "fp16"][3].reshape(nblk, nlev, 2048)
    g_spike = res["spike", "fp16"][3].reshape(nblk, nlev, 2048)
    assert np.array_equal(g_clean[early].view(np.uint32), g_spike[early].view(np.uint32))
    assert not np.array_equal(g_clean[~early].view(np.uint32), g_spike[~early].view(np.uint32))


def test_features_wait_for_the_chunked_copy():
    import torch
    amps, N, dt = synth.survey_config(seed=6)
    namps = len(amps)
    d = torch.from_numpy(amps.view(np.float32).copy()).cuda()
    dev = cs.Engine(_params("fp16"))
    dev.set_spectrum_device(d.data_ptr(), namps, N, dt, keep=d)
    want = dev.block_features(BAND[0], BAND[1], 100, 2048)
    pinned = torch.from_numpy(amps.view(np.float32).copy()).pin_memory()
    eng = cs.Engine(_params("fp16"))
    eng.set_spectrum_host(pinned.data_ptr(), namps, N, dt)
    got = eng.block_features(BAND[0], BAND[1], 100, 2048)
    assert np.array_equal(got.cpu().numpy(), want.cpu().numpy())


def _pair(seed, nsamp=1 << 22, dt=64e-6):
    """A spectrum with one pulsar, on the device and in pinned host memory."""
    import torch
    amps = synth.make_spectrum(nsamp, dt, [synth.Pulsar(11.0 + seed, 0.05, 25.0, 0.3)], seed)
    d = torch.from_numpy(amps.view(np.float32).copy()).cuda()
    h = torch.from_numpy(amps.view(np.float32).copy()).pin_memory()
    return amps, d, h, nsamp, dt


def test_overlapped_copy_with_waves_block_lists_and_a_new_stream():
    """The first search after a chunked copy splits only its first wave's
    interpolation; later waves, block-list searches, a second spectrum copied
    before any search, and a search on another stream all see the whole copy."""
    import torch
    amps, d, h, N, dt = _pair(1)
    band = (1.0, 60.0)
    dev = cs.Engine(_params("fp16"))
    dev.set_spectrum_device(d.data_ptr(), len(amps), N, dt, keep=d)
    want = dev.search_raw(band[0], band[1], 100, 2048, THR)
    nblk = dev.stats()["blocks"]
    blist = np.arange(3, nblk, 7)
    want_blocks = dev.search_blocks_raw(blist, band[0], band[1], 100, 2048, THR)
    assert len(want) > 0 and len(want_blocks) > 0

    # several waves under a memory cap: the spectrum (16 MiB) and a few blocks
    eng = cs.Engine(_params("fp16"))
    eng.set_memory_limit(len(amps) * 8 + (24 << 20))
    eng.set_spectrum_host(h.data_ptr(), len(amps), N, dt)
    got = eng.search_raw(band[0], band[1], 100, 2048, THR)
    assert eng.stats()["waves"] > 1
    assert np.array_equal(got, want)

    # a block list as the first search after the copy
    eng = cs.Engine(_params("fp16"))
    eng.set_spectrum_host(h.data_ptr(), len(amps), N, dt)
    assert np.array_equal(eng.search_blocks_raw(blist, band[0], band[1], 100, 2048, THR), want_blocks)

    # two copies before any search: the second spectrum is the one searched
    amps2, d2, h2, _, _ = _pair(2)
    dev.set_spectrum_device(d2.data_ptr(), len(amps2), N, dt, keep=d2)
    want2 = dev.search_raw(band[0], band[1], 100, 2048, THR)
    assert not np.array_equal(want2, want)
    eng = cs.Engine(_params("fp16"))
    eng.set_spectrum_host(h.data_ptr(), len(amps), N, dt)
    eng.set_spectrum_host(h2.data_ptr(), len(amps2), N, dt)
    assert np.array_equal(eng.search_raw(band[0], band[1], 100, 2048, THR), want2)

    # the copy issued while the handle used its own stream, the search on another
    side = torch.cuda.Stream()
    eng = cs.Engine(_params("fp16"))
    eng.set_spectrum_host(h.data_ptr(), len(amps), N, dt)
    eng.set_stream(side.cuda_stream)
    assert np.array_equal(eng.search_raw(band[0], band[1], 100, 2048, THR), want)
    side.synchronize()
