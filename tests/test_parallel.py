"""The multi-rank path on CPU: two ``gloo`` ranks shard one search by contiguous
block ranges and gather their candidates; the union must equal the
single-process search, record for record.  No GPU here, so each rank's block
search is the oracle's C port; the sharding, the band bookkeeping, the
candidate gather and the max-over-ranks timing are the library's own
(``cohsearch.parallel``), as ``bench.py`` and a multi-GPU caller use them."""
import datetime
import math
import os
import socket

import numpy as np
import pytest

from cohsearch import decimation_set, parallel
from tests.fixtures import multi_spectrum

NHARMS, M, HIDR, BLOCK, THR = 32, 16, 0.5, 2048, 7.0
BAND = (1.0, 60.0)


def _band():
    amps, N, dt = multi_spectrum()
    T = N * dt
    lodr = HIDR / NHARMS
    r_lo = BAND[0] * T
    total = int(math.floor((BAND[1] * T - r_lo) / lodr)) + 1
    return amps, N, dt, r_lo, total


def _oracle_blocks(b0, b1):
    from oracle import cs_cpu
    amps, N, dt, r_lo, total = _band()
    dec = decimation_set(NHARMS, 4)
    return cs_cpu.search_blocks(amps, N, dt, NHARMS, M, HIDR, dec, r_lo, total, BLOCK, b0, b1 - b0, THR, 2)


def _sorted(c):
    return np.sort(c, order=["blk", "k", "j"])


def test_block_shards_tile_the_band():
    for nb in (0, 1, 2, 5, 17, 3930):
        for world in (1, 2, 3, 4, 8):
            shards = [parallel.block_shard(nb, r, world) for r in range(world)]
            assert shards[0][0] == 0 and shards[-1][1] == nb
            assert all(shards[r][1] == shards[r + 1][0] for r in range(world - 1))
            sizes = [b - a for a, b in shards]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        parallel.block_shard(10, 2, 2)


def test_band_blocks_matches_search_bookkeeping():
    amps, N, dt, r_lo, total = _band()
    assert parallel.band_blocks(N, dt, HIDR, NHARMS, BAND[0], BAND[1], 100, BLOCK) == -(-total // BLOCK)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        amps, N, dt, r_lo, total = _band()
        nb = parallel.band_blocks(N, dt, HIDR, NHARMS, BAND[0], BAND[1], 100, BLOCK)
        b0, b1 = parallel.block_shard(nb, rank, world)
        res = _oracle_blocks(b0, b1)
        allc = parallel.gather_records(res["cands"])
        slowest = parallel.max_over_ranks([res["seconds"], float(rank)])
        np.save(os.path.join(out_dir, f"cands_{rank}.npy"), allc)
        np.save(os.path.join(out_dir, f"max_{rank}.npy"), np.array(slowest))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_shard_and_gather(tmp_path):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    amps, N, dt, r_lo, total = _band()
    whole = _oracle_blocks(0, -(-total // BLOCK))["cands"]
    assert len(whole) > 0
    for r in range(2):
        got = np.load(tmp_path / f"cands_{r}.npy")
        assert np.array_equal(_sorted(got), _sorted(whole))
        mx = np.load(tmp_path / f"max_{r}.npy")
        assert mx[1] == 1.0 and mx[0] > 0.0


def test_file_shard_balances_whole_spectra():
    """cfg4 sharding: every spectrum on exactly one rank, loads within one
    spectrum of each other (longest first to the least-loaded rank)."""
    rng = np.random.default_rng(7)
    for world in (1, 2, 3, 8):
        for trials in ([0], [5, 3, 8, 1, 9, 2], list(rng.integers(1, 10**7, 64)),
                       [1 << 21] * 16 + [1 << 22] * 16 + [1 << 23] * 16 + [1 << 24] * 16):
            parts = [parallel.file_shard(trials, r, world) for r in range(world)]
            assert sorted(i for p in parts for i in p) == list(range(len(trials)))
            loads = [sum(trials[i] for i in p) for p in parts]
            assert max(loads) - min(loads) <= max(trials)
            assert all(p == sorted(p) for p in parts)
    with pytest.raises(ValueError):
        parallel.file_shard([1, 2], 2, 2)


class _FakeBatchEngine:
    """Stands in for Engine.search_batch_raw on CPU: each spectrum yields
    (index-dependent) records, in the record layout the library returns."""

    def __init__(self):
        from cohsearch import SearchParams
        self.params = SearchParams(nharms=NHARMS, m=M)

    def search_batch_raw(self, spectra, lofreq, hifreq, lobin, blocksize, threshold, on_device=False):
        from cohsearch import _lib
        recs, owner = [], []
        for i, (tag, N, dt) in enumerate(spectra):
            n = int(tag) % 4
            r = np.zeros(n, _lib.CAND_DTYPE)
            r["trial"] = np.arange(n) * 1000 + int(tag)
            r["k"] = 1 + np.arange(n) % 3
            r["metric"] = 8.0 + int(tag) + np.arange(n)
            recs.append(r)
            owner += [i] * n
        raw = np.concatenate(recs) if recs else np.zeros(0, _lib.CAND_DTYPE)
        return raw, np.asarray(owner, np.int32)


def _batch_spectra():
    lengths = [1 << 21, 1 << 22, 1 << 23, 1 << 24]
    return [(i, lengths[i % 4], 64e-6) for i in range(13)]


def _metric_values():
    """Per rank, per (k, window), seeded metric values (block-sharded search)."""
    rng = np.random.default_rng(11)
    vals = {}
    for k in (1, 2, 3):
        for w in (1, 2, 3):
            v = rng.gamma(2.0, 1.5, 900)
            v[:5] = [-1.0, 0.0, 64.0, 70.0, 3.3]       # under, edges, over
            vals[(k, w)] = v
    return vals


def _stats_of(values_by_key, part, world):
    """MetricStats holding the part-th of `world` shares of every window's values."""
    from cohsearch.metricstats import BlockMetricStats, MetricHistogram, MetricStats, merge_hists
    ms = MetricStats(hist_lo=0.0, hist_hi=64.0, hist_nb=320, nwin=3)
    for k in (1, 2, 3):
        wins = []
        for w in (1, 2, 3):
            v = values_by_key[(k, w)]
            v = v[part::world] if world > 1 else v
            c, _ = np.histogram(v[(v >= 0.0) & (v < 64.0)], bins=320, range=(0.0, 64.0))
            h = MetricHistogram(k, 60 // k, 2 * (60 // k), w, float(w), float(w + 1), 0.0, 64.0, 320 / 64.0,
                                c.astype(np.int64), int(np.sum(v < 0.0)), int(np.sum(v >= 64.0)), len(v),
                                float(np.sum(v)), float(np.sum(v * v)), float(v.min()), float(v.max()))
            wins.append(h)
        ms.whists.extend(wins)
        ms.hists.append(merge_hists(wins, 0, 1.0, 4.0))
        nblk = 6
        for b in range(part, nblk, world) if world > 1 else range(nblk):
            ms.blocks.append(BlockMetricStats(b + 1, k, 60 // k, 2 * (60 // k), 1.0, 1.0, 2.0, 100, 0.1, 1.0,
                                              1.1, 0.5, 9.0 + b))
    return ms


def _rank_main_batch(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = parallel.search_batch_sharded(_FakeBatchEngine(), _batch_spectra(), 0.1, 125.0, rank, world)
        np.save(os.path.join(out_dir, f"batch_{rank}.npy"), got)
        red = parallel.reduce_metricstats(_stats_of(_metric_values(), rank, world))
        import pickle
        with open(os.path.join(out_dir, f"ms_{rank}.pkl"), "wb") as f:
            pickle.dump(red, f)
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_batch_shard_and_metricstats(tmp_path):
    """cfg4 across ranks: the sharded batch's gathered records equal one
    process's (spectrum-major order, global spectrum index); and the metric
    statistics of block-sharded ranks reduce to the whole search's: counts,
    tails and extremes exactly, FP64 sums to rounding, blocks in (block, k)
    order."""
    import multiprocessing as mp
    import pickle
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main_batch, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    raw, owner = _FakeBatchEngine().search_batch_raw(_batch_spectra(), 0.1, 125.0, 100, 2048, None)
    for r in range(2):
        got = np.load(tmp_path / f"batch_{r}.npy")
        assert np.array_equal(got["file"], owner)
        for name in raw.dtype.names:
            assert np.array_equal(got[name], raw[name])
    want = _stats_of(_metric_values(), 0, 1)
    for r in range(2):
        with open(tmp_path / f"ms_{r}.pkl", "rb") as f:
            red = pickle.load(f)
        assert len(red.whists) == len(want.whists) and len(red.hists) == len(want.hists)
        for a, b in zip(red.whists + red.hists, want.whists + want.hists):
            assert (a.k, a.win) == (b.k, b.win)
            assert np.array_equal(a.counts, b.counts)
            assert (a.under, a.over, a.total, a.vmin, a.vmax) == (b.under, b.over, b.total, b.vmin, b.vmax)
            assert a.sum == pytest.approx(b.sum, rel=1e-12) and a.sumsq == pytest.approx(b.sumsq, rel=1e-12)
        assert [(x.block, x.k) for x in red.blocks] == sorted((x.block, x.k) for x in want.blocks)
        assert [x.max for x in red.blocks] == [x.max for x in sorted(want.blocks, key=lambda x: (x.block, x.k))]
