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
