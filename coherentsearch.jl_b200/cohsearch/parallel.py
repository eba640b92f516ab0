"""Multi-GPU plumbing for the search: one process per GPU over torch.distributed.

The search shards without any data-path collective.  A rank searches either a
spectrum of its own (one ``.fft`` per DM trial: weak scaling) or a contiguous
range of whole blocks of one shared spectrum (``Engine.search_raw(blocks=...)``,
i.e. ``cs_search_range``).  Blocks are independent given the band's global
trial anchoring (src/directinterp.jl:498-504, chunk invariance pinned by
test/test_search.jl:234-276), and sigma is per (block, k), so a block range
reproduces that part of the whole search exactly.  The only exchanges are on
results: candidate records gathered to every rank, and timings reduced by max.
They work with the ``gloo`` backend on CPU tensors and ``nccl`` on CUDA tensors.
"""
import math

import numpy as np


def band_blocks(N, dt, hidr, nharms, lofreq, hifreq, lobin=100, blocksize=2048):
    """Number of blocksize-trial blocks of a band: the bookkeeping of `search`
    (src/search.jl:2016-2027) with the FP64 expressions cs_search uses."""
    T = float(N) * float(dt)
    lodr = float(hidr) / float(nharms)
    r_lo = float(lofreq) * T if lobin == 100 else float(lobin)
    r_hi = float(hifreq) * T
    total = max(0, int(math.floor((r_hi - r_lo) / lodr)) + 1)
    return -(-total // blocksize)


def block_shard(nblocks, rank, world):
    """Contiguous block range [b0, b1) of `rank`: sizes differ by at most one and
    the ranges of ranks 0..world-1 tile [0, nblocks) in order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(nblocks), int(world))
    b0 = rank * base + min(rank, extra)
    return b0, b0 + base + (1 if rank < extra else 0)


def gather_records(arr, device="cpu", group=None):
    """All-gather a 1-D structured numpy array of any length from every rank;
    every rank returns the concatenation in rank order.  Counts go first, then
    the records as bytes padded to the longest."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    arr = np.ascontiguousarray(arr)
    n = torch.tensor([len(arr)], dtype=torch.int64, device=device)
    counts = [torch.zeros(1, dtype=torch.int64, device=device) for _ in range(world)]
    dist.all_gather(counts, n, group=group)
    counts = [int(c.item()) for c in counts]
    isz = arr.dtype.itemsize
    width = max(1, max(counts)) * isz
    buf = np.zeros(width, np.uint8)
    raw = arr.view(np.uint8).reshape(-1)
    buf[:raw.size] = raw
    mine = torch.from_numpy(buf).to(device)
    parts = [torch.zeros(width, dtype=torch.uint8, device=device) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    out = [p.cpu().numpy()[:c * isz].view(arr.dtype) for p, c in zip(parts, counts)]
    return np.concatenate(out) if out else arr[:0]


def max_over_ranks(values, device="cpu", group=None):
    """Element-wise maximum of a list of floats over all ranks (FP64)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(x) for x in t.cpu().tolist()]


def search_sharded(engine, N, dt, lofreq, hifreq, rank, world, lobin=100, blocksize=2048, threshold=None,
                   device="cpu", group=None):
    """Whole-band raw detections with this rank searching only its block
    range; every rank returns the full list, in the order cs_search emits."""
    p = engine.params
    nb = band_blocks(N, dt, p.hidr, p.nharms, lofreq, hifreq, lobin, blocksize)
    b0, b1 = block_shard(nb, rank, world)
    mine = engine.search_raw(lofreq, hifreq, lobin, blocksize, threshold, blocks=(b0, b1))
    return gather_records(mine, device=device, group=group)
