"""Multi-GPU plumbing for the search: one process per GPU over torch.distributed.

The search shards without any data-path collective.  A rank searches either
whole spectra of a batch (one ``.fft`` per DM trial, balanced by trial count:
``file_shard`` / ``search_batch_sharded``) or a contiguous range of whole blocks
of one shared spectrum (``Engine.search_raw(blocks=...)``, i.e.
``cs_search_range``).  Blocks are independent given the band's global
trial anchoring (src/directinterp.jl:498-504, chunk invariance pinned by
test/test_search.jl:234-276), and sigma is per (block, k), so a block range
reproduces that part of the whole search exactly.  The only exchanges are on
results: candidate records gathered to every rank, and timings reduced by max.
Block-sharded metric statistics are merged by ``reduce_metricstats`` (histogram
counts and moments summed, extremes reduced by min/max, block records
gathered).  They work with the ``gloo`` backend on CPU tensors and ``nccl`` on
CUDA tensors.
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


def file_shard(trials, rank, world):
    """Indices (ascending) of the whole spectra `rank` searches in a batch whose
    spectra have trials[i] trials: longest first, each to the least-loaded rank
    (ties to the lower rank), so every rank's load is within one spectrum of
    the mean.  Deterministic: every rank computes the same assignment."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    order = sorted(range(len(trials)), key=lambda i: (-int(trials[i]), i))
    load = [0] * world
    owner = [0] * len(trials)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += int(trials[i])
    return [i for i in range(len(trials)) if owner[i] == rank]


def search_batch_sharded(engine, spectra, lofreq, hifreq, rank, world, lobin=100, blocksize=2048, threshold=None,
                         on_device=False, device="cpu", group=None):
    """A batch of spectra (the `Engine.search_batch_raw` list of (amps, N, dt))
    with this rank searching its `file_shard` of them; every rank returns the
    whole batch's raw detections with a ``file`` field (the spectrum's index
    in `spectra`), ordered as one process would emit them: by spectrum, then
    in each spectrum's own order."""
    p = engine.params
    trials = [band_blocks(N, dt, p.hidr, p.nharms, lofreq, hifreq, lobin, blocksize) * blocksize
              for (_, N, dt) in spectra]
    mine = file_shard(trials, rank, world)
    if mine:
        raw, owner = engine.search_batch_raw([spectra[i] for i in mine], lofreq, hifreq, lobin, blocksize,
                                             threshold, on_device=on_device)
    else:
        raw, owner = engine.search_batch_raw([], lofreq, hifreq, lobin, blocksize, threshold, on_device=on_device)
    return _tag_and_gather(raw, np.asarray(mine, np.int64)[owner] if len(raw) else np.zeros(0, np.int64),
                           device, group)


def _tag_and_gather(raw, gfile, device, group):
    """Gather records tagged with their global spectrum index; stable sort by it."""
    dt = np.dtype(raw.dtype.descr + [("file", np.int32)])
    rec = np.zeros(len(raw), dt)
    for name in raw.dtype.names:
        rec[name] = raw[name]
    rec["file"] = gfile
    allr = gather_records(rec, device=device, group=group)
    return allr[np.argsort(allr["file"], kind="stable")]


def reduce_metricstats(ms, device="cpu", group=None):
    """Merge the metric statistics of block-sharded ranks into the whole
    search's, on every rank (a new MetricStats; `ms` is left as it was).

    Every rank searched the same band with the same histogram settings, so its
    per-(k, window) histograms share k, windows and edges: counts, tails,
    totals and the exact FP64 sums add (all_reduce SUM), extremes reduce by
    MIN / MAX, and the per-k merges are rebuilt from the summed windows
    (src/search.jl:1419-1473).  The per-(block, k) records are gathered and
    sorted by (block, k).  The FP64 sums are added in a different order than
    one process adds them (rank partials first), so they agree to rounding."""
    import torch
    import torch.distributed as dist
    from .metricstats import BlockMetricStats, MetricHistogram, MetricStats, merge_hists
    wh = sorted(ms.whists, key=lambda h: (h.k, h.win))
    nh = len(wh)
    nb = int(ms.hist_nb)
    n_all = torch.tensor([nh], dtype=torch.int64, device=device)
    dist.all_reduce(n_all, op=dist.ReduceOp.MAX, group=group)
    if int(n_all.item()) != nh:
        raise ValueError("ranks hold different histogram sets; every rank must search the same band")
    counts = torch.from_numpy(np.stack([h.counts for h in wh]).astype(np.int64) if nh else
                              np.zeros((0, nb), np.int64)).to(device)
    tails = torch.tensor([[h.under, h.over, h.total] for h in wh] or np.zeros((0, 3)), dtype=torch.int64,
                         device=device)
    sums = torch.tensor([[h.sum, h.sumsq] for h in wh] or np.zeros((0, 2)), dtype=torch.float64, device=device)
    vmin = torch.tensor([h.vmin for h in wh], dtype=torch.float64, device=device)
    vmax = torch.tensor([h.vmax for h in wh], dtype=torch.float64, device=device)
    for t, op in ((counts, dist.ReduceOp.SUM), (tails, dist.ReduceOp.SUM), (sums, dist.ReduceOp.SUM),
                  (vmin, dist.ReduceOp.MIN), (vmax, dist.ReduceOp.MAX)):
        dist.all_reduce(t, op=op, group=group)
    counts, tails, sums = counts.cpu().numpy(), tails.cpu().numpy(), sums.cpu().numpy()
    vmin, vmax = vmin.cpu().numpy(), vmax.cpu().numpy()
    out = MetricStats(hist_lo=ms.hist_lo, hist_hi=ms.hist_hi, hist_nb=ms.hist_nb, nwin=ms.nwin)
    for i, h in enumerate(wh):
        out.whists.append(MetricHistogram(h.k, h.Hk, h.nbins, h.win, h.flo, h.fhi, h.lo, h.hi, h.invw,
                                          counts[i].copy(), int(tails[i, 0]), int(tails[i, 1]), int(tails[i, 2]),
                                          float(sums[i, 0]), float(sums[i, 1]), float(vmin[i]), float(vmax[i])))
    for k in sorted({h.k for h in out.whists}):
        wins = [h for h in out.whists if h.k == k]
        out.hists.append(merge_hists(wins, 0, wins[0].flo, wins[-1].fhi))
    # the per-(block, k) records, as a structured array through the record gather
    fields = [("block", np.int64), ("k", np.int32), ("Hk", np.int32), ("nbins", np.int32), ("ngoodbins", np.float64),
              ("flo", np.float64), ("fhi", np.float64), ("n", np.int64), ("min", np.float64),
              ("median", np.float64), ("mean", np.float64), ("std", np.float64), ("max", np.float64)]
    rec = np.zeros(len(ms.blocks), np.dtype(fields))
    for j, b in enumerate(ms.blocks):
        rec[j] = tuple(getattr(b, f) for f, _ in fields)
    allb = gather_records(rec, device=device, group=group)
    allb = allb[np.lexsort((allb["k"], allb["block"]))]
    for r in allb:
        out.blocks.append(BlockMetricStats(int(r["block"]), int(r["k"]), int(r["Hk"]), int(r["nbins"]),
                                           float(r["ngoodbins"]), float(r["flo"]), float(r["fhi"]), int(r["n"]),
                                           float(r["min"]), float(r["median"]), float(r["mean"]), float(r["std"]),
                                           float(r["max"])))
    return out
