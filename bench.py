#!/usr/bin/env python
"""Throughput of the coherent-search hot path on B200: fundamental trials/s.

Workload (the default CLI survey of one spectrum): 2^23 real samples at
dt = 64 us (T = 537 s, 2^22 complex64 bins = 32 MiB) of seeded unit-variance
noise with six injected pulsars (0.37-702 Hz, duty 2-20%, nominal S/N 7-25);
nharms = 60, decimations = decimation_set(60, 6), 0.1-125 Hz fundamentals,
threshold 8, blocksize 2048: 8,046,622 trials.  One step = one full search of
that band through the C ABI (every decimation level, candidates copied back).

  value  trials/s with the spectrum already resident on the device;
  e2e    trials/s through the same C-ABI call with the spectrum in pinned host
         memory, its host->device copy and the candidates' device->host copy
         inside the timed region.
The 32 MiB spectrum fits in L2, so L2 is flushed (a 256 MiB write) before every
timed step; steps are timed with CUDA events on the engine's stream.

Under torchrun (N > 1) every rank searches its own seeded spectrum (one file
per GPU, no data-path collective): weak scaling, value = all ranks' trials /
max-over-ranks time.  ``--impl reference`` times the CPU restatement of the
reference's search (the C port, all host threads) on a bounded sample of the
same workload.
"""
import argparse
import gc
import json
import math
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "coherentsearch.jl_b200"))
sys.path.insert(0, ROOT)

METRIC = "trials/s at nharms=60 (plain vs mixed/learned GPU) at >=99.5% recall of S/N>=8"
NHARMS, MAXDECIM, LOF, HIF, THR, BLOCK = 60, 6, 0.1, 125.0, 8.0, 2048


def workload_config(synth_mode):
    return {"workload": "survey: 2^23 samples @64us, 6 injected pulsars, nharms=60, "
                        "decimation_set(60,6), 0.1-125 Hz, threshold 8, blocksize 2048",
            "trials_per_step": None, "synth": synth_mode, "l2": "flushed (256 MiB write) before each step",
            "parallelism": "one spectrum per GPU (weak)"}


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock, power and clock-event reasons of this process's GPU, polled
    through NVML every 5 ms while the timed region runs (nvidia-smi's 100 ms
    loop would see a few samples of a sub-second region at most)."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.samples = []
        self.stop = threading.Event()
        self.thread = None
        self.max_mhz = None
        self.nvml = None

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.cuda_index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def _poll(self, nv, h):
        masks = [(n, getattr(nv, c)) for n, c in self.REASONS]
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), [n for n, m in masks if rs & m]))
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        try:
            nv, h = self._handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.nvml = nv
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.thread:
            self.thread.join(timeout=5)
        if self.nvml:
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0, "source": "nvml"}
        reasons = sorted({r for _, rs in self.samples for r in rs})
        return {"sm_mhz": float(np.median([s for s, _ in self.samples])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "nvml, 5 ms poll"}


# ---------------------------------------------------------------------------
# work per trial (algorithmic), used by the roofline figures
# ---------------------------------------------------------------------------
def level_list():
    from cohsearch import decimation_set
    ks = decimation_set(NHARMS, MAXDECIM)
    return [(k, NHARMS // k) for k in ks]


def synth_flops_per_trial(frac_valid):
    """Real inverse DFT by the symmetric direct form: per level (Hk+1)(Hk-1)
    FMA pairs (E and O) = 4(Hk+1)(Hk-1) flops, weighted by the valid fraction."""
    return sum(4.0 * (Hk + 1) * (Hk - 1) * frac_valid.get(k, 1.0) for k, Hk in level_list())


def interp_flops_per_trial(m=16):
    return NHARMS * (4 * m + 6)   # m real-times-complex FMAs + one complex product


def tensor_flops_per_trial():
    """Dense contraction of the Re/Im amplitude stack against every level's
    cos/sin rows: 2 * sum_k (2 Hk)^2 flops."""
    return sum(2 * (2 * Hk) ** 2 for _, Hk in level_list())


# boxcar gate per trial (prefix sums + a subtract and a max per start and width, all levels)
GATE_OPS_PER_TRIAL = 2922


def sigma_flops_per_block():
    """FP32 synthesis of the pooled sigma columns of one block, all levels: per
    level min(2048, 8192 // nbins) columns of 4(Hk+1)(Hk-1) flops."""
    return sum(min(BLOCK, 8192 // (2 * Hk)) * 4.0 * (Hk + 1) * (Hk - 1) for _, Hk in level_list())


# DRAM bytes (read + write) per trial of one launch, from the ncu captures
# summarised under profiles/ (small survey case, 1,282,048 trials; the traffic
# of these kernels grows in proportion to the trial count).
NCU_BYTES_PER_TRIAL = {"k_interp": 294.9, "k_synth_tc": 260.1, "k_sigma": 100.9, "k_rescue": 0.44}


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return pk, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
                "sm_max_mhz": 1965.0}, "fallback"


# ---------------------------------------------------------------------------
# our engine
# ---------------------------------------------------------------------------
def run_dmsweep(args, rank, local_rank):
    """The batched DM-sweep workload: 64 spectra (16 each of 2^21..2^24 samples)
    searched at nharms=60, maxdecim 6, 0.1-125 Hz, through cs_search_batch.
    `value`: spectra resident on the device; `e2e`: from pinned host memory,
    copies overlapped with the searches."""
    import torch
    from cohsearch import Engine, SearchParams, decimation_set, synth
    torch.cuda.set_device(local_rank)
    files = synth.dmsweep_config(seed=4 + rank)
    params = SearchParams(nharms=NHARMS, m=16, decimations=decimation_set(NHARMS, MAXDECIM), threshold=THR,
                          synth=args.synth)
    eng = Engine(params, device=local_rank)
    # a stream of its own (the legacy default stream cannot be captured):
    # device-resident batches replay one captured graph (cs_set_batch_graph)
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    eng.set_batch_graph(not args.no_graph)
    dev = [torch.from_numpy(a.view(np.float32).copy()).cuda() for a, _, _ in files]
    pin = [torch.from_numpy(a.view(np.float32).copy()).pin_memory() for a, _, _ in files]
    on_dev = [((d.data_ptr(), len(a)), N, dt) for d, (a, N, dt) in zip(dev, files)]
    on_host = [(p.numpy().view(np.complex64), N, dt) for p, (a, N, dt) in zip(pin, files)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    lof, hif = args.band if args.band else (LOF, HIF)

    def timed(spectra, on_device, k):
        tot, launches, trials, ncand, d2h = 0.0, 0, 0, 0, 0
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            raw, _ = eng.search_batch_raw(spectra, lof, hif, 100, BLOCK, THR, on_device=on_device)
            e1.record(stream)
            e1.synchronize()
            tot += e0.elapsed_time(e1)
            st = eng.stats()
            launches += st["launches"]
            trials = st["trials"]
            ncand = len(raw)
            d2h = st["d2h_bytes"]
        return tot, launches, trials, ncand, d2h

    for _ in range(args.warmup):
        timed(on_dev, True, 1)
    torch.cuda.synchronize()
    gc.disable()
    with ClockSampler(local_rank) as clk:
        ms, launches, trials, ncand, _ = timed(on_dev, True, args.steps)
        torch.cuda.synchronize()
    timed(on_host, False, 1)   # (pinned host spectra: the ordinary run and the graph capture)
    ms_e2e, _, _, _, d2h = timed(on_host, False, args.steps)
    gc.enable()
    h2d = sum(a.nbytes for a, _, _ in files)
    return {"ms": ms, "ms_e2e": ms_e2e, "launches": launches, "trials": trials, "ncand": ncand,
            "clocks": clk.summary(), "nfiles": len(files), "h2d": h2d, "d2h": d2h}


def run_learned(args, local_rank):
    """The learned block proposal on a 2^24-sample spectrum.  Training: separately
    seeded 2^24-sample spectra with 200 injections each (f 0.1-750 Hz, duty
    1-20 %, S/N 6-20, frequency-domain synthesis), every block of the survey
    band labelled by the coherent search's own candidates (S/N > 8; the mixed
    FP16 search reports exactly the plain candidates), until --train-blocks.
    The score cut keeps 99.5 % of the positive blocks of 4 validation spectra.
    Evaluation spectrum: another such spectrum.  Timed (wall clock, each stage
    ending in a device sync, every arm alike): the plain FP32 full search, the
    mixed FP16 full search, and the learned path -- features, scores, plain
    FP32 re-search of the blocks at or above the cut (and its mixed variant)."""
    import torch
    from cohsearch import Engine, FFTFile, SearchParams, decimation_set, learned, synth
    torch.cuda.set_device(local_rank)
    nsamp, dt = 1 << 24, 64e-6
    dec = decimation_set(NHARMS, MAXDECIM)
    plain = Engine(SearchParams(nharms=NHARMS, m=16, decimations=dec, threshold=THR, synth="fp32"), device=local_rank)
    mixed = Engine(SearchParams(nharms=NHARMS, m=16, decimations=dec, threshold=THR, synth="fp16"), device=local_rank)

    def spectrum(seed):
        rng = np.random.default_rng(seed)
        ps = synth.random_pulsars(rng, 200, 0.1, 750.0, 0.01, 0.20, 6.0, 20.0)
        return synth.make_spectrum_fd(nsamp, dt, ps, seed)

    def labelled(seed):
        mixed.set_spectrum(FFTFile.from_array(spectrum(seed), nsamp, dt))
        X = mixed.block_features(LOF, HIF, 100, BLOCK)
        raw = mixed.search_raw(LOF, HIF, 100, BLOCK, THR)
        return X, torch.from_numpy(learned.block_labels(raw, X.shape[0], BLOCK, THR))

    t0 = time.perf_counter()
    xs, ys, seed, nb = [], [], 10_000, 0
    while nb < args.train_blocks:
        X, Y = labelled(seed)
        xs.append(X)
        ys.append(Y)
        nb += X.shape[0]
        seed += 1
    Xt, Yt = torch.cat(xs), torch.cat(ys)
    del xs, ys
    t_data = time.perf_counter() - t0
    mlp = learned.ProposalMLP(Xt.shape[1], 256, seed=0, device=local_rank)
    t0 = time.perf_counter()
    hist = mlp.fit(Xt, Yt, epochs=10, batch=4096, lr=1e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    val = [labelled(s) for s in (20_000, 20_001, 20_002, 20_003)]
    sv = np.concatenate([mlp.scores(X) for X, _ in val])
    tau = learned.choose_threshold(sv, np.concatenate([Y.numpy() for _, Y in val]), 0.995)

    ev = spectrum(30_000)
    for e in (plain, mixed):
        e.set_spectrum(FFTFile.from_array(ev, nsamp, dt))

    def wall(fn, k):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(k):
            out = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t) * 1e3 / k, out

    gc.disable()
    ms_plain, full = wall(lambda: plain.search_raw(LOF, HIF, 100, BLOCK, THR), args.steps)
    ms_mixed, _ = wall(lambda: mixed.search_raw(LOF, HIF, 100, BLOCK, THR), args.steps)
    ms_learn, res = wall(lambda: learned.learned_search(plain, mlp, tau, LOF, HIF, 100, BLOCK, THR), args.steps)
    ms_learn_mixed, res_m = wall(lambda: learned.learned_search(mixed, mlp, tau, LOF, HIF, 100, BLOCK, THR),
                                 args.steps)
    gc.enable()
    T = nsamp * dt
    lodr = 0.5 / NHARMS
    total = int(np.floor((HIF * T - LOF * T) / lodr)) + 1
    return {"ms_plain": ms_plain, "ms_mixed": ms_mixed, "ms_learned": ms_learn, "ms_learned_mixed": ms_learn_mixed,
            "recall": learned.recall_of(res.cands, full, THR), "recall_mixed": learned.recall_of(res_m.cands, full, THR),
            "frac_blocks": len(res.blocks) / res.nblocks, "nblocks": res.nblocks, "trials": total,
            "stage_ms": {"features": res.ms_features, "scores": res.ms_scores, "research": res.ms_search},
            "train_blocks": int(Xt.shape[0]), "train_pos": int(Yt.sum().item()), "nfeat": int(Xt.shape[1]),
            "loss": [round(h, 4) for h in hist], "tau": tau, "t_data_s": t_data, "t_train_s": t_train,
            "ncand_full": int(np.sum(full["metric"] > THR))}


def run_ours(args, rank, world, local_rank):
    import torch
    from cohsearch import Engine, SearchParams, decimation_set, synth

    torch.cuda.set_device(local_rank)
    amps, N, dt = synth.survey_config(seed=2 + rank)
    namps = len(amps)
    params = SearchParams(nharms=NHARMS, m=16, decimations=decimation_set(NHARMS, MAXDECIM),
                          threshold=THR, synth=args.synth)
    eng = Engine(params, device=local_rank)
    # the engine's work and the timing events on one stream of our own
    stream = torch.cuda.Stream()
    eng.set_stream(stream.cuda_stream)
    d_amps = torch.from_numpy(amps.view(np.float32).copy()).cuda()
    h_amps = torch.from_numpy(amps.view(np.float32).copy()).pin_memory()
    eng.set_spectrum_device(d_amps.data_ptr(), namps, N, dt, keep=d_amps)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    lof, hif = args.band if args.band else (LOF, HIF)
    # launch shapes from the autotuner (setup, outside the timed region)
    if args.shapes:
        # fixed launch shapes (reproducible profiling runs): no tuner launches
        i_k, s_k, d0, d1, db = args.shapes
        eng.set_launch_shapes(interp_kernel=i_k, sigma_kernel=s_k, tc_double_buffer=db, tc_div=(d0, d1))
    tune = None if (args.no_tune or args.shapes) else eng.autotune(lof, hif, 100, BLOCK, nsample=4096)

    # Device-resident step: the search of the resident spectrum through the
    # batch entry point with its captured graph (cs_set_batch_graph): the
    # first warm-up call runs it the ordinary way and captures it, every later
    # call replays it -- no host round trip between the kernels.
    dev_batch = [((d_amps.data_ptr(), namps), N, dt)]
    eng.set_batch_graph(not args.no_graph)

    def step_device():
        return eng.search_batch_raw(dev_batch, lof, hif, 100, BLOCK, THR, on_device=True)[0]

    def step_e2e():
        eng.set_spectrum_host(h_amps.data_ptr(), namps, N, dt)
        return eng.search_raw(lof, hif, 100, BLOCK, THR)

    for _ in range(args.warmup):
        cands = step_device()

    def timed(fn, k):
        total_ms, launches, h2d, d2h, ncand = 0.0, 0, 0, 0, 0
        for _ in range(k):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            c = fn()
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            s = eng.stats()
            launches += s["launches"]
            h2d += s["h2d_bytes"]
            d2h += s["d2h_bytes"]
            ncand = len(c)
        return total_ms, launches, h2d, d2h, ncand

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    gc.disable()   # no collector pauses inside the timed regions
    with ClockSampler(local_rank) as clk:
        ms, launches, _, _, ncand = timed(step_device, args.steps)
        torch.cuda.synchronize()
    ms_e2e, _, h2d, d2h, _ = timed(step_e2e, args.steps)
    torch.cuda.synchronize()
    gc.enable()
    # per-kernel times (CUDA events between the kernels of ordinary searches
    # of the same workload; a replayed graph has none), for the roofline
    stage = {"ms_interp": 0.0, "ms_synth": 0.0, "ms_sigma": 0.0, "ms_rescue": 0.0}
    nst = 3
    for _ in range(nst):
        with torch.cuda.stream(stream):
            flush.zero_()
        eng.search_raw(lof, hif, 100, BLOCK, THR)
        s_ = eng.stats()
        for key in stage:
            stage[key] += s_[key] / nst
    st = eng.stats()
    trials = st["trials"]
    plain = None
    if args.synth != "fp32" and not args.no_plain:
        # the plain FP32 GPU form on the same data, for the mixed-vs-plain comparison
        eng32 = Engine(SearchParams(nharms=NHARMS, m=16, decimations=decimation_set(NHARMS, MAXDECIM),
                                    threshold=THR, synth="fp32"), device=local_rank)
        eng32.set_stream(stream.cuda_stream)
        eng32.set_spectrum_device(d_amps.data_ptr(), namps, N, dt, keep=d_amps)
        if not args.no_tune:
            eng32.autotune(lof, hif, 100, BLOCK, nsample=4096)
        eng32.set_batch_graph(not args.no_graph)
        for _ in range(2):
            c32 = eng32.search_batch_raw(dev_batch, lof, hif, 100, BLOCK, THR, on_device=True)[0]
        ms32 = 0.0
        for _ in range(max(1, args.steps)):
            with torch.cuda.stream(stream):
                flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            c32 = eng32.search_batch_raw(dev_batch, lof, hif, 100, BLOCK, THR, on_device=True)[0]
            e1.record(stream)
            e1.synchronize()
            ms32 += e0.elapsed_time(e1)
        same = bool(np.array_equal(c32, cands)) if len(cands) == len(c32) else False
        plain = {"ms": ms32 / max(1, args.steps), "same_candidates": same, "ncand": int(len(c32))}
        del eng32
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms, ms_e2e], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_e2e = float(t[0]), float(t[1])
    res = {"ms": ms, "ms_e2e": ms_e2e, "namps": namps, "tune": tune, "stage": stage, "stage_is_mean": True,
           "launches": launches, "h2d": h2d, "d2h": d2h,
           "trials": trials, "ncand": ncand, "clocks": clk.summary(), "stats": st, "plain": plain}
    del eng
    return res


# ---------------------------------------------------------------------------
# CPU restatement (reference arm and cpu_baseline)
# ---------------------------------------------------------------------------
_CPU_SPECTRUM = {}


def cpu_band_run(nthreads, nblocks=None, seed=2, first_block=None):
    """Time the C port of the reference search (oracle/cs_cpu.c, all given
    threads, blocks dealt round-robin as the reference's tasks take chunks) on
    the survey workload: the whole band by default, else `nblocks` blocks from
    `first_block` (mid-band when not given).  The port's c2r transform is its
    own mixed-radix FP64 FFT where the reference calls FFTW."""
    from oracle import cs_cpu
    if seed not in _CPU_SPECTRUM:
        from cohsearch import synth
        _CPU_SPECTRUM[seed] = synth.survey_config(seed=seed)
    amps, N, dt = _CPU_SPECTRUM[seed]
    T = N * dt
    lodr = 0.5 / NHARMS
    r_lo = LOF * T
    total = int(math.floor((HIF * T - r_lo) / lodr)) + 1
    nblk_all = -(-total // BLOCK)
    if nblocks is None:
        first_block, nblocks = 0, nblk_all
    elif first_block is None:
        first_block = max(0, nblk_all // 2 - nblocks // 2)
    return cs_cpu.search_blocks(amps, N, dt, NHARMS, 16, 0.5, [k for k, _ in level_list()], r_lo, total,
                                BLOCK, first_block, nblocks, THR, nthreads)


CPU_PORT_NOTE = ("C restatement of the reference's production search (Float32-weight interpolation, FP64 "
                 "profiles, block sigma, batched FP32 gate, exact rescan); its c2r transform is its own "
                 "mixed-radix FP64 FFT where the reference calls FFTW")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--synth", default="fp16", choices=["fp32", "bf16", "fp16", "bf16_split", "fp16_split"])
    ap.add_argument("--cpu-blocks", type=int, default=None,
                    help="CPU port legs: N mid-band blocks per step instead of the whole band (a quick check)")
    ap.add_argument("--workload", choices=["survey", "dmsweep", "learned"], default="survey",
                    help="survey: one 2^23-sample spectrum (the headline); dmsweep: 64 spectra of "
                         "2^21..2^24 samples through the batch entry point; learned: the learned block "
                         "proposal on a 2^24-sample spectrum with 200 injections")
    ap.add_argument("--no-graph", action="store_true",
                    help="search device-resident spectra the ordinary way (a host round trip per search), not by "
                         "a replayed CUDA graph")
    ap.add_argument("--train-blocks", type=int, default=1_000_000,
                    help="learned workload: labelled training blocks (separately seeded spectra)")
    ap.add_argument("--band", type=float, nargs=2, default=None,
                    help="search only [LO, HI] Hz (a smaller case of the same kernels, for profiling)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison run")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch shapes (no autotuner)")
    ap.add_argument("--shapes", type=int, nargs=5, default=None, metavar=("INTERP", "SIGMA", "DIV0", "DIV1", "DBUF"),
                    help="fixed launch shapes instead of the autotuner (cs_set_launch_shapes): interpolation kernel "
                         "(0 per item, 1 persistent), sigma kernel (0 or 1), epilogue divisors, TMEM double buffer")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return 0
        nthreads = os.cpu_count() or 1
        # warm-up on a sliver of the band (the reference's own timing method,
        # bench/thread_scaling.jl:83-97), then every timed step searches the
        # whole band, as the GPU arm's step does
        for _ in range(args.warmup):
            cpu_band_run(nthreads, nblocks=2 * nthreads)
        times, trials, nblk = [], 0, 0
        for _ in range(args.steps):
            r = cpu_band_run(nthreads, nblocks=args.cpu_blocks)
            times.append(r["seconds"])
            trials, nblk = r["trials"], r["blocks"]
        v = trials * len(times) / sum(times)
        what = "whole band" if args.cpu_blocks is None else "mid-band sample"
        sample = (f"{what} per step ({nblk} blocks x {BLOCK} trials, {trials} trials), {nthreads} threads; "
                  + CPU_PORT_NOTE)
        cfg = workload_config("cpu")
        cfg["trials_per_step"] = trials
        print(json.dumps({
            "impl": "reference", "metric": METRIC, "value": v, "unit": "trials/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": "trials/s", "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": v, "unit": "trials/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return 0

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    if args.workload == "learned":
        if world > 1 or rank != 0:
            return 0
        r = run_learned(args, local_rank)
        cfg = {"workload": "learned proposal: 2^24 samples @64us, 200 injections (f 0.1-750 Hz, duty 1-20%, S/N "
                           "6-20), nharms=60, decimation_set(60,6), 0.1-125 Hz, threshold 8; network "
                           f"{r['nfeat']}-256-256-1 BF16 weights, trained on {r['train_blocks']} labelled blocks",
               "trials_per_step": r["trials"], "blocks": r["nblocks"], "blocks_researched": r["frac_blocks"],
               "recall_vs_plain": r["recall"], "recall_mixed_research": r["recall_mixed"],
               "plain_fp32_ms": r["ms_plain"], "mixed_fp16_ms": r["ms_mixed"],
               "learned_plain_research_ms": r["ms_learned"], "learned_mixed_research_ms": r["ms_learned_mixed"],
               "speedup_vs_plain": r["ms_plain"] / r["ms_learned"],
               "speedup_mixed_research_vs_plain": r["ms_plain"] / r["ms_learned_mixed"],
               "learned_stage_ms": r["stage_ms"], "train_positive_blocks": r["train_pos"],
               "train_loss_per_epoch": r["loss"], "score_cut": r["tau"], "candidates_full": r["ncand_full"],
               "data_s": r["t_data_s"], "train_s": r["t_train_s"], "timing": "wall clock, device-synced, all arms"}
        print(json.dumps({
            "metric": METRIC, "value": r["trials"] / (r["ms_learned"] / 1000.0), "unit": "trials/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_learned"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16", "data": "synthetic", "config": cfg}))
        return 0
    if args.workload == "dmsweep":
        r = run_dmsweep(args, rank, local_rank)
        if world > 1:
            import torch
            import torch.distributed as dist
            t = torch.tensor([r["ms"], r["ms_e2e"]], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            r["ms"], r["ms_e2e"] = float(t[0]), float(t[1])
            dist.barrier()
            dist.destroy_process_group()
        if rank != 0:
            return 0
        K = args.steps
        cfg = {"workload": "batched DM sweep: 64 spectra, 16 each of 2^21/2^22/2^23/2^24 samples @64us, "
                           "0-3 injected pulsars each, nharms=60, decimation_set(60,6), 0.1-125 Hz, threshold 8",
               "trials_per_step": r["trials"], "files": r["nfiles"], "synth": args.synth,
               "l2": "flushed (256 MiB write) before each step", "parallelism": "one sweep per GPU (weak)",
               "batch_graph": not args.no_graph,
               "candidates_per_step": r["ncand"]}
        print(json.dumps({
            "metric": METRIC, "value": world * r["trials"] * K / (r["ms"] / 1000.0), "unit": "trials/s",
            "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": r["ms"] / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.synth == "fp32" else args.synth, "data": "synthetic", "config": cfg,
            "e2e": {"value": world * r["trials"] * K / (r["ms_e2e"] / 1000.0), "unit": "trials/s",
                    "h2d_bytes_per_step": r["h2d"], "d2h_bytes_per_step": r["d2h"]},
            "gpu_launches": r["launches"], "clocks": r["clocks"]}))
        return 0
    res = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    K = args.steps
    trials = res["trials"]
    value = world * trials * K / (res["ms"] / 1000.0)
    e2e = world * trials * K / (res["ms_e2e"] / 1000.0)
    peaks, psrc = load_peaks()
    stage = dict(res["stage"])   # per search already
    st = res["stats"]
    # Roofline of the dominant kernel, on the algorithmic work per trial of the
    # hot path (one fundamental trial through every harmonic and level):
    #   interpolation  nharms*(4m+6) = 4,200 FP32 flops (FP32 SIMT pipe);
    #   profiles       2*sum_k (2 Hk)^2 = 42,952 dense-contraction flops (tensor pipe);
    #   gate scan      ~2,922 FP32 ops (boxcar prefix sums and maxima);
    #   spectrum       the 32 MiB spectrum read once: ~4.2 B per trial (L2-resident).
    # `traffic` is the kernel's measured DRAM bytes (ncu), and
    # `traffic_over_algorithmic` how far it lies above that one spectrum read.
    dom = max(stage, key=stage.get)
    mhz = peaks.get("sm_max_mhz", 1965.0)
    fp32_peak = 148 * 128 * 2 * mhz * 1e6 / 1e12   # TFLOP/s, nominal (no measured FP32 figure exists)
    tc_peak = peaks["bf16_tflops"]
    kname = {"ms_interp": "k_interp", "ms_synth": "k_synth_tc" if args.synth != "fp32" else "k_synth_fp32",
             "ms_sigma": "k_sigma", "ms_rescue": "k_rescue"}[dom]
    alg_bytes = 8.0 * res["namps"] / trials        # the spectrum, read once, per trial
    traffic = NCU_BYTES_PER_TRIAL.get(kname)
    traffic = traffic * trials if traffic is not None else None
    f_interp = interp_flops_per_trial()
    f_tc = tensor_flops_per_trial()
    f_box = GATE_OPS_PER_TRIAL
    fp32_src = (f"nominal FP32 rate 148 SM x 128 lanes x 2 flops x {mhz:.0f} MHz (no measured FP32 peak); "
                "of nominal")
    if kname in ("k_synth_tc",):
        work, unit, peak, bound = f_tc, "TFLOP/s", tc_peak, "tensor"
        wnote = "2*sum_k (2 Hk)^2 = %d tensor flops per trial (dense profile contraction)" % f_tc
        psrc_k = f"MEASURED_PEAKS.json bf16_tflops ({psrc}); of measured" if psrc == "measured" else \
            "fallback 1,590 TFLOP/s; of fallback"
    elif kname == "k_synth_fp32":
        work, unit, peak, bound = synth_flops_per_trial({1: 1.0}) + f_box, "TFLOP/s", fp32_peak, "fp32"
        wnote = "symmetric real DFT 4(Hk+1)(Hk-1) per level + gate scan, FP32 flops per trial"
        psrc_k = fp32_src
    elif kname == "k_interp":
        work, unit, peak, bound = f_interp, "TFLOP/s", fp32_peak, "fp32"
        wnote = "nharms*(4m+6) = %d FP32 flops per trial (16-tap Eqn-30 sums + phase factor)" % f_interp
        psrc_k = fp32_src
    else:   # k_sigma / k_rescue: FP32 profile synthesis of the pooled columns, per trial of the step
        work = sigma_flops_per_block() / BLOCK
        unit, peak, bound = "TFLOP/s", fp32_peak, "fp32"
        wnote = "FP32 synthesis flops of the pooled sigma columns, per trial"
        psrc_k = fp32_src
    achieved = work * trials / (stage[dom] / 1000.0) / 1e12
    roof = {"kernel": kname, "bound": bound, "achieved": achieved, "peak": peak, "unit": unit,
            "frac": achieved / peak, "traffic": traffic,
            "traffic_over_algorithmic": (traffic / (alg_bytes * trials)) if traffic else None,
            "algorithmic_bytes_per_trial": alg_bytes, "work": wnote, "peak_source": psrc_k}
    # the whole step against the path's bound: the slower of the FP32 SIMT work
    # (interpolation + gate scan) and the tensor contraction
    t_bound = max((f_interp + f_box) * trials / (fp32_peak * 1e12), f_tc * trials / (tc_peak * 1e12))
    roof["step"] = {"bound_ms": t_bound * 1e3, "measured_ms": res["ms"] / K,
                    "frac": t_bound * 1e3 / (res["ms"] / K),
                    "work": "max((4,200 + 2,922) FP32 flops / FP32 peak, 42,952 tensor flops / BF16 peak) "
                            "per trial"}
    roof["stage_ms"] = stage
    cpu = None
    try:
        if args.no_cpu:
            raise RuntimeError("skipped (--no-cpu)")
        nthreads = os.cpu_count() or 1
        cpu_band_run(nthreads, nblocks=2 * nthreads)   # warm-up on a sliver of the band
        runs = [cpu_band_run(nthreads, nblocks=args.cpu_blocks) for _ in range(3)]
        secs = sorted(r["seconds"] for r in runs)
        r = runs[0]
        what = "whole band" if args.cpu_blocks is None else "mid-band sample"
        cpu = {"value": r["trials"] / secs[1], "unit": "trials/s", "cores": r["threads"], "kind": "port",
               "sample": f"{what} ({r['blocks']} blocks, {r['trials']} trials), median of 3 runs; "
                         + CPU_PORT_NOTE}
        # and one thread alone, on 32 mid-band blocks (the per-core rate)
        one = [cpu_band_run(1, nblocks=32) for _ in range(3)]
        s1 = sorted(o["seconds"] for o in one)
        cpu["value_1thread"] = one[0]["trials"] / s1[1]
        cpu["sample_1thread"] = f"{one[0]['blocks']} mid-band blocks, {one[0]['trials']} trials, median of 3 runs"
    except Exception as e:  # the baseline is reported, never required
        cpu = {"value": None, "unit": "trials/s", "cores": 0, "kind": "port", "sample": f"failed: {e}"}
    cfg = workload_config(args.synth)
    cfg["trials_per_step"] = trials
    cfg["profiles_per_step"] = st["profiles"]
    cfg["candidates_per_step"] = res["ncand"]
    cfg["rescued_per_step"] = st["rescued"]
    cfg["device_step"] = ("replayed CUDA graph of the search (cs_set_batch_graph)" if not args.no_graph
                          else "ordinary search call")
    cfg["stage_ms_source"] = "CUDA events between the kernels of 3 ordinary searches of the same workload"
    if res.get("tune"):
        cfg["autotuned"] = res["tune"]
    if args.band:
        cfg["band_hz"] = list(args.band)
    if res["plain"]:
        p = res["plain"]
        cfg["plain_fp32_trials_per_s"] = world * trials / (p["ms"] / 1000.0)
        cfg["plain_fp32_ms_per_step"] = p["ms"]
        cfg["mixed_vs_plain_speedup"] = p["ms"] / (res["ms"] / K)
        cfg["recall_vs_plain"] = 1.0 if p["same_candidates"] else None
        cfg["candidates_identical_to_plain"] = p["same_candidates"]
    out = {"metric": METRIC, "value": value, "unit": "trials/s", "n_gpus": world, "steps": K,
           "warmup": args.warmup, "ms_per_step": res["ms"] / K, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.synth == "fp32" else args.synth,
           "data": "synthetic", "config": cfg,
           "e2e": {"value": e2e, "unit": "trials/s", "h2d_bytes_per_step": res["h2d"] // K,
                   "d2h_bytes_per_step": res["d2h"] // K},
           "gpu_launches": res["launches"], "clocks": res["clocks"], "roofline": roof,
           "peaks_source": psrc, "cpu_baseline": cpu}
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
