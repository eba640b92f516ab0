"""Error against the FP64 oracle, stated per configuration: the small plain
search (one 7.3 Hz pulsar, nharms 32, 1-50 Hz), the precision study (the
same noise with 40 injections, f 0.1-750 Hz, duty 1-30 %, S/N 6-20), and at
nharms 60 with decimation_set(60, 6) over 0.1-125 Hz the survey spectrum
(2^23 samples, six pulsars), a DM-sweep spectrum (2^24 samples) and the
learned-proposal spectrum (2^24 samples, 200 injections).  The amplitude and
S/N samples are chunks across the band, both edges included.

  * amplitudes: the device's FP32 interpolation (Float32 weights, FP32 tap
    chain) against Float64 weights and FP64 accumulation, relative to the RMS
    amplitude of the chunk;
  * S/N: chunk_metrics (FP32 profiles, exact median rescan) against the FP64
    oracle's, |dS/N| / max(S/N, 1);
  * 16-bit gates: the tensor-core (BF16 / FP16) zero-baseline gate against the
    FP32 one over the whole band, |dg| / max(|g|, 1), with single operands and
    with each amplitude split hi + lo into two 16-bit operands.

The bounds asserted are the ones the design states; the measured values are
printed (pytest -s) for the record.
"""
import numpy as np
import pytest

from oracle import cs_ref as o

pytestmark = pytest.mark.gpu


def _configs():
    from cohsearch import synth
    amps1, N, dt = synth.small_config()
    rng = np.random.default_rng(33)
    ps = synth.random_pulsars(rng, 40, 0.1, 750.0, 0.01, 0.30, 6.0, 20.0)
    amps3 = synth.make_spectrum(N, dt, ps, 31)
    return {"config 1 (plain, small)": (amps1, N, dt), "config 3 (40 injections)": (amps3, N, dt)}


def _wide_configs():
    """nharms 60 workloads: (amps, N, dt) per name, built on demand."""
    from cohsearch import synth

    def survey():
        return synth.survey_config(seed=2)

    def dmsweep():
        return [f for f in synth.dmsweep_config(seed=4, per_length=1) if f[1] == 1 << 24][0]

    def learned():
        rng = np.random.default_rng(30_000)
        ps = synth.random_pulsars(rng, 200, 0.1, 750.0, 0.01, 0.20, 6.0, 20.0)
        return synth.make_spectrum_fd(1 << 24, 64e-6, ps, 30_000), 1 << 24, 64e-6

    return {"config 2 (survey)": survey, "config 4 (DM sweep, 2^24 samples)": dmsweep,
            "config 5 (learned, 200 injections)": learned}


def _stats(err):
    err = np.abs(np.asarray(err, np.float64))
    return float(err.max()), float(np.sqrt(np.mean(err ** 2)))


@pytest.mark.parametrize("name", list(_configs()))
def test_error_vs_fp64_oracle(name):
    import cohsearch as cs
    amps, N, dt = _configs()[name]
    T = N * dt
    params = cs.SearchParams(nharms=32, m=16)
    op = o.SearchParams(nharms=32, m=16)
    eng = cs.Engine(params)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    lodr = params.hidr / params.nharms
    amp_err, snr_err = [], []
    for f0 in (1.3, 7.29, 19.0, 33.3, 48.0):
        rstart = f0 * T
        n = 512
        # amplitudes of one chunk: device FP32 vs Float64 weights, FP64 accumulation
        dev = eng.interp_chunk(rstart, 0, n)
        plans = o.build_direct_plans(op, rstart, np.float64)
        ref = o.chunk_stack(plans, amps, op, 0, n, N, np.float64)[:, 1:].T   # (nharms, n)
        scale = np.sqrt(np.mean(np.abs(ref) ** 2))
        amp_err.append(np.abs(dev.astype(np.complex128) - ref).ravel() / scale)
        # exact S/N
        got = eng.chunk_metrics(rstart, n)
        want = o.chunk_metrics(amps, N, op, rstart, n, weights=np.float64)
        snr_err.append((got - want) / np.maximum(np.abs(want), 1.0))
    amax, arms = _stats(np.concatenate(amp_err))
    smax, srms = _stats(np.concatenate(snr_err))
    # 16-bit gates against the FP32 gate, whole band, every level
    dec = cs.decimation_set(32, 4)
    gates = {}
    modes = ("bf16", "fp16", "bf16_split", "fp16_split")
    for mode in ("fp32",) + modes:
        e = cs.Engine(cs.SearchParams(nharms=32, m=16, decimations=dec, synth=mode))
        e.set_diagnostics(2)
        e.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
        e.search_raw(1.0, 50.0, 100, 2048, 8.0)
        gates[mode] = e.gate_values()
    g32 = gates["fp32"]
    live = g32 != 0
    gerr = {m: _stats((gates[m][live] - g32[live]) / np.maximum(np.abs(g32[live]), 1.0)) for m in modes}
    print(f"\n| {name} | amplitude max/RMS {amax:.2e}/{arms:.2e} | S/N max/RMS {smax:.2e}/{srms:.2e} | " +
          " | ".join(f"{m.upper()} gate {gerr[m][0]:.2e}/{gerr[m][1]:.2e}" for m in modes) + " |")
    assert amax < 1e-5
    assert smax <= 1e-3
    assert gerr["fp16"][0] < 2e-2 and gerr["bf16"][0] < 8e-2
    # the split gates sit closer to the FP32 gate; what remains is the
    # twiddle operand's own 16-bit rounding, which the amplitude split leaves
    assert gerr["bf16_split"][0] < gerr["bf16"][0] and gerr["bf16_split"][1] < gerr["bf16"][1]
    assert gerr["fp16_split"][0] < gerr["fp16"][0] and gerr["fp16_split"][1] < gerr["fp16"][1]


@pytest.mark.parametrize("name", list(_wide_configs()))
def test_error_vs_fp64_oracle_nharms60(name):
    """Amplitudes of every harmonic and the exact S/N (base fold, the ladder's
    widths) on chunks from the band's bottom edge (0.1 Hz) to its top (125 Hz,
    whose 60th harmonic sits near Nyquist/1.04), against Float64 weights and
    FP64 accumulation; the 16-bit gates against the FP32 gate over the whole
    band, every level."""
    import cohsearch as cs
    amps, N, dt = _wide_configs()[name]()
    T = N * dt
    dec = cs.decimation_set(60, 6)
    params = cs.SearchParams(nharms=60, m=16, decimations=dec)
    op = o.SearchParams(nharms=60, m=16, decimations=list(dec))
    eng = cs.Engine(params)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    amp_err, snr_err = [], []
    n = 256
    for f0 in (0.1, 3.1, 29.0, 117.0, 125.0 - n * 0.5 / 60 / T):
        rstart = f0 * T
        dev = eng.interp_chunk(rstart, 0, n)
        plans = o.build_direct_plans(op, rstart, np.float64)
        ref = o.chunk_stack(plans, amps, op, 0, n, N, np.float64)[:, 1:].T   # (nharms, n)
        live = np.any(ref != 0, axis=1)        # rows the range guard keeps
        assert np.array_equal(live, np.any(dev != 0, axis=1))
        scale = np.sqrt(np.mean(np.abs(ref[live]) ** 2))
        amp_err.append(np.abs(dev[live].astype(np.complex128) - ref[live]).ravel() / scale)
        got = eng.chunk_metrics(rstart, n)
        want = o.chunk_metrics(amps, N, op, rstart, n, weights=np.float64)
        snr_err.append((got - want) / np.maximum(np.abs(want), 1.0))
    amax, arms = _stats(np.concatenate(amp_err))
    smax, srms = _stats(np.concatenate(snr_err))
    gates = {}
    modes = ("bf16", "fp16", "bf16_split", "fp16_split")
    e32 = cs.Engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth="fp32"))
    e32.set_diagnostics(2)
    e32.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    e32.search_raw(0.1, 125.0, 100, 2048, 8.0)
    g32 = e32.gate_values()
    del e32
    live = g32 != 0
    gerr = {}
    for mode in modes:
        e = cs.Engine(cs.SearchParams(nharms=60, m=16, decimations=dec, synth=mode))
        e.set_diagnostics(2)
        e.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
        e.search_raw(0.1, 125.0, 100, 2048, 8.0)
        g = e.gate_values()
        gerr[mode] = _stats((g[live] - g32[live]) / np.maximum(np.abs(g32[live]), 1.0))
        del e, g
    print(f"\n| {name} | amplitude max/RMS {amax:.2e}/{arms:.2e} | S/N max/RMS {smax:.2e}/{srms:.2e} | " +
          " | ".join(f"{m.upper()} gate {gerr[m][0]:.2e}/{gerr[m][1]:.2e}" for m in modes) + " |")
    assert amax < 1e-5
    assert smax <= 1e-3
    assert gerr["fp16"][0] < 2e-2 and gerr["bf16"][0] < 8e-2
    assert gerr["fp16_split"][1] < gerr["fp16"][1] and gerr["bf16_split"][1] < gerr["bf16"][1]
