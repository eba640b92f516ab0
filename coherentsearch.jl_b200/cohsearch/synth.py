"""Seeded synthetic PRESTO spectra with injected pulsars.

The time series is white Gaussian noise (unit variance) plus, per pulsar, a
train of Gaussian pulses of full width at half maximum ``duty`` (as a
fraction of the period) at frequency ``f`` and phase ``phase``.  Its real FFT
is normalised so that noise bins have E|X|^2 = 1 (Re, Im variance 1/2) and
packed as PRESTO does (``amps[0]`` = DC.re + i*Nyquist.re, N/2 values).

The pulse amplitude is set from a nominal coherent S/N:
``A = snr / sqrt(N * 1.0645 * duty)`` -- the boxcar matched-filter S/N of a
Gaussian pulse folded from N samples (1.0645*duty is its area in periods).
The S/N the search reports is lower by the interpolation, grid and
harmonic-truncation losses.
"""
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np


@dataclass
class Pulsar:
    freq: float        # Hz
    duty: float        # FWHM as a fraction of the period
    snr: float         # nominal coherent S/N
    phase: float = 0.0


def gaussian_train(n: int, dt: float, p: Pulsar, amp: float, chunk: int = 1 << 22) -> np.ndarray:
    sig = p.duty / (2.0 * np.sqrt(2.0 * np.log(2.0)))
    out = np.empty(n, dtype=np.float64)
    for s in range(0, n, chunk):
        t = np.arange(s, min(n, s + chunk), dtype=np.float64) * dt
        ph = p.freq * t + p.phase
        d = ph - np.round(ph)
        out[s:s + len(t)] = amp * np.exp(-0.5 * (d / sig) ** 2)
    return out


def make_spectrum(nsamp: int, dt: float, pulsars: Sequence[Pulsar] = (), seed: int = 0) -> np.ndarray:
    """Return the packed complex64 spectrum (nsamp // 2 values)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(nsamp)
    for p in pulsars:
        amp = p.snr / np.sqrt(nsamp * 1.0645 * p.duty)
        x += gaussian_train(nsamp, dt, p, amp)
    X = np.fft.rfft(x) / np.sqrt(nsamp)
    amps = X[: nsamp // 2].astype(np.complex64)
    amps[0] = np.complex64(complex(X[0].real, X[nsamp // 2].real))
    return amps


def make_spectrum_fd(nsamp: int, dt: float, pulsars: Sequence[Pulsar] = (), seed: int = 0,
                     halfwidth: int = 8) -> np.ndarray:
    """The make_spectrum model synthesised in the frequency domain, in
    milliseconds instead of seconds (training sets of many spectra): bins of
    unit-variance complex Gaussian noise (E|X|^2 = 1), plus for each pulsar and
    harmonic h the Gaussian train's Fourier coefficient
    a_h = amp * 1.0645 * duty * exp(-(pi h duty)^2 / (4 ln 2)) * exp(2 pi i h phase)
    (amp as in make_spectrum) times sqrt(nsamp) times the response of a
    finite-length sinusoid at fractional bin r = h f T, sinc(r - k) e^{i pi (r - k)},
    over the `halfwidth` bins either side of r."""
    rng = np.random.default_rng(seed)
    nb = nsamp // 2
    amps = ((rng.standard_normal(nb) + 1j * rng.standard_normal(nb)) * np.sqrt(0.5)).astype(np.complex128)
    T = nsamp * dt
    for p in pulsars:
        amp = p.snr / np.sqrt(nsamp * 1.0645 * p.duty)
        hmax = int(min(np.floor((nb - halfwidth - 1) / (p.freq * T)),
                       np.ceil(3.0 * np.sqrt(4.0 * np.log(2.0)) / (np.pi * p.duty))))
        if hmax < 1:
            continue
        h = np.arange(1, hmax + 1)
        ah = (amp * 1.0645 * p.duty * np.exp(-(np.pi * h * p.duty) ** 2 / (4.0 * np.log(2.0)))
              * np.exp(2j * np.pi * h * p.phase) * np.sqrt(nsamp))
        r = h * p.freq * T
        k = np.floor(r)[:, None].astype(np.int64) + np.arange(-halfwidth + 1, halfwidth + 1)[None, :]
        d = r[:, None] - k
        resp = np.sinc(d) * np.exp(1j * np.pi * d)
        ok = (k >= 1) & (k < nb)
        np.add.at(amps, k[ok], (ah[:, None] * resp)[ok])
    return amps.astype(np.complex64)


def random_pulsars(rng: np.random.Generator, n: int, fmin: float, fmax: float, dmin: float,
                   dmax: float, smin: float, smax: float) -> List[Pulsar]:
    """Log-uniform frequency and duty, uniform S/N and phase."""
    f = np.exp(rng.uniform(np.log(fmin), np.log(fmax), n))
    d = np.exp(rng.uniform(np.log(dmin), np.log(dmax), n))
    s = rng.uniform(smin, smax, n)
    ph = rng.uniform(0, 1, n)
    return [Pulsar(float(a), float(b), float(c), float(e)) for a, b, c, e in zip(f, d, s, ph)]


# The configurations the benchmarks and tests use (sizes, pulsars, bands).
def small_config(seed: int = 1):
    """2^21 samples at 64 us, one 7.3 Hz 5%-duty pulsar (nominal S/N 15);
    searched with nharms=32, no decimation, 1-50 Hz, threshold 8."""
    nsamp, dt = 1 << 21, 64e-6
    amps = make_spectrum(nsamp, dt, [Pulsar(7.3, 0.05, 15.0, 0.25)], seed)
    return amps, nsamp, dt


def survey_config(seed: int = 2):
    """2^23 samples at 64 us with six pulsars (0.37-702 Hz, duty 2-20%, S/N
    7-25); searched with nharms=60, decimation_set(60, 6), 0.1-125 Hz, threshold 8."""
    nsamp, dt = 1 << 23, 64e-6
    psr = [Pulsar(0.37, 0.02, 25.0, 0.1), Pulsar(3.1, 0.05, 12.0, 0.3), Pulsar(29.0, 0.10, 7.0, 0.5),
           Pulsar(117.0, 0.08, 15.0, 0.7), Pulsar(341.0, 0.15, 20.0, 0.2), Pulsar(702.0, 0.20, 10.0, 0.9)]
    amps = make_spectrum(nsamp, dt, psr, seed)
    return amps, nsamp, dt


def dmsweep_config(seed: int = 4, lengths=(1 << 21, 1 << 22, 1 << 23, 1 << 24), per_length: int = 16,
                   dt: float = 64e-6):
    """A batched DM sweep: `per_length` spectra of each length, each with 0-3
    pulsars drawn like the precision study (f log-uniform 0.1-750 Hz, duty
    log-uniform 1-30 %, S/N uniform 6-20).  Returns [(amps, N, dt)]."""
    rng = np.random.default_rng(seed)
    files = []
    for n in lengths:
        for _ in range(per_length):
            ps = random_pulsars(rng, int(rng.integers(0, 4)), 0.1, 750.0, 0.01, 0.30, 6.0, 20.0)
            files.append((make_spectrum(n, dt, ps, int(rng.integers(1 << 31))), n, dt))
    return files
