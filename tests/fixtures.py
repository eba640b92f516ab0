"""Seeded synthetic spectra shared by the tests.

``pulsar_spectrum`` stands in for the reference's data-gated fixture
``harmonics_hi.fft`` (a 10.0123456789123 Hz fake pulsar, N = 1,000,000,
dt = 1 ms; test/test_fileio.jl:12-14), which is not available here: same
frequency, sample time and (rounded to 2^20) length, strong narrow pulses on
unit-variance noise.
"""
import functools

import numpy as np

from cohsearch import synth

PSR_F = 10.0123456789123


@functools.lru_cache(maxsize=None)
def pulsar_spectrum(nsamp=1 << 20, dt=1e-3, snr=60.0, duty=0.03, seed=11):
    amps = synth.make_spectrum(nsamp, dt, [synth.Pulsar(PSR_F, duty, snr, 0.2)], seed)
    amps.setflags(write=False)
    return amps, nsamp, dt


@functools.lru_cache(maxsize=None)
def noise_spectrum(nsamp=1 << 18, dt=64e-6, seed=5):
    amps = synth.make_spectrum(nsamp, dt, [], seed)
    amps.setflags(write=False)
    return amps, nsamp, dt


@functools.lru_cache(maxsize=None)
def multi_spectrum(nsamp=1 << 19, dt=64e-6, seed=7):
    """A few pulsars across the band, for decimation and candidate tests."""
    psr = [synth.Pulsar(3.3, 0.05, 18.0, 0.1), synth.Pulsar(41.7, 0.10, 14.0, 0.6),
           synth.Pulsar(123.4, 0.2, 16.0, 0.3)]
    amps = synth.make_spectrum(nsamp, dt, psr, seed)
    amps.setflags(write=False)
    return amps, nsamp, dt
