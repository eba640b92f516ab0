"""PRESTO ``.inf``/``.fft`` input (mirrors src/fileio.jl) and a writer.

``FFTFile`` maps the ``.fft`` amplitudes (complex64, ``amps[0]`` = DC.re +
i*Nyquist) and reads ``N`` and ``dt`` from the ``.inf``, as
``FFTFile(path)`` does in src/fileio.jl:64-78.
"""
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np


@dataclass
class SimpleInf:
    """The ``.inf`` fields the search needs (src/fileio.jl:12-40)."""
    path: str
    object: Optional[str] = None
    epoch: Optional[float] = None
    N: Optional[int] = None
    dt: Optional[float] = None
    DM: Optional[float] = None

    @classmethod
    def read(cls, path):
        if not os.path.isfile(path):
            raise FileNotFoundError(f"The .inf file '{path}' was not found.")
        out = cls(path=str(path))
        with open(path) as f:
            for line in f:
                val = line.split("=")[-1].strip()
                if line.startswith(" Object being observed"):
                    out.object = val
                elif line.startswith(" Epoch"):
                    out.epoch = float(val)
                elif line.startswith(" Number of bins"):
                    out.N = int(val)
                elif line.startswith(" Width of each time series bin"):
                    out.dt = float(val)
                elif line.startswith(" Dispersion measure"):
                    out.DM = float(val)
        return out


class FFTFile:
    """A memory-mapped PRESTO ``.fft`` plus its ``.inf`` (src/fileio.jl:51-78)."""

    def __init__(self, path):
        path = str(path)
        inf_path = path[:-4] + ".inf"
        inf = SimpleInf.read(inf_path)
        if inf.N is None:
            raise ValueError(f"Missing 'Number of bins' in {inf_path}")
        if inf.dt is None:
            raise ValueError(f"Missing 'Width of each time series bin' in {inf_path}")
        nbytes = os.path.getsize(path)
        n = nbytes // 8
        self.amps = np.memmap(path, dtype=np.complex64, mode="r", shape=(n,)) if n else \
            np.zeros(0, np.complex64)
        self.path = path
        self.inf = inf
        self.N = int(inf.N)
        self.T = self.N * inf.dt
        self.df = 1.0 / self.T
        self.dereddened = "_red.fft" in path
        self.detrended = self.dereddened
        self.DC = float(self.amps[0].real) if n else 0.0
        self.Nyquist = float(self.amps[0].imag) if n else 0.0

    @classmethod
    def from_array(cls, amps, N, dt, path="<memory>"):
        """An in-memory spectrum with the same attributes (no files)."""
        self = cls.__new__(cls)
        self.amps = np.ascontiguousarray(amps, dtype=np.complex64)
        self.path = path
        self.inf = SimpleInf(path=path, N=int(N), dt=float(dt))
        self.N = int(N)
        self.T = self.N * float(dt)
        self.df = 1.0 / self.T
        self.dereddened = self.detrended = False
        self.DC = float(self.amps[0].real) if len(self.amps) else 0.0
        self.Nyquist = float(self.amps[0].imag) if len(self.amps) else 0.0
        return self

    @property
    def dt(self):
        return self.inf.dt

    def freqs(self):
        """Fourier frequencies of bins 0 .. N/2-1 (src/fileio.jl:85)."""
        return np.arange(self.N // 2) * self.df


def freqs(ft):
    return ft.freqs()


def write_fft(stem, amps, N, dt, obj="SYNTH", epoch=50000.0, dm=0.0):
    """Write ``stem.fft`` (raw little-endian complex64) and ``stem.inf``."""
    amps = np.ascontiguousarray(amps, dtype="<c8")
    amps.tofile(stem + ".fft")
    with open(stem + ".inf", "w") as f:
        f.write(f" Object being observed                      =  {obj}\n")
        f.write(f" Epoch of observation (MJD)                 =  {epoch}\n")
        f.write(f" Number of bins in the time series          =  {int(N)}\n")
        f.write(f" Width of each time series bin (sec)        =  {dt!r}\n")
        f.write(f" Dispersion measure (cm-3 pc)               =  {dm}\n")
    return stem + ".fft"
