"""PRESTO .fft/.inf input and the command line's output naming, on the host
(src/fileio.jl:12-85, src/cli.jl:263-270; test/test_cli.jl:28-43).

A synthetic observation is written to disk with ``write_fft`` and read back
with ``FFTFile(path)``: the amplitudes bit for bit, ``amps[0]`` packing DC and
Nyquist, N, T = N*dt and the Fourier frequencies.
"""
import os

import numpy as np
import pytest

import cohsearch as cs


def _synthetic(N=1 << 15, bin0=210):
    """The reference's on-disk fixture (test/test_cli.jl:12-28): flat
    0.5 + 0.5i amplitudes plus a bright harmonic series at bin0*h."""
    nfreq = N // 2
    amps = np.full(nfreq, 0.5 + 0.5j, np.complex64)
    for h in range(1, 9):
        b = bin0 * h
        if b < nfreq:
            amps[b] = np.complex64(60.0 / h)
    return amps


def test_fft_inf_round_trip(tmp_path):
    N, dt = 1 << 15, 1.0e-4
    amps = _synthetic(N)
    amps[0] = np.complex64(123.25 - 7.5j)        # DC.re + i*Nyquist
    path = cs.write_fft(str(tmp_path / "synth"), amps, N, dt)
    ft = cs.FFTFile(path)
    assert ft.N == N and ft.dt == dt and ft.T == N * dt
    assert len(ft.amps) == N // 2
    assert np.array_equal(np.asarray(ft.amps).view(np.uint64), amps.view(np.uint64))
    assert ft.DC == 123.25 and ft.Nyquist == -7.5
    assert ft.inf.object == "SYNTH" and ft.inf.DM == 0.0
    assert np.array_equal(ft.freqs(), np.arange(N // 2) / (N * dt))
    assert not ft.dereddened


def test_truncated_fft_reads_what_is_there(tmp_path):
    """A .fft holding fewer than N/2 amplitudes (namps < N/2) keeps N from the
    .inf: T and the Nyquist bin follow N, the amplitudes what the file holds."""
    N, dt = 1 << 15, 1.0e-4
    amps = _synthetic(N)[: 5000]
    ft = cs.FFTFile(cs.write_fft(str(tmp_path / "short"), amps, N, dt))
    assert ft.N == N and len(ft.amps) == 5000 and ft.T == N * dt


def test_missing_inf_fields_raise(tmp_path):
    stem = str(tmp_path / "bad")
    np.zeros(8, np.complex64).tofile(stem + ".fft")
    with open(stem + ".inf", "w") as f:
        f.write(" Object being observed                      =  X\n")
    with pytest.raises(ValueError):
        cs.FFTFile(stem + ".fft")
    with pytest.raises(FileNotFoundError):
        cs.FFTFile(str(tmp_path / "nothing.fft"))


def test_output_path_resolution():
    """test/test_cli.jl:28-43."""
    assert cs.output_path("/data/obs_DM12.fft", "", "", 1) == ""
    assert cs.output_path("/data/obs_DM12.fft", "cands.txt", "", 1) == "cands.txt"
    assert cs.output_path("/data/obs_DM12.fft", "", "", 3) == "/data/obs_DM12.cohout"
    assert cs.output_path("/data/obs_DM12.fft", "", "/out", 1) == "/out/obs_DM12.cohout"
    assert cs.output_path("/data/obs_DM12.fft", "", "/out", 3) == "/out/obs_DM12.cohout"
    assert cs.output_path("/d/PM0063_DM445.0_red.fft", "", "", 2) == "/d/PM0063_DM445.0_red.cohout"


def test_cohout_table_format(tmp_path):
    """write_candidates (src/cli.jl:317-340): header, then fixed-width rows;
    an unmeasured duty cycle prints as '-'."""
    cands = [cs.Candidate(7.3, 15.254, 3920.0, 32, 0.0625), cs.Candidate(123.0, 9.0, 66059.0, 8)]
    out = str(tmp_path / "x.cohout")
    cs.write_candidates(cands, out, 8.0)
    lines = open(out).read().splitlines()
    assert lines[0] == "#       'S/N'      Frequency (Hz)        Period (ms)    #Harm  Ducy(%)"
    assert lines[1] == f"1        15.25  {7.3:18.12f}  {1000.0 / 7.3:18.12f}    32     6.25"
    assert lines[2].split() == ["2", "9.00", f"{123.0:.12f}", f"{1000.0 / 123.0:.12f}", "8", "-"]
    assert len(lines) == 3


def test_several_files_reject_one_output_name(tmp_path):
    paths = [cs.write_fft(str(tmp_path / f"obs_DM{d}.0"), _synthetic(), 1 << 15, 1e-4) for d in (10, 20)]
    with pytest.raises(ValueError):
        cs.search_files(paths, cs.SearchParams(nharms=8), outputfilenm=str(tmp_path / "x.txt"))
    assert not os.path.exists(str(tmp_path / "x.txt"))
