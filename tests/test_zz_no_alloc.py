"""cs_chunk_metrics_static -- chunk metrics that allocate no device memory --
against cs_chunk_metrics, through the C ABI.

The file name makes pytest collect it last, so in a full run it executes after
every other test in the same process; it also passes alone in a fresh process.
Tolerance: the S/N tolerance of the device parity tests, |dS/N| <= 1e-3 S/N.
"""
import ctypes

import numpy as np
import pytest

from tests.fixtures import pulsar_spectrum

pytestmark = pytest.mark.gpu

SNR_RTOL = 1e-3
CS_ERR_INVALID_ARGUMENT = 1
CS_ERR_CAPACITY = 3


def _lib():
    from cohsearch import _lib
    return _lib.load()


def _device_spectrum(amps):
    import torch
    return torch.from_numpy(np.ascontiguousarray(amps).view(np.float32).copy()).cuda()


def _static(params, d_amps, namps, N, rstart, n):
    """One call of the allocation-free entry point; NaN-filled output so that
    an unwritten trial cannot pass."""
    import torch
    out = torch.full((int(n),), float("nan"), dtype=torch.float32, device="cuda")
    err = ctypes.create_string_buffer(512)
    cp = params.to_c()
    st = _lib().cs_chunk_metrics_static(ctypes.byref(cp), d_amps.data_ptr(), int(namps), int(N), float(rstart),
                                        int(n), out.data_ptr(), torch.cuda.current_stream().cuda_stream,
                                        err, len(err))
    torch.cuda.synchronize()
    return st, out.cpu().numpy().astype(np.float64), err.value.decode()


def _handle_metrics(params, amps, N, dt, rstart, n):
    import cohsearch as cs
    eng = cs.Engine(params)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    return eng.chunk_metrics(rstart, n)


def test_static_matches_chunk_metrics_two_calls():
    """Two calls in a row with different plans and lengths (the second
    overwrites the first's tables in the shared array), each against the
    handle-based entry point on the same inputs."""
    import cohsearch as cs
    amps, N, dt = pulsar_spectrum()
    d_amps = _device_spectrum(amps)
    cases = [(cs.SearchParams(nharms=60, m=16), 5000.0, 2048),
             (cs.SearchParams(nharms=32, m=32), 10010.0, 256)]
    for params, rstart, n in cases:
        st, got, msg = _static(params, d_amps, len(amps), N, rstart, n)
        assert st == 0, msg
        want = _handle_metrics(params, amps, N, dt, rstart, n)
        assert np.all(np.isfinite(got))
        assert np.all(np.abs(got - want) <= SNR_RTOL * np.maximum(np.abs(want), 1.0))


def test_static_call_allocates_no_device_memory():
    """After a first call (which looks up the array's address), a second call
    leaves the device's free memory exactly as it was: no cudaMalloc, no
    allocating library routine on the path."""
    import torch
    import cohsearch as cs
    amps, N, dt = pulsar_spectrum()
    d_amps = _device_spectrum(amps)
    params = cs.SearchParams(nharms=60, m=16)
    cp = params.to_c()
    out = torch.empty(2048, dtype=torch.float32, device="cuda")
    err = ctypes.create_string_buffer(512)
    lib = _lib()

    def call():
        return lib.cs_chunk_metrics_static(ctypes.byref(cp), d_amps.data_ptr(), len(amps), int(N), 5000.0, 2048,
                                           out.data_ptr(), torch.cuda.current_stream().cuda_stream, err, len(err))

    assert call() == 0, err.value.decode()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    assert call() == 0, err.value.decode()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.all(np.isfinite(out.cpu().numpy()))


def test_static_rejects_oversize_requests():
    import cohsearch as cs
    amps, N, dt = pulsar_spectrum()
    d_amps = _device_spectrum(amps)
    # Trial grid 1/4999: 8 harmonics x 4999 phase rows x 32 taps of FP32
    # weights is 5.1 MB of plan tables, above the 4 MiB array.
    big = cs.SearchParams(nharms=8, m=32, hidr=8.0 / 4999.0)
    st, _, msg = _static(big, d_amps, len(amps), N, 5000.0, 64)
    assert st == CS_ERR_CAPACITY and "scratch" in msg
    st, _, msg = _static(cs.SearchParams(nharms=32, m=32), d_amps, len(amps), N, 5000.0, (1 << 16) + 1)
    assert st == CS_ERR_INVALID_ARGUMENT
    # a start with no bin: NaN, infinite or negative
    for bad in (float("nan"), float("inf"), -1.0):
        st, _, msg = _static(cs.SearchParams(nharms=32, m=32), d_amps, len(amps), N, bad, 256)
        assert st == CS_ERR_INVALID_ARGUMENT and "rstart" in msg
    # the array is still usable after a rejected call
    st, got, msg = _static(cs.SearchParams(nharms=32, m=32), d_amps, len(amps), N, 10010.0, 256)
    assert st == 0, msg
    want = _handle_metrics(cs.SearchParams(nharms=32, m=32), amps, N, dt, 10010.0, 256)
    assert np.all(np.abs(got - want) <= SNR_RTOL * np.maximum(np.abs(want), 1.0))
