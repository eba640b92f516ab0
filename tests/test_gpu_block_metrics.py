"""block_metrics over arbitrary trial fundamentals on the device (the reference
path, src/search.jl:933-1097) against the numpy FP64 oracle.

Tolerance: both sides are FP64; they differ by the order of the FP64 sums, the
device's sinpi/cospi against the oracle's exact-reduction ones and, for the
`:fft` kernel, the FFT correlation's rounding against the device's direct grid
sums -- |dS/N| <= 1e-9 * max(S/N, 1).  The production relation the reference
pins (chunk_metrics vs block_metrics(:direct), test/test_search.jl) is checked
at the FP32 path's tolerance, 1e-3.
"""
import numpy as np
import pytest

from oracle import cs_ref as o
from tests.fixtures import PSR_F, pulsar_spectrum

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _cs():
    import cohsearch
    return cohsearch


def _close(got, want, tol):
    return np.all(np.abs(got - want) <= tol * np.maximum(np.abs(want), 1.0))


@pytest.mark.parametrize("kernel", ["fft", "direct"])
@pytest.mark.parametrize("nharms,m", [(32, 16), (60, 32)])
def test_block_metrics_vs_oracle(kernel, nharms, m):
    cs = _cs()
    amps, N, dt = pulsar_spectrum()
    T = N * dt
    rng = np.random.default_rng(nharms + m)
    # off-grid fundamentals around the pulsar and a few tens of bins either side
    r0 = PSR_F * T
    rfund = np.sort(np.concatenate([r0 + rng.uniform(-3.0, 3.0, 200), r0 + rng.uniform(-60.0, 60.0, 56)]))
    params = cs.SearchParams(nharms=nharms, m=m)
    got = cs.block_metrics(cs.FFTFile.from_array(amps, N, dt), rfund, params, kernel=kernel)
    want = o.block_metrics(amps, N, rfund, o.SearchParams(nharms=nharms, m=m), kernel=kernel)
    assert got.shape == want.shape
    assert _close(got, want, TOL), np.max(np.abs(got - want))


def test_block_metrics_widths_and_search_block():
    cs = _cs()
    amps, N, dt = pulsar_spectrum()
    T = N * dt
    rfund = PSR_F * T + np.linspace(-2.0, 2.0, 300)
    params = cs.SearchParams(nharms=32, m=16)
    ft = cs.FFTFile.from_array(amps, N, dt)
    op = o.SearchParams(nharms=32, m=16)
    widths = [1, 2, 4, 8, 16]
    got = cs.block_metrics(ft, rfund, params, kernel="direct", widths=widths)
    want = o.block_metrics(amps, N, rfund, op, kernel="direct", widths=widths)
    assert _close(got, want, TOL)
    cands = cs.search_block(ft, rfund, params, threshold=8.0)
    ref = o.search_block(amps, N, T, rfund, op, threshold=8.0)
    assert [c.r for c in cands] == [c.r for c in ref]
    assert all(abs(a.metric - b.metric) <= TOL * max(abs(b.metric), 1.0) for a, b in zip(cands, ref))
    assert any(abs(c.freq - PSR_F) < 1e-3 for c in cands)


def test_block_metrics_direct_pins_chunk_metrics():
    """chunk_metrics (production FP32 path) equals block_metrics(:direct) on the
    same trial grid, the equivalence the reference's optimised path is pinned to."""
    cs = _cs()
    amps, N, dt = pulsar_spectrum()
    params = cs.SearchParams(nharms=32, m=16)
    lodr = params.hidr / params.nharms
    rstart, n = 10010.0, 256
    eng = cs.Engine(params)
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    chunk = eng.chunk_metrics(rstart, n)
    ref = eng.block_metrics(rstart + np.arange(n) * lodr, kernel="direct")
    assert _close(chunk, ref, 1e-3)


def test_block_metrics_errors():
    cs = _cs()
    amps, N, dt = pulsar_spectrum()
    eng = cs.Engine(cs.SearchParams(nharms=32, m=16))
    eng.set_spectrum(cs.FFTFile.from_array(amps, N, dt))
    with pytest.raises(ValueError):
        eng.block_metrics(np.array([-1.0, 5.0]), kernel="direct")
    with pytest.raises(ValueError):
        eng.block_metrics(np.array([100.0]), kernel="fast")
    assert eng.block_metrics(np.zeros(0)).size == 0
