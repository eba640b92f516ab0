"""Cross-pins of the CPU oracle, restating the reference's data-gated tests
(test/test_search.jl:152-535) on a seeded synthetic pulsar spectrum.

The numpy oracle (FP64) and the C oracle (the Float32-weight production
arithmetic) are independent restatements; agreeing with each other and with
the per-point exact kernel ``fourier_interp`` is what pins them.
"""
import math

import numpy as np
import pytest

from oracle import cs_cpu, cs_ref as o
from tests.fixtures import PSR_F, pulsar_spectrum

PIN_TOL = 1e-8   # test/test_search.jl:20 at the :f64 profile precision


@pytest.fixture(scope="module")
def psr():
    return pulsar_spectrum()


def test_optimised_path_reproduces_exact_kernel_reference(psr):
    """test/test_search.jl:155-199."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=32, m=32)
    lodr = p.hidr / p.nharms
    rstart = 10010.0
    n = 256
    rfund = rstart + np.arange(n) * lodr
    ref = o.block_metrics(amps, N, rfund, p, kernel="direct")
    opt = o.chunk_metrics(amps, N, p, rstart, n, weights=np.float64)
    rel = np.max(np.abs(opt - ref)) / np.max(np.abs(ref))
    assert rel < PIN_TOL
    opt32 = o.chunk_metrics(amps, N, p, rstart, n, weights=np.float32)
    assert np.max(np.abs(opt32 - ref)) / np.max(np.abs(ref)) < 1e-6
    reffft = o.block_metrics(amps, N, rfund, p, kernel="fft")
    assert np.max(np.abs(opt - reffft)) / np.max(np.abs(reffft)) > 1e3 * rel


def test_direct_interp_is_exact_kernel(psr):
    """test/test_search.jl:201-232, for both weight precisions (C oracle = Float32)."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=60, m=32)
    lodr = p.hidr / p.nharms
    rstart, n = 5000.0, 256
    st64 = o.chunk_stack(o.build_direct_plans(p, rstart, np.float64), amps, p, 0, n, N)
    st32 = cs_cpu.interp_chunk(amps, N, 60, 32, p.hidr, rstart, 0, n)
    for stk, tol in ((lambda h, j: st64[j, h], 1e-7), (lambda h, j: st32[h - 1, j], 1e-6)):
        worst = 0.0
        for h in (1, 2, 7, 15, 30, 59, 60):
            for j in (0, 1, 96, n - 1):
                r = h * (rstart + j * lodr)
                v = o.fourier_interp(r, amps, p.m)
                worst = max(worst, abs(stk(h, j) - v) / abs(v))
        assert worst < tol


def test_direct_interp_chunk_invariance(psr):
    """test/test_search.jl:234-276: bit-identical across chunkings, both oracles."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=32, m=32)
    r_lo = 10010.0
    plans = o.build_direct_plans(p, r_lo, np.float32)
    nbig = 384
    big64 = o.chunk_stack(plans, amps, p, 0, nbig, N, np.float32)
    big32 = cs_cpu.interp_chunk(amps, N, 32, 32, p.hidr, r_lo, 0, nbig)
    misaligned = 0
    for nsm in (128, 100, 37, 51):
        misaligned += nsm % o.DIRECT_GROUP_V != 0
        t0 = 0
        while t0 + nsm <= nbig:
            a = o.chunk_stack(plans, amps, p, t0, nsm, N, np.float32)
            assert np.array_equal(a[:, [1, 5, 32]], big64[t0:t0 + nsm][:, [1, 5, 32]])
            c = cs_cpu.interp_chunk(amps, N, 32, 32, p.hidr, r_lo, t0, nsm)
            assert np.array_equal(c, big32[:, t0:t0 + nsm])
            t0 += nsm
    assert misaligned == 3


def test_c_oracle_matches_numpy_oracle_float32(psr):
    """The two restatements of the Float32-weight path agree to FP32 rounding."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=60, m=16)
    r_lo = 4321.7
    st = o.chunk_stack(o.build_direct_plans(p, r_lo, np.float64), amps, p, 777, 300, N)[:, 1:].T
    c = cs_cpu.interp_chunk(amps, N, 60, 16, p.hidr, r_lo, 777, 300)
    scale = np.abs(st).max(axis=1, keepdims=True)
    assert np.max(np.abs(c - st) / scale) < 2e-6
    for h in (1, 7, 60):
        P, W, A, carry = cs_cpu.plan_tables(60, 16, p.hidr, r_lo, h)
        pl = o.build_direct_plans(p, r_lo, np.float32)[h - 1]
        assert P == pl.P and np.array_equal(carry, pl.carry)
        assert np.array_equal(W, pl.W)
        assert np.max(np.abs(A - pl.A)) <= 1e-7


def test_guard_zeroes_rows_past_nyquist(psr):
    """Whole rows stay zero once the chunk's last trial crosses Nyquist
    (src/directinterp.jl:483-496)."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=32, m=16)
    r_lo = N / 2 / 32 - 20.0     # harmonic 32 runs past Nyquist inside the chunk
    c = cs_cpu.interp_chunk(amps, N, 32, 16, p.hidr, r_lo, 0, 4096)
    st = o.chunk_stack(o.build_direct_plans(p, r_lo, np.float32), amps, p, 0, 4096, N)
    zero_c = [h for h in range(1, 33) if not np.any(c[h - 1])]
    zero_o = [h for h in range(1, 33) if not np.any(st[:, h])]
    assert zero_c == zero_o and 32 in zero_c and 1 not in zero_c


def test_decimation_pass_equals_native_fold(psr):
    """test/test_search.jl:445-485."""
    amps, N, dt = psr
    for k in (2, 3, 4):
        nh = 60
        Hk = nh // k
        p = o.SearchParams(nharms=nh, m=32, decimations=[1, k])
        lodr = p.hidr / nh
        rstart, n = 5000.0, 64
        rfund = rstart + np.arange(n) * lodr
        pnat = o.SearchParams(nharms=Hk, m=32)
        wk = o.ladder_boxcar_widths(2 * Hk, k, p)
        ref = o.block_metrics(amps, N, k * rfund, pnat, kernel="direct", widths=wk)
        st = o.chunk_stack(o.build_direct_plans(p, rstart, np.float64), amps, p, 0, n, N)
        dprofs = o.brfft(o.decimated_stack(st, k, nh), 2 * Hk)
        sig = o.block_sigma(dprofs, 2 * Hk, n)
        got = o.profile_boxcar(dprofs, wk, 2 * Hk, 1.0 / sig)
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < PIN_TOL


def test_decimated_stack_is_the_gather(psr):
    """test/test_search.jl:487-510."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=60, decimations=[1, 2, 3, 4, 5, 6])
    st = o.chunk_stack(o.build_direct_plans(p, 5000.0, np.float32), amps, p, 0, 128, N)
    for k in range(2, 7):
        Hk = 60 // k
        want = np.zeros((128, Hk + 1), complex)
        for j in range(1, Hk + 1):
            want[:, j] = st[:, j * k]
        assert np.array_equal(o.decimated_stack(st, k, 60), want)


def test_block_sigma_zero_vs_median_center(psr):
    """test/test_search.jl:311-343."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=60, m=32, decimations=o.decimation_set(60, 6))
    n = 512
    for rstart in (10010.0, 20010.0, 40010.0):
        st = o.chunk_stack(o.build_direct_plans(p, rstart, np.float32), amps, p, 0, n, N)
        for k in p.decimations:
            Hk = 60 // k
            P = o.brfft(o.decimated_stack(st, k, 60), 2 * Hk)
            s0 = o.block_sigma(P, 2 * Hk, n)
            sm = o.block_sigma(P, 2 * Hk, n, center="median")
            assert s0 > 0 and abs(s0 - sm) <= 0.02 * abs(sm)
            assert abs(np.median(P)) < 0.1 * sm


def test_batched_gate_matches_scalar_gate(psr):
    """test/test_search.jl:345-373."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=60, m=32)
    nb, n = 120, 500
    st = o.chunk_stack(o.build_direct_plans(p, 10010.0, np.float32), amps, p, 0, n, N)
    profs = o.brfft(st, nb)
    inv = 1.0 / o.block_sigma(profs, nb, n)
    widths = o.ladder_boxcar_widths(nb, 1, p)
    got = o.boxcar_gate(profs, n, widths, nb, inv)
    want = o.boxcar_scan(o.boxcar_psum(profs, nb, widths[-1], 0.0), widths, nb, inv)
    assert np.max(np.abs(got - want)) < 1e-3 * p.boxcar_medmargin
    tail = n - (n // o.BC_BATCH) * o.BC_BATCH
    assert np.array_equal(got[n - tail:], want[n - tail:])


def test_gate_does_not_change_candidates(psr):
    """test/test_search.jl:287-309: gated and exact searches give identical lists."""
    amps, N, dt = psr
    kw = dict(lofreq=9.9, hifreq=10.1, threshold=6.0, blocksize=512)
    g = o.search(amps, N, dt, o.SearchParams(nharms=60, m=32, decimations=o.decimation_set(60, 4)), **kw)
    e = o.search(amps, N, dt, o.SearchParams(nharms=60, m=32, decimations=o.decimation_set(60, 4),
                                             boxcar_medmargin=math.inf), **kw)
    assert len(g) == len(e) and len(g) > 0
    assert all(a.freq == b.freq and a.nharm == b.nharm and a.metric == b.metric for a, b in zip(g, e))


def test_oracle_detects_the_pulsar(psr):
    """test/test_search.jl:378-385 and :560-582 (dedup keeps the strongest)."""
    amps, N, dt = psr
    p = o.SearchParams(nharms=32, m=32)
    c = o.search(amps, N, dt, p, lofreq=9.9, hifreq=10.1, threshold=8.0)
    best = max(c, key=lambda x: x.metric)
    assert abs(best.freq - PSR_F) < 1e-2
    raw = o.search(amps, N, dt, p, lofreq=9.9, hifreq=10.1, threshold=8.0, remove=False,
                   harm_remove=False)
    assert len(c) < len(raw)
    rb = max(raw, key=lambda x: x.metric)
    dd = o.remove_duplicates(raw)
    db = max(dd, key=lambda x: x.metric)
    assert db.freq == rb.freq and db.metric == rb.metric


@pytest.mark.parametrize("nharms,maxdecim,band", [(32, 4, (1.0, 60.0)), (60, 6, (0.1, 3.0)),
                                                  (32, 4, (3890.0, 3920.0)), (20, 3, (5.0, 12.0))])
def test_c_port_search_equals_numpy_oracle(nharms, maxdecim, band):
    """The two restatements of `_search_region!` (src/search.jl:1768-1894) over
    every block of a band: the C port (the timed CPU baseline and the checker
    of the full-size GPU runs: threaded, batched FP32 gate, its own c2r
    transform) and the numpy oracle (one task, numpy's irfft).  Their FP32
    interpolations round differently (sequential fmaf against numpy's float32
    sums), so: valid trial counts exact, block sigma and S/N within 1e-5,
    candidate (block, k, trial) sets equal outside |S/N - thr| < 1e-5 thr.
    The bands cover the decimated levels' Nyquist cut
    (3890-3920 Hz: 2f crosses N/2 mid-band, every harmonic from the 2nd up
    lies beyond the spectrum), the six bin counts 120..20 of nharms 60, and
    nharms 20 (profiles of 40, 20 and 12 bins)."""
    from tests.fixtures import multi_spectrum
    amps, N, dt = multi_spectrum()
    dec = o.decimation_set(nharms, maxdecim)
    thr = 7.0
    op = o.SearchParams(nharms=nharms, m=16, decimations=dec, threshold=thr)
    T, lodr, r_lo, r_hi, total, Nprof = o.search_setup(N, dt, op, band[0], band[1], 100, 2048)
    cands, blocks = o.search_region(amps, N, T, op, r_lo, r_hi, total, Nprof, thr, thr - op.boxcar_medmargin,
                                    keep_blocks=True)
    port = cs_cpu.search_blocks_ex(amps, N, dt, nharms, 16, op.hidr, dec, r_lo, total, 2048, thr, 3)
    levk = [1] + [k for k in dec if k > 1]
    nblk = -(-total // 2048)
    nv = np.zeros((nblk, len(levk)), np.int32)
    sig = np.zeros((nblk, len(levk)))
    for b in blocks:
        nv[b.block, levk.index(b.k)] = b.nvalid
        sig[b.block, levk.index(b.k)] = b.sigma
    assert np.array_equal(port["nvalid"], nv)
    assert np.any(nv[:, -1] < np.minimum(2048, total - 2048 * np.arange(nblk))) == (band[0] > 1000)
    assert np.allclose(port["sigma"], sig, rtol=1e-5, atol=0.0)
    want = {(c[0], c[1], c[2]): c[3].metric for c in cands}
    got = {(int(c["blk"]), int(c["k"]), int(c["j"])): float(c["metric"]) for c in port["cands"]}
    assert len(want) > 0
    edge = thr * (1 + 1e-5)
    for key in set(want) ^ set(got):
        assert max(want.get(key, 0.0), got.get(key, 0.0)) < edge, key
    for key in set(want) & set(got):
        assert abs(got[key] - want[key]) <= 1e-5 * want[key], (key, got[key], want[key])


@pytest.mark.parametrize("H", [1, 2, 3, 4, 5, 6, 7, 8, 10, 11, 12, 15, 16, 20, 30, 32, 45, 60, 64, 120])
def test_c_port_transform_equals_irfft(H):
    """The C port's profile-stage transform (mixed-radix FFT; direct DFT for
    lengths with a prime factor above 5) against numpy's irfft: the
    unnormalised brfft of (0, X[1..H]) with the imaginary part of Nyquist
    dropped (src/search.jl:1291, :1675), for lane counts below, at and above
    the port's lane tile."""
    rng = np.random.default_rng(H)
    for n in (1, 63, 64, 65, 200):
        X = rng.standard_normal((H + 1, n)) + 1j * rng.standard_normal((H + 1, n))
        got, nst = cs_cpu.c2r(X)
        X[0] = 0.0
        want = np.fft.irfft(X, 2 * H, axis=0) * (2 * H)
        assert np.max(np.abs(got - want)) <= 1e-14 * np.max(np.abs(want)), (H, n)
        smooth = all(f in (2, 3, 5) for f in _factors(H))
        assert (nst > 0) == (smooth and H > 1), (H, nst)


def _factors(n):
    out, f = [], 2
    while n > 1:
        while n % f == 0:
            out.append(f)
            n //= f
        f += 1
    return out


@pytest.mark.parametrize("e", [17, -36])
def test_c_port_search_is_scale_invariant(e):
    """The checker of the device's scale tests: the C port's search of a
    spectrum scaled by 2^e returns the unscaled spectrum's records bit for bit
    (a power of two scales every FP32 and FP64 value of the search exactly,
    and the S/N is a ratio)."""
    from tests.fixtures import multi_spectrum
    amps, N, dt = multi_spectrum()
    dec = o.decimation_set(60, 6)
    op = o.SearchParams(nharms=60, m=16, decimations=dec)
    T, lodr, r_lo, r_hi, total, Nprof = o.search_setup(N, dt, op, 0.2, 30.0, 100, 2048)
    scaled = (np.asarray(amps) * np.float32(2.0 ** e)).astype(np.complex64)
    runs = [cs_cpu.search_blocks_ex(a, N, dt, 60, 16, op.hidr, dec, r_lo, total, 2048, 8.0, 2)
            for a in (amps, scaled)]
    want, got = (np.sort(r["cands"], order=["blk", "k", "j"]) for r in runs)
    assert len(want) > 0 and np.array_equal(got, want)
    assert np.array_equal(runs[1]["sigma"], runs[0]["sigma"] * 2.0 ** e)
