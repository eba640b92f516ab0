"""CPU oracle for the coherent-search hot path -- TEST INFRASTRUCTURE ONLY.

A numpy FP64 restatement of CoherentSearch.jl's search hot path, written from
the reference's source and used only as the checker: by ``tests/``, by
``__graft_entry__.smoke()`` and by ``bench.py``'s ``cpu_baseline`` leg.  The
product (``libcohsearch_cuda.so`` and the ``cohsearch`` host package) never
imports it and has no CPU fallback.

Parity is pinned against the known-answer vectors of the reference's own test
suite (``test/test_fourierinterp.jl``, ``test/test_search.jl``), which
``tests/golden/make_reference_kats.py`` extracts into ``tests/golden/``; the
reference itself (Julia) cannot run on this machine.

Conventions.  Spectra are 0-based numpy ``complex64``/``complex128`` vectors
(``amps[0]`` packs DC.re + i*Nyquist, as PRESTO writes them).  Profile
matrices are ``(n, nbins)`` row-major -- one profile per row -- which has the
same linear order as the reference's column-major ``(nbins, n)`` matrices, so
the block-sigma subsample indices carry over unchanged.  Every function cites
the reference file:line it restates.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

# ---------------------------------------------------------------------------
# Parameters  (src/search.jl:131-167)
# ---------------------------------------------------------------------------


@dataclass
class SearchParams:
    """Restates ``SearchParams`` (src/search.jl:131-144); same defaults."""
    nharms: int = 32
    m: int = 16
    numbetween: int = 16
    hidr: float = 0.5
    threshold: float = 8.0
    boxcar_fsp: float = 1.5
    boxcar_maxfrac: float = 0.3
    boxcar_medmargin: float = 2.0
    decimations: List[int] = field(default_factory=lambda: [1])
    precision: str = "f64"


def proftype(params: SearchParams):
    """src/search.jl:152-156."""
    if params.precision == "f64":
        return np.float64
    if params.precision == "f32":
        return np.float32
    raise ValueError(f"precision must be f64 or f32, got {params.precision}")


def decimation_set(nharms: int, maxdecim: int) -> List[int]:
    """src/search.jl:166-167: k in 1:max(1,maxdecim) with fld(nharms,k) >= 2."""
    return [k for k in range(1, max(1, maxdecim) + 1) if nharms // k >= 2]


# ---------------------------------------------------------------------------
# Exact-reduction sin(pi x) / cos(pi x): Julia's sinpi/cispi/sinc are accurate
# near integers (where the interpolation weights blow up), so the oracle
# reduces x - round(x) exactly before multiplying by pi.
# ---------------------------------------------------------------------------


def sinpi(x):
    x = np.asarray(x, dtype=np.float64)
    n = np.rint(x)
    f = x - n
    sgn = np.where(np.fmod(np.abs(n), 2.0) == 1.0, -1.0, 1.0)
    return sgn * np.sin(np.pi * f)


def cospi(x):
    x = np.asarray(x, dtype=np.float64)
    n = np.rint(x)
    f = x - n
    sgn = np.where(np.fmod(np.abs(n), 2.0) == 1.0, -1.0, 1.0)
    return sgn * np.cos(np.pi * f)


def cispi(x):
    return cospi(x) + 1j * sinpi(x)


def sinc(x):
    x = np.asarray(x, dtype=np.float64)
    safe = np.where(x == 0.0, 1.0, x)
    return np.where(x == 0.0, 1.0, sinpi(safe) / (np.pi * safe))


# ---------------------------------------------------------------------------
# Exact Fourier interpolation  (src/fourierinterp.jl)
# ---------------------------------------------------------------------------


def finterp_coeffs(dr: float, m: int) -> np.ndarray:
    """src/fourierinterp.jl:23-31: sinc(dr-j)*cispi(dr-j), j = -m/2+1 .. m/2."""
    if m % 2:
        raise ValueError("m must be even")
    if not (0.0 <= dr < 1.0):
        raise ValueError("dr must be in [0.0, 1.0)")
    off = dr - np.arange(-(m // 2) + 1, m // 2 + 1, dtype=np.float64)
    return sinc(off) * cispi(off)


def nearby_fourier_bin_range(r: float, m: int) -> Tuple[int, int]:
    """src/fourierinterp.jl:44-50, as a 0-based half-open slice ``[lo, hi)``.

    The reference returns the 1-based inclusive range ``(lo+1):hi``.
    """
    if m % 2:
        raise ValueError("m must be even")
    r_int = math.floor(r + 1e-15) + 1
    return r_int - m // 2, r_int + m // 2


def nearby_fourier_bins(r: float, ft: np.ndarray, m: int) -> np.ndarray:
    """src/fourierinterp.jl:57-59."""
    lo, hi = nearby_fourier_bin_range(r, m)
    return ft[lo:hi]


def fourier_interp(r: float, ft: np.ndarray, m: int) -> complex:
    """src/fourierinterp.jl:66-74: sum conj(coeffs) .* bins."""
    if r < 0:
        raise ValueError("r must be non-negative")
    if m % 2:
        raise ValueError("m must be even")
    coeffs = finterp_coeffs(math.fmod(r, 1.0), m)
    bins = nearby_fourier_bins(r, ft, m).astype(np.complex128)
    return complex(np.sum(np.conj(coeffs) * bins))


def finterp_multi(rs: Sequence[float], ft: np.ndarray, m: int) -> np.ndarray:
    """src/fourierinterp.jl:82-97."""
    rs = np.asarray(rs, dtype=np.float64)
    if m % 2:
        raise ValueError("m must be even")
    lo = math.floor(rs.min() + 1e-15)
    hi = math.floor(rs.max() + 1e-15)
    if hi != lo:
        raise ValueError("rs must all be between 2 Fourier bins")
    off = np.fmod(rs, 1.0)[:, None] - np.arange(-(m // 2) + 1, m // 2 + 1)[None, :]
    coeffs = sinc(off) * cispi(off)
    bins = nearby_fourier_bins(rs[0], ft, m).astype(np.complex128)
    return np.conj(coeffs) @ bins


def next_pow_of_2(n: int) -> int:
    """src/fourierinterp.jl:104-107."""
    if n <= 0:
        raise ValueError("n must be a positive integer")
    return 1 << (int(n) - 1).bit_length()


def is_smooth(n: int) -> bool:
    """src/fourierinterp.jl:115-123."""
    if n <= 0:
        return False
    for f in (2, 3, 5, 7):
        while n % f == 0:
            n //= f
    return n == 1


def next_smooth(n: int) -> int:
    """src/fourierinterp.jl:141-149."""
    if n <= 0:
        raise ValueError("n must be a positive integer")
    if n <= 4:
        return int(n)
    k = int(n)
    while not is_smooth(k):
        k += 1
    return k


def finterp_fft_coeffs(numbetween: int, m: int, fftlen: int) -> np.ndarray:
    """src/fourierinterp.jl:161-174."""
    if m % 2:
        raise ValueError("m must be even")
    if fftlen < numbetween * m:
        raise ValueError("fftlen must be >= numbetween * m")
    c = np.zeros(fftlen, dtype=np.complex128)
    n = (numbetween * m) // 2
    off = np.arange(n) / numbetween
    c[:n] = sinc(off) * cispi(-off)
    off2 = (-(off + 1.0 / numbetween))[::-1]
    c[fftlen - n:] = sinc(off2) * cispi(-off2)
    return np.conj(np.fft.fft(c))


def finterp_fft(lobin: int, numbins: int, numbetween: int, ft: np.ndarray, m: int,
                fftlen: Optional[int] = None) -> np.ndarray:
    """src/fourierinterp.jl:190-212 (FFT-correlation interpolator)."""
    m2 = m // 2
    numftbins = (numbins + m) * numbetween
    if fftlen is None:
        fftlen = next_pow_of_2(numftbins)
    if fftlen < numftbins:
        raise ValueError("fftlen must be >= (numbins+m)*numbetween")
    coeffs = finterp_fft_coeffs(numbetween, m, fftlen)
    arr = np.zeros(fftlen, dtype=np.complex128)
    src = ft[lobin - m2:lobin + numbins + m2].astype(np.complex128)
    arr[np.arange(numbins + m) * numbetween] = src
    corr = np.fft.ifft(np.fft.fft(arr) * coeffs)
    return corr[m2 * numbetween:(m2 + numbins) * numbetween]


def finterp_direct(r0: float, n: int, step: float, ft: np.ndarray, m: int) -> np.ndarray:
    """src/directinterp.jl:71-101 (factored exact kernel, FP64)."""
    if m % 2:
        raise ValueError("m must be even")
    m2 = m // 2
    out = np.empty(n, dtype=np.complex128)
    jj = np.arange(1, m + 1) - m2          # Julia i - m2 for i = 1..m
    for k in range(n):
        r = r0 + k * step
        rint = math.floor(r + 1e-15) + 1
        dr = math.fmod(r, 1.0)
        base = rint - m2                  # Julia ft[base+i] -> 0-based base+i-1
        if dr == 0.0:
            out[k] = complex(ft[base + m2 - 1])
            continue
        w = 1.0 / (dr - jj)
        a = ft[base:base + m].astype(np.complex128)
        s = np.sum(w * a.real) + 1j * np.sum(w * a.imag)
        A = np.conj(sinpi(dr) * cispi(dr) / math.pi)
        out[k] = A * s
    return out


# ---------------------------------------------------------------------------
# Direct interpolation plans  (src/directinterp.jl:111-418)
# ---------------------------------------------------------------------------

DIRECT_QMAX = 1 << 16          # src/directinterp.jl:111
DIRECT_GROUP_V = 32            # src/directinterp.jl:151


def trial_grid_rational(lodr: float) -> Optional[Tuple[int, int]]:
    """src/directinterp.jl:217-225.

    ``rationalize(Int, lodr; tol=1e-13)`` returns the smallest-denominator
    rational within 1e-13; the reference then accepts it only when
    ``q <= DIRECT_QMAX``, ``p >= 1`` and ``|p/q - lodr| <= 8 eps(lodr)``.  Two
    distinct rationals with denominators <= 2^16 are >= 2^-32 apart, so the
    accepted rational, when one exists, is the unique smallest-``q`` rational
    with ``q <= DIRECT_QMAX`` passing the 8-eps test -- found here by scanning
    ``q``.
    """
    if not lodr > 0:
        return None
    eps8 = 8.0 * np.spacing(float(lodr))
    qs = np.arange(1, DIRECT_QMAX + 1, dtype=np.float64)
    ps = np.rint(lodr * qs)
    ok = (ps >= 1) & (np.abs(ps / qs - lodr) <= eps8)
    idx = np.flatnonzero(ok)
    if idx.size == 0:
        return None
    q = int(qs[idx[0]])
    p = int(ps[idx[0]])
    g = math.gcd(p, q)
    return p // g, q // g


@dataclass
class DirectPlan:
    """Per-harmonic phase tables (src/directinterp.jl:179-204), no group tables.

    The reference additionally builds trials-axis group tables
    (``build_group_table``, src/directinterp.jl:237-282); their product is the
    same per-trial sequential tap sum, because the extra entries are exact
    zeros, so the oracle evaluates the sum per trial.
    """
    h: int
    m: int
    q: int
    s: int
    base_adv: int
    pnum: int
    rfloor0: int
    dr0: float
    P: int
    row: np.ndarray        # (q,) residue -> phase row, -1 if unvisited
    W: np.ndarray          # (P, m) weights 1/(dr - j)
    A: np.ndarray          # (P,) conj(sin(pi dr) cispi(dr) / pi)
    carry: np.ndarray      # (P,) bool


def build_direct_plans(params: SearchParams, r_lo: float, wt=np.float64) -> List[DirectPlan]:
    """src/directinterp.jl:345-405.  ``wt`` is the weight storage type; every
    entry is computed in FP64 and rounded once (src/directinterp.jl:375-378)."""
    lodr = params.hidr / params.nharms
    rq = trial_grid_rational(lodr)
    m = params.m
    if m % 2:
        raise ValueError("m must be even")
    m2 = m // 2
    ct = np.complex64 if wt == np.float32 else np.complex128
    plans = []
    for h in range(1, params.nharms + 1):
        hr = h * float(r_lo)
        rfloor0 = math.floor(hr)
        dr0 = hr - rfloor0
        if rq is None:
            plans.append(DirectPlan(h, m, 1, 0, 0, 1, rfloor0, dr0, 0,
                                    np.zeros(0, np.int64), np.zeros((0, m), wt),
                                    np.zeros(0, ct), np.zeros(0, bool)))
            continue
        pnum, q = rq
        step = h * pnum
        s = step % q
        base_adv = step // q
        P = q // math.gcd(step, q)
        row = np.full(q, -1, dtype=np.int64)
        W = np.empty((P, m), dtype=wt)
        A = np.empty(P, dtype=ct)
        carry = np.empty(P, dtype=bool)
        res = 0
        jj = np.arange(1, m + 1) - m2
        for p in range(P):
            row[res] = p
            u = dr0 + res / q
            carry[p] = u >= 1.0
            dr = u - 1.0 if carry[p] else u
            if dr == 0.0:
                A[p] = 1.0
                W[p] = 0.0
                W[p, m2 - 1] = 1.0
            else:
                a64 = np.conj(complex(sinpi(dr) * cispi(dr)) / math.pi)
                A[p] = a64
                W[p] = (1.0 / (dr - jj)).astype(wt)
            res += s
            if res >= q:
                res -= q
        plans.append(DirectPlan(h, m, q, s, base_adv, pnum, rfloor0, dr0, P, row, W, A, carry))
    return plans


def direct_chunk_state(dp: DirectPlan, t0):
    """src/directinterp.jl:414-418: (res, qint) = divrem(t0*h*pnum, q), exact.

    Accepts a Python int (arbitrary precision) or an int64 array of trials."""
    if np.ndim(t0):
        T = np.asarray(t0, dtype=np.int64) * np.int64(dp.h * dp.pnum)
        return T % dp.q, T // dp.q
    T = int(t0) * dp.h * dp.pnum
    return T % dp.q, T // dp.q


def harmonic_guard(dp: DirectPlan, t0: int, n: int, Nhalf: int, namps: int) -> bool:
    """Range guard on the TRUE trial range of a rational-grid plan,
    src/directinterp.jl:490-496."""
    m2 = dp.m // 2
    res, qint = direct_chunk_state(dp, t0)
    lo_trial = dp.rfloor0 + qint + int(dp.carry[dp.row[res]]) + 2 - m2
    resl, qintl = direct_chunk_state(dp, t0 + n - 1)
    hi_trial = dp.rfloor0 + qintl + int(dp.carry[dp.row[resl]]) + 1 + m2
    return lo_trial >= 1 and hi_trial <= namps and (dp.rfloor0 + qintl) < Nhalf


def fill_harmonic_row(dp: DirectPlan, amps: np.ndarray, params: SearchParams,
                      t0: int, n: int, N: int, acc=np.float64) -> np.ndarray:
    """One harmonic row of the amplitude stack for trials ``t0 .. t0+n-1``.

    Restates ``fill_harmonic_row_direct!`` (src/directinterp.jl:470-572) and its
    per-trial fallback ``_fill_row_direct_slow!`` (:623-661).  Returns zeros
    when the guard rejects the row.  ``acc`` is the tap-sum precision (FP64 is
    the accuracy anchor; the bit-exact FP32 form lives in ``cs_cpu.c``).
    """
    out = np.zeros(n, dtype=np.complex128)
    if n < 1:
        return out
    m = dp.m
    m2 = m // 2
    Nhalf = N // 2
    namps = len(amps)
    if dp.P == 0:
        return _fill_row_slow(dp, amps, params, t0, n, N)
    if not harmonic_guard(dp, t0, n, Nhalf, namps):
        return out
    t = np.arange(t0, t0 + n, dtype=np.int64)
    res, qint = direct_chunk_state(dp, t)
    p = dp.row[res]
    fl = dp.rfloor0 + qint + dp.carry[p].astype(np.int64)     # floor(h*r_t)
    base = fl + 1 - m2                                        # 0-based first tap
    idx = base[:, None] + np.arange(m)[None, :]
    win = amps[idx]
    W = dp.W[p].astype(acc)
    sre = np.sum(W * win.real.astype(acc), axis=1)
    sim = np.sum(W * win.imag.astype(acc), axis=1)
    A = dp.A[p]
    return (A.astype(np.complex128) * (sre.astype(np.float64) + 1j * sim.astype(np.float64)))


def _fill_row_slow(dp: DirectPlan, amps, params: SearchParams, t0: int, n: int, N: int):
    """src/directinterp.jl:623-661 (non-rational trial step)."""
    h, m = dp.h, dp.m
    m2 = m // 2
    lodr = params.hidr / params.nharms
    hr_lo = dp.rfloor0 + dp.dr0
    dh = h * lodr
    Nhalf = N // 2
    namps = len(amps)
    out = np.zeros(n, dtype=np.complex128)
    rfirst = hr_lo + t0 * dh
    rlast = hr_lo + (t0 + n - 1) * dh
    lo = math.floor(rfirst + 1e-15) + 2 - m2
    hi = math.floor(rlast + 1e-15) + 1 + m2
    if not (lo >= 1 and hi <= namps and math.floor(rlast) < Nhalf):
        return out
    jj = np.arange(1, m + 1) - m2
    for k in range(n):
        r = hr_lo + (t0 + k) * dh
        rint = math.floor(r + 1e-15) + 1
        dr = math.fmod(r, 1.0)
        base = rint - m2
        if dr == 0.0:
            out[k] = complex(amps[base + m2 - 1])
            continue
        w = 1.0 / (dr - jj)
        a = amps[base:base + m].astype(np.complex128)
        s = np.sum(w * a.real) + 1j * np.sum(w * a.imag)
        out[k] = np.conj(sinpi(dr) * cispi(dr) / math.pi) * s
    return out


def direct_window_size(params: SearchParams, Nprof: int) -> int:
    """src/directinterp.jl:673-674."""
    return math.ceil((Nprof - 1 + 2 * DIRECT_GROUP_V) * params.hidr) + params.m + 4


# ---------------------------------------------------------------------------
# Profile synthesis  (src/search.jl:964-965, 1280-1293, 1664-1675)
# ---------------------------------------------------------------------------


def brfft(stack: np.ndarray, nbins: int) -> np.ndarray:
    """Unnormalised complex->real inverse transform along the harmonic axis.

    ``stack`` is ``(n, H+1)`` (DC first); returns ``(n, nbins)``.  FFTW's c2r
    and numpy's ``irfft`` both ignore Im of DC and Nyquist
    (test/test_fourierinterp.jl:128-143), and brfft = nbins * irfft.
    """
    return np.fft.irfft(stack, n=nbins, axis=1) * nbins


def chunk_stack(plans: Sequence[DirectPlan], amps, params: SearchParams, t0: int, n: int,
                N: int, acc=np.float64) -> np.ndarray:
    """``fill_chunk_profiles!`` amplitude stage (src/search.jl:1280-1290):
    ``(n, nharms+1)`` complex stack, DC column zero."""
    st = np.zeros((n, params.nharms + 1), dtype=np.complex128)
    for dp in plans:
        st[:, dp.h] = fill_harmonic_row(dp, amps, params, t0, n, N, acc)
    return st


def decimated_stack(stack: np.ndarray, k: int, nharms: int) -> np.ndarray:
    """The stride-k view ``ftprofs[1:k:Hk*k+1, :]`` (src/search.jl:1174-1190)."""
    Hk = nharms // k
    return stack[:, 0:Hk * k + 1:k]


# ---------------------------------------------------------------------------
# Boxcar matched-filter metric  (src/search.jl:235-904)
# ---------------------------------------------------------------------------

BOXCAR_SIGMA_SAMPLES = 8192      # src/search.jl:462
BC_BATCH = 128                   # src/search.jl:677
LADDER_WMAX = 6                  # src/search.jl:399


def median_exact(v: np.ndarray) -> float:
    """``_median!`` (src/search.jl:295-305): middle order statistic, or the
    mean of the two central ones for even length."""
    n = len(v)
    half = n >> 1
    if n % 2:
        return np.partition(v, half)[half]
    part = np.partition(v, [half - 1, half])
    t = v.dtype.type
    return t(0.5) * (part[half - 1] + part[half])


def boxcar_widths(nbins: int, fsp: float = 1.5, maxfrac: float = 0.3) -> List[int]:
    """src/search.jl:387-396."""
    wmax = max(1, math.floor(maxfrac * nbins))
    ws = []
    w = 1
    while w <= wmax:
        ws.append(w)
        w = max(math.floor(fsp * w), w + 1)
    return ws


def ladder_boxcar_widths(nbins: int, k: int, params: SearchParams) -> List[int]:
    """src/search.jl:443-459."""
    ws = boxcar_widths(nbins, params.boxcar_fsp, params.boxcar_maxfrac)
    ks = sorted(params.decimations)
    if len(ks) <= 1:
        return ws
    if not all(ks[i + 1] <= (LADDER_WMAX // 2) * ks[i] for i in range(len(ks) - 1)):
        return ws
    kmin, kmax = ks[0], ks[-1]
    pruned = [w for w in ws if (w >= 2 or k == kmin) and (w <= LADDER_WMAX or k == kmax)]
    return ws if not pruned else pruned


def sigma_subsample(M: np.ndarray, nbins: int, n: int, cap: int = BOXCAR_SIGMA_SAMPLES) -> np.ndarray:
    """The samples ``_block_sigma`` pools (src/search.jl:494-537): every bin
    when ``nbins*n <= cap``, else ``ncol`` whole profiles, evenly spaced."""
    flat = M[:n].reshape(-1)
    N = nbins * n
    if N <= cap:
        return flat[:N].copy()
    ncol = min(n, max(1, cap // nbins))
    out = []
    ns = 0
    for c in range(1, ncol + 1):
        j = 1 + ((c - 1) * n) // ncol
        take = min(nbins, cap - ns)
        if take == 0:
            break
        out.append(flat[(j - 1) * nbins:(j - 1) * nbins + take])
        ns += take
    return np.concatenate(out)


def sigma_subsample_columns(nbins: int, n: int, cap: int = BOXCAR_SIGMA_SAMPLES) -> np.ndarray:
    """0-based profile indices the block sigma reads (all when nbins*n <= cap)."""
    if nbins * n <= cap:
        return np.arange(n)
    ncol = min(n, max(1, cap // nbins))
    return np.array([((c - 1) * n) // ncol for c in range(1, ncol + 1)], dtype=np.int64)


def block_sigma(M: np.ndarray, nbins: int, n: int, cap: int = BOXCAR_SIGMA_SAMPLES,
                center: str = "zero") -> float:
    """``_block_sigma`` (src/search.jl:490-566): 1.4826 * median(|x|) over the
    subsample (``center='zero'``), or the classic MAD (``'median'``)."""
    if nbins * n == 0:
        return M.dtype.type(0)
    buf = sigma_subsample(M, nbins, n, cap)
    t = buf.dtype.type
    if center == "median":
        med = median_exact(buf.copy())
        buf = np.abs(buf - med)
    else:
        buf = np.abs(buf)
    return t(1.4826) * median_exact(buf)


def boxcar_psum(cols: np.ndarray, nbins: int, wmax: int, b) -> np.ndarray:
    """``_boxcar_psum!`` (src/search.jl:571-578) for a batch of profiles
    ``cols`` (n, nbins): wrapped prefix sums of ``col - b``, shape (n, nbins+wmax+1)."""
    n = cols.shape[0]
    t = cols.dtype.type
    idx = np.arange(nbins + wmax) % nbins
    x = cols[:, idx] - np.asarray(b, dtype=cols.dtype).reshape(-1, 1)
    ps = np.zeros((n, nbins + wmax + 1), dtype=cols.dtype)
    ps[:, 1:] = np.cumsum(x, axis=1, dtype=cols.dtype)
    return ps


def boxcar_scan(ps: np.ndarray, widths: Sequence[int], nbins: int, invsigma) -> np.ndarray:
    """``_boxcar_scan`` (src/search.jl:585-598), vectorised over rows."""
    t = ps.dtype.type
    best = np.full(ps.shape[0], -np.inf, dtype=ps.dtype)
    for w in widths:
        invsw = t(invsigma) / np.sqrt(t(w))
        d = ps[:, w:w + nbins] - ps[:, 0:nbins]
        m = d.max(axis=1)
        cand = m * invsw
        best = np.where(cand > best, cand, best)
    return best


def boxcar_exact(profs: np.ndarray, widths: Sequence[int], nbins: int, invsigma) -> np.ndarray:
    """``_boxcar_exact`` (src/search.jl:893-904): median baseline, then scan."""
    if profs.shape[0] == 0:
        return np.zeros(0, dtype=profs.dtype)
    med = np.median(profs, axis=1).astype(profs.dtype)
    ps = boxcar_psum(profs, nbins, widths[-1], med)
    return boxcar_scan(ps, widths, nbins, invsigma)


def profile_boxcar(profs: np.ndarray, widths, nbins: int, invsigma) -> np.ndarray:
    """``_profile_boxcar`` with ``medcut = -Inf`` (src/search.jl:875-888)."""
    if not invsigma > 0:
        return np.zeros(profs.shape[0], dtype=profs.dtype)
    return boxcar_exact(profs, widths, nbins, invsigma)


def boxcar_gate(profs: np.ndarray, n: int, widths, nbins: int, invsigma) -> np.ndarray:
    """``_boxcar_gate!`` (src/search.jl:784-807): Float32 zero-baseline scan
    over full 128-profile tiles, the profile-precision scalar scan for the tail."""
    out = np.empty(n, dtype=np.float64)
    nfull = (n // BC_BATCH) * BC_BATCH
    if nfull:
        tile = profs[:nfull].astype(np.float32)
        ps = boxcar_psum(tile, nbins, widths[-1], np.float32(0))
        out[:nfull] = boxcar_scan(ps, widths, nbins, np.float32(invsigma)).astype(np.float64)
    if n > nfull:
        tail = profs[nfull:n]
        ps = boxcar_psum(tail, nbins, widths[-1], tail.dtype.type(0))
        out[nfull:n] = boxcar_scan(ps, widths, nbins, invsigma).astype(np.float64)
    return out


def boxcar_metrics(profs: np.ndarray, n: int, widths, nbins: int, invsigma,
                   medcut: float) -> Tuple[np.ndarray, np.ndarray]:
    """``boxcar_metrics!`` (src/search.jl:825-843).  Returns the per-trial metric
    and the mask of trials that took the exact (median-baseline) path."""
    if medcut == -math.inf or not invsigma > 0:
        return profile_boxcar(profs[:n], widths, nbins, invsigma).astype(np.float64), np.ones(n, bool)
    m = boxcar_gate(profs, n, widths, nbins, invsigma)
    resc = m >= medcut
    if resc.any():
        m[resc] = boxcar_exact(profs[:n][resc], widths, nbins, invsigma).astype(np.float64)
    return m, resc


def boxcar_best_width(prof: np.ndarray, fsp: float = 1.5, maxfrac: float = 0.3) -> Tuple[int, float]:
    """src/search.jl:617-638."""
    col = np.asarray(prof, dtype=np.float64)
    nbins = len(col)
    if nbins < 1:
        raise ValueError("profile must be non-empty")
    widths = boxcar_widths(nbins, fsp, maxfrac)
    med = median_exact(col.copy())
    ps = boxcar_psum(col[None, :], nbins, widths[-1], med)[0]
    best, bestw = -math.inf, widths[0]
    for w in widths:
        m = ps[w] - ps[0]
        for p in range(1, nbins):
            m = max(m, ps[p + w] - ps[p])
        cand = m * (1.0 / math.sqrt(w))
        if cand > best:
            best, bestw = cand, w
    return bestw, bestw / nbins


def snr_metrics(profs: np.ndarray, boxcar_fsp=1.5, boxcar_maxfrac=0.3,
                sigma_samples: int = 2**62, sigma_center: str = "zero",
                widths=None) -> np.ndarray:
    """src/search.jl:933-951.  ``profs`` is ``(L, nbins)``."""
    P = np.asarray(profs, dtype=np.float64)
    L, nbins = P.shape
    if widths is None:
        widths = boxcar_widths(nbins, boxcar_fsp, boxcar_maxfrac)
    sig = block_sigma(P, nbins, L, cap=min(nbins * L, sigma_samples), center=sigma_center)
    invsigma = 1.0 / sig if sig > 0 else 0.0
    return profile_boxcar(P, list(widths), nbins, invsigma)


# ---------------------------------------------------------------------------
# Reference (allocating) path  (src/search.jl:964-1097)
# ---------------------------------------------------------------------------


def uniform_linear_interp(r: float, lobin: int, numbetween: int, amps: np.ndarray) -> complex:
    """src/search.jl:974-986."""
    K = len(amps)
    p = (r - lobin) * numbetween
    if p <= 0:
        return complex(amps[0])
    if p >= K - 1:
        return complex(amps[K - 1])
    i0 = math.floor(p)
    f = p - i0
    return complex(amps[i0]) * (1 - f) + complex(amps[i0 + 1]) * f


def reference_profiles(amps: np.ndarray, N: int, rfund: np.ndarray, params: SearchParams,
                       kernel: str = "fft") -> np.ndarray:
    """src/search.jl:1011-1049.  Returns ``(L, 2*nharms)`` normalised irfft profiles."""
    if kernel not in ("fft", "direct"):
        raise ValueError(f"kernel must be fft or direct, got {kernel}")
    nh, m, nb = params.nharms, params.m, params.numbetween
    m2 = m // 2
    rfund = np.asarray(rfund, dtype=np.float64)
    L = len(rfund)
    Nhalf = N // 2
    namps = len(amps)
    st = np.zeros((L, nh + 1), dtype=np.complex128)
    for h in range(1, nh + 1):
        rmin = rfund[0] * h
        rmax = rfund[-1] * h
        lobin = math.floor(rmin)
        hibin = math.ceil(rmax) + 1
        numbins = hibin - lobin
        if not (lobin >= m2 and (lobin + numbins + m2) <= namps and hibin < Nhalf):
            continue
        if kernel == "fft":
            grid = finterp_fft(lobin, numbins, nb, amps, m)
            for j in range(L):
                st[j, h] = uniform_linear_interp(rfund[j] * h, lobin, nb, grid)
        else:
            for j in range(L):
                st[j, h] = fourier_interp(rfund[j] * h, amps, m)
    return np.fft.irfft(st, n=2 * nh, axis=1)


def block_metrics(amps, N, rfund, params: SearchParams, kernel="fft", widths=None) -> np.ndarray:
    """src/search.jl:1061-1079."""
    nbins = 2 * params.nharms
    profs = reference_profiles(amps, N, rfund, params, kernel)
    if widths is None:
        widths = ladder_boxcar_widths(nbins, 1, params)
    return snr_metrics(profs, params.boxcar_fsp, params.boxcar_maxfrac,
                       sigma_samples=BOXCAR_SIGMA_SAMPLES, widths=widths)


def candidate_profile(amps: np.ndarray, N: int, r: float, nharm: int, m: int = 64) -> np.ndarray:
    """candidate_profile (src/candidate.jl:37-61): contiguous harmonics while
    their m-bin window fits below Nyquist and inside the file, each an exact
    fourier_interp; irfft of [0, amps...] to 2H bins (two zeros if H = 0)."""
    if nharm < 1:
        raise ValueError("nharm must be >= 1")
    if m % 2:
        raise ValueError("m must be even")
    m2 = m // 2
    Nhalf = N // 2
    namps = len(amps)
    out = []
    for h in range(1, nharm + 1):
        rh = r * h
        rint = math.floor(rh + 1e-15) + 1
        if not (rint - m2 >= 0 and rint + m2 <= namps and rh < Nhalf):
            break
        out.append(fourier_interp(rh, amps, m))
    H = len(out)
    if H < 1:
        return np.zeros(2)
    stack = np.zeros(H + 1, dtype=np.complex128)
    stack[1:] = out
    return np.fft.irfft(stack, 2 * H)


def measure_ducy(amps: np.ndarray, N: int, rs, nharms, params: "SearchParams", m: int = 64) -> np.ndarray:
    """measure_ducy (src/candidate.jl:63-99): per candidate (r, nharm) the duty
    cycle of the best boxcar of its refolded profile; NaN when nharm < 1 or r <= 0."""
    res = []
    for r, nh in zip(rs, nharms):
        d = math.nan
        if nh >= 1 and r > 0:
            prof = candidate_profile(amps, N, r, nh, m)
            if len(prof) >= 2:
                _, d = boxcar_best_width(prof, params.boxcar_fsp, params.boxcar_maxfrac)
        res.append(d)
    return np.array(res)


@dataclass
class Candidate:
    """src/search.jl:179-191."""
    freq: float
    metric: float
    r: float
    nharm: int
    ducy: float = math.nan


def search_block(amps, N, T, rfund, params: SearchParams, threshold=None) -> List[Candidate]:
    """src/search.jl:1087-1097."""
    thr = params.threshold if threshold is None else threshold
    met = block_metrics(amps, N, rfund, params)
    return [Candidate(rfund[j] / T, float(met[j]), float(rfund[j]), params.nharms)
            for j in range(len(rfund)) if met[j] > thr]


# ---------------------------------------------------------------------------
# Production path  (src/search.jl:1280-1293, 1664-1755, 1768-1894, 2002-2111)
# ---------------------------------------------------------------------------


def chunk_metrics(amps, N, params: SearchParams, rstart: float, n: int, lodr=None,
                  weights=np.float32) -> np.ndarray:
    """src/search.jl:1740-1755 (global trial 0 = ``rstart``; exact median for all)."""
    nh = params.nharms
    nbins = 2 * nh
    plans = build_direct_plans(params, rstart, weights)
    acc = np.float32 if weights == np.float32 else np.float64
    st = chunk_stack(plans, amps, params, 0, n, N, acc)
    P = proftype(params)
    profs = brfft(st, nbins).astype(P)
    sig = block_sigma(profs, nbins, n)
    inv = P(1) / sig if sig > 0 else P(0)
    widths = ladder_boxcar_widths(nbins, 1, params)
    return profile_boxcar(profs, widths, nbins, inv).astype(np.float64)


@dataclass
class BlockResult:
    """Per (block, k) intermediate values the parity tests compare."""
    block: int
    k: int
    nvalid: int
    sigma: float
    metrics: np.ndarray
    rescued: np.ndarray


def search_region(amps, N, T, params: SearchParams, r_lo: float, r_hi: float, total: int,
                  Nprof: int, threshold: float, medcut: float, plans=None,
                  weights=np.float32, keep_blocks: bool = False, block_range=None):
    """The chunk loop of ``_search_region!`` (src/search.jl:1768-1894) run on
    one task, which fixes the candidate order: per block, the base pass
    (ascending trial) then each decimation factor in ``params.decimations``
    order (src/search.jl:1809-1859, :1695-1708)."""
    lodr = params.hidr / params.nharms
    nh = params.nharms
    nbins = 2 * nh
    P = proftype(params)
    if plans is None:
        plans = build_direct_plans(params, r_lo, weights)
    acc = np.float32 if weights == np.float32 else np.float64
    nchunks = -(-total // Nprof)
    widths1 = ladder_boxcar_widths(nbins, 1, params)
    decims = [k for k in params.decimations if k > 1]
    cands: List[Tuple[int, int, int, Candidate]] = []
    blocks: List[BlockResult] = []
    nyq = N / 2
    rng = range(nchunks) if block_range is None else block_range
    for c in rng:
        i0 = c * Nprof
        n = min(Nprof, total - i0)
        rstart = r_lo + i0 * lodr
        st = chunk_stack(plans, amps, params, i0, n, N, acc)
        profs = brfft(st, nbins).astype(P)
        sig = block_sigma(profs, nbins, n)
        inv = P(1) / sig if sig > 0 else P(0)
        mv, resc = boxcar_metrics(profs, n, widths1, nbins, inv, medcut)
        if keep_blocks:
            blocks.append(BlockResult(c, 1, n, float(sig), mv, resc))
        for j in range(n):
            if mv[j] > threshold:
                rf = rstart + j * lodr
                cands.append((c, 1, j, Candidate(rf / T, float(mv[j]), rf, nh)))
        for k in decims:
            Hk = nh // k
            nb = 2 * Hk
            dprofs = brfft(decimated_stack(st, k, nh), nb).astype(P)
            nvalid = 0
            while nvalid < n and k * (rstart + nvalid * lodr) < nyq:
                nvalid += 1
            sig = block_sigma(dprofs, nb, nvalid)
            inv = P(1) / sig if sig > 0 else P(0)
            wk = ladder_boxcar_widths(nb, k, params)
            mv, resc = boxcar_metrics(dprofs, nvalid, wk, nb, inv, medcut)
            if keep_blocks:
                blocks.append(BlockResult(c, k, nvalid, float(sig), mv, resc))
            for j in range(n):
                r_dec = k * (rstart + j * lodr)
                if not r_dec < nyq:
                    continue
                if mv[j] > threshold:
                    cands.append((c, k, j, Candidate(r_dec / T, float(mv[j]), r_dec, Hk)))
    return cands, blocks


def search_setup(N: int, dt: float, params: SearchParams, lofreq=0.1, hifreq=100.0, lobin=100,
                 blocksize=2048):
    """Band bookkeeping of ``search`` (src/search.jl:2016-2027)."""
    T = N * dt
    lodr = params.hidr / params.nharms
    r_lo = lofreq * T
    if lobin != 100:
        r_lo = float(lobin)
    r_hi = hifreq * T
    total = max(0, math.floor((r_hi - r_lo) / lodr) + 1)
    Nprof = max(1, int(blocksize))
    return T, lodr, r_lo, r_hi, total, Nprof


def search(amps, N, dt, params: SearchParams, lofreq=0.1, hifreq=100.0, lobin=100,
           blocksize=2048, threshold=None, remove=True, dr_tol=1.0, harm_remove=True,
           numharm=16, harm_tol=1.0, exact_all=False) -> List[Candidate]:
    """src/search.jl:2002-2111 (no metricstats/normalize)."""
    thr = params.threshold if threshold is None else threshold
    T, lodr, r_lo, r_hi, total, Nprof = search_setup(N, dt, params, lofreq, hifreq, lobin, blocksize)
    if total == 0:
        return []
    medcut = -math.inf if exact_all else thr - params.boxcar_medmargin
    raw, _ = search_region(amps, N, T, params, r_lo, r_hi, total, Nprof, thr, medcut)
    cands = [c for (_, _, _, c) in raw]
    if remove:
        cands = remove_duplicates(cands, dr_tol)
    else:
        cands = sorted(cands, key=lambda c: c.freq)
    if harm_remove:
        cands = remove_harmonics(cands, numharm, harm_tol)
    return cands


def remove_duplicates(cands: Sequence[Candidate], dr_tol: float = 1.0) -> List[Candidate]:
    """src/search.jl:2148-2167 (stable sort by r; keep first strict max per run)."""
    if not cands:
        return []
    order = sorted(range(len(cands)), key=lambda i: cands[i].r)
    kept = []
    best = cands[order[0]]
    prev_r = best.r
    for i in order[1:]:
        c = cands[i]
        if c.r - prev_r <= dr_tol:
            if c.metric > best.metric:
                best = c
        else:
            kept.append(best)
            best = c
        prev_r = c.r
    kept.append(best)
    return sorted(kept, key=lambda c: c.freq)


def harmonically_related(r1: float, r2: float, numharm: int, tol: float) -> bool:
    """src/search.jl:2179-2188."""
    lo, hi = min(r1, r2), max(r1, r2)
    if not lo > 0:
        return False
    for m in range(1, numharm + 1):
        n = _round_half_even(m * hi / lo)
        if not (1 <= n <= numharm):
            continue
        if abs(m * hi - n * lo) <= tol * m:
            return True
    return False


def _round_half_even(x: float) -> int:
    """Julia ``round(Int, x)`` rounds ties to even, as Python's ``round``."""
    return int(round(x))


def remove_harmonics(cands: Sequence[Candidate], numharm: int = 16, tol: float = 1.0) -> List[Candidate]:
    """src/search.jl:2202-2214 (stable sort by metric, strongest first)."""
    if not cands:
        return []
    order = sorted(range(len(cands)), key=lambda i: -cands[i].metric)
    kept: List[Candidate] = []
    for i in order:
        c = cands[i]
        if not any(harmonically_related(c.r, k.r, numharm, tol) for k in kept):
            kept.append(c)
    return sorted(kept, key=lambda c: c.freq)
