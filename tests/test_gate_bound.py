"""The window-energy bound behind the tensor epilogue's gate skip (host-side
check of its arithmetic; no GPU).

k_synth_tc skips a warp's boxcar scan when, for every trial, the bound

    B = (sqrt(L + 2^-13 q) + 2^-13 sqrt(pw q)) * (1 + 2^-16)

falls below the medcut cut, where q is the FP32 running sum of x^2 over the
unit's pw columns (one fused multiply-add per column) and L the largest FP32
width-W window of it.  The skip is exact only if B is at least the gate value
the full FP32 scan would compute: the largest (ps[s+w] - ps[s]) * rsqrt(w) over
the unit's starts s and widths w <= W, ps the FP32 running sum of x.  These
tests emulate both scans in FP32, in the kernels' order of operations, on
profiles built to stress the rounding: noise, bright pulses, large common
offsets (cancelling prefix sums) and alternating +-1e4 columns.
"""
import zlib

import numpy as np
import pytest

F = np.float32


def _gate_fp32(x, nstart, widths):
    """The full scan: sequential FP32 prefix sums, FP32 differences, max per
    width times the FP32 1/sqrt(w), then the max over widths."""
    n, pw = x.shape
    ps = np.zeros((n, pw + 1), F)
    ps[:, 1:] = np.cumsum(x, axis=1, dtype=F)   # sequential FP32 accumulation
    best = np.full(n, -np.inf, F)
    for w in widths:
        s = np.arange(nstart)
        ok = s + w <= pw
        d = (ps[:, s[ok] + w] - ps[:, s[ok]]).astype(F)
        best = np.maximum(best, (d.max(axis=1) * F(1.0 / np.sqrt(w))).astype(F))
    return best


def _fma32(a, b, c):
    # a*b is exact in FP64 for FP32 inputs; one FP64 add, then the FP32 rounding
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(F)


def _bound_fp32(x, W):
    """The pre-pass: q by fused multiply-adds, every width-W window inside the
    pw columns, and B with the kernel's margins, in FP32."""
    n, pw = x.shape
    q = np.zeros((n, pw + 1), F)
    for e in range(pw):
        q[:, e + 1] = _fma32(x[:, e], x[:, e], q[:, e])
    d = (q[:, W:] - q[:, :-W]).astype(F)
    mx = d.max(axis=1)
    qt = q[:, pw]
    a = np.sqrt((mx + qt * F(2.0 ** -13)).astype(F)).astype(F)
    b = (F(2.0 ** -13) * np.sqrt((F(pw) * qt).astype(F)).astype(F)).astype(F)
    return ((a + b).astype(F) * F(1.0 + 2.0 ** -16)).astype(F)


def _profiles(kind, n, pw, rng):
    x = rng.standard_normal((n, pw))
    if kind == "pulse":
        p = rng.integers(0, pw, n)
        x[np.arange(n), p] += rng.uniform(5, 60, n)
        x[np.arange(n), (p + 1) % pw] += rng.uniform(0, 30, n)
    elif kind == "offset":
        x += rng.choice([-1.0, 1.0], (n, 1)) * 10.0 ** rng.uniform(2, 5, (n, 1))
    elif kind == "alternating":
        x += 1e4 * np.where(np.arange(pw) % 2 == 0, 1.0, -1.0)[None, :]
    elif kind == "tiny":
        x *= 1e-20
    elif kind == "huge":
        x *= 1e15
    return x.astype(F)


LADDER_BASE = [1, 2, 3, 4, 6]
LADDER_DEEP = [2, 3, 4, 6]
GEOMETRIC = [1, 2, 3, 4, 6, 9, 13, 19]


@pytest.mark.parametrize("kind", ["noise", "pulse", "offset", "alternating", "tiny", "huge"])
@pytest.mark.parametrize("widths,nstart,pw", [
    (LADDER_BASE, 40, 48),      # a third of the base level (120 bins, wmax 6)
    (LADDER_BASE, 120, 128),    # the whole base level
    (LADDER_DEEP, 60, 72),      # decimation 2
    (LADDER_DEEP, 20, 32),      # decimation 6
    (GEOMETRIC, 64, 96),        # the plain bank: pw a multiple of 32
])
def test_energy_bound_covers_the_fp32_gate(kind, widths, nstart, pw):
    rng = np.random.default_rng(zlib.crc32(f"{kind}-{nstart}-{pw}".encode()))
    x = _profiles(kind, 4000, pw, rng)
    g = _gate_fp32(x, nstart, widths)
    B = _bound_fp32(x, max(widths))
    assert np.all(np.isfinite(B))
    assert np.all(g <= B), (kind, float(np.max(g - B)))


def test_energy_bound_prunes_noise():
    """On unit-variance noise with the survey's cut (medcut 6 less the FP16
    slack) the bound clears nearly every trial -- the skip is worth having."""
    rng = np.random.default_rng(7)
    x = _profiles("noise", 20000, 48, rng)
    B = _bound_fp32(x, 6)
    cut = 6.0 - (0.02 * 6.0 + 0.05)
    assert np.mean(B < cut) > 0.999


# ---------------------------------------------------------------------------
# The plain FP32 synthesis (k_synth_fp32) bounds its gate from the stored
# wrapped prefix rows themselves: y_e = ps[e+1] - ps[e] over the nbins + W - 1
# columns whose width-W window starts below nbins, an FMA prefix of y^2 with a
# W-slot ring, and the same margins.  Its gate is max over widths w and starts
# p < nbins of (ps[p+w] - ps[p]) * rsqrt(w) with ps[nbins+u] = ps[nbins] + ps[u].
# ---------------------------------------------------------------------------
def _wrapped_ps(x, wmax):
    n, nbins = x.shape
    ps = np.zeros((n, nbins + wmax + 1), F)
    ps[:, 1:nbins + 1] = np.cumsum(x, axis=1, dtype=F)
    for u in range(1, wmax + 1):
        ps[:, nbins + u] = (ps[:, nbins] + ps[:, u]).astype(F)
    return ps


def _plain_gate(ps, nbins, widths):
    best = np.full(ps.shape[0], -np.inf, F)
    for w in widths:
        d = (ps[:, w:w + nbins] - ps[:, :nbins]).astype(F)
        best = np.maximum(best, (d.max(axis=1) * F(1.0 / np.sqrt(w))).astype(F))
    return best


def _plain_bound(ps, nbins, W):
    n = ps.shape[0]
    ne = nbins + W - 1
    y = (ps[:, 1:ne + 1] - ps[:, :ne]).astype(F)
    q = np.zeros((n, ne + 1), F)
    for e in range(ne):
        q[:, e + 1] = _fma32(y[:, e], y[:, e], q[:, e])
    d = (q[:, W:] - q[:, :-W]).astype(F)     # windows starting at p = 0 .. nbins - 1
    mx = d.max(axis=1)
    qt = q[:, ne]
    a = np.sqrt((mx + qt * F(2.0 ** -13)).astype(F)).astype(F)
    b = (F(2.0 ** -13) * np.sqrt((F(nbins + W) * qt).astype(F)).astype(F)).astype(F)
    return ((a + b).astype(F) * F(1.0 + 2.0 ** -16)).astype(F)


@pytest.mark.parametrize("kind", ["noise", "pulse", "offset", "alternating", "tiny", "huge"])
@pytest.mark.parametrize("widths,nbins", [(LADDER_BASE, 120), (LADDER_DEEP, 60), (LADDER_DEEP, 20),
                                          ([1, 2, 3, 4, 6, 8], 64)])
def test_plain_energy_bound_covers_the_fp32_gate(kind, widths, nbins):
    rng = np.random.default_rng(zlib.crc32(f"plain-{kind}-{nbins}".encode()))
    x = _profiles(kind, 4000, nbins, rng)
    W = max(widths)
    ps = _wrapped_ps(x, W)
    g = _plain_gate(ps, nbins, widths)
    B = _plain_bound(ps, nbins, W)
    assert np.all(np.isfinite(B))
    assert np.all(g <= B), (kind, float(np.max(g - B)))


def test_plain_energy_bound_prunes_noise():
    rng = np.random.default_rng(8)
    x = _profiles("noise", 20000, 120, rng)
    B = _plain_bound(_wrapped_ps(x, 6), 120, 6)
    assert np.mean(B < 6.0) > 0.99
