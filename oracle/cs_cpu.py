"""ctypes binding of the C oracle ``libcs_cpu.so`` (test infrastructure only)."""
import ctypes
import os

import numpy as np

from . import build as _build

_lib = None


def load():
    global _lib
    if _lib is None:
        path = _build.build()
        lib = ctypes.CDLL(path)
        lib.csref_interp_chunk.restype = ctypes.c_int
        lib.csref_interp_chunk.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int64,
                                           ctypes.c_int64, ctypes.c_void_p]
        lib.csref_plan_tables.restype = ctypes.c_int
        lib.csref_plan_tables.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int]
        lib.csref_search_blocks.restype = ctypes.c_int64
        lib.csref_search_blocks.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_double,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_int, ctypes.c_int64,
            ctypes.c_int64, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
            ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)]
        lib.csref_search_blocks_ex.restype = ctypes.c_int64
        lib.csref_search_blocks_ex.argtypes = [
            ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_double,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int64, ctypes.c_int, ctypes.c_int64,
            ctypes.c_int64, ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_int64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p,
            ctypes.c_void_p]
        lib.csref_c2r.restype = ctypes.c_int
        lib.csref_c2r.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _lib = lib
    return _lib


def interp_chunk(amps, N, nharms, m, hidr, r_lo, t0, n):
    """(nharms, n) complex64 amplitude stack, FP32-weight production arithmetic."""
    lib = load()
    a = np.ascontiguousarray(amps, dtype=np.complex64)
    out = np.zeros((nharms, n), np.complex64)
    rc = lib.csref_interp_chunk(a.ctypes.data, len(a), int(N), int(nharms), int(m), float(hidr),
                                float(r_lo), int(t0), int(n), out.ctypes.data)
    if rc != 0:
        raise ValueError("csref_interp_chunk: bad arguments")
    return out


def c2r(X):
    """The port's profile-stage transform of harmonic stacks X, complex (H+1, n)
    (row j = harmonic j of n trials; row 0 unused): the (2H, n) FP64 profiles
    and the number of FFT stages used (0: the direct DFT)."""
    lib = load()
    X = np.asarray(X, np.complex128)
    H, n = X.shape[0] - 1, X.shape[1]
    re = np.ascontiguousarray(X.real)
    im = np.ascontiguousarray(X.imag)
    prof = np.zeros((2 * H, n), np.float64)
    nst = lib.csref_c2r(re.ctypes.data, im.ctypes.data, int(H), int(n), prof.ctypes.data)
    if nst < 0:
        raise ValueError("csref_c2r: bad arguments")
    return prof, nst


def plan_tables(nharms, m, hidr, r_lo, h, cap=1 << 16):
    lib = load()
    W = np.zeros((cap, m), np.float32)
    A = np.zeros(cap, np.complex64)
    c = np.zeros(cap, np.uint8)
    P = lib.csref_plan_tables(int(nharms), int(m), float(hidr), float(r_lo), int(h), W.ctypes.data,
                              A.ctypes.data, c.ctypes.data, cap)
    return P, W[:P], A[:P], c[:P].astype(bool)


CAND_DTYPE = np.dtype([("blk", "<i4"), ("k", "<i4"), ("j", "<i4"), ("pad", "<f4"), ("metric", "<f8")])


def search_blocks(amps, N, dt, nharms, m, hidr, decimations, r_lo, total, blocksize, first_block, nblocks,
                  threshold, nthreads, exact_all=False, cap=1 << 20):
    """Run the C port of the production search on blocks [first_block,
    first_block+nblocks) with `nthreads` threads.  Returns a dict with the
    candidates (block, k, j, metric), wall seconds and counts."""
    lib = load()
    a = np.ascontiguousarray(amps, dtype=np.complex64)
    dec = np.ascontiguousarray(decimations, dtype=np.int32)
    out = np.zeros(cap, CAND_DTYPE)
    sec = ctypes.c_double()
    resc = ctypes.c_int64()
    n = lib.csref_search_blocks(a.ctypes.data, len(a), int(N), int(nharms), int(m), float(hidr),
                                dec.ctypes.data, len(dec), float(r_lo), int(total), int(blocksize),
                                int(first_block), int(nblocks), float(threshold), int(bool(exact_all)),
                                int(nthreads), out.ctypes.data, cap, ctypes.byref(sec), ctypes.byref(resc))
    nblk_real = max(0, min(nblocks, -(-total // blocksize) - first_block))
    trials = max(0, min(total, (first_block + nblk_real) * blocksize) - first_block * blocksize)
    return {"cands": out[:min(n, cap)], "ncand": int(n), "seconds": sec.value, "rescued": resc.value,
            "threads": int(nthreads), "blocks": int(nblk_real), "trials": int(trials)}


def search_blocks_ex(amps, N, dt, nharms, m, hidr, decimations, r_lo, total, blocksize, threshold, nthreads,
                     blocks=None, first_block=0, nblocks=None, exact_all=False, cap=1 << 22):
    """search_blocks over a block range, or over the listed `blocks` (global
    block indices of the band's grid), also returning each searched block's
    per-level sigma and valid-trial count: arrays [len(blocks), nlevels],
    levels in search order (k = 1 first, then the other factors as given)."""
    lib = load()
    a = np.ascontiguousarray(amps, dtype=np.complex64)
    dec = np.ascontiguousarray(decimations, dtype=np.int32)
    nlev = 1 + sum(1 for k in decimations if k > 1)
    if blocks is not None:
        bl = np.ascontiguousarray(blocks, dtype=np.int64)
        nb = len(bl)
        bptr = bl.ctypes.data
    else:
        nb = -(-total // blocksize) - first_block if nblocks is None else nblocks
        bl, bptr = None, None
    out = np.zeros(cap, CAND_DTYPE)
    sig = np.zeros((max(nb, 1), nlev), np.float64)
    nv = np.zeros((max(nb, 1), nlev), np.int32)
    sec = ctypes.c_double()
    resc = ctypes.c_int64()
    n = lib.csref_search_blocks_ex(a.ctypes.data, len(a), int(N), int(nharms), int(m), float(hidr),
                                   dec.ctypes.data, len(dec), float(r_lo), int(total), int(blocksize),
                                   int(first_block), int(nb), bptr, float(threshold), int(bool(exact_all)),
                                   int(nthreads), out.ctypes.data, cap, ctypes.byref(sec), ctypes.byref(resc),
                                   sig.ctypes.data, nv.ctypes.data)
    if n > cap:
        raise RuntimeError(f"{n} candidates exceed the oracle's capacity {cap}")
    return {"cands": out[:n], "ncand": int(n), "seconds": sec.value, "rescued": resc.value,
            "sigma": sig[:nb], "nvalid": nv[:nb], "threads": int(nthreads)}
