// cs_kernels.cu -- sm_100a kernels of the coherent-search hot path, in launch order.
//
//   k_interp       Eqn-30 direct interpolation of every harmonic's complex
//                  amplitude (fill_harmonic_row_direct!, src/directinterp.jl:470-572;
//                  per-trial fallback _fill_row_direct_slow!, :623-661); writes
//                  X rows (plain form) or 16-bit A tiles (tensor form) and the
//                  exact amplitudes of the columns the block sigma pools.
//   k_sigma        block sigma (_block_sigma, src/search.jl:490-566): exact FP32
//                  profiles of the pooled columns and their exact median.
//   k_synth_fp32   profile synthesis for every decimation level (the brfft of
//                  src/search.jl:1291 and :1675) + zero-baseline boxcar gate
//                  (_boxcar_gate!, src/search.jl:784-807) + medcut test
//                  (boxcar_metrics!, src/search.jl:825-843).  The tcgen05 form
//                  of this stage is k_synth_tc (cs_synth_tc.cu).
//   k_rescue       exact median-baseline rescan (_boxcar_exact, src/search.jl:893-904)
//                  and candidate emission (src/search.jl:1827-1838, :1695-1708).
#include "cs_internal.h"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <math.h>

#include <algorithm>
#include <math_constants.h>

namespace cs {

// ---------------------------------------------------------------------------
// Interpolation
// ---------------------------------------------------------------------------

// Rational trial grid.  One CTA per (block, harmonic).  The block's bin window
// is staged in shared memory; each thread walks trials j = tid, tid+256, ...
// carrying the exact integer state (phase row p = t mod P and the integer bin
// count (t*h*pnum) div q) incrementally.  The tap sum is a sequential FP32 FMA
// chain over the m taps, and the final complex product is unfused, which is the
// arithmetic of the reference's Float32-weight group kernel
// (src/directinterp.jl:584-605, whose zero-padded extra taps add exact zeros).
__device__ __forceinline__ float2 cmul_unfused(float2 a, float2 s) {
    // Complex{Float32} product a*s without contraction: (a.x*s.x - a.y*s.y, a.x*s.y + a.y*s.x).
    return make_float2(__fsub_rn(__fmul_rn(a.x, s.x), __fmul_rn(a.y, s.y)),
                       __fadd_rn(__fmul_rn(a.x, s.y), __fmul_rn(a.y, s.x)));
}

// ---------------------------------------------------------------------------
// Exact amplitudes on demand (block sigma samples and rescans)
// ---------------------------------------------------------------------------

// The range guard of k_interp for harmonic hp over the block's true trial
// range [t0, t0+n) (src/directinterp.jl:490-496, :633-637).
__device__ bool harm_guard(const WaveArgs& a, const DevHarm& hp, int64_t t0, int n) {
    const int m2 = a.m / 2;
    if (hp.P == 0) {
        const double rfirst = __dadd_rn(hp.hr_lo, __dmul_rn((double)t0, hp.dh));
        const double rlast = __dadd_rn(hp.hr_lo, __dmul_rn((double)(t0 + n - 1), hp.dh));
        const int64_t lo = (int64_t)floor(__dadd_rn(rfirst, 1e-15)) + 2 - m2;
        const int64_t hi = (int64_t)floor(__dadd_rn(rlast, 1e-15)) + 1 + m2;
        return lo >= 1 && hi <= a.namps && (int64_t)floor(rlast) < a.Nhalf;
    }
    const int64_t hpn = (int64_t)hp.h * hp.pnum;
    const int64_t qint0 = (t0 * hpn) / hp.q;
    const int64_t tl = t0 + n - 1;
    const int64_t qintl = (tl * hpn) / hp.q;
    const uint8_t* ct = a.ctab + hp.a_off;
    const int64_t fl0 = hp.rfloor0 + qint0 + ct[(int)(t0 % hp.P)];
    const int64_t fll = hp.rfloor0 + qintl + ct[(int)(tl % hp.P)];
    return (fl0 + 2 - m2 >= 1) && (fll + 1 + m2 <= a.namps) && (hp.rfloor0 + qintl < a.Nhalf);
}

// Amplitude of harmonic hp at global trial t (guard assumed passed), with the
// arithmetic of k_interp: bit-identical to the value k_interp writes.
// t_div_q / t_mod_q are t / q and t % q of the rational grid.
__device__ float2 exact_amp(const WaveArgs& a, const DevHarm& hp, int64_t t, int64_t t_div_q, int t_mod_q) {
    const int m = a.m, m2 = m / 2;
    if (hp.P == 0) {
        const double r = __dadd_rn(hp.hr_lo, __dmul_rn((double)t, hp.dh));
        const int64_t rint = (int64_t)floor(__dadd_rn(r, 1e-15)) + 1;
        const double dr = fmod(r, 1.0);
        const int64_t base = rint - m2;
        if (dr == 0.0) return a.amps[base + m2 - 1];
        double sre = 0.0, sim = 0.0;
        for (int i = 0; i < m; ++i) {
            const double w = 1.0 / (dr - (double)(i + 1 - m2));
            const float2 x = a.amps[base + i];
            sre = fma(w, (double)x.x, sre);
            sim = fma(w, (double)x.y, sim);
        }
        const double sn = sinpi(dr), c = cospi(dr);
        const double ar = __ddiv_rn(__dmul_rn(sn, c), M_PI);
        const double ai = -__ddiv_rn(__dmul_rn(sn, sn), M_PI);
        return make_float2((float)__dsub_rn(__dmul_rn(ar, sre), __dmul_rn(ai, sim)),
                           (float)__dadd_rn(__dmul_rn(ar, sim), __dmul_rn(ai, sre)));
    }
    // t*h*pnum = t*base_adv*q + t*s, and t*s = t_div_q*q*s + t_mod_q*s.
    const uint32_t ts = (uint32_t)t_mod_q * (uint32_t)hp.s;
    const int64_t qint = t * (int64_t)hp.base_adv + t_div_q * (int64_t)hp.s + (int64_t)(ts / (uint32_t)hp.q);
    const int p = t_mod_q % hp.P;   // P divides q
    const int64_t base = hp.rfloor0 + qint + a.ctab[hp.a_off + p] + 1 - m2;
    const float* w = a.wtab + hp.w_off;
    const float2* x = a.amps + base;
    float sre = 0.0f, sim = 0.0f;
    for (int i = 0; i < m; ++i) {
        const float wi = __ldg(w + i * hp.P + p);
        const float2 xi = __ldg(x + i);
        sre = fmaf(wi, xi.x, sre);
        sim = fmaf(wi, xi.y, sim);
    }
    return cmul_unfused(__ldg(a.atab + hp.a_off + p), make_float2(sre, sim));
}

__device__ __forceinline__ void tq_split(const DevHarm& hp, int64_t t, int64_t* t_div_q, int* t_mod_q) {
    if (hp.P == 0) { *t_div_q = 0; *t_mod_q = 0; return; }
    *t_div_q = t / hp.q;
    *t_mod_q = (int)(t - *t_div_q * hp.q);
}

constexpr int kHG = 4;   // harmonics per interpolation CTA: one 16-byte K chunk of an A tile

// Emit a block's staged rows for harmonics hidx0 .. hidx0+ng-1: FP32 rows
// (plain synthesis) or one 16-byte K chunk per trial of the block's A tiles
// (tensor synthesis), and the exact FP32 amplitudes of the columns each
// level's block sigma pools.
// pair_jh[g*nlev + l]: the index jh of harmonic hidx0+g+1 among level l's
// harmonics (h/k - 1), or -1 when the level does not fold it; pair_ncap[l] =
// max(1, kSigmaCap/nbins).  Both optional (nullptr: computed per pair here).
__device__ __forceinline__ void emit_rows(const WaveArgs& a, const float2* xo, int Nst, int blk, int hidx0,
                                          int ng, int n, float sc, const short* pair_jh = nullptr,
                                          const int* pair_ncap = nullptr) {
    if (a.X) {
        for (int g = 0; g < ng; ++g) {
            float2* xrow = a.X + ((int64_t)blk * a.nharms + hidx0 + g) * a.Nprof;
            for (int j = threadIdx.x; j < n; j += blockDim.x) xrow[j] = xo[g * Nst + j];
        }
    }
    if (a.Atile) {
        // A tile (block, j/128), row r = j%128, K chunk hidx0/4 holds (Re, Im) of
        // the 4 harmonics: SWIZZLE_NONE K-major core matrices, each K chunk's 16
        // row groups contiguous (2 KB per chunk, chunks 2 KB apart).  Split
        // tiles: the tile of residuals x - hi follows each tile.
        const int tsz = a.asplit * kATileBytes;
        uint8_t* base = a.Atile + (int64_t)blk * a.tiles_per_blk * tsz + (hidx0 >> 2) * 2048;
        const float2* x1 = xo + Nst;
        const float2* x2 = xo + 2 * Nst;
        const float2* x3 = xo + 3 * Nst;
        const float2 z = make_float2(0.0f, 0.0f);
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const float2 v0 = xo[j];
            const float2 v1 = ng > 1 ? x1[j] : z;
            const float2 v2 = ng > 2 ? x2[j] : z;
            const float2 v3 = ng > 3 ? x3[j] : z;
            uint4 pk;
            const uint32_t off = (uint32_t)(j >> 7) * (uint32_t)tsz + ((uint32_t)(j & 127) >> 3) * 128u +
                                 (uint32_t)(j & 7) * 16u;
            if (a.asplit == 2) {
                const float2 vv[4] = {v0, v1, v2, v3};
                uint32_t hw[4], lw[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (a.fp16) {
                        const float xr = vv[q].x * sc, xi = vv[q].y * sc;
                        const __half2 h = __floats2half2_rn(xr, xi);
                        const __half2 lo = __floats2half2_rn(xr - __low2float(h), xi - __high2float(h));
                        hw[q] = *reinterpret_cast<const uint32_t*>(&h);
                        lw[q] = *reinterpret_cast<const uint32_t*>(&lo);
                    } else {
                        const __nv_bfloat162 h = __floats2bfloat162_rn(vv[q].x, vv[q].y);
                        const __nv_bfloat162 lo =
                            __floats2bfloat162_rn(vv[q].x - __low2float(h), vv[q].y - __high2float(h));
                        hw[q] = *reinterpret_cast<const uint32_t*>(&h);
                        lw[q] = *reinterpret_cast<const uint32_t*>(&lo);
                    }
                }
                *reinterpret_cast<uint4*>(base + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                *reinterpret_cast<uint4*>(base + off + kATileBytes) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                continue;
            }
            if (a.fp16) {
                __half2 h0 = __floats2half2_rn(v0.x * sc, v0.y * sc), h1 = __floats2half2_rn(v1.x * sc, v1.y * sc);
                __half2 h2 = __floats2half2_rn(v2.x * sc, v2.y * sc), h3 = __floats2half2_rn(v3.x * sc, v3.y * sc);
                pk = make_uint4(*reinterpret_cast<uint32_t*>(&h0), *reinterpret_cast<uint32_t*>(&h1),
                                *reinterpret_cast<uint32_t*>(&h2), *reinterpret_cast<uint32_t*>(&h3));
            } else {
                __nv_bfloat162 h0 = __floats2bfloat162_rn(v0.x, v0.y), h1 = __floats2bfloat162_rn(v1.x, v1.y);
                __nv_bfloat162 h2 = __floats2bfloat162_rn(v2.x, v2.y), h3 = __floats2bfloat162_rn(v3.x, v3.y);
                pk = make_uint4(*reinterpret_cast<uint32_t*>(&h0), *reinterpret_cast<uint32_t*>(&h1),
                                *reinterpret_cast<uint32_t*>(&h2), *reinterpret_cast<uint32_t*>(&h3));
            }
            *reinterpret_cast<uint4*>(base + off) = pk;
        }
    }
    if (!a.samp) return;
    // One warp per (harmonic, level) pair whose level folds this harmonic;
    // lanes over its pooled columns j_c = (c*nv) div ncs (src/search.jl:528-537).
    const int lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    const int npair = ng * a.nlev;
    for (int e = threadIdx.x >> 5; e < npair; e += nwarps) {
        int g = 0, l = e;
        while (l >= a.nlev) {
            l -= a.nlev;
            ++g;
        }
        const DevLevel& L = a.levels[l];
        int jh;
        if (pair_jh) {
            jh = pair_jh[e];
        } else {
            const int h = hidx0 + g + 1;
            jh = (h % L.k == 0 && h / L.k <= L.Hk) ? h / L.k - 1 : -1;
        }
        if (jh < 0) continue;
        const int nv = a.nvalid[blk * a.nlev + l];
        if (nv <= 0) continue;
        const bool all = (int64_t)L.nbins * nv <= kSigmaCap;
        const int ncap = pair_ncap ? pair_ncap[l] : max(1, kSigmaCap / L.nbins);
        const int ncs = all ? nv : min(nv, ncap);
        float2* dst = a.samp + ((int64_t)blk * a.nlev + l) * kSampStride + (int64_t)jh * ncs;
        const float2* src = xo + g * Nst;
        if (all || ncs == 1) {
            for (int c = lane; c < ncs; c += 32) dst[c] = src[all ? c : 0];
        } else if ((int64_t)ncs * nv < (1 << 24) && nv < (1 << 22)) {
            // c*nv < 2^24 is exact in FP32, and c*nv/ncs < 2^22 carries an
            // error below 1 through the rounded reciprocal and the truncating
            // product, so one correction step either way gives the quotient.
            const uint32_t un = (uint32_t)ncs;
            const float inv = __frcp_rn((float)ncs);
            for (int c = lane; c < ncs; c += 32) {
                const uint32_t x = (uint32_t)c * (uint32_t)nv;
                uint32_t q = __float2uint_rz(__fmul_rz((float)x, inv));
                if (q * un > x) --q;
                else if ((q + 1u) * un <= x) ++q;
                dst[c] = src[q];
            }
        } else {
            // the division by ncs as a multiply-high by ceil(2^64/ncs), exact
            // for every 32-bit dividend
            const uint64_t mg = 0xFFFFFFFFFFFFFFFFull / (uint64_t)ncs + 1ull;
            for (int c = lane; c < ncs; c += 32) {
                const uint32_t x = (uint32_t)c * (uint32_t)nv;
                dst[c] = src[(int)__umul64hi((uint64_t)x, mg)];
            }
        }
    }
}

// Packed FP32 pairs (sm_100): fma.rn.f32x2 is two IEEE fmaf, lane by lane, so
// a (re, im) tap pair costs one instruction and rounds exactly like fmaf.
__device__ __forceinline__ unsigned long long f2_pack(float lo, float hi) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 f2_unpack(unsigned long long v) {
    float lo, hi;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
    return make_float2(lo, hi);
}
__device__ __forceinline__ unsigned long long f2_fma(unsigned long long a, unsigned long long b,
                                                     unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Outputs of one phase class: trials j = jc + P*u, u in [u0, u1), whose phase
// row p and window start b0 (+ u*Hs) are fixed, so the m weights and the
// complex factor stay in registers.  Same sequential FMA chain and unfused
// complex product per trial as the reference's Float32 kernel.
template <int M>
__device__ __forceinline__ void class_run(const float* __restrict__ wt, int P, int p, float2 A,
                                          const float2* __restrict__ win, int b0, int Hs, int jc, int u0,
                                          int u1, float2* xo, int m) {
    if (M > 0) {
        constexpr int MW = M > 0 ? M : 1;
        unsigned long long w2[MW];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const float wi = __ldg(wt + i * P + p);
            w2[i] = f2_pack(wi, wi);
        }
        const unsigned long long* x = reinterpret_cast<const unsigned long long*>(win + b0 + u0 * Hs);
        float2* o = xo + jc + P * u0;
#pragma unroll 2
        for (int u = u0; u < u1; ++u) {
            unsigned long long acc = 0ull;   // (+0, +0)
#pragma unroll
            for (int i = 0; i < M; ++i) acc = f2_fma(w2[i], x[i], acc);
            *o = cmul_unfused(A, f2_unpack(acc));
            x += Hs;
            o += P;
        }
    } else {
        for (int u = u0; u < u1; ++u) {
            const float2* x = win + b0 + u * Hs;
            float sre = 0.0f, sim = 0.0f;
            for (int i = 0; i < m; ++i) {
                const float wi = __ldg(wt + i * P + p);
                const float2 xi = x[i];
                sre = fmaf(wi, xi.x, sre);
                sim = fmaf(wi, xi.y, sim);
            }
            xo[jc + P * u] = cmul_unfused(A, make_float2(sre, sim));
        }
    }
}

// class_run for 16 taps when consecutive trials of the class sit HS < 16 bins
// apart: the 16 window values live in a register ring and each trial loads
// only its HS new ones.  Element i of trial it (counted from u0) sits in slot
// (i + it*HS) mod 16; after a trial the HS oldest slots take the next values.
// The ring offsets repeat after 16/gcd(16, HS) trials, the unrolled period.
// Same chain, same order of taps as class_run.
template <int HS>
__device__ __forceinline__ void slide_run(const float* __restrict__ wt, int P, int p, float2 A,
                                          const float2* __restrict__ win, int b0, int jc, int u0, int u1,
                                          float2* xo) {
    constexpr int M = 16;
    constexpr int G = (HS % 16 == 0) ? 16 : (HS % 8 == 0) ? 8 : (HS % 4 == 0) ? 4 : (HS % 2 == 0) ? 2 : 1;
    constexpr int PERIOD = M / G;
    unsigned long long w2[M], r[M];
#pragma unroll
    for (int i = 0; i < M; ++i) {
        const float wi = __ldg(wt + i * P + p);
        w2[i] = f2_pack(wi, wi);
    }
    const unsigned long long* xn = reinterpret_cast<const unsigned long long*>(win + b0 + u0 * HS);
#pragma unroll
    for (int i = 0; i < M; ++i) r[i] = xn[i];
    xn += M;
    float2* o = xo + jc + P * u0;
    int u = u0;
    while (true) {
#pragma unroll
        for (int it = 0; it < PERIOD; ++it) {
            unsigned long long acc = 0ull;   // (+0, +0)
#pragma unroll
            for (int i = 0; i < M; ++i) acc = f2_fma(w2[i], r[(i + it * HS) % M], acc);
            *o = cmul_unfused(A, f2_unpack(acc));
            o += P;
            if (++u >= u1) return;
#pragma unroll
            for (int j = 0; j < HS; ++j) r[(it * HS + j) % M] = xn[j];
            xn += HS;
        }
    }
}

__device__ __forceinline__ bool slide_dispatch(int Hs, const float* __restrict__ wt, int P, int p, float2 A,
                                               const float2* __restrict__ win, int b0, int jc, int u0, int u1,
                                               float2* xo) {
    switch (Hs) {
        case 1: slide_run<1>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 2: slide_run<2>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 3: slide_run<3>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 4: slide_run<4>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 5: slide_run<5>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 6: slide_run<6>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 7: slide_run<7>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 8: slide_run<8>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 9: slide_run<9>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 10: slide_run<10>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 11: slide_run<11>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        case 12: slide_run<12>(wt, P, p, A, win, b0, jc, u0, u1, xo); return true;
        default: return false;
    }
}

// One CTA per (group of 4 harmonics, block).  Per harmonic: the range guard on
// the block's TRUE trial range (src/directinterp.jl:490-496), the bin window
// staged in shared memory, then every phase class of the block's trials --
// trials t and t+P share the phase row (t mod P) and sit exactly
// Hs = P*h*pnum/q bins apart -- split into runs over the threads.  Three CTAs
// per SM (74 KB of shared memory each, registers capped to match) hide the
// shared-memory latency of the tap loads.
template <int M>
__global__ void __launch_bounds__(256, 3) k_interp(WaveArgs a, int win_max, int Nst, int* err) {
    extern __shared__ float2 sm_i[];
    float2* win = sm_i;
    float2* xo = sm_i + win_max;            // [kHG][Nst] staged outputs
    // Per-harmonic state of the group, computed by one thread per harmonic.
    __shared__ int s_ok[kHG], s_nw[kHG], s_p0[kHG], s_res0[kHG], s_Ub[kHG], s_chunk[kHG], s_Tc[kHG],
        s_small[kHG], s_Hs[kHG];
    __shared__ long long s_lo[kHG], s_base[kHG];   // s_base = rfloor0 + qint0 - lo + 1 - m2
    __shared__ unsigned long long s_qm[kHG];       // ceil(2^64 / q): (n div q) = mulhi(n, s_qm) for n < 2^32
    __shared__ unsigned s_pm[kHG];                 // ceil(2^24 / P): (task div P) for task * P < 2^24
    __shared__ uint32_t s_am[kMaxSpecChunks];      // FP16 A tiles: the spectrum chunks' maxima
    __shared__ int s_cidx;                         // and the block's last chunk: its scale 2^-s
    __shared__ short s_jh[kHG * kMaxLevels];       // per (harmonic, level) pair: emit_rows' pair_jh
    __shared__ int s_ncap[kMaxLevels];             // per level: emit_rows' pair_ncap

    // harmonic groups fastest: the CTAs filling one block's A tiles (each a
    // 128-byte piece of every 2 KB row group) run together
    const int hidx0 = blockIdx.x * kHG;
    const int ng = min(kHG, a.nharms - hidx0);
    const int blk = a.blk_first + (int)blockIdx.y;
    const int m = M > 0 ? M : a.m;
    const int m2 = m / 2;
    const int64_t t0 = blk_t0(a, blk);
    const int n = (int)min((int64_t)a.Nprof, a.total - t0);
    if (n <= 0) return;

    // (loaded by warps 1-2 beside warp 0's per-harmonic set-up, not after it)
    if (threadIdx.x >= 32 && threadIdx.x < 32 + kMaxSpecChunks)
        s_am[threadIdx.x - 32] = a.amax_bits ? a.amax_bits[threadIdx.x - 32] : 0u;
    if (threadIdx.x == 32 + kMaxSpecChunks) s_cidx = a.blk_cidx ? a.blk_cidx[blk] : kMaxSpecChunks - 1;
    // the sigma samples' per-pair bookkeeping, once per CTA by warps 2-3 (its
    // integer divisions off the emission's path)
    if (threadIdx.x >= 64 && threadIdx.x < 64 + ng * a.nlev) {
        const int e = (int)threadIdx.x - 64;
        int g = 0, l = e;
        while (l >= a.nlev) {
            l -= a.nlev;
            ++g;
        }
        const int h = hidx0 + g + 1, k = a.levels[l].k;
        s_jh[e] = (short)((h % k == 0 && h / k <= a.levels[l].Hk) ? h / k - 1 : -1);
    }
    if (threadIdx.x >= 160 && threadIdx.x < 160 + a.nlev)
        s_ncap[threadIdx.x - 160] = max(1, kSigmaCap / a.levels[threadIdx.x - 160].nbins);
    if (threadIdx.x < ng) {
        // Range guard on the TRUE trial range (src/directinterp.jl:490-496),
        // with the Julia 1-based bounds translated to 0-based windows.
        const int g = threadIdx.x;
        const DevHarm hp = a.harms[hidx0 + g];
        if (hp.P == 0) {
            s_ok[g] = harm_guard(a, hp, t0, n) ? 2 : 0;   // 2: per-trial FP64 path
        } else {
            const uint8_t* ct = a.ctab + hp.a_off;
            const int64_t hpn = (int64_t)hp.h * hp.pnum;
            const int64_t T0 = t0 * hpn;
            const int64_t qint0 = T0 / hp.q;
            const int p0 = (int)(t0 % hp.P);
            const int64_t tl = t0 + n - 1;
            const int64_t qintl = (tl * hpn) / hp.q;
            const int pl = (int)(tl % hp.P);
            const int64_t fl0 = hp.rfloor0 + qint0 + ct[p0];
            const int64_t fll = hp.rfloor0 + qintl + ct[pl];
            const bool ok = (fl0 + 2 - m2 >= 1) && (fll + 1 + m2 <= a.namps) &&
                            (hp.rfloor0 + qintl < a.Nhalf);
            const int64_t lo = fl0 + 1 - m2;
            const int64_t nw = fll + m2 - lo + 1;
            s_ok[g] = ok && nw <= win_max ? 1 : 0;
            if (ok && nw > win_max) atomicExch(err, 1);
            s_lo[g] = lo;
            s_nw[g] = (int)min(nw, (int64_t)win_max);
            s_p0[g] = p0;
            s_res0[g] = (int)(T0 % hp.q);
            s_base[g] = hp.rfloor0 + qint0 - lo + 1 - m2;
            // task split of the phase classes (see below)
            const int P = hp.P;
            const int Tc = P >= (int)blockDim.x ? 1 : (int)blockDim.x / P;
            const int Ub = n / P;                       // classes jc < n - Ub*P get Ub+1 trials
            s_Ub[g] = Ub;
            s_Tc[g] = Tc;
            s_chunk[g] = (Ub + 1 + Tc - 1) / Tc;
            // res0 + jc*h*pnum < 2^32 for every class: the window start fits 32-bit math
            // (q > 1: ceil(2^64/q) must fit 64 bits)
            s_small[g] = ((uint64_t)hp.q + (uint64_t)P * (uint64_t)hpn) < 0xFFFFFFFFull && hp.q > 1;
            s_Hs[g] = (int)(((int64_t)P * hpn) / hp.q);   // bins between trials t and t+P
            s_qm[g] = hp.q > 1 ? 0xFFFFFFFFFFFFFFFFull / (uint64_t)hp.q + 1ull : 0ull;
            s_pm[g] = (unsigned)((((uint64_t)1 << 24) + (uint64_t)P - 1) / (uint64_t)P);
        }
    }
    __syncthreads();

    for (int g = 0; g < ng; ++g) {
        const DevHarm& hp = a.harms[hidx0 + g];
        float2* xg = xo + g * Nst;
        if (s_ok[g] != 1) {
            // guarded-off row, or the per-trial FP64 fallback for a non-rational
            // trial step (_fill_row_direct_slow!, src/directinterp.jl:623-661)
            const bool slow = s_ok[g] == 2;
            for (int j = threadIdx.x; j < n; j += blockDim.x)
                xg[j] = slow ? exact_amp(a, hp, t0 + j, 0, 0) : make_float2(0.0f, 0.0f);
            continue;
        }
        const float* __restrict__ wt = a.wtab + hp.w_off;
        const float2* __restrict__ at = a.atab + hp.a_off;
        const uint8_t* __restrict__ ct = a.ctab + hp.a_off;
        const int64_t hpn = (int64_t)hp.h * hp.pnum;
        const int nw = s_nw[g];
        const float2* __restrict__ src = a.amps + s_lo[g];
        __syncthreads();   // the previous harmonic's window reads are done
        for (int i = threadIdx.x; i < nw; i += blockDim.x) win[i] = src[i];
        __syncthreads();
        const int P = hp.P, q = hp.q, Hs = s_Hs[g];
        // Runs: class jc (first trial j = jc, phase (p0 + jc) mod P), part `part`
        // of its u range; classes below n - Ub*P have Ub+1 trials, the rest Ub.
        const int Tc = s_Tc[g], Ub = s_Ub[g], chunk = s_chunk[g], p0 = s_p0[g], res0 = s_res0[g];
        const int small = s_small[g];
        const long long base = s_base[g];
        const int ntask = P >= (int)blockDim.x ? P : P * Tc;
        const int nlong = n - Ub * P;
        const unsigned long long qm = s_qm[g];
        const unsigned pm = s_pm[g];
        for (int task = threadIdx.x; task < ntask; task += blockDim.x) {
            // task < 256 and P <= 256 when Tc > 1, so task * P < 2^24 and the
            // multiply by ceil(2^24/P) gives the exact quotient
            const int part = Tc > 1 ? (int)(((uint64_t)task * pm) >> 24) : 0;
            const int jc = task - part * P;
            if (jc >= n) continue;
            const int U = Ub + (jc < nlong ? 1 : 0);
            const int u0 = part * chunk, u1 = min(U, u0 + chunk);
            if (u0 >= u1) continue;
            int p = p0 + jc;
            if (p >= P) p -= P;
            const int64_t qv = small ? (int64_t)__umul64hi((uint64_t)((uint32_t)res0 + (uint32_t)jc * (uint32_t)hpn), qm)
                                     : ((int64_t)res0 + (int64_t)jc * hpn) / q;
            const int b0 = (int)(base + qv + ct[p]);
            const float2 A = __ldg(at + p);
            if (M == 16 && u1 - u0 >= 2 && slide_dispatch(Hs, wt, P, p, A, win, b0, jc, u0, u1, xg)) continue;
            class_run<M>(wt, P, p, A, win, b0, Hs, jc, u0, u1, xg, m);
        }
    }
    __syncthreads();
    const float sc = a.fp16 && a.Atile ? pow2f(-ascale_exp(s_am, s_cidx)) : 1.0f;   // exact power of two
    emit_rows(a, xo, Nst, blk, hidx0, ng, n, sc, s_jh, s_ncap);
}

// ---------------------------------------------------------------------------
// Persistent form of k_interp for the common case (m = 16, rational trial
// grid, every phase cycle P <= 256).  Two CTAs per SM walk the work items
// (block, group of 4 harmonics), group fastest.  An item's four bin windows
// arrive by bulk copy (cp.async.bulk, 16-byte aligned body; the odd first and
// last bins by plain loads) into a staging buffer, issued by warp 0 as soon as
// the previous item's taps are done, so the copy runs under that item's
// emission of A tiles and sigma samples.  Two barriers per item: after the
// taps (the staging buffer and the staged rows are complete) and after the
// emission (the rows are free, the next windows have landed).  The tap
// arithmetic is k_interp's, bit for bit.
// ---------------------------------------------------------------------------
constexpr int kI2Threads = 256;

struct HarmStage {
    int ok;             // 1: computed; 0: zero row
    int head;           // window element 0 sits at stage + head (1 when its address is not 16-byte aligned)
    int p0, res0, Ub, Tc, chunk, small, Hs;
    unsigned pm;        // ceil(2^24 / P)
    float sc;           // FP16 A tiles: the block's scale 2^-s (exact), the same in every slot
    long long base;     // rfloor0 + qint0 - lo + 1 - m2
    unsigned long long qm;   // ceil(2^64 / q), q > 1
};

__device__ __forceinline__ int i2_wstride(int win_max) { return (win_max + 3) & ~1; }

// Warp 0: the per-harmonic state of `item` into st[], its windows' plain-loaded
// edge bins, and the bulk copies of their bodies, completing on *bar.
__device__ void i2_prepare(const WaveArgs& a, int item, int ngroups, int win_max, float2* stage, HarmStage* st,
                           uint64_t* bar, int* err) {
    const int lane = threadIdx.x & 31;
    const int bi = item / ngroups, grp = item - bi * ngroups;   // harmonic groups fastest
    const int blk = a.blk_first + bi;
    const int hidx0 = grp * kHG;
    const int ng = min(kHG, a.nharms - hidx0);
    const int64_t t0 = blk_t0(a, blk);
    const int n = (int)min((int64_t)a.Nprof, a.total - t0);
    const int m2 = 8;
    const int wstride = i2_wstride(win_max);
    uint32_t body_bytes = 0;
    int head = 0, body = 0, tail = 0;
    int64_t lo = 0;
    if (lane < ng) {
        const DevHarm hp = a.harms[hidx0 + lane];
        const uint8_t* ct = a.ctab + hp.a_off;
        const int64_t hpn = (int64_t)hp.h * hp.pnum;
        const int64_t T0 = t0 * hpn;
        const int64_t qint0 = T0 / hp.q;
        const int p0 = (int)(t0 % hp.P);
        const int64_t tl = t0 + n - 1;
        const int64_t qintl = (tl * hpn) / hp.q;
        const int pl = (int)(tl % hp.P);
        const int64_t fl0 = hp.rfloor0 + qint0 + ct[p0];
        const int64_t fll = hp.rfloor0 + qintl + ct[pl];
        // range guard on the TRUE trial range (src/directinterp.jl:490-496)
        const bool ok = (fl0 + 2 - m2 >= 1) && (fll + 1 + m2 <= a.namps) && (hp.rfloor0 + qintl < a.Nhalf) && n > 0;
        lo = fl0 + 1 - m2;
        const int64_t nw = fll + m2 - lo + 1;
        HarmStage h{};
        h.ok = ok && nw <= win_max ? 1 : 0;
        if (ok && nw > win_max) atomicExch(err, 1);
        if (h.ok) {
            head = (reinterpret_cast<uintptr_t>(a.amps + lo) & 15u) ? 1 : 0;
            body = ((int)nw - head) & ~1;
            tail = (int)nw - head - body;
            body_bytes = (uint32_t)body * 8u;
        }
        h.head = head;
        h.p0 = p0;
        h.res0 = (int)(T0 % hp.q);
        h.base = hp.rfloor0 + qint0 - lo + 1 - m2;
        const int P = hp.P;
        const int Tc = P >= kI2Threads ? 1 : kI2Threads / P;
        const int Ub = n / P;                       // classes jc < n - Ub*P get Ub+1 trials
        h.Ub = Ub;
        h.Tc = Tc;
        h.chunk = (Ub + 1 + Tc - 1) / Tc;
        h.small = ((uint64_t)hp.q + (uint64_t)P * (uint64_t)hpn) < 0xFFFFFFFFull && hp.q > 1;
        h.sc = a.fp16 && a.Atile ? pow2f(-ascale_exp_blk(a, blk)) : 1.0f;
        h.Hs = (int)(((int64_t)P * hpn) / hp.q);   // bins between trials t and t+P
        h.qm = hp.q > 1 ? 0xFFFFFFFFFFFFFFFFull / (uint64_t)hp.q + 1ull : 0ull;
        h.pm = (unsigned)((((uint64_t)1 << 24) + (uint64_t)P - 1) / (uint64_t)P);
        st[lane] = h;
    }
    uint32_t total = body_bytes;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    if (lane == 0) mbar_expect_tx(bar, total);   // the one arrival of the phase, with every copy's bytes
    __syncwarp();
    if (lane < ng && (head | body | tail)) {
        float2* win = stage + lane * wstride + head;
        const float2* src = a.amps + lo;
        if (head) win[0] = src[0];
        if (tail) win[head + body] = src[head + body];
        if (body) bulk_copy(smem_u32(win + head), src + head, (uint32_t)body * 8u, bar);
    }
}

__global__ void __launch_bounds__(kI2Threads, 2) k_interp2(WaveArgs a, int win_max, int Nst, int nitems, int* err) {
    extern __shared__ __align__(16) float2 sm_i2[];
    float2* xo = sm_i2;                                  // [kHG][Nst] staged rows
    float2* stage = sm_i2 + kHG * Nst;                   // [kHG][wstride] bin windows
    const int wstride = i2_wstride(win_max);
    __shared__ HarmStage st[2][kHG];
    __shared__ __align__(8) uint64_t wbar;
    const int ngroups = (a.nharms + kHG - 1) / kHG;
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        mbar_init(&wbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int item = blockIdx.x;
    uint32_t pend = 0;   // parity of the latest phase copies were issued on
    if (item < nitems && warp == 0) i2_prepare(a, item, ngroups, win_max, stage, st[0], &wbar, err);
    bool ok = __syncthreads_or(item < nitems && !mbar_wait(&wbar, 0)) == 0;
    if (!ok && threadIdx.x == 0) atomicExch(err, 4);
    for (int it = 0; item < nitems && ok; item += gridDim.x, ++it) {
        const HarmStage* S = st[it & 1];
        const int bi = item / ngroups, grp = item - bi * ngroups;
        const int blk = a.blk_first + bi;
        const int hidx0 = grp * kHG;
        const int ng = min(kHG, a.nharms - hidx0);
        const int64_t t0 = blk_t0(a, blk);
        const int n = (int)min((int64_t)a.Nprof, a.total - t0);
        for (int g = 0; g < ng; ++g) {
            float2* xg = xo + g * Nst;
            const HarmStage h = S[g];
            if (h.ok != 1) {
                for (int j = threadIdx.x; j < n; j += blockDim.x) xg[j] = make_float2(0.0f, 0.0f);
                continue;
            }
            const DevHarm& hp = a.harms[hidx0 + g];
            const float* __restrict__ wt = a.wtab + hp.w_off;
            const float2* __restrict__ at = a.atab + hp.a_off;
            const uint8_t* __restrict__ ct = a.ctab + hp.a_off;
            const float2* __restrict__ win = stage + g * wstride + h.head;
            const int64_t hpn = (int64_t)hp.h * hp.pnum;
            const int P = hp.P, q = hp.q, Hs = h.Hs;
            const int Tc = h.Tc, Ub = h.Ub, chunk = h.chunk;
            const int ntask = P >= kI2Threads ? P : P * Tc;
            const int nlong = n - Ub * P;
            for (int task = threadIdx.x; task < ntask; task += blockDim.x) {
                // task < 256 and P <= 256 when Tc > 1: task * P < 2^24, exact quotient
                const int part = Tc > 1 ? (int)(((uint64_t)task * h.pm) >> 24) : 0;
                const int jc = task - part * P;
                if (jc >= n) continue;
                const int U = Ub + (jc < nlong ? 1 : 0);
                const int u0 = part * chunk, u1 = min(U, u0 + chunk);
                if (u0 >= u1) continue;
                int p = h.p0 + jc;
                if (p >= P) p -= P;
                const int64_t qv = h.small ? (int64_t)__umul64hi((uint64_t)((uint32_t)h.res0 + (uint32_t)jc * (uint32_t)hpn), h.qm)
                                           : ((int64_t)h.res0 + (int64_t)jc * hpn) / q;
                const int b0 = (int)(h.base + qv + ct[p]);
                const float2 A = __ldg(at + p);
                if (u1 - u0 >= 2 && slide_dispatch(Hs, wt, P, p, A, win, b0, jc, u0, u1, xg)) continue;
                class_run<16>(wt, P, p, A, win, b0, Hs, jc, u0, u1, xg, 16);
            }
        }
        __syncthreads();   // taps done: the staging buffer is free, the rows complete
        const int nxt = item + (int)gridDim.x;
        if (nxt < nitems && warp == 0) i2_prepare(a, nxt, ngroups, win_max, stage, st[(it + 1) & 1], &wbar, err);
        if (nxt < nitems) pend = (uint32_t)((it + 1) & 1);
        emit_rows(a, xo, Nst, blk, hidx0, ng, n, S[0].sc);
        // rows emitted; the next item's windows have landed (bounded wait)
        ok = __syncthreads_or(nxt < nitems && !mbar_wait(&wbar, (uint32_t)((it + 1) & 1))) == 0;
        if (!ok && threadIdx.x == 0) atomicExch(err, 4);
    }
    if (!ok && threadIdx.x == 0) mbar_wait(&wbar, pend);   // bounded: lets a late copy land before exit
}

size_t interp2_smem(int win_max, int Nprof) {
    return (size_t)(kHG * Nprof + kHG * ((win_max + 3) & ~1)) * sizeof(float2);
}

cudaError_t launch_interp2(const WaveArgs& a, cudaStream_t st, int win_max, int* err, int num_sms) {
    const int ngroups = (a.nharms + kHG - 1) / kHG;
    const int nitems = ngroups * a.nblk;
    const size_t smem = interp2_smem(win_max, a.Nprof);
    cudaFuncSetAttribute(k_interp2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int grid = std::min(nitems, 2 * num_sms);
    k_interp2<<<grid, kI2Threads, smem, st>>>(a, win_max, a.Nprof, nitems, err);
    return cudaGetLastError();
}

// The largest |Re| or |Im| of each chunk of a spectrum (NaN ignored), for the
// FP16 A-tile scale: one chunk per grid row, grid-stride maximum, warp
// reduction, one atomicMax on the float bits (non-negative floats order like
// their bits) per warp into out[chunk].
__global__ void __launch_bounds__(256) k_amax(const float2* __restrict__ amps, int64_t n, int64_t unit,
                                               uint32_t* out) {
    const int64_t c0 = spec_chunk_lo(unit, (int)blockIdx.y);
    const int64_t c1 = spec_chunk_hi(unit, (int)blockIdx.y, n);
    float mx = 0.0f;
    for (int64_t i = c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c1;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float2 x = amps[i];
        mx = fmaxf(mx, fmaxf(fabsf(x.x), fabsf(x.y)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out + blockIdx.y, __float_as_uint(mx));
}

cudaError_t launch_amax(const float2* amps, int64_t n, int64_t unit, int nchunk, uint32_t* out, cudaStream_t st,
                        int num_sms) {
    if (nchunk < 1 || nchunk > kMaxSpecChunks || unit < 1) return cudaErrorInvalidValue;
    // every chunk gets the full grid row (the last holds half the bins; the
    // small ones leave most of theirs idle), so the largest chunk has enough
    // loads in flight
    k_amax<<<dim3(num_sms * 4, nchunk), 256, 0, st>>>(amps, n, unit, out);
    return cudaGetLastError();
}

size_t interp_smem(int win_max, int Nprof) { return (size_t)(win_max + kHG * Nprof) * sizeof(float2); }

cudaError_t launch_interp(const WaveArgs& a, cudaStream_t st, int win_max, int* err) {
    dim3 grid((a.nharms + kHG - 1) / kHG, a.nblk);
    const size_t smem = interp_smem(win_max, a.Nprof);
    const int Nst = a.Nprof;
    switch (a.m) {
        case 16:
            cudaFuncSetAttribute(k_interp<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<16><<<grid, 256, smem, st>>>(a, win_max, Nst, err);
            break;
        case 32:
            cudaFuncSetAttribute(k_interp<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<32><<<grid, 256, smem, st>>>(a, win_max, Nst, err);
            break;
        case 8:
            cudaFuncSetAttribute(k_interp<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<8><<<grid, 256, smem, st>>>(a, win_max, Nst, err);
            break;
        default:
            cudaFuncSetAttribute(k_interp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<0><<<grid, 256, smem, st>>>(a, win_max, Nst, err);
            break;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Profile synthesis (FP32 SIMT) + zero-baseline gate + sigma samples
// ---------------------------------------------------------------------------
//
// Level k folds base harmonics k, 2k, ..., Hk*k into nbins = 2*Hk bins.  The
// unnormalised c2r transform with DC = 0 is
//   prof[n] = E[n] + O[n],  prof[N-n] = E[n] - O[n],
//   E[n] = sum_{j<Hk} a_j*2cos(2 pi j n/N) + a_Hk*(-1)^n,  O[n] = -sum_{j<Hk} b_j*2sin(2 pi j n/N)
// (Im of the Nyquist term ignored, as FFTW's c2r does).  The twiddle rows C2/S2
// are the host-rounded FP32 values of those FP64 cosines/sines.

// Profile values E[n0..n0+7] +- O: shared by the tile kernel and the rescan.
__device__ __forceinline__ void synth_chunk8(const float2* __restrict__ xs, int xstride,
                                             const float* __restrict__ C2,
                                             const float* __restrict__ S2, int np, int k, int Hk,
                                             int n0, float E[8], float O[8]) {
    // adjacent outputs (u, u+1) as one packed fma.rn.f32x2: per output the
    // same sequential fmaf chain
    unsigned long long e[4], o[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) e[v] = o[v] = f2_pack(0.0f, 0.0f);
#pragma unroll 4
    for (int jh = 1; jh < Hk; ++jh) {
        const float2 x = xs[(jh * k - 1) * xstride];
        const ulonglong2 c01 = *reinterpret_cast<const ulonglong2*>(C2 + jh * np + n0);
        const ulonglong2 c23 = *reinterpret_cast<const ulonglong2*>(C2 + jh * np + n0 + 4);
        const ulonglong2 s01 = *reinterpret_cast<const ulonglong2*>(S2 + jh * np + n0);
        const ulonglong2 s23 = *reinterpret_cast<const ulonglong2*>(S2 + jh * np + n0 + 4);
        const unsigned long long xr = f2_pack(x.x, x.x), xi = f2_pack(x.y, x.y);
        e[0] = f2_fma(xr, c01.x, e[0]);
        e[1] = f2_fma(xr, c01.y, e[1]);
        e[2] = f2_fma(xr, c23.x, e[2]);
        e[3] = f2_fma(xr, c23.y, e[3]);
        o[0] = f2_fma(xi, s01.x, o[0]);
        o[1] = f2_fma(xi, s01.y, o[1]);
        o[2] = f2_fma(xi, s23.x, o[2]);
        o[3] = f2_fma(xi, s23.y, o[3]);
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float2 ev = f2_unpack(e[v]), ov = f2_unpack(o[v]);
        E[2 * v] = ev.x;
        E[2 * v + 1] = ev.y;
        O[2 * v] = ov.x;
        O[2 * v + 1] = ov.y;
    }
    const float ny = xs[(Hk * k - 1) * xstride].x;
#pragma unroll
    for (int u = 0; u < 8; ++u) E[u] = E[u] + (((n0 + u) & 1) ? -ny : ny);
}

// synth_chunk8 for two columns sharing each twiddle load; per output the same
// sequential FMA chain, hence the same values.  Adjacent outputs (u, u+1) go
// as one packed fma.rn.f32x2 (two IEEE fmaf), the twiddle pair loaded as one
// 64-bit operand.
__device__ __forceinline__ void synth_chunk8x2(const float2* __restrict__ xa, const float2* __restrict__ xb,
                                               int xstride, const float* __restrict__ C2,
                                               const float* __restrict__ S2, int np, int Hk, int n0,
                                               float Ea[8], float Oa[8], float Eb[8], float Ob[8]) {
    unsigned long long ea[4], oa[4], eb[4], ob[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) ea[v] = oa[v] = eb[v] = ob[v] = f2_pack(0.0f, 0.0f);
#pragma unroll 2
    for (int jh = 1; jh < Hk; ++jh) {
        const float2 x = xa[(jh - 1) * xstride];
        const float2 y = xb[(jh - 1) * xstride];
        const ulonglong2 c01 = *reinterpret_cast<const ulonglong2*>(C2 + jh * np + n0);
        const ulonglong2 c23 = *reinterpret_cast<const ulonglong2*>(C2 + jh * np + n0 + 4);
        const ulonglong2 s01 = *reinterpret_cast<const ulonglong2*>(S2 + jh * np + n0);
        const ulonglong2 s23 = *reinterpret_cast<const ulonglong2*>(S2 + jh * np + n0 + 4);
        const unsigned long long c[4] = {c01.x, c01.y, c23.x, c23.y};
        const unsigned long long sv[4] = {s01.x, s01.y, s23.x, s23.y};
        const unsigned long long xr = f2_pack(x.x, x.x), xi = f2_pack(x.y, x.y);
        const unsigned long long yr = f2_pack(y.x, y.x), yi = f2_pack(y.y, y.y);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            ea[v] = f2_fma(xr, c[v], ea[v]);
            oa[v] = f2_fma(xi, sv[v], oa[v]);
            eb[v] = f2_fma(yr, c[v], eb[v]);
            ob[v] = f2_fma(yi, sv[v], ob[v]);
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float2 e0 = f2_unpack(ea[v]), o0 = f2_unpack(oa[v]), e1 = f2_unpack(eb[v]), o1 = f2_unpack(ob[v]);
        Ea[2 * v] = e0.x; Ea[2 * v + 1] = e0.y;
        Oa[2 * v] = o0.x; Oa[2 * v + 1] = o0.y;
        Eb[2 * v] = e1.x; Eb[2 * v + 1] = e1.y;
        Ob[2 * v] = o1.x; Ob[2 * v + 1] = o1.y;
    }
    const float nya = xa[(Hk - 1) * xstride].x;
    const float nyb = xb[(Hk - 1) * xstride].x;
#pragma unroll
    for (int u = 0; u < 8; ++u) {
        Ea[u] = Ea[u] + (((n0 + u) & 1) ? -nya : nya);
        Eb[u] = Eb[u] + (((n0 + u) & 1) ? -nyb : nyb);
    }
}

// Window-energy bound of the gate (the FP32 form of the tensor epilogue's
// skip).  Over the stored prefix rows ps[0 .. nbins+W] of trial column t,
// with y_e = ps[e+1] - ps[e], every gate term ps[p+w] - ps[p] (w <= W) is a
// sum of w of the y, so by Cauchy-Schwarz (ps[p+w] - ps[p]) / sqrt(w) is at
// most the root of the largest sum of y^2 over W consecutive columns from a
// start p < nbins.  Returned: that largest sum (FP32, fused multiply-add
// prefix of y^2 and a W-slot ring of it) and the total of y^2 for the
// rounding slack.
template <int W>
__device__ __forceinline__ float ps_window_energy(const float* buf, int TT, int t, int nbins, float* qtot) {
    float ring[W];
#pragma unroll
    for (int d = 0; d < W; ++d) ring[d] = INFINITY;   // no window starts before column 0
    ring[0] = 0.0f;
    float q = 0.0f, mx = -INFINITY, prev = buf[t];
    const int ne = nbins + W - 1;   // columns e whose window [e+1-W, e+1) starts at p < nbins
    for (int e0 = 0; e0 < ne; e0 += W) {
#pragma unroll
        for (int u = 0; u < W; ++u) {
            if (e0 + u < ne) {
                const float cur = buf[(e0 + u + 1) * TT + t];
                const float y = cur - prev;
                prev = cur;
                q = fmaf(y, y, q);
                // Q[e+1] and Q[e+1-W] share ring slot (u+1) mod W
                mx = fmaxf(mx, q - ring[(u + 1) % W]);
                ring[(u + 1) % W] = q;
            }
        }
    }
    *qtot = q;
    return mx;
}

__device__ __forceinline__ float ps_energy_bound(const float* buf, int TT, int t, int nbins, int W) {
    float q = 0.0f, mx;
    switch (W) {
        case 1: mx = ps_window_energy<1>(buf, TT, t, nbins, &q); break;
        case 2: mx = ps_window_energy<2>(buf, TT, t, nbins, &q); break;
        case 3: mx = ps_window_energy<3>(buf, TT, t, nbins, &q); break;
        case 4: mx = ps_window_energy<4>(buf, TT, t, nbins, &q); break;
        case 5: mx = ps_window_energy<5>(buf, TT, t, nbins, &q); break;
        case 6: mx = ps_window_energy<6>(buf, TT, t, nbins, &q); break;
        case 7: mx = ps_window_energy<7>(buf, TT, t, nbins, &q); break;
        case 8: mx = ps_window_energy<8>(buf, TT, t, nbins, &q); break;
        default: return INFINITY;   // wider boxcars: no bound, the full scan runs
    }
    // slack: 2^-13 of the total for the prefix roundings of both scans and the
    // differences of the stored rows, then a relative 2^-16 for the rest
    return (sqrtf(mx + q * 0x1p-13f) + 0x1p-13f * sqrtf((float)(nbins + W) * q)) * (1.0f + 0x1p-16f);
}

__global__ void __launch_bounds__(2 * kTileTrials) k_synth_fp32(WaveArgs a) {
    constexpr int TT = kTileTrials;
    extern __shared__ float4 smem4[];
    float2* Xs = reinterpret_cast<float2*>(smem4);               // [nharms][TT]
    float* buf = reinterpret_cast<float*>(Xs + a.nharms * TT);   // [nbuf][TT]
    __shared__ float red[2][TT];
    __shared__ int skip_sh[TT];

    const int tile = blockIdx.x;
    const int blk = blockIdx.y;
    const int t = threadIdx.x % TT;
    const int half = threadIdx.x / TT;
    const int j = tile * TT + t;

    for (int idx = threadIdx.x; idx < a.nharms * TT; idx += blockDim.x) {
        const int hh = idx / TT, tt = idx % TT, jj = tile * TT + tt;
        Xs[idx] = jj < a.Nprof ? a.X[((int64_t)blk * a.nharms + hh) * a.Nprof + jj]
                               : make_float2(0.0f, 0.0f);
    }
    __syncthreads();

    for (int l = 0; l < a.nlev; ++l) {
        const DevLevel& L = a.levels[l];
        const int k = L.k, Hk = L.Hk, nbins = L.nbins, wmax = L.wmax, np = L.np, nw = L.nw;
        const int nv = a.nvalid[blk * a.nlev + l];
        if (tile * TT >= nv) continue;  // uniform: nothing valid in this tile
        const float invsig = inv_sigma(a.sigma[blk * a.nlev + l]);   // used by the medcut test below
        const int OFF = wmax + 1;
        const float* C2 = a.tw + L.tw_off;
        const float* S2 = C2 + (int64_t)Hk * np;
        const int nch = (Hk + 1 + 7) / 8;
        for (int ch = half; ch < nch; ch += 2) {
            const int n0 = ch * 8;
            float E[8], O[8];
            synth_chunk8(Xs + t, TT, C2, S2, np, k, Hk, n0, E, O);
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int nn = n0 + u;
                if (nn <= Hk) buf[(OFF + nn) * TT + t] = E[u] + O[u];
                if (nn >= 1 && nn < Hk) buf[(OFF + 2 * Hk - nn) * TT + t] = E[u] - O[u];
            }
        }
        __syncthreads();
        if (half == 0) {
            // Wrapped prefix sums in place: ps[i] lands in row i, reading prof
            // from row OFF+i >= i+1 before it is overwritten.
            float s = 0.0f;
            buf[t] = 0.0f;
            for (int i = 0; i < nbins; ++i) {
                s += buf[(OFF + i) * TT + t];
                buf[(i + 1) * TT + t] = s;
            }
            for (int u = 1; u <= wmax; ++u) buf[(nbins + u) * TT + t] = s + buf[u * TT + t];
            // skip the full gate scan when the window-energy bound keeps this
            // trial's gate below both the medcut test and the threshold (its
            // gate is then -inf: neither flagged nor a candidate); never with
            // the exact gate values requested
            const float c = fminf(a.medcut_gate, a.threshold);
            bool skip = false;
            if (!a.Q0 && invsig > 0.0f && c > 0.0f)
                skip = ps_energy_bound(buf, TT, t, nbins, wmax) < (c / invsig) * (1.0f - 0x1p-16f);
            skip_sh[t] = skip;
        }
        __syncthreads();
        float best = -INFINITY;
        if (!skip_sh[t]) for (int wi = half; wi < nw; wi += 2) {
            const int w = L.widths[wi];
            float mm = buf[w * TT + t] - buf[t];
            for (int p = 1; p < nbins; ++p) mm = fmaxf(mm, buf[(p + w) * TT + t] - buf[p * TT + t]);
            best = fmaxf(best, mm * L.rsqrtw[wi]);
        }
        red[half][t] = best;
        __syncthreads();
        if (half == 0 && j < nv) {
            const float g = fmaxf(red[0][t], red[1][t]);
            if (a.Q0) a.Q0[((int64_t)blk * a.nlev + l) * a.Nprof + j] = g;
            gate_flag(a, blk, l, j, g, invsig);
        }
        __syncthreads();
    }
}

size_t synth_fp32_smem(int nharms, int maxbins, int maxwmax) {
    return (size_t)nharms * kTileTrials * sizeof(float2) +
           (size_t)(maxbins + maxwmax + 1) * kTileTrials * sizeof(float);
}

cudaError_t launch_synth_fp32(const WaveArgs& a, cudaStream_t st, int smem_bytes) {
    dim3 grid((a.Nprof + kTileTrials - 1) / kTileTrials, a.nblk);
    cudaFuncSetAttribute(k_synth_fp32, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    k_synth_fp32<<<grid, 2 * kTileTrials, smem_bytes, st>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Block sigma: exact FP32 profiles of the pooled columns, then the exact median
// ---------------------------------------------------------------------------

// Block-wide exclusive prefix sum of one int per thread (blockDim.x <= 1024).
__device__ __forceinline__ int block_excl_scan(int v, int* warp_tot, int* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        int incl = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_tot[lane] = incl - w;
        if (lane == 31) *total = incl;
    }
    __syncthreads();
    const int r = warp_tot[wid] + x - v;
    __syncthreads();
    return r;
}

// k-th smallest (0-based) of ns non-negative floats given as bit patterns
// (non-negative IEEE floats order like their unsigned bits): three radix
// passes of 11/11/10 bits with a parallel bucket search.
__device__ uint32_t radix_select(const uint32_t* vals, int ns, int kth, uint32_t* hist, int* sh, int* wtot) {
    uint32_t prefix = 0, mask = 0;
    int kk = kth;
    const int shifts[3] = {21, 10, 0};
    const int bits[3] = {11, 11, 10};
    for (int pass = 0; pass < 3; ++pass) {
        const int shift = shifts[pass], nb = 1 << bits[pass];
        for (int i = threadIdx.x; i < nb; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const uint32_t v = vals[i];
            if ((v & mask) == prefix) atomicAdd(&hist[(v >> shift) & (uint32_t)(nb - 1)], 1u);
        }
        __syncthreads();
        const int per = (nb + (int)blockDim.x - 1) / (int)blockDim.x;
        const int b0 = min(nb, (int)threadIdx.x * per), b1 = min(nb, b0 + per);
        int local = 0;
        for (int b = b0; b < b1; ++b) local += (int)hist[b];
        const int excl = block_excl_scan(local, wtot, sh + 2);
        if (excl <= kk && kk < excl + local) {
            int c = excl;
            for (int b = b0; b < b1; ++b) {
                const int hb = (int)hist[b];
                if (c + hb > kk) {
                    sh[0] = b;
                    sh[1] = kk - c;
                    break;
                }
                c += hb;
            }
        }
        __syncthreads();
        prefix |= (uint32_t)sh[0] << shift;
        mask |= (uint32_t)(nb - 1) << shift;
        kk = sh[1];
        __syncthreads();
    }
    return prefix;
}

// radix_select with fewer barriers, for the block sigma: two histogram
// buffers (the next pass's is cleared while this pass counts) and two slots
// for the scan's warp totals and the pass result, so that nothing written in
// one pass is overwritten before every thread has read it.  Four barriers per
// pass.  hist2 holds 2 x 2048 bins; wtot2 2 x 32 ints; sh2 2 x 4 ints.
// With `next`, also the (kth+1)-th smallest value into *next (written by
// thread 0 before the last barrier) when the last pass's histogram holds it,
// that is when it shares the kth's top 22 bits; else 0xFFFFFFFF, and the
// caller finds it itself.
__device__ uint32_t radix_select_2buf(const uint32_t* vals, int ns, int kth, uint32_t* hist2, int* sh2, int* wtot2,
                                      uint32_t* next = nullptr) {
    uint32_t prefix = 0, mask = 0;
    int kk = kth;
    const int shifts[3] = {21, 10, 0};
    const int bits[3] = {11, 11, 10};
    const int nthr = (int)blockDim.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < 2048; i += nthr) hist2[i] = 0;
    __syncthreads();
    for (int pass = 0; pass < 3; ++pass) {
        const int shift = shifts[pass], nb = 1 << bits[pass];
        uint32_t* hist = hist2 + (pass & 1) * 2048;
        uint32_t* hnext = hist2 + ((pass + 1) & 1) * 2048;
        int* wtot = wtot2 + (pass & 1) * 32;
        int* sh = sh2 + (pass & 1) * 4;
        if (next && pass == 2 && threadIdx.x == 0) sh[2] = -1;   // read only after the barriers below
        for (int i = threadIdx.x; i < ns; i += nthr) {
            const uint32_t v = vals[i];
            if ((v & mask) == prefix) atomicAdd(&hist[(v >> shift) & (uint32_t)(nb - 1)], 1u);
        }
        if (pass < 2)
            for (int i = threadIdx.x; i < 2048; i += nthr) hnext[i] = 0;
        __syncthreads();
        const int per = (nb + nthr - 1) / nthr;
        const int b0 = min(nb, (int)threadIdx.x * per), b1 = min(nb, b0 + per);
        int local = 0;
        for (int b = b0; b < b1; ++b) local += (int)hist[b];
        // block exclusive scan of `local`
        int x = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wtot[wid] = x;
        __syncthreads();
        if (wid == 0) {
            const int w = lane < (nthr >> 5) ? wtot[lane] : 0;
            int incl = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            if (lane < (nthr >> 5)) wtot[lane] = incl - w;
        }
        __syncthreads();
        const int excl = wtot[wid] + x - local;
        if (excl <= kk && kk < excl + local) {
            int c = excl;
            for (int b = b0; b < b1; ++b) {
                const int hb = (int)hist[b];
                if (c + hb > kk) {
                    sh[0] = b;
                    sh[1] = kk - c;
                    break;
                }
                c += hb;
            }
        }
        // last pass: the bin of rank kk+1 as well
        if (next && pass == 2 && excl <= kk + 1 && kk + 1 < excl + local) {
            int c = excl;
            for (int b = b0; b < b1; ++b) {
                const int hb = (int)hist[b];
                if (c + hb > kk + 1) {
                    sh[2] = b;
                    break;
                }
                c += hb;
            }
        }
        __syncthreads();
        if (next && pass == 2 && threadIdx.x == 0)
            *next = sh[2] >= 0 ? (prefix | (uint32_t)sh[2]) : 0xFFFFFFFFu;
        prefix |= (uint32_t)sh[0] << shift;
        mask |= (uint32_t)(nb - 1) << shift;
        kk = sh[1];
    }
    return prefix;
}

// One CTA per (block, level).  The columns _block_sigma pools
// (src/search.jl:528-537): every valid column when nbins*nv <= 8192, else ncol
// whole columns spaced evenly.  k_interp leaves their exact FP32 amplitudes in
// `samp`; their profiles are built here with synth_chunk8 -- the arithmetic of
// the FP32 synthesis and of the rescan -- so sigma is identical in every
// synthesis mode.  sigma = 1.4826 * median(|x|), _median! semantics.
// Two forms, picked by the autotuner: NT = 384 threads with the level's
// twiddle rows copied into shared memory beside the samples (two CTAs per SM),
// or NT = 256 with the twiddles read through L1 from global memory (less
// shared memory: three CTAs per SM).  Same arithmetic, same sigma.
template <int NT, bool TWS>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 2) k_sigma(WaveArgs a, int* err) {
    extern __shared__ float4 ss4[];
    __shared__ int sh[4];
    __shared__ int wtot[32];
    __shared__ int sh2[8];      // radix_select_2buf's two result slots
    __shared__ int wtot2[64];   // and its two scan slots
    __shared__ uint32_t red[32];
    __shared__ __align__(8) uint64_t sbar;
    __shared__ __align__(8) uint64_t never;   // test hook: a barrier no thread or copy completes
    const int bl = blockIdx.x;
    const int l = bl % a.nlev;
    const DevLevel& L = a.levels[l];
    const int Hk = L.Hk, nbins = L.nbins, np = L.np;
    const int nv = a.nvalid[bl];
    if (nv <= 0) {
        if (threadIdx.x == 0) a.sigma[bl] = 0.0f;
        return;
    }
    const bool all = (int64_t)nbins * nv <= kSigmaCap;
    const int ncs = all ? nv : min(nv, max(1, kSigmaCap / nbins));
    const int ns = ncs * nbins;
    float2* Xs = reinterpret_cast<float2*>(ss4);                    // [Hk][ncs], <= kSampStride
    uint32_t* hist = reinterpret_cast<uint32_t*>(ss4);              // 2 x 2048 bins: reuses Xs once profiles exist
    uint32_t* vals = reinterpret_cast<uint32_t*>(Xs + kSampStride);  // [ns]
    float* tws = reinterpret_cast<float*>(vals + kSigmaCap);        // the level's C2 then S2 rows (TWS)
    const float* C2 = TWS ? tws : a.tw + L.tw_off;
    const float* S2 = C2 + Hk * np;
    const float2* samp = a.samp + (int64_t)bl * kSampStride;
    // The samples arrive by one bulk copy (rounded up to 16 bytes, still inside
    // this (block, level)'s kSampStride slot) instead of dependent loads.
    if (threadIdx.x == 0) {
        mbar_init(&sbar, 1);
        mbar_init(&never, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // the level's twiddle rows come along (2*Hk*np floats, a multiple of 64 bytes)
        const uint32_t xb = (uint32_t)((Hk * ncs * (int)sizeof(float2) + 15) & ~15);
        const uint32_t tb = TWS ? (uint32_t)(2 * Hk * np * (int)sizeof(float)) : 0u;
        mbar_expect_tx(&sbar, xb + tb);
        bulk_copy(smem_u32(Xs), samp, xb, &sbar);
        if (TWS) bulk_copy(smem_u32(tws), a.tw + L.tw_off, tb, &sbar);
    }
    if (__syncthreads_or(!mbar_wait(&sbar, 0))) {
        // give up (every thread alike) with an error status, after the copy in
        // flight (bounded again)
        mbar_wait(&sbar, 0);
        if (threadIdx.x == 0) {
            atomicExch(err, 3);
            a.sigma[bl] = 0.0f;
        }
        return;
    }
    // Test hook of the bounded waits: block 0 waits on a barrier whose phase
    // never completes (no arrival is ever made on it; the sample copy above has
    // landed), gives up after stall_ns and takes the error exit.
    if (a.stall_ns > 0 && bl == 0) {
        const bool done = mbar_wait(&never, 0, (uint64_t)a.stall_ns);
        if (__syncthreads_or(!done)) {
            if (threadIdx.x == 0) {
                atomicExch(err, 3);
                a.sigma[bl] = 0.0f;
            }
            return;
        }
    }
    // Two columns per thread share each twiddle load (read through L1) when
    // the pairs fit one pass of the CTA; otherwise one column per thread, so
    // that the pass count, not a thin second pass, sets the time.
    const int nch = (Hk + 1 + 7) / 8;
    const int npairs = (ncs + 1) / 2;
    if (npairs * nch > (int)blockDim.x) {
        for (int idx = threadIdx.x; idx < ncs * nch; idx += blockDim.x) {
            const int sl = idx % ncs, ch = idx / ncs;
            const int n0 = ch * 8;
            float E[8], O[8];
            synth_chunk8(Xs + sl, ncs, C2, S2, np, 1, Hk, n0, E, O);
            uint32_t* d = vals + sl * nbins;
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int nn = n0 + u;
                if (nn <= Hk) d[nn] = __float_as_uint(fabsf(E[u] + O[u]));
                if (nn >= 1 && nn < Hk) d[2 * Hk - nn] = __float_as_uint(fabsf(E[u] - O[u]));
            }
        }
    } else for (int idx = threadIdx.x; idx < npairs * nch; idx += blockDim.x) {
        const int pr = idx % npairs, ch = idx / npairs;
        const int sa = 2 * pr, sb = min(2 * pr + 1, ncs - 1);
        const int n0 = ch * 8;
        float Ea[8], Oa[8], Eb[8], Ob[8];
        synth_chunk8x2(Xs + sa, Xs + sb, ncs, C2, S2, np, Hk, n0, Ea, Oa, Eb, Ob);
        uint32_t* da = vals + sa * nbins;
        uint32_t* db = vals + sb * nbins;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int nn = n0 + u;
            if (nn <= Hk) {
                da[nn] = __float_as_uint(fabsf(Ea[u] + Oa[u]));
                db[nn] = __float_as_uint(fabsf(Eb[u] + Ob[u]));
            }
            if (nn >= 1 && nn < Hk) {
                da[2 * Hk - nn] = __float_as_uint(fabsf(Ea[u] - Oa[u]));
                db[2 * Hk - nn] = __float_as_uint(fabsf(Eb[u] - Ob[u]));
            }
        }
    }
    __syncthreads();
    const int half = ns >> 1;
    float med;
    if (ns & 1) {
        med = __uint_as_float(radix_select_2buf(vals, ns, half, hist, sh2, wtot2));
    } else {
        // _median! (src/search.jl:295-305): mean of the two central order statistics.
        __shared__ uint32_t hi_sh;
        const uint32_t lo = radix_select_2buf(vals, ns, half - 1, hist, sh2, wtot2, &hi_sh);
        __syncthreads();
        const uint32_t hi = hi_sh;
        if (hi != 0xFFFFFFFFu) {
            med = 0.5f * (__uint_as_float(lo) + __uint_as_float(hi));
            if (threadIdx.x == 0) a.sigma[bl] = 1.4826f * med;
            return;
        }
        int le = 0;
        uint32_t above = 0xFFFFFFFFu;
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const uint32_t v = vals[i];
            le += v <= lo;
            if (v > lo && v < above) above = v;
        }
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            le += __shfl_xor_sync(0xffffffffu, le, o);
            above = min(above, __shfl_xor_sync(0xffffffffu, above, o));
        }
        if (lane == 0) { wtot[wid] = le; red[wid] = above; }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tle = 0;
            uint32_t tab = 0xFFFFFFFFu;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { tle += wtot[w]; tab = min(tab, red[w]); }
            sh[3] = (int)(tle >= half + 1 ? lo : tab);
        }
        __syncthreads();
        med = 0.5f * (__uint_as_float(lo) + __uint_as_float((uint32_t)sh[3]));
    }
    if (threadIdx.x == 0) a.sigma[bl] = 1.4826f * med;
}

size_t sigma_smem(int max_hk, int max_np, int variant) {
    return (size_t)kSampStride * sizeof(float2) + (size_t)kSigmaCap * sizeof(uint32_t) +
           (variant == 1 ? 0 : (size_t)2 * max_hk * max_np * sizeof(float));
}

cudaError_t launch_sigma(const WaveArgs& a, cudaStream_t st, int max_hk, int max_np, int* err, int variant) {
    const size_t smem = sigma_smem(max_hk, max_np, variant);
    if (variant == 1) {
        cudaFuncSetAttribute(k_sigma<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_sigma<256, false><<<a.nblk * a.nlev, 256, smem, st>>>(a, err);
    } else {
        cudaFuncSetAttribute(k_sigma<kSigmaThreads, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_sigma<kSigmaThreads, true><<<a.nblk * a.nlev, kSigmaThreads, smem, st>>>(a, err);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Gate test and exact rescan
// ---------------------------------------------------------------------------

// In-situ normalisation (_normalize, src/search.jl:1638-1643; the candidate
// test of decim_pass!/_search_region!, :1704-1707, :1834-1837): the trial's
// searched frequency f = k*(rstart + j*lodr)/T in FP64 (the host's expressions,
// no contraction), its window w = clamp(searchsortedlast(edges, f), 1, nwin),
// and z = (M - loc[w]) / scale[w] against the threshold.
__device__ bool norm_pass(const WaveArgs& a, int blk, int l, int k, int j, float metric) {
    const int64_t i0 = blk_t0(a, blk);
    const double rstart = __dadd_rn(a.r_lo, __dmul_rn((double)i0, a.lodr));
    const double rf = __dadd_rn(rstart, __dmul_rn((double)j, a.lodr));
    const double r = k == 1 ? rf : __dmul_rn((double)k, rf);
    const double f = __ddiv_rn(r, a.T);
    const int nw = a.norm_nwin;
    const double* e = a.norm_edges + (int64_t)l * (nw + 1);
    int w = 0;
    for (int i = 0; i <= nw; ++i) w += e[i] <= f;   // searchsortedlast: edges <= f
    w = min(max(w, 1), nw) - 1;
    const double z = __ddiv_rn(__dsub_rn((double)metric, a.norm_loc[l * nw + w]), a.norm_scale[l * nw + w]);
    return z > a.norm_thr;
}

constexpr int kRescueWarps = 4;

// One warp per (block, level, trial).  Lanes recompute the exact amplitudes of
// the level's harmonics, then the FP32 profile chunks (synth_chunk8, the
// arithmetic of the FP32 synthesis), then:
//  * when the gate was a 16-bit one, the FP32 zero-baseline gate exactly as
//    k_synth_fp32 forms it, against medcut -- so the rescanned set is the
//    plain form's;
//  * the exact metric: median baseline (order statistics by rank counting),
//    sequential wrapped prefix sums, max over phase and width
//    (src/search.jl:571-598, :893-904).
__global__ void __launch_bounds__(32 * kRescueWarps) k_rescue(WaveArgs a) {
    __shared__ float2 xs_all[kRescueWarps][kMaxBins / 2 + 8];
    __shared__ float prof_all[kRescueWarps][kMaxBins];
    __shared__ float ps_all[kRescueWarps][2 * kMaxBins + 2];
    __shared__ float med_all[kRescueWarps][2];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* xs = xs_all[wid];
    float* prof = prof_all[wid];
    float* ps = ps_all[wid];
    const int64_t count = a.exact_all ? (int64_t)a.nblk * a.nlev * a.Nprof
                                      : (int64_t)min(*a.n_items, a.cap_items);
    const int64_t gwarps = (int64_t)gridDim.x * kRescueWarps;
    for (int64_t idx = blockIdx.x * (int64_t)kRescueWarps + wid; idx < count; idx += gwarps) {
        int blk, l, j;
        if (a.exact_all) {
            j = (int)(idx % a.Nprof);
            const int bl = (int)(idx / a.Nprof);
            if (j >= a.nvalid[bl]) continue;   // warp-uniform
            l = bl % a.nlev;
            blk = bl / a.nlev;
        } else {
            const DevItem it = a.items[idx];
            blk = it.blk;
            l = it.lev;
            j = it.j;
        }
        const float invsig = inv_sigma(a.sigma[blk * a.nlev + l]);
        const DevLevel& L = a.levels[l];
        const int k = L.k, Hk = L.Hk, nbins = L.nbins, np = L.np, nw = L.nw, wmax = L.wmax;
        float metric = 0.0f;
        if (invsig > 0.0f) {
            const int64_t t0 = blk_t0(a, blk);
            const int n = (int)min((int64_t)a.Nprof, a.total - t0);
            const int64_t t = t0 + j;
            for (int jh = 1 + lane; jh <= Hk; jh += 32) {
                const DevHarm& hp = a.harms[jh * k - 1];
                float2 v = make_float2(0.0f, 0.0f);
                if (harm_guard(a, hp, t0, n)) {
                    int64_t tdq;
                    int tmq;
                    tq_split(hp, t, &tdq, &tmq);
                    v = exact_amp(a, hp, t, tdq, tmq);
                }
                xs[jh - 1] = v;
            }
            __syncwarp();
            const float* C2 = a.tw + L.tw_off;
            const float* S2 = C2 + (int64_t)Hk * np;
            const int nch = (Hk + 1 + 7) / 8;
            if (lane < nch) {
                const int n0 = lane * 8;
                float E[8], O[8];
                synth_chunk8(xs, 1, C2, S2, np, 1, Hk, n0, E, O);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int nn = n0 + u;
                    if (nn <= Hk) prof[nn] = E[u] + O[u];
                    if (nn >= 1 && nn < Hk) prof[2 * Hk - nn] = E[u] - O[u];
                }
            }
            __syncwarp();
            bool exact = true;
            if (a.verify_gate) {
                // k_synth_fp32's gate: sequential prefix, wrap as ps[nbins] + ps[u].
                if (lane == 0) {
                    float s = 0.0f;
                    ps[0] = 0.0f;
                    for (int i = 0; i < nbins; ++i) { s += prof[i]; ps[i + 1] = s; }
                    for (int u = 1; u <= wmax; ++u) ps[nbins + u] = s + ps[u];
                }
                __syncwarp();
                float best = -INFINITY;
                for (int wi = 0; wi < nw; ++wi) {
                    const int w = L.widths[wi];
                    float mm = -INFINITY;
                    for (int p = lane; p < nbins; p += 32) mm = fmaxf(mm, ps[p + w] - ps[p]);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, o));
                    best = fmaxf(best, mm * L.rsqrtw[wi]);
                }
                const float m0 = best * invsig;
                if (!(m0 >= a.medcut)) {
                    metric = m0;
                    exact = false;
                }
                __syncwarp();
            }
            if (exact) {
                // Median: the values of rank half-1 and half by counting.
                const int half = nbins >> 1;
                for (int i = lane; i < nbins; i += 32) {
                    const float v = prof[i];
                    int lt = 0, le = 0;
                    for (int q2 = 0; q2 < nbins; ++q2) {
                        const float u = prof[q2];
                        lt += u < v;
                        le += u <= v;
                    }
                    if (nbins & 1) {
                        if (lt <= half && half < le) med_all[wid][0] = v;
                    } else {
                        if (lt <= half - 1 && half - 1 < le) med_all[wid][0] = v;
                        if (lt <= half && half < le) med_all[wid][1] = v;
                    }
                }
                __syncwarp();
                const float med = (nbins & 1) ? med_all[wid][0] : 0.5f * (med_all[wid][0] + med_all[wid][1]);
                if (lane == 0) {
                    ps[0] = 0.0f;
                    for (int i = 0; i < nbins + wmax; ++i) {
                        const int id = i >= nbins ? i - nbins : i;
                        ps[i + 1] = ps[i] + (prof[id] - med);
                    }
                }
                __syncwarp();
                float best = -INFINITY;
                for (int wi = 0; wi < nw; ++wi) {
                    const int w = L.widths[wi];
                    const float invsw = invsig / sqrtf((float)w);
                    float mm = -INFINITY;
                    for (int p = lane; p < nbins; p += 32) mm = fmaxf(mm, ps[p + w] - ps[p]);
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) mm = fmaxf(mm, __shfl_xor_sync(0xffffffffu, mm, o));
                    const float cand = mm * invsw;
                    if (cand > best) best = cand;
                }
                metric = best;
            }
        }
        if (lane == 0) {
            if (a.tmetric) a.tmetric[((int64_t)blk * a.nlev + l) * a.Nprof + j] = metric;
            if (a.norm_edges ? norm_pass(a, blk, l, k, j, metric) : metric > a.threshold)
                push_cand(a, blk, l, j, metric);
        }
        __syncwarp();
    }
}

cudaError_t launch_rescue(const WaveArgs& a, cudaStream_t st, int num_sms) {
    k_rescue<<<num_sms * 8, 32 * kRescueWarps, 0, st>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Metric statistics (the opt-in MetricStats sink, src/search.jl:1296-1560)
// ---------------------------------------------------------------------------

constexpr int kMstSmemBins = 8192;   // histograms up to this many bins accumulate in shared memory

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One CTA per (block, level) of an exact_all wave: over the valid trials'
// exact metrics (tmetric), the moments and exact median of _block_stats
// (:1339-1359: two-pass std with n-1, _median! mean of the two central values)
// and the histogram pushes of _hist_push! (:1428-1442) into the (level, window)
// histogram of the block's centre frequency.  Sums are FP64 per block; the host
// adds the blocks in order.
__global__ void __launch_bounds__(256) k_mstats(WaveArgs a) {
    extern __shared__ uint32_t msm[];
    uint32_t* rhist = msm;          // radix histogram (2048)
    uint32_t* hbins = msm + 2048;   // metric histogram when it fits
    __shared__ int sh[4];
    __shared__ int wtot[32];
    __shared__ double dred[4][32];
    __shared__ uint32_t ured[32];
    const int bl = blockIdx.x;
    const int l = bl % a.nlev;
    const int nv = a.nvalid[bl];
    double* out = a.mst + (int64_t)bl * kMstFields;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarp = blockDim.x >> 5;
    if (nv <= 0) {
        if (tid < kMstFields) out[tid] = tid == 0 ? 0.0 : CUDART_NAN;
        return;
    }
    const float* v = a.tmetric + (int64_t)bl * a.Nprof;
    const int nb = a.hist_nb;
    const bool smh = nb <= kMstSmemBins;
    for (int i = tid; i < (smh ? nb : 0); i += blockDim.x) hbins[i] = 0;
    __syncthreads();
    const int w = a.mwin[bl];
    unsigned long long* gcount = a.mhist + ((int64_t)l * a.hist_nwin + w) * nb;
    double s = 0.0, s2 = 0.0, mn = CUDART_INF, mx = -CUDART_INF;
    uint32_t under = 0, over = 0;
    for (int j = tid; j < nv; j += blockDim.x) {
        const double x = (double)v[j];
        s = __dadd_rn(s, x);
        s2 = __dadd_rn(s2, __dmul_rn(x, x));
        mn = fmin(mn, x);
        mx = fmax(mx, x);
        if (x < a.hist_lo) {
            ++under;
        } else if (x >= a.hist_hi) {
            ++over;
        } else {
            int bin = (int)floor(__dmul_rn(__dsub_rn(x, a.hist_lo), a.hist_invw));
            bin = min(bin, nb - 1);
            if (smh) atomicAdd(&hbins[bin], 1u);
            else atomicAdd(&gcount[bin], 1ull);
        }
    }
    s = warp_sum_d(s);
    s2 = warp_sum_d(s2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        under += __shfl_xor_sync(0xffffffffu, under, o);
        over += __shfl_xor_sync(0xffffffffu, over, o);
    }
    if (lane == 0) {
        dred[0][wid] = s;
        dred[1][wid] = s2;
        dred[2][wid] = mn;
        dred[3][wid] = mx;
        wtot[wid] = (int)under;
        ured[wid] = over;
    }
    __syncthreads();
    if (tid == 0) {
        double ts = 0.0, ts2 = 0.0, tmn = CUDART_INF, tmx = -CUDART_INF;
        uint32_t tu = 0, to = 0;
        for (int q = 0; q < nwarp; ++q) {
            ts = __dadd_rn(ts, dred[0][q]);
            ts2 = __dadd_rn(ts2, dred[1][q]);
            tmn = fmin(tmn, dred[2][q]);
            tmx = fmax(tmx, dred[3][q]);
            tu += (uint32_t)wtot[q];
            to += ured[q];
        }
        out[0] = (double)nv;
        out[1] = tmn;
        out[5] = tmx;
        out[6] = ts;
        out[7] = ts2;
        out[3] = ts / (double)nv;
        if (tu) atomicAdd(&a.muo[((int64_t)l * a.hist_nwin + w) * 2 + 0], (unsigned long long)tu);
        if (to) atomicAdd(&a.muo[((int64_t)l * a.hist_nwin + w) * 2 + 1], (unsigned long long)to);
    }
    __syncthreads();
    for (int i = tid; i < (smh ? nb : 0); i += blockDim.x)
        if (hbins[i]) atomicAdd(&gcount[i], (unsigned long long)hbins[i]);
    // second pass: sum of squared deviations from the mean
    const double mean = out[3];
    double ss = 0.0;
    for (int j = tid; j < nv; j += blockDim.x) {
        const double d = __dsub_rn((double)v[j], mean);
        ss = __dadd_rn(ss, __dmul_rn(d, d));
    }
    ss = warp_sum_d(ss);
    __syncthreads();
    if (lane == 0) dred[0][wid] = ss;
    __syncthreads();
    if (tid == 0) {
        double t = 0.0;
        for (int q = 0; q < nwarp; ++q) t = __dadd_rn(t, dred[0][q]);
        out[4] = nv > 1 ? sqrt(t / (double)(nv - 1)) : 0.0;
    }
    // exact median (metrics are non-negative, so their bit patterns order like them)
    const uint32_t* vb = reinterpret_cast<const uint32_t*>(v);
    const int half = nv >> 1;
    double med;
    if (nv & 1) {
        med = (double)__uint_as_float(radix_select(vb, nv, half, rhist, sh, wtot));
    } else {
        const uint32_t lo = radix_select(vb, nv, half - 1, rhist, sh, wtot);
        int le = 0;
        uint32_t above = 0xFFFFFFFFu;
        for (int i = tid; i < nv; i += blockDim.x) {
            const uint32_t x = vb[i];
            le += x <= lo;
            if (x > lo && x < above) above = x;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            le += __shfl_xor_sync(0xffffffffu, le, o);
            above = min(above, __shfl_xor_sync(0xffffffffu, above, o));
        }
        __syncthreads();
        if (lane == 0) { wtot[wid] = le; ured[wid] = above; }
        __syncthreads();
        if (tid == 0) {
            int tle = 0;
            uint32_t tab = 0xFFFFFFFFu;
            for (int q = 0; q < nwarp; ++q) { tle += wtot[q]; tab = min(tab, ured[q]); }
            sh[3] = (int)(tle >= half + 1 ? lo : tab);
        }
        __syncthreads();
        med = 0.5 * ((double)__uint_as_float(lo) + (double)__uint_as_float((uint32_t)sh[3]));
    }
    if (tid == 0) out[2] = med;
}

size_t mstats_smem(int nprof, int hist_nb) {
    (void)nprof;
    return (size_t)2048 * sizeof(uint32_t) + (hist_nb <= kMstSmemBins ? (size_t)hist_nb * sizeof(uint32_t) : 0);
}

cudaError_t launch_mstats(const WaveArgs& a, cudaStream_t st) {
    const size_t smem = mstats_smem(a.Nprof, a.hist_nb);
    cudaFuncSetAttribute(k_mstats, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_mstats<<<a.nblk * a.nlev, 256, smem, st>>>(a);
    return cudaGetLastError();
}

}  // namespace cs
