// cs_kernels.cu -- sm_100a kernels of the coherent-search hot path.
//
//   k_interp       Eqn-30 direct interpolation of every harmonic's complex
//                  amplitude (fill_harmonic_row_direct!, src/directinterp.jl:470-572;
//                  per-trial fallback _fill_row_direct_slow!, :623-661).
//   k_synth_fp32   profile synthesis for every decimation level (the brfft of
//                  src/search.jl:1291 and :1675) + zero-baseline boxcar gate
//                  (_boxcar_gate!, src/search.jl:784-807) + the |x| samples the
//                  block sigma pools (_block_sigma, src/search.jl:490-566).
//   k_sigma        exact median of the pooled samples per (block, level).
//   k_flag         medcut test of the gate (boxcar_metrics!, src/search.jl:825-843).
//   k_rescue       exact median-baseline rescan (_boxcar_exact, src/search.jl:893-904)
//                  and candidate emission (src/search.jl:1827-1838, :1695-1708).
#include "cs_internal.h"

#include <math.h>

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
template <int M>
__device__ __forceinline__ float2 tap_sum(const float* __restrict__ w, int P, int p,
                                          const float2* __restrict__ x, int m) {
    float sre = 0.0f, sim = 0.0f;
    if (M > 0) {
#pragma unroll
        for (int i = 0; i < M; ++i) {
            const float wi = __ldg(w + i * P + p);
            const float2 xi = x[i];
            sre = fmaf(wi, xi.x, sre);
            sim = fmaf(wi, xi.y, sim);
        }
    } else {
        for (int i = 0; i < m; ++i) {
            const float wi = __ldg(w + i * P + p);
            const float2 xi = x[i];
            sre = fmaf(wi, xi.x, sre);
            sim = fmaf(wi, xi.y, sim);
        }
    }
    return make_float2(sre, sim);
}

__device__ __forceinline__ float2 cmul_unfused(float2 a, float2 s) {
    // Complex{Float32} product a*s without contraction: (a.x*s.x - a.y*s.y, a.x*s.y + a.y*s.x).
    return make_float2(__fsub_rn(__fmul_rn(a.x, s.x), __fmul_rn(a.y, s.y)),
                       __fadd_rn(__fmul_rn(a.x, s.y), __fmul_rn(a.y, s.x)));
}

template <int M>
__global__ void __launch_bounds__(256) k_interp(WaveArgs a, int win_max, int* err) {
    extern __shared__ float2 win[];
    __shared__ int s_ok, s_nw, s_p0, s_res0;
    __shared__ long long s_lo, s_base;  // s_base = rfloor0 + qint0 - lo + 1 - m2

    const int blk = blockIdx.x;
    const int hidx = blockIdx.y;
    const DevHarm hp = a.harms[hidx];
    const int m = M > 0 ? M : a.m;
    const int m2 = m / 2;
    const int64_t t0 = a.t_first + (int64_t)blk * a.Nprof;
    const int n = (int)min((int64_t)a.Nprof, a.total - t0);
    if (n <= 0) return;
    float2* __restrict__ xrow = a.X + ((int64_t)blk * a.nharms + hidx) * a.Nprof;

    if (hp.P == 0) {
        // Per-trial FP64 fallback for a non-rational trial step
        // (_fill_row_direct_slow!, src/directinterp.jl:623-661).  Julia does not
        // contract, so the FP64 expressions are evaluated with explicit rounding.
        const double rfirst = __dadd_rn(hp.hr_lo, __dmul_rn((double)t0, hp.dh));
        const double rlast = __dadd_rn(hp.hr_lo, __dmul_rn((double)(t0 + n - 1), hp.dh));
        const int64_t lo = (int64_t)floor(__dadd_rn(rfirst, 1e-15)) + 2 - m2;
        const int64_t hi = (int64_t)floor(__dadd_rn(rlast, 1e-15)) + 1 + m2;
        const bool ok = lo >= 1 && hi <= a.namps && (int64_t)floor(rlast) < a.Nhalf;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            float2 out = make_float2(0.0f, 0.0f);
            if (ok) {
                const double r = __dadd_rn(hp.hr_lo, __dmul_rn((double)(t0 + j), hp.dh));
                const int64_t rint = (int64_t)floor(__dadd_rn(r, 1e-15)) + 1;
                const double dr = fmod(r, 1.0);
                const int64_t base = rint - m2;  // 0-based tap i at base + i
                if (dr == 0.0) {
                    out = a.amps[base + m2 - 1];
                } else {
                    double sre = 0.0, sim = 0.0;
                    for (int i = 0; i < m; ++i) {
                        const double w = 1.0 / (dr - (double)(i + 1 - m2));
                        const float2 x = a.amps[base + i];
                        sre = fma(w, (double)x.x, sre);
                        sim = fma(w, (double)x.y, sim);
                    }
                    const double s = sinpi(dr), c = cospi(dr);
                    const double ar = __ddiv_rn(__dmul_rn(s, c), M_PI);
                    const double ai = -__ddiv_rn(__dmul_rn(s, s), M_PI);
                    out.x = (float)__dsub_rn(__dmul_rn(ar, sre), __dmul_rn(ai, sim));
                    out.y = (float)__dadd_rn(__dmul_rn(ar, sim), __dmul_rn(ai, sre));
                }
            }
            xrow[j] = out;
        }
        return;
    }

    const float* __restrict__ wt = a.wtab + hp.w_off;
    const float2* __restrict__ at = a.atab + hp.a_off;
    const uint8_t* __restrict__ ct = a.ctab + hp.a_off;
    const int64_t hpn = (int64_t)hp.h * hp.pnum;
    if (threadIdx.x == 0) {
        // Range guard on the TRUE trial range (src/directinterp.jl:490-496),
        // with the Julia 1-based bounds translated to 0-based windows.
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
        s_ok = ok && nw <= win_max;
        if (ok && nw > win_max) atomicExch(err, 1);
        s_lo = lo;
        s_nw = (int)min(nw, (int64_t)win_max);
        s_p0 = p0;
        s_res0 = (int)(T0 % hp.q);
        s_base = hp.rfloor0 + qint0 - lo + 1 - m2;
    }
    __syncthreads();
    if (!s_ok) {
        for (int j = threadIdx.x; j < n; j += blockDim.x) xrow[j] = make_float2(0.0f, 0.0f);
        return;
    }
    const int nw = s_nw;
    const float2* __restrict__ src = a.amps + s_lo;
    for (int i = threadIdx.x; i < nw; i += blockDim.x) win[i] = src[i];
    __syncthreads();

    const int P = hp.P, q = hp.q;
    const int step = blockDim.x;
    // Trial j: p = (p0 + j) mod P;  (res0 + j*hpn) = qv*q + rv.
    int j = threadIdx.x;
    int p = (int)((s_p0 + (int64_t)j) % P);
    const int pstep = step % P;
    int64_t v = (int64_t)s_res0 + (int64_t)j * hpn;
    int64_t qv = v / q;
    int rv = (int)(v % q);
    const int64_t dv = (int64_t)step * hpn;
    const int64_t dq = dv / q;
    const int drr = (int)(dv % q);
    const int64_t base0 = s_base;
    for (; j < n; j += step) {
        const int b = (int)(base0 + qv + ct[p]);   // window index of tap 0
        const float2 s = tap_sum<M>(wt, P, p, win + b, m);
        xrow[j] = cmul_unfused(at[p], s);
        p += pstep;
        if (p >= P) p -= P;
        qv += dq;
        rv += drr;
        if (rv >= q) { rv -= q; qv += 1; }
    }
}

cudaError_t launch_interp(const WaveArgs& a, cudaStream_t st, int win_max, int* err) {
    dim3 grid(a.nblk, a.nharms);
    const size_t smem = (size_t)win_max * sizeof(float2);
    switch (a.m) {
        case 16:
            cudaFuncSetAttribute(k_interp<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<16><<<grid, 256, smem, st>>>(a, win_max, err);
            break;
        case 32:
            cudaFuncSetAttribute(k_interp<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<32><<<grid, 256, smem, st>>>(a, win_max, err);
            break;
        case 8:
            cudaFuncSetAttribute(k_interp<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<8><<<grid, 256, smem, st>>>(a, win_max, err);
            break;
        default:
            cudaFuncSetAttribute(k_interp<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            k_interp<0><<<grid, 256, smem, st>>>(a, win_max, err);
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
#pragma unroll
    for (int u = 0; u < 8; ++u) { E[u] = 0.0f; O[u] = 0.0f; }
    for (int jh = 1; jh < Hk; ++jh) {
        const float2 x = xs[(jh * k - 1) * xstride];
        const float4 c0 = *reinterpret_cast<const float4*>(C2 + jh * np + n0);
        const float4 c1 = *reinterpret_cast<const float4*>(C2 + jh * np + n0 + 4);
        const float4 s0 = *reinterpret_cast<const float4*>(S2 + jh * np + n0);
        const float4 s1 = *reinterpret_cast<const float4*>(S2 + jh * np + n0 + 4);
        E[0] = fmaf(x.x, c0.x, E[0]); E[1] = fmaf(x.x, c0.y, E[1]);
        E[2] = fmaf(x.x, c0.z, E[2]); E[3] = fmaf(x.x, c0.w, E[3]);
        E[4] = fmaf(x.x, c1.x, E[4]); E[5] = fmaf(x.x, c1.y, E[5]);
        E[6] = fmaf(x.x, c1.z, E[6]); E[7] = fmaf(x.x, c1.w, E[7]);
        O[0] = fmaf(x.y, s0.x, O[0]); O[1] = fmaf(x.y, s0.y, O[1]);
        O[2] = fmaf(x.y, s0.z, O[2]); O[3] = fmaf(x.y, s0.w, O[3]);
        O[4] = fmaf(x.y, s1.x, O[4]); O[5] = fmaf(x.y, s1.y, O[5]);
        O[6] = fmaf(x.y, s1.z, O[6]); O[7] = fmaf(x.y, s1.w, O[7]);
    }
    const float ny = xs[(Hk * k - 1) * xstride].x;
#pragma unroll
    for (int u = 0; u < 8; ++u) E[u] = E[u] + (((n0 + u) & 1) ? -ny : ny);
}

// Slot of profile column j among the columns _block_sigma pools for a
// (block, level) with nv valid columns (src/search.jl:528-537), or -1.
__device__ __forceinline__ int sigma_slot(int j, int nv, int nbins) {
    if ((int64_t)nbins * nv <= kSigmaCap) return j < nv ? j : -1;
    const int ncol = min(nv, max(1, kSigmaCap / nbins));
    const int c = (int)(((int64_t)j * ncol + nv - 1) / nv);  // ceil(j*ncol/nv)
    if (c < ncol && (int)(((int64_t)c * nv) / ncol) == j) return c;
    return -1;
}

__global__ void __launch_bounds__(2 * kTileTrials) k_synth_fp32(WaveArgs a) {
    constexpr int TT = kTileTrials;
    extern __shared__ float4 smem4[];
    float2* Xs = reinterpret_cast<float2*>(smem4);               // [nharms][TT]
    float* buf = reinterpret_cast<float*>(Xs + a.nharms * TT);   // [nbuf][TT]
    __shared__ float red[2][TT];

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
        if (j < nv) {
            const int slot = sigma_slot(j, nv, nbins);
            if (slot >= 0) {
                float* dst = a.sub + ((int64_t)blk * a.nlev + l) * kSigmaCap + (int64_t)slot * nbins;
                for (int i = half; i < nbins; i += 2) dst[i] = fabsf(buf[(OFF + i) * TT + t]);
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
        }
        __syncthreads();
        float best = -INFINITY;
        for (int wi = half; wi < nw; wi += 2) {
            const int w = L.widths[wi];
            float mm = buf[w * TT + t] - buf[t];
            for (int p = 1; p < nbins; ++p) mm = fmaxf(mm, buf[(p + w) * TT + t] - buf[p * TT + t]);
            best = fmaxf(best, mm * L.rsqrtw[wi]);
        }
        red[half][t] = best;
        __syncthreads();
        if (half == 0 && j < nv)
            a.Q0[((int64_t)blk * a.nlev + l) * a.Nprof + j] = fmaxf(red[0][t], red[1][t]);
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
// Block sigma: exact median of the pooled |x| samples (radix select)
// ---------------------------------------------------------------------------

// k-th smallest (0-based) of ns non-negative floats given as bit patterns;
// non-negative IEEE floats order like their unsigned bit patterns.
__device__ uint32_t radix_select(const uint32_t* vals, int ns, int kth, uint32_t* hist, int* sh) {
    uint32_t prefix = 0, mask = 0;
    int kk = kth;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < ns; i += blockDim.x) {
            const uint32_t v = vals[i];
            if ((v & mask) == prefix) atomicAdd(&hist[(v >> shift) & 255u], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int cum = 0, d = 0;
            for (; d < 255; ++d) {
                const int c = (int)hist[d];
                if (cum + c > kk) break;
                cum += c;
            }
            sh[0] = d;
            sh[1] = kk - cum;
        }
        __syncthreads();
        prefix |= (uint32_t)sh[0] << shift;
        mask |= 255u << shift;
        kk = sh[1];
        __syncthreads();
    }
    return prefix;
}

__global__ void __launch_bounds__(256) k_sigma(WaveArgs a) {
    __shared__ uint32_t vals[kSigmaCap];
    __shared__ uint32_t hist[256];
    __shared__ int sh[2];
    const int bl = blockIdx.x;
    const int l = bl % a.nlev;
    const int nbins = a.levels[l].nbins;
    const int nv = a.nvalid[bl];
    const int64_t N = (int64_t)nbins * nv;
    int ns;
    if (N <= kSigmaCap) ns = (int)N;
    else ns = min(nv, max(1, kSigmaCap / nbins)) * nbins;
    if (ns == 0) {
        if (threadIdx.x == 0) a.sigma[bl] = 0.0f;
        return;
    }
    const float* src = a.sub + (int64_t)bl * kSigmaCap;
    for (int i = threadIdx.x; i < ns; i += blockDim.x) vals[i] = __float_as_uint(src[i]);
    __syncthreads();
    const int half = ns >> 1;
    float med;
    if (ns & 1) {
        med = __uint_as_float(radix_select(vals, ns, half, hist, sh));
    } else {
        const float lo = __uint_as_float(radix_select(vals, ns, half - 1, hist, sh));
        const float hi = __uint_as_float(radix_select(vals, ns, half, hist, sh));
        med = 0.5f * (lo + hi);
    }
    if (threadIdx.x == 0) a.sigma[bl] = 1.4826f * med;
}

cudaError_t launch_sigma(const WaveArgs& a, cudaStream_t st) {
    k_sigma<<<a.nblk * a.nlev, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Gate test and exact rescan
// ---------------------------------------------------------------------------

__device__ __forceinline__ void push_cand(const WaveArgs& a, int blk, int l, int j, float metric) {
    const int pos = atomicAdd(a.n_cands, 1);
    if (pos < a.cap_cands) {
        DevCand c;
        c.blk = a.blk_base + blk;
        c.lev = l;
        c.j = j;
        c.metric = metric;
        a.cands[pos] = c;
    }
}

__device__ __forceinline__ float inv_sigma(float sig) { return sig > 0.0f ? 1.0f / sig : 0.0f; }

__global__ void __launch_bounds__(256) k_flag(WaveArgs a) {
    const int64_t n_all = (int64_t)a.nblk * a.nlev * a.Nprof;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n_all;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int j = (int)(idx % a.Nprof);
        const int bl = (int)(idx / a.Nprof);
        if (j >= a.nvalid[bl]) continue;
        const int l = bl % a.nlev, blk = bl / a.nlev;
        const float invsig = inv_sigma(a.sigma[bl]);
        if (!(invsig > 0.0f)) {
            if (0.0f > a.threshold) push_cand(a, blk, l, j, 0.0f);
            continue;
        }
        const float m0 = a.Q0[idx] * invsig;
        if (m0 >= a.medcut) {
            const int pos = atomicAdd(a.n_items, 1);
            if (pos < a.cap_items) {
                DevItem it;
                it.blk = blk;
                it.lev = l;
                it.j = j;
                it.pad = 0;
                a.items[pos] = it;
            }
        } else if (m0 > a.threshold) {
            push_cand(a, blk, l, j, m0);
        }
    }
}

cudaError_t launch_flag(const WaveArgs& a, cudaStream_t st) {
    const int64_t n_all = (int64_t)a.nblk * a.nlev * a.Nprof;
    const int grid = (int)(((n_all + 255) / 256) < 148 * 16 ? ((n_all + 255) / 256) : 148 * 16);
    k_flag<<<grid, 256, 0, st>>>(a);
    return cudaGetLastError();
}

// Exact metric of one (block, level, trial): the profile recomputed with the
// tile kernel's arithmetic, its median as baseline, sequential wrapped prefix
// sums, and the width/phase scan (src/search.jl:571-598, :893-904).
__device__ float exact_metric(const WaveArgs& a, int blk, int l, int j, float invsig) {
    const DevLevel& L = a.levels[l];
    const int k = L.k, Hk = L.Hk, nbins = L.nbins, wmax = L.wmax, np = L.np;
    float prof[kMaxBins];
    float srt[kMaxBins];
    float ps[kMaxBins + kMaxBins + 1];
    const float2* xs = a.X + (int64_t)blk * a.nharms * a.Nprof + j;
    const float* C2 = a.tw + L.tw_off;
    const float* S2 = C2 + (int64_t)Hk * np;
    for (int n0 = 0; n0 <= Hk; n0 += 8) {
        float E[8], O[8];
        synth_chunk8(xs, a.Nprof, C2, S2, np, k, Hk, n0, E, O);
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int nn = n0 + u;
            if (nn <= Hk) prof[nn] = E[u] + O[u];
            if (nn >= 1 && nn < Hk) prof[2 * Hk - nn] = E[u] - O[u];
        }
    }
    for (int i = 0; i < nbins; ++i) {
        const float x = prof[i];
        int q = i - 1;
        while (q >= 0 && srt[q] > x) { srt[q + 1] = srt[q]; --q; }
        srt[q + 1] = x;
    }
    const int half = nbins >> 1;
    const float med = (nbins & 1) ? srt[half] : 0.5f * (srt[half - 1] + srt[half]);
    ps[0] = 0.0f;
    for (int i = 0; i < nbins + wmax; ++i) {
        const int idx = i >= nbins ? i - nbins : i;
        ps[i + 1] = ps[i] + (prof[idx] - med);
    }
    float best = -INFINITY;
    for (int wi = 0; wi < L.nw; ++wi) {
        const int w = L.widths[wi];
        const float invsw = invsig / sqrtf((float)w);
        float mm = ps[w] - ps[0];
        for (int p = 1; p < nbins; ++p) mm = fmaxf(mm, ps[p + w] - ps[p]);
        const float cand = mm * invsw;
        if (cand > best) best = cand;
    }
    return best;
}

__global__ void __launch_bounds__(128) k_rescue(WaveArgs a) {
    const int64_t count = a.exact_all ? (int64_t)a.nblk * a.nlev * a.Nprof
                                      : (int64_t)min(*a.n_items, a.cap_items);
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < count;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int blk, l, j;
        if (a.exact_all) {
            j = (int)(idx % a.Nprof);
            const int bl = (int)(idx / a.Nprof);
            if (j >= a.nvalid[bl]) continue;
            l = bl % a.nlev;
            blk = bl / a.nlev;
        } else {
            const DevItem it = a.items[idx];
            blk = it.blk;
            l = it.lev;
            j = it.j;
        }
        const float invsig = inv_sigma(a.sigma[blk * a.nlev + l]);
        const float metric = invsig > 0.0f ? exact_metric(a, blk, l, j, invsig) : 0.0f;
        if (a.tmetric) a.tmetric[((int64_t)blk * a.nlev + l) * a.Nprof + j] = metric;
        if (metric > a.threshold) push_cand(a, blk, l, j, metric);
    }
}

cudaError_t launch_rescue(const WaveArgs& a, cudaStream_t st, int num_sms) {
    k_rescue<<<num_sms * 8, 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace cs
