// cs_block.cu -- the reference / equivalence path on the device:
// block_metrics over arbitrary trial fundamentals (reference_profiles,
// coherent_profiles, snr_metrics; src/search.jl:933-1079), FP64 throughout.
//
//   k_bm_amps    the (trial, harmonic) amplitudes: `:direct` evaluates Eqn 30
//                (fourier_interp, src/fourierinterp.jl:64-74) at r = h*rfund[j];
//                `:fft` reproduces finterp_fft + uniform_linear_interp
//                (src/fourierinterp.jl:187-212, src/search.jl:974-986): the
//                FFT correlation's grid values at lobin + i/numbetween are the
//                same m-bin Eqn-30 sums, so the two grid neighbours of r are
//                evaluated directly and interpolated linearly -- no FFT, the
//                same numbers up to FP64 rounding.
//   k_bm_prof    normalised irfft to 2*nharms bins (coherent_profiles, DC zero,
//                Nyquist real part only).
//   k_bm_sigma   1.4826 * median(|x|) over the pooled profiles (_block_sigma).
//   k_bm_metric  exact median-baseline boxcar S/N per profile (_profile_boxcar,
//                medcut = -Inf).
#include "cs_internal.h"

#include <math.h>
#include <math_constants.h>

namespace cs {

namespace {

__device__ __forceinline__ double sinc_d(double x) {
    return x == 0.0 ? 1.0 : sinpi(x) / (CUDART_PI * x);
}

// fourier_interp(r, amps, m): sum over the m bins around r of conj(c) * bin,
// c = sinc(x) * cispi(x), x = dr - o for o = -m/2+1 .. m/2, dr = mod(r, 1),
// bins from 0-based r_int - m/2 with r_int = floor(r + 1e-15) + 1.
__device__ double2 fourier_interp_d(double r, const float2* __restrict__ amps, int64_t namps, int m) {
    const int m2 = m / 2;
    const int64_t r_int = (int64_t)floor(r + 1e-15) + 1;
    const double dr = fmod(r, 1.0);
    double re = 0.0, im = 0.0;
    for (int i = 0; i < m; ++i) {
        const double x = dr - (double)(i - m2 + 1);
        const double s = sinc_d(x);
        const double cr = s * cospi(x), ci = s * sinpi(x);
        const int64_t b = r_int - m2 + i;
        if (b < 0 || b >= namps) continue;   // outside the file: the guard keeps every used window inside
        const float2 v = amps[b];
        re += cr * (double)v.x + ci * (double)v.y;
        im += cr * (double)v.y - ci * (double)v.x;
    }
    return make_double2(re, im);
}

__global__ void k_bm_amps(const double* __restrict__ rfund, int L, const BmHarm* __restrict__ hm, int nh, int m,
                          int nb, int kernel, const float2* __restrict__ amps, int64_t namps,
                          double2* __restrict__ st) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)L * nh) return;
    const int j = (int)(idx / nh), h = (int)(idx % nh) + 1;
    const BmHarm H = hm[h - 1];
    double2 v = make_double2(0.0, 0.0);
    if (H.ok) {
        const double r = rfund[j] * (double)h;
        if (kernel == 1) {
            v = fourier_interp_d(r, amps, namps, m);
        } else {
            const double p = (r - (double)H.lobin) * (double)nb;
            const int64_t K = H.K;
            auto grid = [&](int64_t i) {
                return fourier_interp_d((double)H.lobin + (double)i / (double)nb, amps, namps, m);
            };
            if (p <= 0.0) {
                v = grid(0);
            } else if (p >= (double)(K - 1)) {
                v = grid(K - 1);
            } else {
                const int64_t i0 = (int64_t)floor(p);
                const double f = p - (double)i0;
                const double2 a = grid(i0), b = grid(i0 + 1);
                v = make_double2(a.x * (1.0 - f) + b.x * f, a.y * (1.0 - f) + b.y * f);
            }
        }
    }
    st[idx] = v;   // [trial][harmonic - 1]
}

// prof[n] = (1/N) (sum_{h<nh} 2 Re(X_h e^{2 pi i h n / N}) + Re(X_nh) (-1)^n), N = 2 nh.
__global__ void k_bm_prof(const double2* __restrict__ st, int L, int nh, double* __restrict__ prof) {
    const int N = 2 * nh;
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (idx >= (int64_t)L * N) return;
    const int j = (int)(idx / N), n = (int)(idx % N);
    const double2* x = st + (int64_t)j * nh;
    double s = 0.0;
    for (int h = 1; h < nh; ++h) {
        const double ang = 2.0 * (double)(((int64_t)h * n) % N) / (double)N;   // in units of pi
        s += 2.0 * (x[h - 1].x * cospi(ang) - x[h - 1].y * sinpi(ang));
    }
    s += (n & 1) ? -x[nh - 1].x : x[nh - 1].x;
    prof[idx] = s / (double)N;
}

constexpr int kBmSortMax = 8192;

// One CTA: the pooled |x| (every bin when nbins*L <= 8192, else whole profiles
// j = ((c-1)*L) div ncol), bitonic-sorted in shared memory, then the median.
__global__ void __launch_bounds__(1024) k_bm_sigma(const double* __restrict__ prof, int L, int nbins,
                                                   double* __restrict__ sigma) {
    extern __shared__ double v[];   // kBmSortMax
    const bool all = (int64_t)nbins * L <= kBmSortMax;
    const int ncol = all ? L : min(L, max(1, kBmSortMax / nbins));
    const int ns = ncol * nbins;
    int npow = 1;
    while (npow < ns) npow <<= 1;
    for (int i = threadIdx.x; i < npow; i += blockDim.x) {
        double x = CUDART_INF;
        if (i < ns) {
            const int c = i / nbins, b = i % nbins;
            const int col = all ? c : (int)(((int64_t)c * L) / ncol);
            x = fabs(prof[(int64_t)col * nbins + b]);
        }
        v[i] = x;
    }
    __syncthreads();
    for (int k = 2; k <= npow; k <<= 1) {
        for (int jj = k >> 1; jj > 0; jj >>= 1) {
            for (int i = threadIdx.x; i < npow; i += blockDim.x) {
                const int ixj = i ^ jj;
                if (ixj > i) {
                    const bool up = (i & k) == 0;
                    const double a = v[i], b = v[ixj];
                    if ((a > b) == up) {
                        v[i] = b;
                        v[ixj] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        const int half = ns >> 1;
        const double med = (ns & 1) ? v[half] : 0.5 * (v[half - 1] + v[half]);
        *sigma = ns > 0 ? 1.4826 * med : 0.0;
    }
}

// One warp per profile: exact median (rank counting), wrapped prefix sums of
// (x - median) by lane 0, then max over widths of max_p (ps[p+w] - ps[p]) * invsigma / sqrt(w).
__global__ void __launch_bounds__(128) k_bm_metric(const double* __restrict__ prof, int L, int nbins,
                                                   const int* __restrict__ widths, int nw,
                                                   const double* __restrict__ sigma, double* __restrict__ out) {
    __shared__ double ps_all[4][2 * kMaxBins + 2];
    __shared__ double med_all[4][2];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = blockIdx.x * 4 + wid;
    if (j >= L) return;
    const double* x = prof + (int64_t)j * nbins;
    double* ps = ps_all[wid];
    const double sg = *sigma;
    const double invsig = sg > 0.0 ? 1.0 / sg : 0.0;
    if (!(invsig > 0.0)) {
        if (lane == 0) out[j] = 0.0;
        return;
    }
    const int half = nbins >> 1;
    for (int i = lane; i < nbins; i += 32) {
        const double v = x[i];
        int lt = 0, le = 0;
        for (int q = 0; q < nbins; ++q) {
            lt += x[q] < v;
            le += x[q] <= v;
        }
        if (nbins & 1) {
            if (lt <= half && half < le) med_all[wid][0] = v;
        } else {
            if (lt <= half - 1 && half - 1 < le) med_all[wid][0] = v;
            if (lt <= half && half < le) med_all[wid][1] = v;
        }
    }
    __syncwarp();
    const double med = (nbins & 1) ? med_all[wid][0] : (med_all[wid][0] + med_all[wid][1]) / 2.0;
    const int wmax = widths[nw - 1];
    if (lane == 0) {
        ps[0] = 0.0;
        for (int i = 0; i < nbins + wmax; ++i) ps[i + 1] = ps[i] + (x[i % nbins] - med);
    }
    __syncwarp();
    double best = -CUDART_INF;
    for (int wi = 0; wi < nw; ++wi) {
        const int w = widths[wi];
        const double invsw = invsig / sqrt((double)w);
        double mm = -CUDART_INF;
        for (int p = lane; p < nbins; p += 32) mm = fmax(mm, ps[p + w] - ps[p]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mm = fmax(mm, __shfl_xor_sync(0xffffffffu, mm, o));
        const double cand = mm * invsw;
        if (cand > best) best = cand;
    }
    if (lane == 0) out[j] = best;
}

}  // namespace

cudaError_t run_block_metrics(const double* d_rfund, int L, const BmHarm* d_hm, int nh, int m, int nb, int kernel,
                              const float2* amps, int64_t namps, double2* d_st, double* d_prof,
                              const int* d_widths, int nw, double* d_sigma, double* d_out, cudaStream_t st) {
    const int64_t na = (int64_t)L * nh;
    k_bm_amps<<<(unsigned)((na + 127) / 128), 128, 0, st>>>(d_rfund, L, d_hm, nh, m, nb, kernel, amps, namps, d_st);
    const int64_t np = (int64_t)L * 2 * nh;
    k_bm_prof<<<(unsigned)((np + 127) / 128), 128, 0, st>>>(d_st, L, nh, d_prof);
    cudaFuncSetAttribute(k_bm_sigma, cudaFuncAttributeMaxDynamicSharedMemorySize, kBmSortMax * (int)sizeof(double));
    k_bm_sigma<<<1, 1024, kBmSortMax * sizeof(double), st>>>(d_prof, L, 2 * nh, d_sigma);
    k_bm_metric<<<(L + 3) / 4, 128, 0, st>>>(d_prof, L, 2 * nh, d_widths, nw, d_sigma, d_out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Candidate refold (candidate_profile / measure_ducy, src/candidate.jl:37-99)
// ---------------------------------------------------------------------------

namespace {

constexpr int kRefoldMaxH = 512;   // harmonics a refold may request

// One CTA per candidate: the contiguous harmonics 1..H that fit (the first
// whose m-bin window crosses Nyquist or the file's end stops the sum), each a
// wide-kernel fourier_interp at r*h; the normalised irfft to 2H bins; then
// boxcar_best_width (src/search.jl:617-638) on that profile for the duty cycle.
__global__ void __launch_bounds__(128) k_refold(const double* __restrict__ rr, const int* __restrict__ nh_in,
                                                int n, int m, double fsp, double maxfrac,
                                                const float2* __restrict__ amps, int64_t namps, int64_t Nhalf,
                                                int maxh, double* __restrict__ prof_out, int* __restrict__ H_out,
                                                double* __restrict__ ducy_out) {
    __shared__ double2 X[kRefoldMaxH];
    __shared__ double prof[2 * kRefoldMaxH];
    __shared__ double ps[4 * kRefoldMaxH + 2];
    __shared__ int sH;
    __shared__ double smed[2];
    const int c = blockIdx.x;
    if (c >= n) return;
    const double r = rr[c];
    const int nharm = nh_in[c];
    const int m2 = m / 2;
    if (!(nharm >= 1 && r > 0.0)) {
        if (threadIdx.x == 0) {
            H_out[c] = -1;
            ducy_out[c] = CUDART_NAN;
        }
        return;
    }
    if (threadIdx.x == 0) {
        int H = 0;
        for (int h = 1; h <= min(nharm, maxh); ++h) {
            const double rh = r * (double)h;
            const int64_t rint = (int64_t)floor(rh + 1e-15) + 1;
            if (!(rint - m2 >= 0 && rint + m2 <= namps && rh < (double)Nhalf)) break;
            H = h;
        }
        sH = H;
    }
    __syncthreads();
    const int H = sH;
    for (int h = threadIdx.x; h < H; h += blockDim.x) X[h] = fourier_interp_d(r * (double)(h + 1), amps, namps, m);
    __syncthreads();
    const int nb = H >= 1 ? 2 * H : 2;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        double s = 0.0;
        if (H >= 1) {
            for (int h = 1; h < H; ++h) {
                const double ang = 2.0 * (double)(((int64_t)h * b) % nb) / (double)nb;
                s += 2.0 * (X[h - 1].x * cospi(ang) - X[h - 1].y * sinpi(ang));
            }
            s += (b & 1) ? -X[H - 1].x : X[H - 1].x;
            s /= (double)nb;
        }
        prof[b] = s;
        if (prof_out) prof_out[(int64_t)c * 2 * maxh + b] = s;
    }
    __syncthreads();
    // exact median by rank counting
    const int half = nb >> 1;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const double v = prof[i];
        int lt = 0, le = 0;
        for (int q = 0; q < nb; ++q) {
            lt += prof[q] < v;
            le += prof[q] <= v;
        }
        if (lt <= half - 1 && half - 1 < le) smed[0] = v;
        if (lt <= half && half < le) smed[1] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double med = (smed[0] + smed[1]) / 2.0;   // nb is even
        // boxcar_widths (src/search.jl:387-396)
        const int wmax = max(1, (int)floor(maxfrac * nb));
        int wlast = 1;
        for (int w = 1; w <= wmax; w = max((int)floor(fsp * w), w + 1)) wlast = w;
        ps[0] = 0.0;
        for (int i = 0; i < nb + wlast; ++i) ps[i + 1] = ps[i] + (prof[i % nb] - med);
        double best = -CUDART_INF;
        int bestw = 1;
        for (int w = 1; w <= wmax; w = max((int)floor(fsp * w), w + 1)) {
            const double invsw = 1.0 / sqrt((double)w);
            double mm = ps[w] - ps[0];
            for (int p = 1; p < nb; ++p) mm = fmax(mm, ps[p + w] - ps[p]);
            const double cand = mm * invsw;
            if (cand > best) {
                best = cand;
                bestw = w;
            }
        }
        H_out[c] = H;
        ducy_out[c] = (double)bestw / (double)nb;
    }
}

}  // namespace

cudaError_t run_refold(const double* d_r, const int* d_nharm, int n, int m, double fsp, double maxfrac,
                       const float2* amps, int64_t namps, int64_t Nhalf, int maxh, double* d_prof, int* d_H,
                       double* d_ducy, cudaStream_t st) {
    if (n > 0)
        k_refold<<<n, 128, 0, st>>>(d_r, d_nharm, n, m, fsp, maxfrac, amps, namps, Nhalf, maxh, d_prof, d_H, d_ducy);
    return cudaGetLastError();
}

}  // namespace cs
