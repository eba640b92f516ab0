// cs_internal.h -- device data layout shared by the host orchestration
// (cs_api.cu) and the kernels (cs_kernels.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cohsearch.h"

#include <vector>

namespace cs {

constexpr int kMaxLevels = 16;     // decimation factors per search
constexpr int kMaxWidths = 64;     // boxcar widths per level
constexpr int kMaxBins = 256;      // profile bins (nharms <= 128)
constexpr int kMaxSpecChunks = 16;  // room for a spectrum's chunk maxima (it has at most 6 chunks)
constexpr int kSigmaCap = 8192;    // _BOXCAR_SIGMA_SAMPLES, src/search.jl:462
constexpr int kTileTrials = 64;    // trials per CTA in the FP32 synthesis kernel
constexpr int kATileBytes = 128 * 128 * 2;  // one 16-bit A tile: 128 trials x 128 K
constexpr int kSampStride = kSigmaCap / 2;  // float2 per (block, level) in `samp`
constexpr int kSigmaThreads = 384;          // k_sigma CTA: one pass over a level's synthesis tasks

// One harmonic's rational trial-grid recipe (DirectPlan, src/directinterp.jl:179-204).
// Global trial t of the search evaluates harmonic h at Fourier frequency
// h*r_lo + t*h*pnum/q; its phase row is p = t mod P, its integer bin is
// floor(h*r_t) = rfloor0 + (t*h*pnum) div q + carry[p].
struct DevHarm {
    int32_t h;
    int32_t P;          // phase-cycle length q / gcd(h*pnum, q); 0 => per-trial FP64 path
    int32_t q;
    int32_t pnum;
    int32_t s;          // (h*pnum) mod q
    int32_t base_adv;   // (h*pnum) div q
    int64_t rfloor0;    // floor(h * r_lo)
    double dr0;         // h*r_lo - rfloor0
    double hr_lo;       // rfloor0 + dr0 (per-trial path)
    double dh;          // h * lodr (per-trial path)
    int64_t w_off;      // W[i][p] at wtab[w_off + i*P + p], i < m
    int64_t a_off;      // A[p] at atab[a_off + p], carry[p] at ctab[a_off + p]
};

// One decimation level k: profiles of nbins = 2*Hk bins from base harmonics k, 2k, ..., Hk*k.
struct DevLevel {
    int32_t k;
    int32_t Hk;
    int32_t nbins;
    int32_t nw;
    int32_t wmax;
    int32_t np;         // padded twiddle row length (multiple of 8, >= Hk+1)
    int64_t tw_off;     // C2[j][n] at tw[tw_off + j*np + n], S2 at tw[tw_off + Hk*np + j*np + n]
    int32_t widths[kMaxWidths];
    float rsqrtw[kMaxWidths];  // 1/sqrt(w), for the gate
};

// Device candidate record: block, level, trial within block, metric.
struct DevCand {
    int32_t blk;
    int32_t lev;
    int32_t j;
    float metric;
};

// Rescue work item (block, level, trial within block).
struct DevItem {
    int32_t blk;
    int32_t lev;
    int32_t j;
    int32_t pad;
};

// Everything one wave of blocks needs; device pointers.
struct WaveArgs {
    const float2* amps;
    int64_t namps;
    int64_t Nhalf;
    int32_t nharms;
    int32_t m;
    int32_t nlev;
    int32_t Nprof;
    int64_t t_first;        // global trial index of the wave's first block
    int64_t total;          // trials in the whole search
    int32_t nblk;           // blocks in this wave
    int32_t blk_base;       // index of the wave's first block in the search
    const int64_t* blk_map; // search of a block list: wave block -> band block (trial anchor 0), or nullptr
    const DevHarm* harms;
    const float* wtab;
    const float2* atab;
    const uint8_t* ctab;
    const DevLevel* levels;
    const float* tw;
    const int32_t* nvalid;  // [nblk][nlev]
    float2* X;              // [nblk][nharms][Nprof] FP32 amplitudes (plain synthesis) or nullptr
    uint8_t* Atile;         // [nblk][tiles_per_blk] 16-bit A tiles (tensor synthesis) or nullptr
    int32_t tiles_per_blk;
    int32_t fp16;           // A-tile format: 1 = FP16, 0 = BF16
    int32_t asplit;         // 1, or 2: each 128-trial A tile is followed by the tile of the
                            // amplitudes' rounding residuals (x - hi), in the same format
    // FP16 A tiles: bits of the largest |Re| or |Im| of each spectrum chunk
    // (k_amax, kMaxSpecChunks entries, unused ones 0).  A block's tiles take a
    // power-of-two scale from the maximum over chunks 0..blk_cidx[blk], which
    // holds every bin the block reads, so the scale is known as soon as those
    // chunks are on the device.  nullptr: no scale (BF16 has FP32's range)
    const uint32_t* amax_bits;
    const int32_t* blk_cidx;  // [nblk]: last spectrum chunk the block reads; nullptr: all chunks
    int32_t blk_first;        // interpolation launches over part of a wave: its first block
    float2* samp;           // [nblk][nlev][kSampStride]: pooled columns' amplitudes, [jh-1][slot]
    float* Q0;              // [nblk][nlev][Nprof] zero-baseline gate (unscaled by 1/sigma); diagnostics only, may be null
    float* sigma;           // [nblk][nlev]
    float* tmetric;         // [nblk][nlev][Nprof] exact metrics (exact_all mode) or nullptr
    DevItem* items;         // rescue list
    int32_t* n_items;
    int32_t cap_items;
    DevCand* cands;
    int32_t* n_cands;
    int32_t cap_cands;
    float threshold;
    float medcut;         // threshold - boxcar_medmargin (the reference's gate)
    float medcut_gate;    // the flag kernel's cut: medcut, less a slack for 16-bit gates
    int32_t verify_gate;  // rescan recomputes the FP32 gate and applies medcut itself
    int32_t exact_all;
    // Metric statistics (exact_all mode; the reference's MetricStats sink):
    // per (block, level) moments and the per-(level, window) histograms.
    double* mst;              // [nblk][nlev][kMstFields] or nullptr
    const int32_t* mwin;      // [nblk][nlev] window of the block's centre frequency
    unsigned long long* mhist;  // [nlev][nwin][hist_nb] counts
    unsigned long long* muo;    // [nlev][nwin][2] under / over
    double hist_lo, hist_hi, hist_invw;
    int32_t hist_nb, hist_nwin;
    // In-situ normalisation (MetricNorm): a trial is a candidate when
    // z = (M - loc[l][w]) / scale[l][w] > threshold, w the window of its
    // searched frequency k*rf/T among norm_edges[l][0..nwin].
    const double* norm_edges;   // [nlev][norm_nwin + 1] or nullptr
    const double* norm_loc;     // [nlev][norm_nwin]
    const double* norm_scale;   // [nlev][norm_nwin]
    int32_t norm_nwin;
    double norm_thr;            // the threshold, in FP64
    double r_lo, lodr, T;       // band anchor, trial step and observation time (FP64 frequencies)
    // Test hook (cs_set_wait_test): > 0 makes thread block 0 of k_sigma wait
    // this many nanoseconds at most on a barrier nothing completes.
    int64_t stall_ns;
};

constexpr int kMstFields = 8;   // n, min, median, mean, std, max, sum, sumsq

// Tensor-core synthesis (cs_synth_tc.cu): per-level TMEM column layout.
struct TcLevel {
    int32_t nbins;
    int32_t ncol;      // nbins + wmax columns with data (bins, then the wrapped first wmax bins)
    int32_t pw;        // columns streamed: ncol padded with zero columns to a multiple of the ring
    int32_t col;       // first TMEM column of the level
    int32_t nunits;    // epilogue units the level's starts are split into
    uint32_t wmask;    // bit w-1 set for each boxcar width w
    float rsq[32];     // 1/sqrt(w) at index w-1
};

// One epilogue work unit: the boxcar starts [p0, p0+nstart) of one level,
// scanned over pw columns from TMEM column col on even tiles, col1 on odd
// ones (they differ for the double-buffered base level).
struct TcUnit {
    int16_t lev;
    int16_t wg;        // epilogue warpgroup (0..3)
    int16_t nstart;
    int16_t pw;
    int16_t col;
    int16_t col1;
    int16_t phase;     // 0: scanned first (decimated levels); 1: after the next tile's product is issued
                       // (split epilogue: 1 = warpgroups 0-1's levels, 0 = warpgroups 2-3's)
    int16_t pad;
};

// One tcgen05.mma column range: B columns [bcol, bcol + n) into TMEM columns
// from tcol (even tiles) or tcol1 (odd tiles).  phase: the split epilogue's
// group that issues it (1: warpgroups 0-1, 0: warpgroups 2-3).
struct TcMma {
    int16_t bcol;
    int16_t n;
    int16_t tcol;
    int16_t tcol1;
    int16_t phase;
    int16_t pad;
};

constexpr int kMaxUnits = 32;
constexpr int kMaxMma = 8;

struct TcArgs {
    TcLevel lev[kMaxLevels];
    TcUnit unit[kMaxUnits];
    TcMma mma[kMaxMma];
    int32_t nunit;
    int32_t nmma;
    int32_t nlev;
    int32_t hm;            // prefix-sum ring size: 8 or 32 (>= widest boxcar)
    int32_t ncols_total;   // B columns of the product (multiple of 16)
    int32_t dbuf;          // 1: the base level has two TMEM slots, so the next tile's product
                           // runs while this tile's base level is scanned; 2: besides, the
                           // levels are split between two pairs of warpgroups that scan side
                           // by side, each pair issuing the products of its own levels
    int32_t fp16;          // operand format: 1 = FP16, 0 = BF16
    int32_t split;         // A tiles per 128 trials: 1, or 2 (hi and lo: K runs over both)
};

struct TcPlanHost {
    TcArgs args;
    std::vector<uint16_t> B;   // ncols_total x 128 twiddles, core-matrix layout
    size_t smem = 0;
};

// Returns 0, or < 0 when the configuration does not fit the tensor path.
// div0/div1 (> 0): the epilogue segment divisor of phase 0 / 1 instead of the
// cost model's choice (one of 2, 3, 4, 5, 6, 8, 10, 12, 16); allow_dbuf = 0: one
// base-level TMEM slot.
int prepare_tc(const DevLevel* dl, int nlev, int nharms, int fp16, int split, TcPlanHost* out, int div0 = 0,
               int div1 = 0, int allow_dbuf = 1);
cudaError_t launch_synth_tc(const WaveArgs& a, const TcPlanHost& tp, const void* dB, int* err,
                            cudaStream_t st, int num_sms);

// Kernel launchers (cs_kernels.cu).  Each returns the launch error.
#ifdef __CUDACC__
// ---------------------------------------------------------------------------
// Shared-memory barriers and plain (non-multicast) bulk copies, used by the
// tensor-core synthesis and the block sigma.
// ---------------------------------------------------------------------------
constexpr uint32_t kWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase: gives up after kWaitLimit polls or
// limit_ns of wall time (about one second by default), whichever comes first.
// The clock is first read after 1024 polls: a wait that ends sooner (nearly
// every one) reads no timer.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns = 1000000000ull) {
    uint64_t t0 = 0;
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if ((it & 1023u) == 1023u) {
            const uint64_t now = global_ns();
            if (t0 == 0) t0 = now;
            else if (now - t0 > limit_ns) return false;
        }
    }
    return false;
}

// Plain (non-multicast) 1-D bulk copy global -> this CTA's shared memory,
// completing `bytes` of transaction on mbarrier `bar` (armed here).
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(smem_u32(bar))
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// The same copy without arming the barrier: the caller arms it once, with
// mbar_expect_tx, for the bytes of all the copies that complete on it.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(dst), "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// ---------------------------------------------------------------------------
// Candidates and the medcut test of a gate value (boxcar_metrics!,
// src/search.jl:825-843), shared by both synthesis kernels' epilogues.
// ---------------------------------------------------------------------------
// Global trial of wave block blk's first trial.
__device__ __forceinline__ int64_t blk_t0(const WaveArgs& a, int blk) {
    return a.blk_map ? a.blk_map[blk] * (int64_t)a.Nprof : a.t_first + (int64_t)blk * a.Nprof;
}

__device__ __forceinline__ void push_cand(const WaveArgs& a, int blk, int l, int j, float metric) {
    const int pos = atomicAdd(a.n_cands, 1);
    if (pos < a.cap_cands) {
        DevCand c;
        c.blk = a.blk_map ? (int32_t)a.blk_map[blk] : a.blk_base + blk;
        c.lev = l;
        c.j = j;
        c.metric = metric;
        a.cands[pos] = c;
    }
}

__device__ __forceinline__ float inv_sigma(float sig) { return sig > 0.0f ? 1.0f / sig : 0.0f; }

// Exponent s of the FP16 A-tile scale 2^-s: the smallest with
// 16 * amax * 2^-s < 65504, so that amax * 2^-s lies in [2047, 4094).  An
// interpolated amplitude is at most about 2.7 * sqrt(2) times the largest |Re|
// or |Im| of the spectrum (the sum of the 16 taps' |sinc| weights), so 16
// leaves a further factor 4 of headroom for the tiles.  s is negative for a
// faint spectrum: its amplitudes are scaled up into FP16's normal range instead
// of rounding to subnormals or zero.  FP16 rounding of normal values and the
// FP32 sums are exact under a power of two, so the gate comes back exactly by
// 2^s and does not depend on the spectrum's overall scale.  |s| <= 100.
__device__ __forceinline__ int ascale_exp(const uint32_t* amax_bits, int cidx) {
    if (!amax_bits) return 0;
    uint32_t mx = 0;   // non-negative floats order as their bits
    for (int c = 0; c <= cidx; ++c) mx = max(mx, amax_bits[c]);
    const float r = __uint_as_float(mx) * (16.0f / 65504.0f);
    if (!(r < 1e30f)) return 100;                 // inf or NaN in the spectrum
    if (!(r > 0.0f)) return 0;                    // every bin read is zero
    int e;
    frexpf(r, &e);                                // r = f * 2^e, f in [0.5, 1): r < 2^e
    return max(min(e, 100), -100);
}
__device__ __forceinline__ float pow2f(int e) { return __int_as_float((127 + e) << 23); }   // |e| <= 126
// The scale exponent of wave block blk's A tiles.
__device__ __forceinline__ int ascale_exp_blk(const WaveArgs& a, int blk) {
    return ascale_exp(a.amax_bits, a.blk_cidx ? a.blk_cidx[blk] : kMaxSpecChunks - 1);
}

// Gate value g (zero-baseline boxcar maximum, not yet divided by sigma) of
// valid trial j: at or above medcut_gate it goes to the rescan list, else its
// gate S/N is final (a candidate only if above threshold).
// invsig = inv_sigma(sigma of (blk, l)), loaded by the caller ahead of time.
__device__ __forceinline__ void gate_flag(const WaveArgs& a, int blk, int l, int j, float g, float invsig) {
    if (!(invsig > 0.0f)) {
        if (0.0f > a.threshold) push_cand(a, blk, l, j, 0.0f);
        return;
    }
    const float m0 = g * invsig;
    if (m0 >= a.medcut_gate) {
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
#endif  // __CUDACC__

cudaError_t launch_interp(const WaveArgs& a, cudaStream_t st, int win_max, int* err);
// Persistent interpolation for m = 16 and phase cycles 1 <= P <= 256 (same values as launch_interp).
cudaError_t launch_interp2(const WaveArgs& a, cudaStream_t st, int win_max, int* err, int num_sms);
size_t interp2_smem(int win_max, int Nprof);
cudaError_t launch_synth_fp32(const WaveArgs& a, cudaStream_t st, int smem_bytes);
// variant 0: 384 threads, twiddles in shared memory; 1: 256 threads, twiddles through L1
size_t sigma_smem(int max_hk, int max_np, int variant = 0);
size_t interp_smem(int win_max, int Nprof);
cudaError_t launch_sigma(const WaveArgs& a, cudaStream_t st, int max_hk, int max_np, int* err, int variant = 0);
cudaError_t launch_rescue(const WaveArgs& a, cudaStream_t st, int num_sms);
cudaError_t launch_mstats(const WaveArgs& a, cudaStream_t st);
// the largest |Re| or |Im| of the spectrum, as float bits, into *out (zeroed by the caller)
cudaError_t launch_features(const float2* amps, int64_t namps, double r_lo, double lodr, int64_t Nprof, int64_t total,
                            const DevLevel* levels, int nlev, int nfeat, float* out, cudaStream_t st);
cudaError_t launch_mlp_forward(const cs_mlp& net, const float* x, int64_t n, float* h1, float* h2, float* z,
                               cudaStream_t st);
cudaError_t launch_mlp_backward(const cs_mlp& net, const float* x, const float* h1, const float* h2, const float* z,
                                const float* y, int64_t n, float pos_weight, float* dz, float* dh1, float* dh2,
                                const cs_mlp_grads& g, float* loss, cudaStream_t st);
cudaError_t launch_adam(const cs_adam_param& p, float lr, float b1, float b2, float eps, int step, cudaStream_t st);
cudaError_t launch_to_bf16(const float* p, uint16_t* pb, int64_t n, cudaStream_t st);
// Bins of chunk c of a spectrum of n bins and chunk unit u: [lo, hi), chunk
// sizes doubling after the first (chunk 0: [0, u); chunk c: [u*2^(c-1), u*2^c)).
__host__ __device__ inline int64_t spec_chunk_lo(int64_t u, int c) { return c == 0 ? 0 : u << (c - 1); }
__host__ __device__ inline int64_t spec_chunk_hi(int64_t u, int c, int64_t n) {
    return (u << c) < n ? (u << c) : n;
}
// Largest |Re| or |Im| of each chunk c < nchunk of a spectrum of n bins and
// chunk unit u, atomically maxed into out[c] (zeroed by the caller).
cudaError_t launch_amax(const float2* amps, int64_t n, int64_t unit, int nchunk, uint32_t* out, cudaStream_t st,
                        int num_sms);

// block_metrics (reference path): per harmonic, the fine-grid origin, its
// length (numbins * numbetween) and the reference's range guard.
struct BmHarm {
    int64_t lobin;
    int64_t K;
    int32_t ok;
    int32_t pad;
};
cudaError_t run_block_metrics(const double* d_rfund, int L, const BmHarm* d_hm, int nh, int m, int nb, int kernel,
                              const float2* amps, int64_t namps, double2* d_st, double* d_prof,
                              const int* d_widths, int nw, double* d_sigma, double* d_out, cudaStream_t st);
cudaError_t run_refold(const double* d_r, const int* d_nharm, int n, int m, double fsp, double maxfrac,
                       const float2* amps, int64_t namps, int64_t Nhalf, int maxh, double* d_prof, int* d_H,
                       double* d_ducy, cudaStream_t st);
size_t mstats_smem(int nprof, int hist_nb);
size_t synth_fp32_smem(int nharms, int maxbins, int maxwmax);

}  // namespace cs
