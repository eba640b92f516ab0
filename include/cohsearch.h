/*
 * cohsearch.h -- C ABI of libcohsearch_cuda.so, the B200 (sm_100a) engine for
 * the coherent harmonic-summing search hot path of CoherentSearch.jl.
 *
 * The reference has no FFI layer: its seam is the Julia function
 * `_search_region!` (src/search.jl:1768-1894) called from `search`
 * (src/search.jl:2002-2111), plus the reference/equivalence entry points
 * `block_metrics` (src/search.jl:1061-1079) and `chunk_metrics`
 * (src/search.jl:1740-1755).  Each entry point below names the reference
 * interface it replaces.  Plain C types only: no CUDA or torch types appear in
 * these signatures, so Julia (`ccall`), Python (`ctypes`) or C can bind them.
 *
 * Error behaviour: every call returns a cs_status; nothing aborts.  Invalid
 * arguments (the reference's ArgumentError cases) return
 * CS_ERR_INVALID_ARGUMENT; device failures return CS_ERR_CUDA with text in
 * cs_last_error().  A handle is not thread-safe (as SearchCache,
 * src/search.jl:1910-1912); distinct handles may be used concurrently.
 */
#ifndef COHSEARCH_H
#define COHSEARCH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cs_handle cs_handle;

typedef enum cs_status {
    CS_OK = 0,
    CS_ERR_INVALID_ARGUMENT = 1, /* bad parameter (reference: ArgumentError) */
    CS_ERR_NO_SPECTRUM = 2,      /* cs_search before a spectrum was attached */
    CS_ERR_CAPACITY = 3,         /* output array too small; *n_out = required */
    CS_ERR_CUDA = 4,             /* CUDA runtime/device error (see cs_last_error) */
    CS_ERR_OUT_OF_MEMORY = 5,    /* device allocation failed */
    CS_ERR_TIMEOUT = 6,          /* a bounded device wait ran out */
    CS_ERR_UNSUPPORTED = 7       /* parameter combination not built */
} cs_status;

enum { CS_MAX_DECIM = 16 };

/* Profile-synthesis arithmetic on the device.  It feeds only the
 * zero-baseline gate; every trial that can reach the threshold is rescored by
 * the exact FP32 path, so candidates and their S/N are the same in all modes. */
typedef enum cs_synth {
    CS_SYNTH_FP32 = 0,   /* plain FP32 SIMT synthesis ("plain FP32 GPU form") */
    CS_SYNTH_BF16 = 1,   /* tcgen05 tensor-core product, BF16 operands, FP32 accumulate */
    CS_SYNTH_FP16 = 2,   /* tcgen05 tensor-core product, FP16 operands, FP32 accumulate */
    CS_SYNTH_BF16_SPLIT = 3,  /* as BF16 with each amplitude split hi + lo (two BF16 operands,
                                 twice the A-tile bytes): about 16 significant bits */
    CS_SYNTH_FP16_SPLIT = 4   /* as FP16 with the hi + lo split: about 22 significant bits */
} cs_synth;

/* Mirrors SearchParams (src/search.jl:131-144). */
typedef struct cs_params {
    int32_t nharms;          /* harmonics coherently summed */
    int32_t m;               /* bins in the interpolation kernel (even) */
    int32_t numbetween;      /* fine-grid oversampling, reference path only */
    int32_t ndecim;          /* entries used in decimations[] */
    int32_t decimations[CS_MAX_DECIM];  /* harmonic-decimation factors k */
    double hidr;             /* Fourier-bin step at the highest harmonic */
    double threshold;
    double boxcar_fsp;
    double boxcar_maxfrac;
    double boxcar_medmargin;
    int32_t precision;       /* reference profile stage: 0 = :f64, 1 = :f32 */
    int32_t synth;           /* cs_synth */
} cs_params;

/* One detection (Candidate, src/search.jl:179-191) plus its provenance. */
typedef struct cs_candidate {
    double freq;     /* Hz: r / T */
    double metric;   /* boxcar matched-filter S/N */
    double r;        /* Fourier frequency in bins (k * fundamental for a k-fold) */
    int32_t nharm;   /* harmonics summed: floor(nharms / k) */
    int32_t k;       /* decimation factor that found it */
    int64_t trial;   /* global index of the fundamental trial */
} cs_candidate;

/* Per-search counters and device timings, filled by cs_search_stats. */
typedef struct cs_stats {
    int64_t trials;          /* fundamental trials searched */
    int64_t blocks;          /* blocks of `blocksize` trials */
    int64_t profiles;        /* scored (trial, k) pairs: sum over k of valid trials */
    int64_t rescued;         /* (trial, k) pairs that took the exact median rescan */
    int64_t candidates;      /* raw above-threshold detections (before dedup) */
    int64_t waves;           /* device passes the blocks were split into */
    int64_t launches;        /* kernels launched by the last call */
    double ms_interp;        /* CUDA-event time of each stage, summed over waves */
    double ms_synth;         /* profile synthesis + gate scan + medcut test */
    double ms_sigma;         /* block sigma (runs before the synthesis) */
    double ms_rescue;        /* exact rescan of the flagged trials */
    double ms_total;         /* first to last event of the call */
    int64_t h2d_bytes;       /* host->device bytes the call copied */
    int64_t d2h_bytes;       /* device->host bytes the call copied */
} cs_stats;

/* Create a handle for `params` on CUDA device `device`.  Replaces the setup
 * half of `search` (plans and workspaces, src/search.jl:2037-2046) and the
 * SearchCache (src/search.jl:1914-1961): one handle per SearchParams. */
cs_status cs_create(cs_handle** out, const cs_params* params, int32_t device);

/* Run the handle's work on `stream` (a cudaStream_t passed as void*; NULL
 * restores the handle's own stream).  Lets a caller order the engine with its
 * own copies and time it with its own events. */
cs_status cs_set_stream(cs_handle* h, void* stream);

/* Release all device memory of the handle. */
cs_status cs_destroy(cs_handle* h);

/* Text of the last error on this handle ("" if none). */
const char* cs_last_error(const cs_handle* h);

/* Attach a spectrum from HOST memory: namps complex64 values, interleaved
 * (re, im), amps[0] = DC.re + i*Nyquist, as FFTFile maps it
 * (src/fileio.jl:64-78); N = time-series length, dt = sample time (s), so
 * T = N*dt.  The data are copied to the device in chunks of doubling size
 * (at most 6) on a copy stream of the handle's.  From page-locked memory the copy is asynchronous
 * and the next search overlaps it, interpolating each run of blocks as soon
 * as the chunks that run reads have landed: keep the buffer unchanged until
 * that search (or any other call that reads the spectrum) has returned.
 * From pageable memory the call returns once the data are staged. */
cs_status cs_set_spectrum(cs_handle* h, const float* amps, int64_t namps, int64_t N, double dt);

/* As cs_set_spectrum, but `d_amps` is already a DEVICE pointer on the
 * handle's device.  Nothing is copied; the caller keeps it alive. */
cs_status cs_set_spectrum_device(cs_handle* h, const float* d_amps, int64_t namps, int64_t N,
                                 double dt);

/* The hot loop: search fundamentals over [lofreq, hifreq] Hz (or from bin
 * `lobin` when lobin != 100, the reference's precedence rule) in blocks of
 * `blocksize` trials, every decimation factor, and write the raw detections
 * above `threshold` to out[0 .. *n_out).  Replaces `_search_region!`
 * (src/search.jl:1768-1894) as called by `search` (src/search.jl:2080-2094);
 * duplicate and harmonic collapse (src/search.jl:2148-2214) stay with the
 * caller.  exact_all = 1 scores every trial with the exact median baseline
 * (the reference's medcut = -Inf); 0 uses the zero-baseline gate with
 * medcut = threshold - boxcar_medmargin.  Candidates come back in the order a
 * single-task reference run produces them: by block, base fold first then each
 * decimation factor, ascending trial.  If cap is too small, returns
 * CS_ERR_CAPACITY with *n_out = the number found (out holds the first cap). */
cs_status cs_search(cs_handle* h, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                    double threshold, int32_t exact_all, cs_candidate* out, int64_t cap,
                    int64_t* n_out);

/* cs_search restricted to blocks [block_begin, block_end) of the band's grid
 * of blocksize-trial blocks (block_end < 0: through the last block).  The
 * trial grid stays anchored at the band's start, so the blocks, their sigmas
 * and the candidates (trial indices global to the band) are exactly those of
 * the whole search: the unit a multi-GPU run shards over (the reference's
 * chunk loop, src/search.jl:1768-1894, over a contiguous range of chunks). */
cs_status cs_search_range(cs_handle* h, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                          double threshold, int32_t exact_all, int64_t block_begin, int64_t block_end,
                          cs_candidate* out, int64_t cap, int64_t* n_out);

/* enable != 0: cs_search_batch over device spectra (on_device = 1), or over
 * host spectra that are all page-locked, runs the batch the ordinary way
 * once, captures it into one CUDA graph -- per spectrum its uploads (for host
 * spectra the copy into a batch buffer, overlapped with the previous
 * spectrum's search), launches and readback, no host round trip between
 * spectra -- and replays that graph while later calls repeat the same batch
 * (same spectrum addresses, lengths, band and threshold; refill the spectra
 * in place between calls).  Any other search on the handle drops the graph.
 * A spectrum needing more than one wave keeps the batch ordinary; one with
 * more than 4096 candidates is searched again the ordinary way.  No
 * counterpart in the reference (its batch is a loop over files,
 * src/cli.jl:237-289). */
cs_status cs_set_batch_graph(cs_handle* h, int32_t enable);

/* cs_search restricted to the listed blocks of the band's grid (strictly
 * ascending indices): each block's sigma and candidates are exactly the whole
 * search's, as with cs_search_range.  The re-search of the blocks a learned
 * proposal picks.  No counterpart in the reference (its chunk loop,
 * src/search.jl:1768-1894, runs over every chunk).  Not with metric
 * statistics or normalisation. */
cs_status cs_search_blocks(cs_handle* h, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                           double threshold, const int64_t* blocks, int64_t nblocks, cs_candidate* out, int64_t cap,
                           int64_t* n_out);

/* ---------------------------------------------------------------------------
 * Learned block proposal.  No counterpart in the reference: a small network
 * scores the band's blocks from cheap incoherent features, and the coherent
 * search re-searches the proposed blocks (cs_search_blocks).  All pointers
 * with a d_ prefix are device memory the caller owns; stream may be null.
 * ------------------------------------------------------------------------- */

/* Per block of the band (blocks of blocksize trials from the band's start, as
 * cs_search), one feature per (decimation level k with Hk harmonics, H = 1..Hk),
 * levels in the handle's order: the incoherent power sum
 * S(r) = sum_{i<=H} |X[rint(i*k*r)]|^2 of the attached (normalised) spectrum at
 * every trial r of the block, as z = (S - H)/sqrt(H), and the feature is
 * asinh(max over the block of z) -- the incoherent counterpart of every sum
 * the coherent search forms.  d_out [nblocks][nfeat]; *nblocks_out and
 * *nfeat_out (sum of Hk) get the sizes; CS_ERR_CAPACITY if the block count
 * exceeds cap_blocks. */
cs_status cs_block_features(cs_handle* h, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                            float* d_out, int64_t cap_blocks, int64_t* nblocks_out, int32_t* nfeat_out);

/* The proposal network: din -> dh -> dh -> 1, ReLU, BF16 weights (bit
 * patterns), FP32 biases; W[j][i] maps input i to unit j. */
typedef struct cs_mlp {
    int32_t din, dh;
    const uint16_t* w1;   /* [dh][din] */
    const float* b1;      /* [dh] */
    const uint16_t* w2;   /* [dh][dh] */
    const float* b2;      /* [dh] */
    const uint16_t* w3;   /* [dh] */
    const float* b3;      /* [1] */
} cs_mlp;

/* FP32 gradients of every parameter of a cs_mlp, same shapes. */
typedef struct cs_mlp_grads {
    float *w1, *b1, *w2, *b2, *w3, *b3;
} cs_mlp_grads;

/* One Adam-updated tensor: FP32 master, optional BF16 copy refreshed after the
 * step, moments m and v, gradient. */
typedef struct cs_adam_param {
    float* master;
    uint16_t* bf16;
    float* m;
    float* v;
    const float* grad;
    int64_t n;
} cs_adam_param;

/* Forward pass over n rows of d_x [n][din]: d_h1, d_h2 [n][dh] (post-ReLU) and
 * the logits d_z [n]; FP32 accumulation. */
cs_status cs_mlp_forward(const cs_mlp* net, const float* d_x, int64_t n, float* d_h1, float* d_h2, float* d_z,
                         void* stream);

/* Weighted binary cross-entropy with logits against labels d_y (0/1), mean
 * over n, weight pos_weight on positives: the loss into *d_loss and the
 * gradients of every parameter into grads (d_dz [n], d_dh1, d_dh2 [n][dh] are
 * scratch). */
cs_status cs_mlp_backward(const cs_mlp* net, const float* d_x, const float* d_h1, const float* d_h2,
                          const float* d_z, const float* d_y, int64_t n, float pos_weight, float* d_dz, float* d_dh1,
                          float* d_dh2, const cs_mlp_grads* grads, float* d_loss, void* stream);

/* One Adam step (bias-corrected, step >= 1) on each listed tensor. */
cs_status cs_adam_step(const cs_adam_param* params, int32_t nparams, float lr, float beta1, float beta2, float eps,
                       int32_t step, void* stream);

/* BF16 (round to nearest even) copies of FP32 weights. */
cs_status cs_mlp_to_bf16(const float* d_src, uint16_t* d_dst, int64_t n, void* stream);

/* ---------------------------------------------------------------------------
 * Metric statistics and in-situ normalisation (the reference's --metricstats
 * and --normalize: MetricStats, BlockMetricStats, MetricHistogram, MetricNorm,
 * src/search.jl:1296-1643, collected in _search_region!/decim_pass!,
 * :1664-1894, driven by search, :2063-2094).
 * ------------------------------------------------------------------------- */

/* One (block, k) record of BlockMetricStats (src/search.jl:1321-1335); block is
 * the reference's 1-based chunk index of the band. */
typedef struct cs_block_stats {
    int64_t block;
    int32_t k, Hk, nbins, pad;
    double ngoodbins, flo, fhi;
    int64_t n;
    double min, median, mean, std, max;
} cs_block_stats;

/* enable != 0: every following cs_search / cs_search_range scores every trial
 * exactly (medcut = -Inf, as the reference does when collecting) and collects
 * the per-(block, k) statistics and the per-(k, window) histograms of the raw
 * metric: hist_nb bins over [hist_lo, hist_hi), nwin log-spaced searched-
 * frequency windows per k (MetricStats defaults: 0, 64, 3200, 16).  Candidates
 * are unchanged. */
cs_status cs_set_metricstats(cs_handle* h, int32_t enable, double hist_lo, double hist_hi, int32_t hist_nb,
                             int32_t nwin);

/* The last search's BlockMetricStats records, sorted by (block, k); if cap is
 * too small, CS_ERR_CAPACITY with *n_out = the number available. */
cs_status cs_get_block_stats(const cs_handle* h, cs_block_stats* out, int64_t cap, int64_t* n_out);

/* The last search's per-(k, window) histograms (MetricHistogram, one per k
 * and window, ks ascending).  *nlev, *nwin, *nb receive the shape; with null
 * arrays only the shape is returned.  ks[nlev]; edges[nlev][nwin+1] (Hz);
 * counts[nlev][nwin][nb]; moments[nlev][nwin][7] = under, over, total, sum,
 * sumsq, vmin, vmax. */
cs_status cs_get_metric_hists(const cs_handle* h, int32_t* nlev, int32_t* nwin, int32_t* nb, int32_t* ks,
                              double* edges, int64_t* counts, double* moments);

/* In-situ normalisation for the following searches (MetricNorm, built by the
 * caller from a stats pass as build_metricnorm does): for decimation ks[i],
 * window edges edges[i][0..nwin] (Hz) and per-window loc/scale[i][0..nwin-1].
 * Every trial is scored exactly and is a candidate when its
 * z = (M - loc) / scale > threshold; the candidate's metric is z.  nlev = 0
 * clears it.  Each k of the handle's levels must be given. */
cs_status cs_set_metricnorm(cs_handle* h, int32_t nlev, int32_t nwin, const int32_t* ks, const double* edges,
                            const double* loc, const double* scale);

/* One spectrum of a batch: complex64 amps [namps] (host or device memory,
 * per cs_search_batch's on_device), N samples at dt seconds. */
typedef struct cs_spectrum {
    const float* amps;
    int64_t namps;
    int64_t N;
    double dt;
} cs_spectrum;

/* `search` over each of nfiles spectra (a DM sweep: many .fft files of uneven
 * length, src/cli.jl:237-246 loops `search_one` over them) with one handle:
 * candidates as cs_search emits them, file by file in order, file_of[c] the
 * index of candidate c's spectrum.  Host spectra (on_device = 0; pinned memory
 * for full overlap) are copied on a second stream, file i+1's copy running
 * under file i's search.  No counterpart takes all files at once in the
 * reference.  cs_search_stats then gives the totals over the batch.  If cap is
 * too small, CS_ERR_CAPACITY with *n_out = the number found. */
cs_status cs_search_batch(cs_handle* h, const cs_spectrum* files, int32_t nfiles, int32_t on_device,
                          double lofreq, double hifreq, int64_t lobin, int64_t blocksize, double threshold,
                          cs_candidate* out, int32_t* file_of, int64_t cap, int64_t* n_out);

/* Counters and stage timings of the last cs_search on this handle. */
cs_status cs_search_stats(const cs_handle* h, cs_stats* out);

/* Equivalence bridge `chunk_metrics` (src/search.jl:1740-1755): the exact
 * metric of each of the n trials rstart + j*lodr (one block, global trial 0
 * at rstart, base fold only), written to out[0..n).  rstart must be finite
 * and >= 0, 1 <= n <= 65536 (else CS_ERR_INVALID_ARGUMENT). */
cs_status cs_chunk_metrics(cs_handle* h, double rstart, int64_t n, double* out);

/* cs_chunk_metrics for callers that may not allocate device memory.  It has
 * no counterpart in the reference: it exists for code that runs inside a host
 * that owns the device memory budget (a pipeline that reserved HBM at start-up
 * and hands out fixed buffers, a runtime whose pool allocator must see every
 * allocation) or that cannot pay the device-wide synchronisation of cudaFree.
 * It creates no handle and calls no cudaMalloc, cudaFree or allocating
 * library routine.  Its scratch (counters, plan tables, sigma samples) lives
 * in a 4 MiB array inside the library that every GPU using the library holds
 * until the process exits; a request whose plan tables need more returns
 * CS_ERR_CAPACITY with the sizes in `err`.
 *
 * Inputs and output are device memory on the current device: d_amps holds
 * namps complex64 amplitudes of an N-sample series (8-byte aligned), d_out
 * receives the n float32 metrics that cs_chunk_metrics returns as doubles
 * (trials rstart + j*lodr, base fold), 1 <= n <= 65536, rstart finite and
 * >= 0.  Work runs on
 * `stream` (NULL = legacy default stream) and the call returns once it has
 * finished.  `err` (may be NULL) receives a message of at most err_cap bytes.
 *
 * The first call on a device looks up the array's device address there
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls on a device share the array and it keeps the last call's
 * contents; the counters are cleared on every call.  Calls whose GPU work
 * overlapped would race on it: the library serialises its own calls per
 * device with a lock and returns, on success and on every error after work
 * was queued, only once that work is done. */
cs_status cs_chunk_metrics_static(const cs_params* params, const float* d_amps, int64_t namps, int64_t N,
                                  double rstart, int64_t n, float* d_out, void* stream, char* err,
                                  int64_t err_cap);

/* Reference path `block_metrics(ft, rfund, params; kernel, widths)`
 * (src/search.jl:1061-1079, with reference_profiles :1011-1049 and snr_metrics
 * :933-951): the coherent-fold S/N of each of the L trial fundamentals rfund
 * (Fourier bins, ascending, >= 0; any values, not a grid), FP64 throughout.
 * kernel 0 = :fft (finterp_fft on the numbetween grid + linear interpolation),
 * 1 = :direct (Eqn 30 at each point).  widths NULL or nw = 0: the base pass's
 * ladder bank. */
cs_status cs_block_metrics(cs_handle* h, const double* rfund, int64_t L, int32_t kernel, const int32_t* widths,
                           int32_t nw, double* out);

/* candidate_profile / measure_ducy (src/candidate.jl:37-99) for n candidates:
 * fundamental Fourier frequency r[i] (bins) and requested harmonics nharm[i]
 * (<= 512).  Each harmonic h = 1, 2, ... is an m-bin (reference default 64)
 * exact fourier_interp at r*h, stopping at the first whose window crosses
 * Nyquist or the file's end; H[i] receives the harmonics used (-1 when
 * nharm < 1 or r <= 0, whose duty cycle is NaN), profiles[i*256 + 0 .. 2H)
 * the normalised irfft profile (NULL: not returned; H = 0 gives two zero bins),
 * ducy[i] the best boxcar width / profile bins (boxcar_best_width,
 * src/search.jl:617-638, with the handle's boxcar_fsp / boxcar_maxfrac). */
cs_status cs_refold(cs_handle* h, const double* r, const int32_t* nharm, int64_t n, int32_t m, int32_t* H,
                    double* profiles, double* ducy);

/* Interpolated amplitude stack of a chunk (the `ftprofs` rows of
 * fill_chunk_profiles!, src/search.jl:1280-1290, and fill_harmonic_row_direct!,
 * src/directinterp.jl:470-572): trials t0 .. t0+n-1 of a search whose global
 * trial 0 sits at Fourier frequency r_lo.  out is (nharms, n) complex64,
 * interleaved, harmonic-major; rows the range guard rejects are zero. */
cs_status cs_interp_chunk(cs_handle* h, double r_lo, int64_t t0, int64_t n, float* out);

/* Diagnostic copies of the last cs_search's per-(block, k) values:
 * sigma[b * nlev + l] (device block sigma) and nvalid[b * nlev + l]; `cap`
 * counts entries; nlev = number of decimation factors, l in params order. */
cs_status cs_search_block_values(const cs_handle* h, float* sigma, int32_t* nvalid, int64_t cap,
                                 int64_t* n_out);

/* Diagnostics kept on the host after each cs_search: 0 = none (default),
 * 1 = per-(block, k) sigma and valid counts, 2 = also every trial's gate
 * value.  Level 2 copies nblocks*nlev*blocksize floats back per search. */
cs_status cs_set_diagnostics(cs_handle* h, int32_t level);

/* Zero-baseline gate value of every (block, k, trial) of the last cs_search
 * run with diagnostics level 2: the `mvals` the reference's batched gate
 * leaves before the exact rescan (_boxcar_gate!, src/search.jl:784-807),
 * out[(b * nlev + l) * blocksize + j]; entries past a block's valid trials
 * are 0. */
cs_status cs_search_gate_values(const cs_handle* h, float* out, int64_t cap, int64_t* n_out);

/* Per-trial metrics of the last cs_search run with exact_all = 1:
 * out[(b * nlev + l) * blocksize + j]. */
cs_status cs_search_trial_metrics(const cs_handle* h, float* out, int64_t cap, int64_t* n_out);

/* What cs_autotune chose, and the stage times it measured on its sample. */
typedef struct cs_tune_report {
    int32_t interp_kernel;        /* 1: persistent kernel with bulk-copied windows; 0: one CTA per item */
    int32_t sigma_kernel;         /* block sigma: 0 = 384 threads, twiddles in shared memory; 1 = 256, via L1 */
    int32_t tc_double_buffer;     /* tensor modes: 0 = one TMEM slot; 1 = base level in two slots,
                                     scanned after the decimated levels; 2 = base level in two
                                     slots, scanned by warpgroups 0-1 beside warpgroups 2-3 on the
                                     decimated levels, each pair issuing its own products */
    int32_t tc_div[2];            /* epilogue segment divisor of each phase (0: FP32 synthesis) */
    int32_t nlev;                 /* decimation levels */
    int32_t nbins[CS_MAX_DECIM];  /* profile bins of each level, in level order */
    int32_t units[CS_MAX_DECIM];  /* epilogue work units (start segments) of each level */
    double ms_interp[2];          /* interpolation stage time of kernel 0 / 1 (-1: not applicable) */
    double ms_sigma[2];           /* block-sigma stage time of kernel 0 / 1 */
    double ms_synth_model;        /* synthesis stage time with the cost model's plan */
    double ms_synth_tuned;        /* ... with the chosen plan */
    int64_t sample_blocks;        /* blocks of the timed sample */
} cs_tune_report;

/* Autotune the handle's launch shapes on its attached spectrum: a sample of
 * nsample blocks from the middle of the band [lofreq, hifreq] (arguments as
 * cs_search) is searched with each candidate -- the interpolation kernel, the
 * block-sigma kernel, and in the tensor modes the epilogue form (one TMEM
 * slot, the base level double-buffered and scanned after the decimated
 * levels, or split between two warpgroup pairs) with, per form, the segment
 * size of each phase per profile bin count -- timed with CUDA events
 * (the least of 3 runs after a warm-up), and the fastest kept on the handle.
 * Every candidate computes the same values, so candidates are unchanged.  The
 * choice is also cached for the device and these parameters: handles created
 * later with the same cs_params on the same device start with it.  An
 * untuned handle runs one CTA per interpolation item, 384-thread sigma and
 * the one-slot epilogue with segment divisors 3 and 2 (the tuner's choice on
 * the nharms-60 survey workload).  No counterpart in the reference. */
cs_status cs_autotune(cs_handle* h, double lofreq, double hifreq, int64_t lobin, int64_t blocksize, int64_t nsample,
                      cs_tune_report* out);

/* Apply launch shapes chosen earlier (a cs_autotune report, e.g. stored by a
 * pipeline at its first run): interp_kernel, sigma_kernel, tc_double_buffer
 * and tc_div are read; the other fields are ignored.  tc_double_buffer is 0,
 * 1 or 2 (2 needs unsplit tiles and decimation levels; otherwise the plan
 * falls back to 1, then 0).  tc_div entries are 0
 * (the cost model's choice) or one of 2, 3, 4, 5, 6, 8, 10, 12, 16.  Every
 * shape computes the same values.  No counterpart in the reference. */
cs_status cs_set_launch_shapes(cs_handle* h, const cs_tune_report* shapes);

/* Cap on the device memory this handle holds (bytes; 0 = no cap, the
 * default).  Searches split their blocks into waves that fit under the cap
 * beside the handle's fixed tables and spectrum; when even one block's
 * working set does not fit, the search returns CS_ERR_OUT_OF_MEMORY and the
 * handle stays usable.  Setting the cap releases the wave buffers (and a
 * captured batch graph), so that later searches reallocate them at the
 * size the cap allows.  No counterpart in the reference (its workspaces are
 * sized per thread, src/search.jl:1170-1265). */
cs_status cs_set_memory_limit(cs_handle* h, int64_t bytes);

/* Test hook of the bounded device waits.  With wait_ns > 0 the next searches
 * make one thread block of the block-sigma kernel wait, for at most wait_ns
 * nanoseconds, on a shared-memory barrier that nothing completes (every
 * other device wait keeps its limit of about one second); the wait gives up,
 * the kernel ends with an error flag and the search returns CS_ERR_TIMEOUT
 * with the handle and the CUDA context still usable.  wait_ns = 0 (the
 * default) turns it off.  No counterpart in the reference. */
cs_status cs_set_wait_test(cs_handle* h, int64_t wait_ns);

/* Library version string. */
const char* cs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* COHSEARCH_H */
