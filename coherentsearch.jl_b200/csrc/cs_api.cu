// cs_api.cu -- host side of libcohsearch_cuda.so: the C ABI of cohsearch.h,
// the FP64 plan tables, the decimation levels and the wave orchestration.
//
// All FP64 bookkeeping that decides bin ranges, trial counts, valid decimated
// trials and candidate frequencies is evaluated here with the reference's own
// expressions (no contraction: built with -ffp-contract=off), so those values
// are bit-identical to the reference's.
#include "cohsearch.h"
#include "cs_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdarg>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

using namespace cs;

namespace {
// FP16 A tiles (plain or split), and A tiles per 128 trials (2: hi and lo)
bool synth_fp16(int s) { return s == CS_SYNTH_FP16 || s == CS_SYNTH_FP16_SPLIT; }
int synth_split(int s) { return (s == CS_SYNTH_BF16_SPLIT || s == CS_SYNTH_FP16_SPLIT) ? 2 : 1; }
}  // namespace

#define CS_VERSION_STRING "cohsearch-b200 0.1.0 (sm_100a)"

namespace {

struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need) {
        if (need == 0) need = 16;
        if (need <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, need);
        if (e == cudaSuccess) bytes = need;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Pinned host staging (grown on demand): copies from and to it are truly
// asynchronous, so a search enqueues its work without host-side stalls.
struct HBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t need) {
        if (need == 0) need = 16;
        if (need <= bytes) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaHostAlloc(&p, need, cudaHostAllocDefault);
        if (e == cudaSuccess) bytes = need;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};


struct LevelHost {
    int k, Hk, nbins;
    std::vector<int> widths;
};

// sin(pi x), cos(pi x) for x in [0, 1), reduced so that pi*x is formed only on
// [0, 1/4]; the reference uses Julia's sinpi/cispi (src/directinterp.jl:392).
double sinpi_d(double x) {
    if (x <= 0.25) return std::sin(M_PI * x);
    if (x <= 0.75) return std::cos(M_PI * (x - 0.5));
    return std::sin(M_PI * (1.0 - x));
}
double cospi_d(double x) {
    if (x <= 0.25) return std::cos(M_PI * x);
    if (x <= 0.75) return -std::sin(M_PI * (x - 0.5));
    return -std::cos(M_PI * (1.0 - x));
}

int64_t gcd64(int64_t a, int64_t b) {
    while (b) {
        int64_t t = a % b;
        a = b;
        b = t;
    }
    return a < 0 ? -a : a;
}

// trial_grid_rational (src/directinterp.jl:217-225): the smallest-denominator
// rational p/q, q <= 2^16, within 8 eps(lodr) of lodr.  Two distinct rationals
// with denominators <= 2^16 are >= 2^-32 apart, so a scan over q finds exactly
// the value `rationalize(Int, lodr; tol=1e-13)` returns whenever the reference
// accepts it.
bool trial_grid_rational(double lodr, int64_t* pnum, int64_t* q) {
    if (!(lodr > 0)) return false;
    const double eps8 = 8.0 * (std::nextafter(lodr, INFINITY) - lodr);
    for (int64_t qq = 1; qq <= (1 << 16); ++qq) {
        const double pp = std::nearbyint(lodr * (double)qq);
        if (pp >= 1 && std::fabs(pp / (double)qq - lodr) <= eps8) {
            const int64_t g = gcd64((int64_t)pp, qq);
            *pnum = (int64_t)pp / g;
            *q = qq / g;
            return true;
        }
    }
    return false;
}

// boxcar_widths (src/search.jl:387-396).
std::vector<int> boxcar_widths(int nbins, double fsp, double maxfrac) {
    const int64_t wmax = std::max<int64_t>(1, (int64_t)std::floor(maxfrac * (double)nbins));
    std::vector<int> ws;
    int64_t w = 1;
    while (w <= wmax) {
        ws.push_back((int)w);
        w = std::max<int64_t>((int64_t)std::floor(fsp * (double)w), w + 1);
        if (ws.size() > 4096) break;
    }
    return ws;
}

// ladder_boxcar_widths (src/search.jl:443-459).
std::vector<int> ladder_widths(int nbins, int k, const cs_params& p) {
    std::vector<int> ws = boxcar_widths(nbins, p.boxcar_fsp, p.boxcar_maxfrac);
    std::vector<int> ks(p.decimations, p.decimations + p.ndecim);
    std::sort(ks.begin(), ks.end());
    if (ks.size() <= 1) return ws;
    for (size_t i = 0; i + 1 < ks.size(); ++i)
        if (!(ks[i + 1] <= 3 * ks[i])) return ws;  // _LADDER_WMAX ÷ 2 = 3
    const int kmin = ks.front(), kmax = ks.back();
    std::vector<int> pr;
    for (int w : ws)
        if ((w >= 2 || k == kmin) && (w <= 6 || k == kmax)) pr.push_back(w);
    return pr.empty() ? ws : pr;
}

struct HostPlans {
    std::vector<DevHarm> harms;
    std::vector<float> w;
    std::vector<float2> a;
    std::vector<uint8_t> c;
};

// build_direct_plans with Float32 weights (src/directinterp.jl:342-405): every
// table entry computed in FP64 and rounded once.  The device indexes W as
// [i][p] so that consecutive trials (consecutive p) read consecutive words.
void build_plans(const cs_params& p, double r_lo, HostPlans& out) {
    const double lodr = p.hidr / (double)p.nharms;
    int64_t pnum = 1, q = 1;
    const bool rq = trial_grid_rational(lodr, &pnum, &q);
    const int m = p.m, m2 = m / 2;
    out.harms.clear();
    out.w.clear();
    out.a.clear();
    out.c.clear();
    for (int h = 1; h <= p.nharms; ++h) {
        const double hr = (double)h * r_lo;
        const double fl = std::floor(hr);
        DevHarm d{};
        d.h = h;
        d.rfloor0 = (int64_t)fl;
        d.dr0 = hr - fl;
        d.hr_lo = (double)d.rfloor0 + d.dr0;
        d.dh = (double)h * lodr;
        if (!rq) {
            d.P = 0;
            d.q = 1;
            d.pnum = 1;
            out.harms.push_back(d);
            continue;
        }
        const int64_t step = (int64_t)h * pnum;
        const int64_t s = step % q;
        const int64_t P = q / gcd64(step, q);
        d.P = (int32_t)P;
        d.q = (int32_t)q;
        d.pnum = (int32_t)pnum;
        d.s = (int32_t)s;
        d.base_adv = (int32_t)(step / q);
        d.w_off = (int64_t)out.w.size();
        d.a_off = (int64_t)out.a.size();
        out.w.resize(out.w.size() + (size_t)m * P);
        out.a.resize(out.a.size() + P);
        out.c.resize(out.c.size() + P);
        int64_t res = 0;
        for (int64_t pp = 0; pp < P; ++pp) {
            const double u = d.dr0 + (double)res / (double)q;
            const bool carry = u >= 1.0;
            const double dr = carry ? u - 1.0 : u;
            out.c[d.a_off + pp] = carry ? 1 : 0;
            if (dr == 0.0) {
                out.a[d.a_off + pp] = make_float2(1.0f, 0.0f);
                for (int i = 0; i < m; ++i) out.w[d.w_off + (int64_t)i * P + pp] = (i == m2 - 1) ? 1.0f : 0.0f;
            } else {
                const double sn = sinpi_d(dr), cs_ = cospi_d(dr);
                const double ar = (sn * cs_) / M_PI;
                const double ai = -((sn * sn) / M_PI);
                out.a[d.a_off + pp] = make_float2((float)ar, (float)ai);
                for (int i = 0; i < m; ++i)
                    out.w[d.w_off + (int64_t)i * P + pp] = (float)(1.0 / (dr - (double)(i + 1 - m2)));
            }
            res += s;
            if (res >= q) res -= q;
        }
        out.harms.push_back(d);
    }
}

}  // namespace

struct cs_handle {
    cs_params p{};
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;      // the stream work is issued on
    cudaStream_t own_stream = nullptr;  // the handle's own stream
    std::string err;
    std::vector<LevelHost> levels;
    int maxbins = 0, maxwmax = 0;
    std::vector<DevLevel> dlev;
    // spectrum
    const float2* amps = nullptr;
    DBuf amps_owned;
    int64_t namps = 0, N = 0;
    double dt = 0.0;
    bool has_spec = false;
    int64_t spec_h2d_bytes = 0;   // bytes of the last host spectrum copy, charged to the next search
    // A host spectrum (cs_set_spectrum) arrives in chunks on the copy stream:
    // chunk c of amps_owned, and its maximum in d_amax_spec[c], are on the
    // device once chunk_ev[c] has completed.  The first search after the copy
    // starts interpolating each run of blocks as soon as the chunks it reads
    // have landed; everything else that reads the spectrum waits for all.
    const float2* chunked_amps = nullptr;   // amps_owned while chunk_ev describes it
    bool chunks_pending = false;            // no search has overlapped with the copy yet
    int spec_nchunk = 0;
    cudaEvent_t chunk_ev[kMaxSpecChunks] = {};
    cudaEvent_t spec_free_ev = nullptr;     // every earlier read of amps_owned, before an overwrite
    DBuf d_amax_spec;
    // device buffers
    TcPlanHost tc;                      // tensor-core synthesis plan (synth != FP32)
    DBuf d_tcB;
    DBuf d_A, d_samp;
    HBuf h_nvalid, h_io;                // pinned: valid counts up; counters + candidate prefix down
    // What h_nvalid holds after a single-wave search of a band: a repeat of
    // the same band on a spectrum of the same size reuses it as it stands.
    struct NvKey {
        double r_lo, lodr, nyq;
        int64_t t_base, t_end, nblocks, namps;
        int32_t Nprof, nlev, nharms, m;
        int64_t profiles;   // its valid-count total (the stats' profile count)
    };
    NvKey nv_key{};
    bool nv_key_ok = false;
    HBuf h_bmap;                        // pinned: a wave's block map (block-list search)
    DBuf d_levels, d_tw, d_nvalid, d_X, d_Q0, d_sigma,
        d_tmetric, d_items, d_counts, d_cands, d_amax, d_bmap;
    // FP64 plan tables of the last anchor r_lo, already on the device
    // FP64 plan tables of recent anchors r_lo, each kept on the device too: a
    // batch of spectra of several lengths alternates between them without
    // re-uploading, and a captured batch graph reads them in place
    struct PlanSet {
        double rlo = 0.0;
        HostPlans host;
        DBuf harms, wtab, atab, ctab;
        void release() {
            harms.release();
            wtab.release();
            atab.release();
            ctab.release();
        }
    };
    std::vector<std::unique_ptr<PlanSet>> plan_sets;
    // batch graph (cs_set_batch_graph): one captured graph of a whole batch of
    // device spectra, replayed while the batch's signature stays the same;
    // any other search drops it (its buffers and plan tables may move)
    bool batch_graph = false;
    bool graph_valid = false;
    bool graph_failed = false;          // the batch of gkey could not be captured: do not retry
    cudaGraphExec_t gexec = nullptr;
    struct GraphSlot {
        HBuf io;           // counters, then the candidate prefix
        HBuf nvalid;       // valid counts the graph uploads
        int64_t launches = 0;
    };
    std::vector<GraphSlot> gslots;
    std::vector<cs_spectrum> gkey;
    double gkey_d[3] = {0, 0, 0};
    int64_t gkey_i[3] = {0, 0, 0};     // lobin, blocksize, spectra on the device
    // a graph of page-locked host spectra: each file's copy into the batch
    // buffer of its parity, on the copy stream forked into the capture
    cudaEvent_t bg_copied_ev[2] = {nullptr, nullptr}, bg_done_ev[2] = {nullptr, nullptr};
    int64_t plan_bytes = 0;
    // metric statistics (MetricStats) and normalisation (MetricNorm)
    bool ms_on = false;
    double ms_lo = 0.0, ms_hi = 64.0;
    int ms_nb = 3200, ms_nwin = 16;
    std::vector<cs_block_stats> ms_blocks;
    std::vector<double> ms_edges;     // [level][nwin+1], handle level order
    std::vector<int64_t> ms_counts;   // [level][nwin][nb]
    std::vector<double> ms_mom;       // [level][nwin][7]: under, over, total, sum, sumsq, vmin, vmax
    int ms_nlev = 0;
    bool norm_on = false;
    int norm_nwin = 0;
    std::vector<double> norm_edges, norm_loc, norm_scale;   // handle level order
    DBuf d_mst, d_mwin, d_mhist, d_muo, d_norm;
    DBuf d_bm_r, d_bm_h, d_bm_st, d_bm_prof, d_bm_w, d_bm_sig, d_bm_out;   // block_metrics
    // batch: spectra copied on a second stream into two alternating buffers
    cudaStream_t copy_stream = nullptr;
    // a second compute stream: the overlapped search's interpolation runs
    // alternate between it and the handle's stream (fork and join events)
    cudaStream_t run_stream = nullptr;
    cudaEvent_t run_fork_ev = nullptr, run_join_ev = nullptr;
    cudaEvent_t copy_ev[2] = {nullptr, nullptr};
    DBuf d_batch[2];
    HBuf h_mwin, h_mst;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cs_stats stats{};
    std::vector<float> last_sigma;
    std::vector<int32_t> last_nvalid;
    std::vector<float> last_tmetric;
    std::vector<float> last_gate;
    int diag = 0;
    size_t mem_limit = 0;   // cs_set_memory_limit: device bytes the handle may hold (0: no cap)
    // launch shapes (cs_autotune): interpolation kernel (-1: by applicability,
    // 0: one CTA per item, 1: persistent), the tensor epilogue's segment
    // divisors per phase (0: cost model) and its form (0 one slot, 1 phased
    // double buffer, 2 split).  The defaults are the shapes the tuner picks on
    // the survey workload (nharms 60, six levels), measured fastest there.
    int tune_interp = 0;
    int tune_div[2] = {3, 2};
    int tune_dbuf = 0;
    int tune_sigma = 0;
    double stats_sigma_min = 0.0;   // cs_autotune: least sigma-stage time of its last timed configuration     // block-sigma kernel: 0 = 384 threads, twiddles in shared memory; 1 = 256, through L1
    bool interp2_used = false, interp2_ok = false;   // the last search's interpolation kernel / its applicability
    int64_t stall_ns = 0;   // cs_set_wait_test
    int last_nlev = 0;
    int last_Nprof = 0;
};

namespace {

cs_status fail(cs_handle* H, cs_status st, const std::string& msg) {
    if (H) H->err = msg;
    return st;
}

cs_status cuda_fail(cs_handle* H, cudaError_t e, const char* where) {
    std::string m = std::string(where) + ": " + cudaGetErrorString(e);
    return fail(H, e == cudaErrorMemoryAllocation ? CS_ERR_OUT_OF_MEMORY : CS_ERR_CUDA, m);
}

#define CS_CUDA(call, where)                                   \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(H, e_, where); \
    } while (0)

// Chunks of a spectrum of namps bins, doubling in size: chunk 0 holds bins
// [0, u), chunk c >= 1 bins [u*2^(c-1), u*2^c), with u = max(namps/32, 64 Ki)
// (rounded up), so at most 6 chunks (spec_chunk_lo/hi, shared with k_amax).
// A block of trials near r reads bins up to about nharms*r, so the blocks in
// frequency order need growing prefixes: each chunk lands before the search
// has interpolated the blocks of the chunks below it.  Host and device spectra
// use the same layout, so a block's FP16 tile scale does not depend on where
// its spectrum came from.
static void spec_chunks(int64_t namps, int64_t* unit, int* nchunk) {
    const int64_t u = std::max<int64_t>((namps + 31) / 32, (int64_t)1 << 16);
    int n = 1;
    while (spec_chunk_hi(u, n - 1, namps) < namps) ++n;
    *unit = u;
    *nchunk = n;
}

// The chunk holding bin x (>= 0) of a spectrum of chunk unit u, at most last.
static int spec_chunk_of(int64_t x, int64_t u, int last) {
    int c = 0;
    while (c < last && x >= spec_chunk_hi(u, c, INT64_MAX)) ++c;
    return c;
}

// Work on H->stream that reads the attached spectrum at once waits for the
// whole of a chunked host copy.
static cudaError_t spec_ready(cs_handle* H) {
    if (H->amps && H->amps == H->chunked_amps)
        return cudaStreamWaitEvent(H->stream, H->chunk_ev[H->spec_nchunk - 1], 0);
    return cudaSuccess;
}

template <class T>
cudaError_t upload(DBuf& b, const std::vector<T>& v, cudaStream_t st) {
    cudaError_t e = b.ensure(v.size() * sizeof(T));
    if (e != cudaSuccess || v.empty()) return e;
    return cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

cs_status validate(const cs_params* p) {
    if (!p) return CS_ERR_INVALID_ARGUMENT;
    if (p->nharms < 1) return CS_ERR_INVALID_ARGUMENT;
    if (p->m < 2 || (p->m % 2) != 0) return CS_ERR_INVALID_ARGUMENT;  // "m must be even"
    if (!(p->hidr > 0)) return CS_ERR_INVALID_ARGUMENT;
    if (p->ndecim < 0 || p->ndecim > CS_MAX_DECIM) return CS_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < p->ndecim; ++i)
        if (p->decimations[i] < 1 || p->nharms / p->decimations[i] < 1) return CS_ERR_INVALID_ARGUMENT;
    if (p->precision != 0 && p->precision != 1) return CS_ERR_INVALID_ARGUMENT;
    if (!(p->boxcar_fsp > 0) || !(p->boxcar_maxfrac > 0)) return CS_ERR_INVALID_ARGUMENT;
    if (p->synth < CS_SYNTH_FP32 || p->synth > CS_SYNTH_FP16_SPLIT)
        return CS_ERR_INVALID_ARGUMENT;
    return CS_OK;
}

// Levels: the base fold k = 1, then every k > 1 of params.decimations in
// order (Workspace.decims, src/search.jl:1251-1254).
// The tensor synthesis plan with the handle's launch shapes, and its twiddles on the device.
cs_status build_tc(cs_handle* H) {
    const cs_params& p = H->p;
    const int rc = prepare_tc(H->dlev.data(), (int)H->dlev.size(), p.nharms, synth_fp16(p.synth) ? 1 : 0,
                              synth_split(p.synth), &H->tc, H->tune_div[0], H->tune_div[1], H->tune_dbuf);
    if (rc != 0)
        return fail(H, CS_ERR_UNSUPPORTED,
                    "tensor-core synthesis needs nharms <= 64, boxcar widths <= 32 and <= 512 TMEM columns");
    CS_CUDA(upload(H->d_tcB, H->tc.B, H->stream), "upload tensor twiddles");
    H->graph_valid = false;   // a captured graph holds the old plan
    return CS_OK;
}

cs_status build_levels(cs_handle* H) {
    const cs_params& p = H->p;
    std::vector<int> ks{1};
    for (int i = 0; i < p.ndecim; ++i)
        if (p.decimations[i] > 1) ks.push_back(p.decimations[i]);
    if ((int)ks.size() > kMaxLevels) return fail(H, CS_ERR_UNSUPPORTED, "more than 16 decimation levels");
    H->levels.clear();
    H->dlev.clear();
    H->maxbins = 0;
    H->maxwmax = 0;
    std::vector<float> tw;
    for (int k : ks) {
        LevelHost L;
        L.k = k;
        L.Hk = p.nharms / k;
        L.nbins = 2 * L.Hk;
        L.widths = ladder_widths(L.nbins, k, p);
        if (L.nbins > kMaxBins) return fail(H, CS_ERR_UNSUPPORTED, "nharms > 128 is not built");
        if ((int)L.widths.size() > kMaxWidths)
            return fail(H, CS_ERR_UNSUPPORTED, "more than 64 boxcar widths per level");
        if (L.widths.back() > kMaxBins)
            return fail(H, CS_ERR_UNSUPPORTED, "boxcar widths wider than 256 bins");
        DevLevel d{};
        d.k = k;
        d.Hk = L.Hk;
        d.nbins = L.nbins;
        d.nw = (int)L.widths.size();
        d.wmax = L.widths.back();
        d.np = ((L.Hk + 1) + 7) / 8 * 8;
        d.tw_off = (int64_t)tw.size();
        for (int i = 0; i < d.nw; ++i) {
            d.widths[i] = L.widths[i];
            d.rsqrtw[i] = (float)(1.0 / std::sqrt((double)L.widths[i]));
        }
        const int Nb = L.nbins;
        tw.resize(tw.size() + 2 * (size_t)L.Hk * d.np, 0.0f);
        float* C2 = tw.data() + d.tw_off;
        float* S2 = C2 + (size_t)L.Hk * d.np;
        for (int j = 1; j < L.Hk; ++j)
            for (int n = 0; n <= L.Hk; ++n) {
                const double ang = 2.0 * M_PI * (double)(((int64_t)j * n) % Nb) / (double)Nb;
                C2[(size_t)j * d.np + n] = (float)(2.0 * std::cos(ang));
                S2[(size_t)j * d.np + n] = (float)(-2.0 * std::sin(ang));
            }
        H->maxbins = std::max(H->maxbins, L.nbins);
        H->maxwmax = std::max(H->maxwmax, d.wmax);
        H->levels.push_back(L);
        H->dlev.push_back(d);
    }
    CS_CUDA(upload(H->d_levels, H->dlev, H->stream), "upload levels");
    CS_CUDA(upload(H->d_tw, tw, H->stream), "upload twiddles");
    if (p.synth != CS_SYNTH_FP32) return build_tc(H);
    return CS_OK;
}

// Number of trials j < n of a block whose k-fold lies below Nyquist: the
// prefix `decim_pass!` scores (src/search.jl:1680-1683), found by bisection
// on the same (monotone) FP64 predicate.
int nvalid_decim(int k, double rstart, double lodr, int n, double nyq) {
    auto ok = [&](int j) { return (double)k * (rstart + (double)j * lodr) < nyq; };
    if (n <= 0 || !ok(0)) return 0;
    if (ok(n - 1)) return n;
    int lo = 0, hi = n - 1;  // ok(lo), !ok(hi)
    while (hi - lo > 1) {
        const int mid = lo + (hi - lo) / 2;
        if (ok(mid)) lo = mid; else hi = mid;
    }
    return hi;
}

struct RunSpec {
    double r_lo;          // plan anchor: global trial 0 sits at r_lo
    double lodr;
    int64_t nblocks;
    int Nprof;
    int64_t t_base;       // global trial of block 0
    int64_t t_end;        // one past the last global trial
    int nlev;             // levels used (prefix of H->levels)
    bool exact_all;
    float threshold;
    float medcut;
    bool interp_only;     // stop after interpolation (cs_interp_chunk)
    bool keep_diag;       // keep sigma/nvalid/tmetric of the run on the host
    bool stats = false;   // collect MetricStats (exact_all)
    bool norm = false;    // normalised candidate test (exact_all)
    double r_hi = 0.0;    // band end (Fourier bins) and observation time, for the
    double T = 0.0;       // frequency windows
    double threshold_d = 0.0;
    const int64_t* blist = nullptr;   // search of a block list: band block indices (ascending), nblocks of them
    // capture into a batch graph: no host syncs; counters and the candidate
    // prefix go to these pinned slots, valid counts come from h_nvalid
    bool capture = false;
    int32_t* cap_io = nullptr;          // 64 bytes of counters, then kCandPrefix DevCands
    int32_t* cap_nvalid = nullptr;      // pinned [nblocks][nlev + 1], filled here
};

// _logedges (src/search.jl:1406-1411): nwin+1 log-spaced edges over [a, b].
void logedges(double a, double b, int nwin, double* e) {
    a = std::max(a, std::numeric_limits<double>::min());
    b = std::max(b, a * (1 + 1e-9));
    const double la = std::log10(a), lb = std::log10(b);
    for (int i = 0; i <= nwin; ++i) e[i] = std::pow(10.0, la + (lb - la) * i / nwin);
}

// _window_index (src/search.jl:1415-1416), 0-based: clamp(searchsortedlast(e, f), 1, nwin) - 1.
int window_index(const double* e, int nwin, double f) {
    int c = 0;
    for (int i = 0; i <= nwin; ++i) c += e[i] <= f;
    return std::min(std::max(c, 1), nwin) - 1;
}

cs_status run_blocks(cs_handle* H, const RunSpec& R, std::vector<DevCand>* cands, float2* x_out) {
    const cs_params& p = H->p;
    if (!R.capture) H->graph_valid = false;   // buffers and plan tables may move
    // The tables depend on r_lo only (params are fixed per handle): a search
    // repeated on the same band, the common case of a pipeline over many
    // spectra, reuses the device copies.
    int64_t plan_bytes = 0;
    cs_handle::PlanSet* ps = nullptr;
    for (auto& e : H->plan_sets)
        if (e->rlo == R.r_lo) ps = e.get();
    if (!ps) {
        if (R.capture) return fail(H, CS_ERR_UNSUPPORTED, "a captured search needs its plan tables on the device");
        if (H->plan_sets.size() >= 8) {
            H->plan_sets.front()->release();
            H->plan_sets.erase(H->plan_sets.begin());
        }
        H->plan_sets.push_back(std::make_unique<cs_handle::PlanSet>());
        ps = H->plan_sets.back().get();
        ps->rlo = R.r_lo;
        build_plans(p, R.r_lo, ps->host);
        const HostPlans& plans = ps->host;
        CS_CUDA(upload(ps->harms, plans.harms, H->stream), "upload plans");
        CS_CUDA(upload(ps->wtab, plans.w, H->stream), "upload weights");
        CS_CUDA(upload(ps->atab, plans.a, H->stream), "upload phases");
        CS_CUDA(upload(ps->ctab, plans.c, H->stream), "upload carries");
        plan_bytes = (int64_t)(plans.harms.size() * sizeof(DevHarm) + plans.w.size() * sizeof(float) +
                               plans.a.size() * sizeof(float2) + plans.c.size());
    }
    for (const DevHarm& d : ps->host.harms) {
        const double lim = 4.6e18;
        if ((double)R.t_end * (double)d.h * (double)d.pnum > lim)
            return fail(H, CS_ERR_UNSUPPORTED, "trial index times harmonic overflows 64-bit phase state");
    }

    const int Nprof = R.Nprof;
    const int win_max = (int)std::ceil((double)(Nprof - 1 + 64) * p.hidr) + p.m + 4;
    if (interp_smem(win_max, Nprof) > 200 * 1024)
        return fail(H, CS_ERR_UNSUPPORTED, "blocksize too large for the shared-memory interpolation row");
    // the persistent interpolation kernel: 16 taps, every phase cycle 1..256,
    // two CTAs' staging within an SM's shared memory, 8-byte aligned bins for
    // its window copies
    bool interp2 = p.m == 16 && interp2_smem(win_max, Nprof) <= 112 * 1024 &&
                   (reinterpret_cast<uintptr_t>(H->amps) & 7u) == 0;
    for (const DevHarm& d : ps->host.harms) interp2 = interp2 && d.P >= 1 && d.P <= 256;
    const bool interp2_ok = interp2;
    if (H->tune_interp == 0) interp2 = false;
    H->interp2_used = interp2;
    H->interp2_ok = interp2_ok;
    int maxbins = 0, maxwmax = 0;
    for (int l = 0; l < R.nlev; ++l) {
        maxbins = std::max(maxbins, H->dlev[l].nbins);
        maxwmax = std::max(maxwmax, H->dlev[l].wmax);
    }
    const size_t smem_synth = synth_fp32_smem(p.nharms, maxbins, maxwmax);
    int max_hk = 0, max_np = 0;
    for (int l = 0; l < R.nlev; ++l) {
        max_hk = std::max(max_hk, H->dlev[l].Hk);
        max_np = std::max(max_np, H->dlev[l].np);
    }
    if (sigma_smem(max_hk, max_np) + 16 * 1024 > 227 * 1024)
        return fail(H, CS_ERR_UNSUPPORTED, "sigma working set exceeds shared memory");
    const bool tensor = p.synth != CS_SYNTH_FP32 && R.nlev == (int)H->dlev.size();
    if (!tensor && smem_synth > 227 * 1024) return fail(H, CS_ERR_UNSUPPORTED, "profile tile exceeds shared memory");

    const int nlev = R.nlev;
    const int tiles_per_blk = (Nprof + 127) / 128;
    const bool want_x = !tensor || R.interp_only;
    const size_t per_blk = (want_x ? (size_t)p.nharms * Nprof * sizeof(float2) : 0) +
                           (tensor ? (size_t)tiles_per_blk * kATileBytes * synth_split(p.synth) : 0) +
                           (size_t)nlev * kSampStride * sizeof(float2) +
                           (size_t)nlev * Nprof * sizeof(float) * (R.exact_all ? 2 : 1) +
                           (size_t)nlev * Nprof * (sizeof(DevItem) + sizeof(DevCand)) + 64;
    // Working set of one wave: up to 16 GiB, and at most half of the free
    // device memory (a full survey band of a 2^24-sample spectrum, ~9 GB, is
    // one wave on a 180 GB part).
    // When the wave buffers the handle holds already cover every block of this
    // run (a repeated search), it is one wave with no query of the free memory
    // (a driver call that costs more host time than the rest of the set-up).
    const int64_t NB = R.nblocks;
    auto holds = [](const DBuf& d, size_t n) { return d.bytes >= n; };
    const bool held_all =
        !H->mem_limit && !R.stats && (!want_x || holds(H->d_X, (size_t)NB * p.nharms * Nprof * sizeof(float2))) &&
        (!(tensor && !R.interp_only) ||
         holds(H->d_A, (size_t)NB * tiles_per_blk * kATileBytes * synth_split(p.synth))) &&
        (R.interp_only ||
         (holds(H->d_samp, (size_t)NB * nlev * kSampStride * sizeof(float2)) &&
          (!(H->diag >= 2 && !R.exact_all) || holds(H->d_Q0, (size_t)NB * nlev * Nprof * sizeof(float))) &&
          holds(H->d_sigma, (size_t)NB * nlev * sizeof(float)) &&
          holds(H->d_nvalid, (size_t)NB * (nlev + 1) * sizeof(int32_t)) &&
          holds(H->d_items, (size_t)NB * nlev * Nprof * sizeof(DevItem)) &&
          holds(H->d_cands, (size_t)NB * nlev * Nprof * sizeof(DevCand)) &&
          (!R.exact_all || holds(H->d_tmetric, (size_t)NB * nlev * Nprof * sizeof(float)))));
    size_t budget = (size_t)16 << 30;
    if (!held_all) {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            // memory this handle already holds for waves counts as free
            const size_t held = H->d_X.bytes + H->d_A.bytes + H->d_samp.bytes + H->d_Q0.bytes +
                                H->d_items.bytes + H->d_cands.bytes + H->d_tmetric.bytes;
            budget = std::min(budget, std::max<size_t>((size_t)512 << 20, (free_b + held) / 2));
        }
    }
    if (H->mem_limit) {
        // the cap covers the wave buffers and everything else the handle holds
        // (spectrum, plan tables, twiddles, batch buffers, block-metric scratch)
        size_t fixed = 0;
        const DBuf* held_fixed[] = {&H->amps_owned, &H->d_tcB, &H->d_levels, &H->d_tw, &H->d_counts, &H->d_amax,
                                    &H->d_bmap, &H->d_batch[0], &H->d_batch[1], &H->d_mst, &H->d_mwin,
                                    &H->d_mhist, &H->d_muo, &H->d_norm, &H->d_bm_r, &H->d_bm_h, &H->d_bm_st,
                                    &H->d_bm_prof, &H->d_bm_w, &H->d_bm_sig, &H->d_bm_out};
        for (const DBuf* b : held_fixed) fixed += b->bytes;
        for (const auto& e : H->plan_sets)
            fixed += e->harms.bytes + e->wtab.bytes + e->atab.bytes + e->ctab.bytes;
        const size_t room = H->mem_limit > fixed + ((size_t)1 << 16) ? H->mem_limit - fixed - ((size_t)1 << 16) : 0;
        if (room < per_blk)
            return fail(H, CS_ERR_OUT_OF_MEMORY,
                        "memory limit " + std::to_string(H->mem_limit) + " B: the handle holds " +
                            std::to_string(fixed) + " B and one block's working set needs " +
                            std::to_string(per_blk) + " B more");
        budget = std::min(budget, room);
    }
    const int64_t WB =
        held_all ? NB : std::max<int64_t>(1, std::min<int64_t>(R.nblocks, (int64_t)(budget / per_blk)));
    if (R.capture) {
        // a captured search runs as one wave on buffers an earlier run sized,
        // without statistics, diagnostics or host round trips
        if (WB < R.nblocks) return fail(H, CS_ERR_UNSUPPORTED, "a captured search must fit one wave");
        if (R.stats || R.norm || R.keep_diag || R.interp_only || R.blist || R.exact_all)
            return fail(H, CS_ERR_UNSUPPORTED, "a captured search carries no statistics, diagnostics or block list");
        auto small = [](const DBuf& d, size_t n) { return d.bytes < n; };
        if ((want_x && small(H->d_X, (size_t)WB * p.nharms * Nprof * sizeof(float2))) ||
            (tensor && small(H->d_A, (size_t)WB * tiles_per_blk * kATileBytes * synth_split(p.synth))) ||
            small(H->d_samp, (size_t)WB * nlev * kSampStride * sizeof(float2)) ||
            small(H->d_sigma, (size_t)WB * nlev * sizeof(float)) ||
            small(H->d_nvalid, (size_t)WB * (nlev + 1) * sizeof(int32_t)) ||
            small(H->d_items, (size_t)WB * nlev * Nprof * sizeof(DevItem)) ||
            small(H->d_cands, (size_t)WB * nlev * Nprof * sizeof(DevCand)) || small(H->d_counts, 4 * sizeof(int32_t)) ||
            (tensor && synth_fp16(p.synth) && small(H->d_amax, kMaxSpecChunks * sizeof(uint32_t))))
            return fail(H, CS_ERR_UNSUPPORTED, "a captured search needs buffers sized by an earlier run");
    }

    if (want_x) CS_CUDA(H->d_X.ensure((size_t)WB * p.nharms * Nprof * sizeof(float2)), "alloc X");
    if (tensor && !R.interp_only) {
        const size_t abytes = (size_t)WB * tiles_per_blk * kATileBytes * synth_split(p.synth);
        if (abytes > H->d_A.bytes) {
            // zero once: the K columns past 2*nharms are never written
            CS_CUDA(H->d_A.ensure(abytes), "alloc A tiles");
            CS_CUDA(cudaMemsetAsync(H->d_A.p, 0, H->d_A.bytes, H->stream), "zero A tiles");
        }
    }
    if (!R.interp_only) {
        CS_CUDA(H->d_samp.ensure((size_t)WB * nlev * kSampStride * sizeof(float2)), "alloc samples");
        if (H->diag >= 2 && !R.exact_all)
            CS_CUDA(H->d_Q0.ensure((size_t)WB * nlev * Nprof * sizeof(float)), "alloc gate values");
        CS_CUDA(H->d_sigma.ensure((size_t)WB * nlev * sizeof(float)), "alloc sigma");
        // valid counts [nb][nlev], then each block's last spectrum chunk [nb]
        CS_CUDA(H->d_nvalid.ensure((size_t)WB * (nlev + 1) * sizeof(int32_t)), "alloc nvalid");
        CS_CUDA(H->d_items.ensure((size_t)WB * nlev * Nprof * sizeof(DevItem)), "alloc items");
        CS_CUDA(H->d_cands.ensure((size_t)WB * nlev * Nprof * sizeof(DevCand)), "alloc cands");
        if (R.exact_all)
            CS_CUDA(H->d_tmetric.ensure((size_t)WB * nlev * Nprof * sizeof(float)), "alloc tmetric");
    }
    CS_CUDA(H->d_counts.ensure(4 * sizeof(int32_t)), "alloc counters");
    const int mnw = H->ms_nwin, mnb = H->ms_nb;
    if (R.stats) {
        H->ms_nlev = nlev;
        H->ms_blocks.clear();
        H->ms_edges.assign((size_t)nlev * (mnw + 1), 0.0);
        H->ms_mom.assign((size_t)nlev * mnw * 7, 0.0);
        for (int l = 0; l < nlev; ++l) {
            const double k = (double)H->dlev[l].k;
            logedges(k * R.r_lo / R.T, k * R.r_hi / R.T, mnw, &H->ms_edges[(size_t)l * (mnw + 1)]);
            for (int w = 0; w < mnw; ++w) {
                H->ms_mom[((size_t)l * mnw + w) * 7 + 5] = INFINITY;
                H->ms_mom[((size_t)l * mnw + w) * 7 + 6] = -INFINITY;
            }
        }
        CS_CUDA(H->d_mhist.ensure((size_t)nlev * mnw * mnb * sizeof(unsigned long long)), "alloc histograms");
        CS_CUDA(H->d_muo.ensure((size_t)nlev * mnw * 2 * sizeof(unsigned long long)), "alloc histogram tails");
        CS_CUDA(cudaMemsetAsync(H->d_mhist.p, 0, (size_t)nlev * mnw * mnb * sizeof(unsigned long long), H->stream),
                "clear histograms");
        CS_CUDA(cudaMemsetAsync(H->d_muo.p, 0, (size_t)nlev * mnw * 2 * sizeof(unsigned long long), H->stream),
                "clear histogram tails");
        CS_CUDA(H->d_mst.ensure((size_t)WB * nlev * kMstFields * sizeof(double)), "alloc block stats");
        CS_CUDA(H->d_mwin.ensure((size_t)WB * nlev * sizeof(int32_t)), "alloc block windows");
        CS_CUDA(H->h_mwin.ensure((size_t)WB * nlev * sizeof(int32_t)), "pinned block windows");
        CS_CUDA(H->h_mst.ensure((size_t)WB * nlev * kMstFields * sizeof(double)), "pinned block stats");
    }
    if (R.norm) {
        const int nw = H->norm_nwin;
        std::vector<double> nd;
        nd.insert(nd.end(), H->norm_edges.begin(), H->norm_edges.begin() + (size_t)nlev * (nw + 1));
        nd.insert(nd.end(), H->norm_loc.begin(), H->norm_loc.begin() + (size_t)nlev * nw);
        nd.insert(nd.end(), H->norm_scale.begin(), H->norm_scale.begin() + (size_t)nlev * nw);
        CS_CUDA(upload(H->d_norm, nd, H->stream), "upload normalisation");
    }

    cs_stats& S = H->stats;
    S = cs_stats{};
    S.h2d_bytes = H->spec_h2d_bytes + plan_bytes;
    H->spec_h2d_bytes = 0;
    S.blocks = R.nblocks;
    if (R.blist) {
        S.trials = 0;
        for (int64_t c = 0; c < R.nblocks; ++c)
            S.trials += std::min<int64_t>(Nprof, R.t_end - R.blist[c] * (int64_t)Nprof);
    } else {
        S.trials = R.t_end - R.t_base;
    }
    if (R.keep_diag) {
        H->last_sigma.assign((size_t)R.nblocks * nlev, 0.0f);
        H->last_nvalid.assign((size_t)R.nblocks * nlev, 0);
        if (R.exact_all) H->last_tmetric.assign((size_t)R.nblocks * nlev * Nprof, 0.0f);
        else H->last_tmetric.clear();
        if (H->diag >= 2 && !R.exact_all) H->last_gate.assign((size_t)R.nblocks * nlev * Nprof, 0.0f);
        else H->last_gate.clear();
        H->last_nlev = nlev;
        H->last_Nprof = Nprof;
    }
    const double nyq = (double)H->N / 2.0;
    // counters, then the first kCandPrefix candidates, come back in one pinned read
    constexpr int kCandPrefix = 4096;
    if (!R.capture) CS_CUDA(H->h_io.ensure(64 + (size_t)kCandPrefix * sizeof(DevCand)), "pinned readback");
    int32_t* counts = R.capture ? R.cap_io : H->h_io.as<int32_t>();
    DevCand* cand_pre = reinterpret_cast<DevCand*>(reinterpret_cast<uint8_t*>(counts) + 64);

    // The spectrum's chunks: a host spectrum still being copied in chunks is
    // interpolated run of blocks by run of blocks as its chunks land (first
    // wave only; later work waits for the whole copy).
    int64_t unit = 0;
    int nch = 0;
    spec_chunks(H->namps, &unit, &nch);
    const bool host_spec = H->amps == H->chunked_amps;
    if (host_spec && nch != H->spec_nchunk) return fail(H, CS_ERR_INVALID_ARGUMENT, "spectrum chunk layout changed");
    bool overlap = host_spec && H->chunks_pending && !R.capture;
    // FP16 A tiles: each spectrum chunk's largest component, for their range
    // scale (a host spectrum's come with its copy)
    const bool fp16_scale = tensor && !R.interp_only && synth_fp16(p.synth);
    const uint32_t* amax = nullptr;
    if (fp16_scale && host_spec) {
        amax = H->d_amax_spec.as<uint32_t>();
    } else if (fp16_scale) {
        if (!R.capture) CS_CUDA(H->d_amax.ensure(kMaxSpecChunks * sizeof(uint32_t)), "alloc chunk maxima");
        CS_CUDA(cudaMemsetAsync(H->d_amax.p, 0, kMaxSpecChunks * sizeof(uint32_t), H->stream), "reset chunk maxima");
        CS_CUDA(launch_amax(H->amps, H->namps, unit, nch, H->d_amax.as<uint32_t>(), H->stream, H->num_sms),
                "maximum launch");
        S.launches += 1;
        amax = H->d_amax.as<uint32_t>();
    }
    if (host_spec && !overlap) CS_CUDA(spec_ready(H), "wait for the spectrum");

    for (int64_t c0 = 0; c0 < R.nblocks; c0 += WB) {
        const int nb = (int)std::min<int64_t>(WB, R.nblocks - c0);
        WaveArgs a{};
        a.amps = H->amps;
        a.namps = H->namps;
        a.Nhalf = H->N / 2;
        a.nharms = p.nharms;
        a.m = p.m;
        a.nlev = nlev;
        a.Nprof = Nprof;
        a.t_first = R.t_base + c0 * (int64_t)Nprof;
        a.total = R.t_end;
        a.nblk = nb;
        a.blk_base = (int32_t)c0;
        a.harms = ps->harms.as<DevHarm>();
        a.wtab = ps->wtab.as<float>();
        a.atab = ps->atab.as<float2>();
        a.ctab = ps->ctab.as<uint8_t>();
        a.levels = H->d_levels.as<DevLevel>();
        a.tw = H->d_tw.as<float>();
        a.nvalid = H->d_nvalid.as<int32_t>();
        a.X = want_x ? H->d_X.as<float2>() : nullptr;
        a.Atile = (tensor && !R.interp_only) ? H->d_A.as<uint8_t>() : nullptr;
        a.tiles_per_blk = tiles_per_blk;
        a.fp16 = synth_fp16(p.synth) ? 1 : 0;
        a.asplit = synth_split(p.synth);
        a.amax_bits = amax;
        a.blk_cidx = nullptr;
        a.blk_first = 0;
        a.samp = R.interp_only ? nullptr : H->d_samp.as<float2>();
        a.Q0 = (H->diag >= 2 && !R.exact_all) ? H->d_Q0.as<float>() : nullptr;   // gate values: diagnostics only
        a.sigma = H->d_sigma.as<float>();
        a.tmetric = R.exact_all ? H->d_tmetric.as<float>() : nullptr;
        a.items = H->d_items.as<DevItem>();
        a.n_items = H->d_counts.as<int32_t>();
        a.cap_items = (int32_t)std::min<int64_t>((int64_t)nb * nlev * Nprof, INT32_MAX);
        a.cands = H->d_cands.as<DevCand>();
        a.n_cands = H->d_counts.as<int32_t>() + 1;
        a.cap_cands = a.cap_items;
        a.threshold = R.threshold;
        a.medcut = R.medcut;
        a.medcut_gate = R.medcut;
        a.verify_gate = 0;
        if (tensor && !R.exact_all) {
            // A 16-bit gate flags with slack below medcut; the rescan re-forms
            // the FP32 gate and applies medcut itself, so the rescanned set --
            // hence every candidate -- is the plain form's.
            // (the split modes keep FP16's slack: their gates are closer still)
            const float rel = p.synth == CS_SYNTH_BF16 ? 0.08f : 0.02f;
            const float ab = p.synth == CS_SYNTH_BF16 ? 0.10f : 0.05f;
            a.medcut_gate = R.medcut - (rel * std::fabs(R.medcut) + ab);
            a.verify_gate = 1;
        }
        a.exact_all = R.exact_all ? 1 : 0;
        a.r_lo = R.r_lo;
        a.lodr = R.lodr;
        a.T = R.T;
        a.norm_thr = R.threshold_d;
        a.stall_ns = H->stall_ns;
        if (R.norm) {
            const int nw = H->norm_nwin;
            const double* nd = H->d_norm.as<double>();
            a.norm_edges = nd;
            a.norm_loc = nd + (size_t)nlev * (nw + 1);
            a.norm_scale = nd + (size_t)nlev * (nw + 1) + (size_t)nlev * nw;
            a.norm_nwin = nw;
        }
        int32_t* mwin = nullptr;
        if (R.stats) {
            a.mst = H->d_mst.as<double>();
            a.mwin = H->d_mwin.as<int32_t>();
            a.mhist = H->d_mhist.as<unsigned long long>();
            a.muo = H->d_muo.as<unsigned long long>();
            a.hist_lo = H->ms_lo;
            a.hist_hi = H->ms_hi;
            a.hist_invw = (double)mnb / (H->ms_hi - H->ms_lo);   // MetricHistogram's nb / (hi - lo)
            a.hist_nb = mnb;
            a.hist_nwin = mnw;
            mwin = H->h_mwin.as<int32_t>();
        }
        int* d_err = H->d_counts.as<int32_t>() + 2;

        if (!R.capture) {
            const size_t had = H->h_nvalid.bytes;
            CS_CUDA(H->h_nvalid.ensure((size_t)nb * (nlev + 1) * sizeof(int32_t)), "pinned valid counts");
            if (H->h_nvalid.bytes != had) H->nv_key_ok = false;
        }
        int32_t* nvalid = R.capture ? R.cap_nvalid : H->h_nvalid.as<int32_t>();
        int32_t* cidx = nvalid + (size_t)nb * nlev;   // each block's last spectrum chunk
        const bool cacheable = !R.capture && !R.blist && !mwin && c0 == 0 && nb == R.nblocks;
        const cs_handle::NvKey key{R.r_lo, R.lodr, nyq, R.t_base, R.t_end, R.nblocks, H->namps,
                                   Nprof, nlev, p.nharms, p.m, 0};
        const cs_handle::NvKey& kk = H->nv_key;
        const bool reuse = cacheable && H->nv_key_ok && kk.r_lo == key.r_lo && kk.lodr == key.lodr &&
                           kk.nyq == key.nyq && kk.t_base == key.t_base && kk.t_end == key.t_end &&
                           kk.nblocks == key.nblocks && kk.namps == key.namps && kk.Nprof == key.Nprof &&
                           kk.nlev == key.nlev && kk.nharms == key.nharms && kk.m == key.m;
        if (!R.capture && !reuse) H->nv_key_ok = false;   // h_nvalid is rewritten below
        const int64_t profiles0 = S.profiles;
        if (reuse) S.profiles += kk.profiles;
        for (int b = 0; b < nb && !reuse; ++b) {
            const int64_t c = c0 + b;
            // global trial of the block's first trial
            const int64_t tb = R.blist ? R.blist[c] * (int64_t)Nprof : R.t_base + c * (int64_t)Nprof;
            const int n = (int)std::min<int64_t>(Nprof, R.t_end - tb);
            const double rstart = R.r_lo + (double)tb * R.lodr;
            // the highest bin any harmonic's window reaches: nharms * r of the
            // block's last trial, m/2 taps past it, and a margin for rounding
            const double top = std::floor((double)p.nharms * (rstart + (double)(n - 1) * R.lodr));
            const int64_t bin_max = top < 0 ? 0 : (top > 4.0e18 ? INT64_MAX / 2 : (int64_t)top) + p.m / 2 + 4;
            cidx[b] = spec_chunk_of(bin_max, unit, nch - 1);
            for (int l = 0; l < nlev; ++l) {
                const int k = H->dlev[l].k;
                nvalid[(size_t)b * nlev + l] = (k == 1) ? n : nvalid_decim(k, rstart, R.lodr, n, nyq);
                S.profiles += nvalid[(size_t)b * nlev + l];
                if (mwin) {
                    // the whole block goes to the window of its centre frequency
                    // (src/search.jl:1825-1826, :1848-1849)
                    const double rmean = rstart + (n - 1) * R.lodr / 2;
                    const double f = k == 1 ? rmean / R.T : (double)k * rmean / R.T;
                    mwin[(size_t)b * nlev + l] =
                        window_index(&H->ms_edges[(size_t)l * (mnw + 1)], mnw, f);
                }
            }
        }
        if (cacheable && !reuse) {
            H->nv_key = key;
            H->nv_key.profiles = S.profiles - profiles0;
            H->nv_key_ok = true;
        }
        if (mwin)
            CS_CUDA(cudaMemcpyAsync(H->d_mwin.p, mwin, (size_t)nb * nlev * sizeof(int32_t), cudaMemcpyHostToDevice,
                                    H->stream),
                    "upload block windows");
        if (R.blist) {
            CS_CUDA(H->h_bmap.ensure((size_t)nb * sizeof(int64_t)), "pinned block map");
            std::copy(R.blist + c0, R.blist + c0 + nb, H->h_bmap.as<int64_t>());
            CS_CUDA(H->d_bmap.ensure((size_t)WB * sizeof(int64_t)), "alloc block map");
            CS_CUDA(cudaMemcpyAsync(H->d_bmap.p, H->h_bmap.p, (size_t)nb * sizeof(int64_t), cudaMemcpyHostToDevice,
                                    H->stream),
                    "upload block map");
            a.blk_map = H->d_bmap.as<int64_t>();
        }
        CS_CUDA(cudaMemsetAsync(H->d_counts.p, 0, 4 * sizeof(int32_t), H->stream), "reset counters");
        if (!R.interp_only) {
            CS_CUDA(cudaMemcpyAsync(H->d_nvalid.p, nvalid, (size_t)nb * (nlev + 1) * sizeof(int32_t),
                                    cudaMemcpyHostToDevice, H->stream),
                    "upload nvalid");
            S.h2d_bytes += (int64_t)nb * (nlev + 1) * (int64_t)sizeof(int32_t);
            a.nvalid = H->d_nvalid.as<int32_t>();
            a.blk_cidx = H->d_nvalid.as<int32_t>() + (size_t)nb * nlev;
        }
        if (!R.capture) CS_CUDA(cudaEventRecord(H->ev[0], H->stream), "event");
        auto interp_launch = [&](const WaveArgs& w, cudaStream_t st) {
            return interp2 ? launch_interp2(w, st, win_max, d_err, H->num_sms) : launch_interp(w, st, win_max, d_err);
        };
        if (overlap) {
            // Runs of blocks by the last chunk they read (the running maximum
            // of cidx): each run starts once that chunk has landed.  The runs
            // write disjoint blocks, so they alternate between the handle's
            // stream and a second one, each run's start overlapping the
            // previous run's tail; the handle's stream joins the second after
            // the last run.
            if (!H->run_stream)
                CS_CUDA(cudaStreamCreateWithFlags(&H->run_stream, cudaStreamNonBlocking), "run stream");
            if (!H->run_fork_ev) CS_CUDA(cudaEventCreateWithFlags(&H->run_fork_ev, cudaEventDisableTiming), "event");
            if (!H->run_join_ev) CS_CUDA(cudaEventCreateWithFlags(&H->run_join_ev, cudaEventDisableTiming), "event");
            CS_CUDA(cudaEventRecord(H->run_fork_ev, H->stream), "event");   // after the uploads above
            CS_CUDA(cudaStreamWaitEvent(H->run_stream, H->run_fork_ev, 0), "fork");
            int s = 0, need = cidx[0], run = 0;
            for (int b = 1; b <= nb; ++b) {
                if (b < nb && cidx[b] <= need) continue;
                WaveArgs w = a;
                w.blk_first = s;
                w.nblk = b - s;
                cudaStream_t st = (run & 1) ? H->run_stream : H->stream;
                CS_CUDA(cudaStreamWaitEvent(st, H->chunk_ev[need], 0), "wait for a spectrum chunk");
                CS_CUDA(interp_launch(w, st), "interp launch");
                S.launches += 1;
                ++run;
                if (b < nb) {
                    s = b;
                    need = cidx[b];
                }
            }
            CS_CUDA(cudaEventRecord(H->run_join_ev, H->run_stream), "event");
            CS_CUDA(cudaStreamWaitEvent(H->stream, H->run_join_ev, 0), "join");
            CS_CUDA(spec_ready(H), "wait for the spectrum");
            H->chunks_pending = false;
            overlap = false;
        } else {
            CS_CUDA(interp_launch(a, H->stream), "interp launch");
            S.launches += 1;
        }
        if (!R.capture) CS_CUDA(cudaEventRecord(H->ev[1], H->stream), "event");
        if (!R.interp_only) {
            // sigma needs only the samples, so it runs first and the synthesis
            // epilogue applies the medcut test itself (no gate pass over HBM);
            // exact_all scores every trial exactly and needs no gate at all
            CS_CUDA(launch_sigma(a, H->stream, max_hk, max_np, d_err, H->tune_sigma), "sigma launch");
            if (!R.capture) CS_CUDA(cudaEventRecord(H->ev[2], H->stream), "event");
            S.launches += 1;
            if (!R.exact_all) {
                if (tensor)
                    CS_CUDA(launch_synth_tc(a, H->tc, H->d_tcB.p, d_err, H->stream, H->num_sms), "synth launch");
                else
                    CS_CUDA(launch_synth_fp32(a, H->stream, (int)smem_synth), "synth launch");
                S.launches += 1;
            }
            if (!R.capture) CS_CUDA(cudaEventRecord(H->ev[3], H->stream), "event");
            CS_CUDA(launch_rescue(a, H->stream, H->num_sms), "rescue launch");
            S.launches += 1;
            if (R.stats) {
                CS_CUDA(launch_mstats(a, H->stream), "stats launch");
                S.launches += 1;
                CS_CUDA(cudaMemcpyAsync(H->h_mst.p, H->d_mst.p, (size_t)nb * nlev * kMstFields * sizeof(double),
                                        cudaMemcpyDeviceToHost, H->stream),
                        "read block stats");
            }
            if (!R.capture) CS_CUDA(cudaEventRecord(H->ev[4], H->stream), "event");
        }
        CS_CUDA(cudaMemcpyAsync(counts, H->d_counts.p, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost,
                                H->stream),
                "read counters");
        const int n_pre = (int)std::min<size_t>((size_t)kCandPrefix, H->d_cands.bytes / sizeof(DevCand));
        if (cands && !R.interp_only && n_pre > 0)
            CS_CUDA(cudaMemcpyAsync(cand_pre, H->d_cands.p, (size_t)n_pre * sizeof(DevCand),
                                    cudaMemcpyDeviceToHost, H->stream),
                    "read candidates");
        if (R.capture) return CS_OK;   // one wave: the caller's graph holds the rest
        CS_CUDA(cudaStreamSynchronize(H->stream), "wave");
        S.d2h_bytes += 4 * sizeof(int32_t);
        if (counts[2] == 1) return fail(H, CS_ERR_CUDA, "interpolation window exceeded its bound");
        if (counts[2] == 2) return fail(H, CS_ERR_TIMEOUT, "tensor-core completion wait ran out");
        if (counts[2] == 3) return fail(H, CS_ERR_TIMEOUT, "sigma sample copy wait ran out");
        if (counts[2] == 4) return fail(H, CS_ERR_TIMEOUT, "interpolation window copy wait ran out");
        float ms = 0.0f;
        CS_CUDA(cudaEventElapsedTime(&ms, H->ev[0], H->ev[1]), "timing");
        S.ms_interp += ms;
        if (!R.interp_only) {
            CS_CUDA(cudaEventElapsedTime(&ms, H->ev[1], H->ev[2]), "timing");
            S.ms_sigma += ms;
            CS_CUDA(cudaEventElapsedTime(&ms, H->ev[2], H->ev[3]), "timing");
            S.ms_synth += ms;
            CS_CUDA(cudaEventElapsedTime(&ms, H->ev[3], H->ev[4]), "timing");
            S.ms_rescue += ms;
            CS_CUDA(cudaEventElapsedTime(&ms, H->ev[0], H->ev[4]), "timing");
            S.ms_total += ms;
        } else {
            S.ms_total += ms;
        }
        S.waves += 1;
        if (R.stats) {
            // BlockMetricStats per (block, k) (src/search.jl:1839-1844, :1710-1717):
            // every base-fold block, decimated blocks with a valid trial; their
            // moments also enter the (k, window) histogram's exact accumulators.
            const double* mst = H->h_mst.as<double>();
            const int64_t gblk0 = R.t_base / Nprof + c0;
            for (int b = 0; b < nb; ++b) {
                const int64_t c = c0 + b;
                const int64_t i0 = c * (int64_t)Nprof;
                const int n = (int)std::min<int64_t>(Nprof, R.t_end - (R.t_base + i0));
                const double rstart = R.r_lo + (double)(R.t_base + i0) * R.lodr;
                const double rmean = rstart + (n - 1) * R.lodr / 2;
                for (int l = 0; l < nlev; ++l) {
                    const int k = H->dlev[l].k, Hk = H->dlev[l].Hk;
                    const int nv = nvalid[(size_t)b * nlev + l];
                    if (k > 1 && nv == 0) continue;
                    const double* m = mst + ((size_t)b * nlev + l) * kMstFields;
                    cs_block_stats r{};
                    r.block = gblk0 + b + 1;
                    r.k = k;
                    r.Hk = Hk;
                    r.nbins = 2 * Hk;
                    const double half_n = (double)H->N / 2;
                    if (k == 1) {
                        r.ngoodbins = std::min(half_n / rmean, (double)p.nharms);
                        r.flo = rstart / R.T;
                        r.fhi = (rstart + (n - 1) * R.lodr) / R.T;
                    } else {
                        r.ngoodbins = std::min(half_n / ((double)k * rmean), (double)Hk);
                        r.flo = (double)k * rstart / R.T;
                        r.fhi = (double)k * (rstart + (nv - 1) * R.lodr) / R.T;
                    }
                    r.n = nv;
                    r.min = m[1];
                    r.median = m[2];
                    r.mean = m[3];
                    r.std = m[4];
                    r.max = m[5];
                    H->ms_blocks.push_back(r);
                    double* mom = &H->ms_mom[((size_t)l * mnw + mwin[(size_t)b * nlev + l]) * 7];
                    mom[2] += nv;
                    mom[3] += m[6];
                    mom[4] += m[7];
                    if (nv > 0) {
                        mom[5] = std::min(mom[5], m[1]);
                        mom[6] = std::max(mom[6], m[5]);
                    }
                }
            }
        }
        if (R.interp_only) {
            if (x_out)
                CS_CUDA(cudaMemcpy(x_out, H->d_X.p, (size_t)nb * p.nharms * Nprof * sizeof(float2),
                                   cudaMemcpyDeviceToHost),
                        "read amplitudes");
            continue;
        }
        const int n_items = counts[0], n_c = counts[1];
        S.rescued += R.exact_all ? 0 : n_items;
        S.candidates += n_c;
        if (!R.exact_all && n_items > a.cap_items) return fail(H, CS_ERR_CAPACITY, "rescue list overflow");
        if (n_c > a.cap_cands) return fail(H, CS_ERR_CAPACITY, "candidate list overflow");
        if (cands && n_c > 0) {
            cands->insert(cands->end(), cand_pre, cand_pre + std::min(n_c, n_pre));
            if (n_c > n_pre) {
                const size_t old_n = cands->size();
                cands->resize(old_n + (size_t)(n_c - n_pre));
                CS_CUDA(cudaMemcpy(cands->data() + old_n, H->d_cands.as<DevCand>() + n_pre,
                                   (size_t)(n_c - n_pre) * sizeof(DevCand), cudaMemcpyDeviceToHost),
                        "read candidates");
            }
            S.d2h_bytes += (int64_t)n_c * (int64_t)sizeof(DevCand);
        }
        if (R.keep_diag) {
            CS_CUDA(cudaMemcpy(H->last_sigma.data() + (size_t)c0 * nlev, H->d_sigma.p,
                               (size_t)nb * nlev * sizeof(float), cudaMemcpyDeviceToHost),
                    "read sigma");
            std::copy(nvalid, nvalid + (size_t)nb * nlev, H->last_nvalid.begin() + (size_t)c0 * nlev);
            S.d2h_bytes += (int64_t)nb * nlev * (int64_t)sizeof(float);
            if (R.exact_all)
                CS_CUDA(cudaMemcpy(H->last_tmetric.data() + (size_t)c0 * nlev * Nprof, H->d_tmetric.p,
                                   (size_t)nb * nlev * Nprof * sizeof(float), cudaMemcpyDeviceToHost),
                        "read metrics");
            if (!H->last_gate.empty()) {
                float* g = H->last_gate.data() + (size_t)c0 * nlev * Nprof;
                CS_CUDA(cudaMemcpy(g, H->d_Q0.p, (size_t)nb * nlev * Nprof * sizeof(float),
                                   cudaMemcpyDeviceToHost),
                        "read gate");
                for (int b = 0; b < nb; ++b)
                    for (int l = 0; l < nlev; ++l) {
                        const float sg = H->last_sigma[(size_t)(c0 + b) * nlev + l];
                        const float inv = sg > 0.0f ? 1.0f / sg : 0.0f;
                        const int nv = nvalid[(size_t)b * nlev + l];
                        float* row = g + ((size_t)b * nlev + l) * Nprof;
                        for (int j = 0; j < Nprof; ++j) row[j] = j < nv ? row[j] * inv : 0.0f;
                    }
            }
        }
    }
    if (R.stats) {
        std::vector<unsigned long long> cnt((size_t)nlev * mnw * mnb), uo((size_t)nlev * mnw * 2);
        CS_CUDA(cudaMemcpy(cnt.data(), H->d_mhist.p, cnt.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
                "read histograms");
        CS_CUDA(cudaMemcpy(uo.data(), H->d_muo.p, uo.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost),
                "read histogram tails");
        H->ms_counts.assign(cnt.begin(), cnt.end());
        for (size_t i = 0; i < (size_t)nlev * mnw; ++i) {
            H->ms_mom[i * 7 + 0] = (double)uo[2 * i];
            H->ms_mom[i * 7 + 1] = (double)uo[2 * i + 1];
        }
        std::stable_sort(H->ms_blocks.begin(), H->ms_blocks.end(), [](const cs_block_stats& x, const cs_block_stats& y) {
            return x.block != y.block ? x.block < y.block : x.k < y.k;
        });
    }
    return CS_OK;
}

}  // namespace

extern "C" {

cs_status cs_set_batch_graph(cs_handle* H, int32_t enable) {
    if (!H) return CS_ERR_INVALID_ARGUMENT;
    H->batch_graph = enable != 0;
    if (!H->batch_graph) H->graph_valid = false;
    return CS_OK;
}

const char* cs_version(void) { return CS_VERSION_STRING; }

const char* cs_last_error(const cs_handle* h) { return h ? h->err.c_str() : "null handle"; }

namespace {
// Launch shapes cs_autotune chose, per device and cs_params (bytewise).
struct TuneEntry {
    int device;
    cs_params p;
    int interp, div0, div1, dbuf, sigma;
};
std::mutex g_tune_mu;
std::vector<TuneEntry> g_tune_cache;

bool tune_lookup(int device, const cs_params& p, TuneEntry* out) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (const TuneEntry& e : g_tune_cache)
        if (e.device == device && std::memcmp(&e.p, &p, sizeof(cs_params)) == 0) {
            *out = e;
            return true;
        }
    return false;
}

void tune_store(const TuneEntry& t) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    for (TuneEntry& e : g_tune_cache)
        if (e.device == t.device && std::memcmp(&e.p, &t.p, sizeof(cs_params)) == 0) {
            e = t;
            return;
        }
    g_tune_cache.push_back(t);
}
}  // namespace

cs_status cs_create(cs_handle** out, const cs_params* params, int32_t device) {
    if (!out) return CS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    cs_status st = validate(params);
    if (st != CS_OK) return st;
    cs_handle* H = new (std::nothrow) cs_handle();
    if (!H) return CS_ERR_OUT_OF_MEMORY;
    H->p = *params;
    H->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&H->own_stream, cudaStreamNonBlocking);
    H->stream = H->own_stream;
    if (e == cudaSuccess) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
            H->num_sms = sms;
        for (auto& ev : H->ev)
            if (e == cudaSuccess) e = cudaEventCreate(&ev);
    }
    if (e != cudaSuccess) {
        cs_destroy(H);
        return CS_ERR_CUDA;
    }
    st = build_levels(H);
    TuneEntry te{};
    if (st == CS_OK && tune_lookup(device, H->p, &te)) {
        // launch shapes an earlier cs_autotune chose for these parameters here
        H->tune_interp = te.interp;
        H->tune_div[0] = te.div0;
        H->tune_div[1] = te.div1;
        H->tune_dbuf = te.dbuf;
        H->tune_sigma = te.sigma;
        if (H->p.synth != CS_SYNTH_FP32) st = build_tc(H);
    }
    if (st != CS_OK) {
        cs_destroy(H);
        return st;
    }
    *out = H;
    return CS_OK;
}

cs_status cs_set_stream(cs_handle* H, void* stream) {
    if (!H) return CS_ERR_INVALID_ARGUMENT;
    H->stream = stream ? static_cast<cudaStream_t>(stream) : H->own_stream;
    return CS_OK;
}

cs_status cs_destroy(cs_handle* H) {
    if (!H) return CS_ERR_INVALID_ARGUMENT;
    cudaSetDevice(H->device);
    if (H->stream) cudaStreamSynchronize(H->stream);
    if (H->own_stream) cudaStreamSynchronize(H->own_stream);
    if (H->copy_stream) cudaStreamSynchronize(H->copy_stream);   // chunk copies still in flight
    for (auto& e : H->plan_sets) e->release();
    H->plan_sets.clear();
    if (H->gexec) cudaGraphExecDestroy(H->gexec);
    H->gexec = nullptr;
    for (auto& g : H->gslots) {
        g.io.release();
        g.nvalid.release();
    }
    DBuf* bufs[] = {&H->d_A, &H->d_samp, &H->d_tcB, &H->amps_owned, &H->d_levels, &H->d_tw, &H->d_amax, &H->d_bmap,
                    &H->d_nvalid, &H->d_X, &H->d_Q0, &H->d_sigma,
                    &H->d_tmetric, &H->d_items, &H->d_counts, &H->d_cands};
    for (DBuf* b : bufs) b->release();
    H->h_nvalid.release();
    H->h_bmap.release();
    H->h_io.release();
    H->h_mwin.release();
    H->h_mst.release();
    if (H->copy_stream) cudaStreamSynchronize(H->copy_stream);
    H->d_batch[0].release();
    H->d_batch[1].release();
    for (auto& e : H->copy_ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : H->chunk_ev)
        if (e) cudaEventDestroy(e);
    if (H->spec_free_ev) cudaEventDestroy(H->spec_free_ev);
    if (H->run_fork_ev) cudaEventDestroy(H->run_fork_ev);
    if (H->run_join_ev) cudaEventDestroy(H->run_join_ev);
    if (H->run_stream) {
        cudaStreamSynchronize(H->run_stream);
        cudaStreamDestroy(H->run_stream);
    }
    H->d_amax_spec.release();
    if (H->copy_stream) cudaStreamDestroy(H->copy_stream);
    DBuf* mbufs[] = {&H->d_mst, &H->d_mwin, &H->d_mhist, &H->d_muo, &H->d_norm, &H->d_bm_r, &H->d_bm_h,
                     &H->d_bm_st, &H->d_bm_prof, &H->d_bm_w, &H->d_bm_sig, &H->d_bm_out};
    for (DBuf* b : mbufs) b->release();
    for (auto& ev : H->ev)
        if (ev) cudaEventDestroy(ev);
    if (H->own_stream) cudaStreamDestroy(H->own_stream);
    delete H;
    return CS_OK;
}

static cs_status check_spec_args(cs_handle* H, const float* amps, int64_t namps, int64_t N, double dt) {
    if (!H) return CS_ERR_INVALID_ARGUMENT;
    if (!amps || namps < 1 || N < 2 || !(dt > 0))
        return fail(H, CS_ERR_INVALID_ARGUMENT, "spectrum needs namps >= 1, N >= 2, dt > 0");
    return CS_OK;
}

cs_status cs_set_spectrum(cs_handle* H, const float* amps, int64_t namps, int64_t N, double dt) {
    cs_status st = check_spec_args(H, amps, namps, N, dt);
    if (st != CS_OK) return st;
    CS_CUDA(cudaSetDevice(H->device), "set device");
    H->has_spec = false;
    H->chunked_amps = nullptr;
    H->chunks_pending = false;
    if (!H->copy_stream) CS_CUDA(cudaStreamCreateWithFlags(&H->copy_stream, cudaStreamNonBlocking), "copy stream");
    if (!H->spec_free_ev) CS_CUDA(cudaEventCreateWithFlags(&H->spec_free_ev, cudaEventDisableTiming), "event");
    for (auto& e : H->chunk_ev)
        if (!e) CS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "event");
    // the copies overwrite amps_owned only after everything issued so far that reads it
    CS_CUDA(cudaEventRecord(H->spec_free_ev, H->stream), "event");
    CS_CUDA(cudaStreamWaitEvent(H->copy_stream, H->spec_free_ev, 0), "order the copy");
    CS_CUDA(H->amps_owned.ensure((size_t)namps * sizeof(float2)), "alloc spectrum");
    CS_CUDA(H->d_amax_spec.ensure(kMaxSpecChunks * sizeof(uint32_t)), "alloc chunk maxima");
    CS_CUDA(cudaMemsetAsync(H->d_amax_spec.p, 0, kMaxSpecChunks * sizeof(uint32_t), H->copy_stream),
            "reset chunk maxima");
    int64_t unit = 0;
    int nch = 0;
    spec_chunks(namps, &unit, &nch);
    float2* dst = H->amps_owned.as<float2>();
    for (int c = 0; c < nch; ++c) {
        const int64_t b0 = spec_chunk_lo(unit, c), nb = spec_chunk_hi(unit, c, namps) - b0;
        CS_CUDA(cudaMemcpyAsync(dst + b0, amps + 2 * b0, (size_t)nb * sizeof(float2), cudaMemcpyHostToDevice,
                                H->copy_stream),
                "copy spectrum");
        // a one-chunk layout of the chunk alone: its maximum into slot c
        CS_CUDA(launch_amax(dst + b0, nb, nb, 1, H->d_amax_spec.as<uint32_t>() + c, H->copy_stream, H->num_sms),
                "chunk maximum launch");
        CS_CUDA(cudaEventRecord(H->chunk_ev[c], H->copy_stream), "event");
    }
    H->spec_nchunk = nch;
    H->chunked_amps = dst;
    H->chunks_pending = true;
    H->spec_h2d_bytes = namps * (int64_t)sizeof(float2);
    H->amps = dst;
    H->namps = namps;
    H->N = N;
    H->dt = dt;
    H->has_spec = true;
    return CS_OK;
}

cs_status cs_set_spectrum_device(cs_handle* H, const float* d_amps, int64_t namps, int64_t N, double dt) {
    cs_status st = check_spec_args(H, d_amps, namps, N, dt);
    if (st != CS_OK) return st;
    if ((reinterpret_cast<uintptr_t>(d_amps) & 7u) != 0)
        return fail(H, CS_ERR_INVALID_ARGUMENT, "device spectrum must be 8-byte aligned");
    H->amps = reinterpret_cast<const float2*>(d_amps);
    H->namps = namps;
    H->N = N;
    H->dt = dt;
    H->has_spec = true;
    return CS_OK;
}

}  // extern "C"

namespace {

// The search of one spectrum over blocks [block_begin, block_end) of the band's
// grid; candidates appended to `outv` in the reference's order.
// The band bookkeeping of `search` (src/search.jl:2016-2027) into a RunSpec;
// *empty when there is nothing to search.
cs_status setup_run(cs_handle* H, double lofreq, double hifreq, int64_t lobin, int64_t blocksize, double threshold,
                    int32_t exact_all, int64_t block_begin, int64_t block_end, const int64_t* blist, int64_t nlist,
                    RunSpec& R, bool* empty) {
    *empty = true;
    if (!H->has_spec) return fail(H, CS_ERR_NO_SPECTRUM, "no spectrum attached");
    CS_CUDA(cudaSetDevice(H->device), "set device");
    const cs_params& p = H->p;
    const double T = (double)H->N * H->dt;
    const double lodr = p.hidr / (double)p.nharms;
    double r_lo = lofreq * T;
    if (lobin != 100) r_lo = (double)lobin;
    const double r_hi = hifreq * T;
    const double span = std::floor((r_hi - r_lo) / lodr);
    if (!(span == span) || span > 4.0e15) return fail(H, CS_ERR_INVALID_ARGUMENT, "band is not finite");
    const int64_t total = std::max<int64_t>(0, (int64_t)span + 1);
    H->stats = cs_stats{};
    if (total == 0) return CS_OK;
    const int Nprof = (int)std::max<int64_t>(1, blocksize);
    if (blocksize > (1 << 16)) return fail(H, CS_ERR_UNSUPPORTED, "blocksize above 65536 is not built");
    // Blocks [block_begin, block_end) of the band's grid (block_end < 0: to the
    // end); the trial anchor stays r_lo, so a range reproduces exactly the
    // blocks, sigmas and candidates of the whole search.
    const int64_t nblk_all = (total + Nprof - 1) / Nprof;
    const int64_t b1 = block_end < 0 ? nblk_all : std::min(block_end, nblk_all);
    if (blist) {
        // a list of the band's blocks: ascending, inside the band
        for (int64_t i = 0; i < nlist; ++i)
            if (blist[i] < 0 || blist[i] >= nblk_all || (i > 0 && blist[i] <= blist[i - 1]))
                return fail(H, CS_ERR_INVALID_ARGUMENT, "block list must ascend strictly within the band's blocks");
        if (H->ms_on || H->norm_on)
            return fail(H, CS_ERR_UNSUPPORTED, "metric statistics and normalisation need contiguous blocks");
        if (nlist == 0) return CS_OK;
        block_begin = 0;
    } else if (block_begin >= b1) {
        return CS_OK;
    }
    R = RunSpec{};
    R.r_lo = r_lo;
    R.lodr = lodr;
    R.Nprof = Nprof;
    R.nblocks = blist ? nlist : b1 - block_begin;
    R.t_base = block_begin * Nprof;
    R.t_end = blist ? total : std::min(total, b1 * Nprof);
    R.blist = blist;
    R.nlev = (int)H->levels.size();
    R.stats = H->ms_on;
    R.norm = H->norm_on;
    // statistics and normalisation need every trial's exact metric (medcut = -Inf)
    R.exact_all = exact_all != 0 || R.stats || R.norm;
    R.threshold = (float)threshold;
    R.threshold_d = threshold;
    R.medcut = R.exact_all ? -INFINITY : (float)(threshold - p.boxcar_medmargin);
    R.keep_diag = H->diag >= 1;
    R.r_hi = r_hi;
    R.T = T;
    *empty = false;
    return CS_OK;
}

// Device records to candidates: the reference order with one task (by block,
// base fold then each decimation level in params order, ascending trial:
// src/search.jl:1809-1859) and its FP64 frequency expressions.
void emit_candidates(cs_handle* H, const RunSpec& R, std::vector<DevCand>& raw, std::vector<cs_candidate>* outv) {
    const cs_params& p = H->p;
    std::sort(raw.begin(), raw.end(), [](const DevCand& x, const DevCand& y) {
        if (x.blk != y.blk) return x.blk < y.blk;
        if (x.lev != y.lev) return x.lev < y.lev;
        return x.j < y.j;
    });
    const int64_t block_begin = R.blist ? 0 : R.t_base / R.Nprof;
    const int64_t n = (int64_t)raw.size();
    outv->reserve(outv->size() + (size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        const DevCand& c = raw[i];
        const LevelHost& L = H->levels[c.lev];
        const int64_t i0 = (block_begin + (int64_t)c.blk) * R.Nprof;
        const double rstart = R.r_lo + (double)i0 * R.lodr;
        cs_candidate o{};
        if (L.k == 1) {
            o.r = rstart + (double)c.j * R.lodr;           // rf, src/search.jl:1833
            o.nharm = p.nharms;
        } else {
            o.r = (double)L.k * (rstart + (double)c.j * R.lodr);  // r_dec, src/search.jl:1696
            o.nharm = L.Hk;
        }
        o.freq = o.r / R.T;
        o.metric = (double)c.metric;
        if (R.norm) {
            // z of the normalised test, with the device's FP64 expressions
            const int nw = H->norm_nwin;
            const int w = window_index(&H->norm_edges[(size_t)c.lev * (nw + 1)], nw, o.freq);
            o.metric = ((double)c.metric - H->norm_loc[(size_t)c.lev * nw + w]) / H->norm_scale[(size_t)c.lev * nw + w];
        }
        o.k = L.k;
        o.trial = i0 + c.j;
        outv->push_back(o);
    }
}

cs_status search_core(cs_handle* H, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                      double threshold, int32_t exact_all, int64_t block_begin, int64_t block_end,
                      std::vector<cs_candidate>* outv, const int64_t* blist = nullptr, int64_t nlist = 0) {
    RunSpec R{};
    bool empty = true;
    cs_status st = setup_run(H, lofreq, hifreq, lobin, blocksize, threshold, exact_all, block_begin, block_end, blist,
                             nlist, R, &empty);
    if (st != CS_OK || empty) return st;
    std::vector<DevCand> raw;
    st = run_blocks(H, R, &raw, nullptr);
    if (st != CS_OK) return st;
    emit_candidates(H, R, raw, outv);
    return CS_OK;
}

constexpr int kGraphPrefix = 4096;   // candidates a captured search reads back per spectrum

// Capture one graph of the whole batch (device spectra, after an ordinary run
// of it sized every buffer): per spectrum the valid-count upload from its
// own pinned slot, the search's launches and the readback of its counters
// and candidate prefix into that slot.  Not an error when a spectrum cannot
// be captured (more than one wave): the batch then stays ordinary.
void capture_batch(cs_handle* H, const cs_spectrum* files, int nfiles, int on_device, double lofreq, double hifreq,
                   int64_t lobin, int64_t blocksize, double threshold) {
    if (H->gexec) cudaGraphExecDestroy(H->gexec);
    H->gexec = nullptr;
    H->graph_valid = false;
    H->graph_failed = true;   // until the capture below succeeds
    H->gkey.assign(files, files + nfiles);
    H->gkey_d[0] = lofreq;
    H->gkey_d[1] = hifreq;
    H->gkey_d[2] = threshold;
    H->gkey_i[0] = lobin;
    H->gkey_i[1] = blocksize;
    H->gkey_i[2] = on_device;
    const cs_stats keep = H->stats;   // the batch's own statistics survive the capture
    struct Restore {
        cs_handle* H;
        cs_stats s;
        ~Restore() { H->stats = s; }
    } restore{H, keep};
    if ((int)H->gslots.size() < nfiles) H->gslots.resize(nfiles);
    const int nlev = (int)H->levels.size();
    // slots and run specs first: no allocation while capturing
    std::vector<RunSpec> specs(nfiles);
    std::vector<char> empty(nfiles, 1);
    for (int i = 0; i < nfiles; ++i) {
        H->amps = on_device ? reinterpret_cast<const float2*>(files[i].amps) : H->d_batch[i & 1].as<float2>();
        H->namps = files[i].namps;
        H->N = files[i].N;
        H->dt = files[i].dt;
        H->has_spec = true;
        bool e = true;
        if (setup_run(H, lofreq, hifreq, lobin, blocksize, threshold, 0, 0, -1, nullptr, 0, specs[i], &e) != CS_OK) return;
        empty[i] = e ? 1 : 0;
        if (e) continue;
        if (H->gslots[i].io.ensure(64 + (size_t)kGraphPrefix * sizeof(DevCand)) != cudaSuccess ||
            H->gslots[i].nvalid.ensure((size_t)specs[i].nblocks * (nlev + 1) * sizeof(int32_t)) != cudaSuccess)
            return;
    }
    if (!on_device) {
        if (!H->copy_stream || !H->copy_ev[0]) return;   // the ordinary run before made them
        for (int b = 0; b < 2; ++b) {
            if (!H->bg_copied_ev[b] && cudaEventCreateWithFlags(&H->bg_copied_ev[b], cudaEventDisableTiming)) return;
            if (!H->bg_done_ev[b] && cudaEventCreateWithFlags(&H->bg_done_ev[b], cudaEventDisableTiming)) return;
        }
    }
    if (cudaStreamBeginCapture(H->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) return;
    bool ok = true;
    // Host spectra: file i lands in batch buffer i&1 by a copy on the copy
    // stream, issued before file i-1's search so that the two overlap; the
    // copy into a buffer waits for the search two files back that read it.
    auto copy_file = [&](int i) -> bool {
        const int b = i & 1;
        if (i >= 2 && cudaStreamWaitEvent(H->copy_stream, H->bg_done_ev[b], 0) != cudaSuccess) return false;
        if (cudaMemcpyAsync(H->d_batch[b].p, files[i].amps, (size_t)files[i].namps * sizeof(float2),
                            cudaMemcpyHostToDevice, H->copy_stream) != cudaSuccess)
            return false;
        return cudaEventRecord(H->bg_copied_ev[b], H->copy_stream) == cudaSuccess;
    };
    if (!on_device && nfiles > 0) {
        // fork the copy stream into the capture
        ok = cudaEventRecord(H->copy_ev[0], H->stream) == cudaSuccess &&
             cudaStreamWaitEvent(H->copy_stream, H->copy_ev[0], 0) == cudaSuccess && copy_file(0);
    }
    for (int i = 0; i < nfiles && ok; ++i) {
        if (!on_device) {
            if (i + 1 < nfiles && !copy_file(i + 1)) {
                ok = false;
                break;
            }
            if (cudaStreamWaitEvent(H->stream, H->bg_copied_ev[i & 1], 0) != cudaSuccess) {
                ok = false;
                break;
            }
        }
        if (empty[i]) {
            if (!on_device) ok = cudaEventRecord(H->bg_done_ev[i & 1], H->stream) == cudaSuccess;
            continue;
        }
        H->amps = on_device ? reinterpret_cast<const float2*>(files[i].amps) : H->d_batch[i & 1].as<float2>();
        H->namps = files[i].namps;
        H->N = files[i].N;
        H->dt = files[i].dt;
        RunSpec R = specs[i];
        R.capture = true;
        R.keep_diag = false;
        R.cap_io = H->gslots[i].io.as<int32_t>();
        R.cap_nvalid = H->gslots[i].nvalid.as<int32_t>();
        std::vector<DevCand> unused;   // (the candidates come back through the slot)
        ok = run_blocks(H, R, &unused, nullptr) == CS_OK;
        H->gslots[i].launches = H->stats.launches;
        if (ok && !on_device) ok = cudaEventRecord(H->bg_done_ev[i & 1], H->stream) == cudaSuccess;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(H->stream, &g);
    if (ok && ec == cudaSuccess && g && cudaGraphInstantiate(&H->gexec, g, 0) == cudaSuccess) {
        H->graph_valid = true;
        H->graph_failed = false;
    } else {
        H->gexec = nullptr;
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();   // a failed capture leaves no sticky state to report
    H->err.clear();
}


}  // namespace

extern "C" {

cs_status cs_search_blocks(cs_handle* H, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                           double threshold, const int64_t* blocks, int64_t nblocks, cs_candidate* out, int64_t cap,
                           int64_t* n_out) {
    if (!H || !n_out || (cap > 0 && !out) || cap < 0 || nblocks < 0 || (nblocks > 0 && !blocks))
        return CS_ERR_INVALID_ARGUMENT;
    *n_out = 0;
    std::vector<cs_candidate> v;
    cs_status st = search_core(H, lofreq, hifreq, lobin, blocksize, threshold, 0, 0, -1, &v, blocks, nblocks);
    if (st != CS_OK) return st;
    const int64_t n = (int64_t)v.size();
    std::copy_n(v.begin(), std::min(n, cap), out);
    *n_out = n;
    if (n > cap) return fail(H, CS_ERR_CAPACITY, "candidate array too small");
    return CS_OK;
}

cs_status cs_block_features(cs_handle* H, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                            float* d_out, int64_t cap_blocks, int64_t* nblocks_out, int32_t* nfeat_out) {
    if (!H || !nblocks_out || !nfeat_out || cap_blocks < 0 || (cap_blocks > 0 && !d_out))
        return CS_ERR_INVALID_ARGUMENT;
    *nblocks_out = 0;
    int nfeat = 0;
    for (const DevLevel& L : H->dlev) nfeat += L.Hk;
    *nfeat_out = nfeat;
    if (!H->has_spec) return fail(H, CS_ERR_NO_SPECTRUM, "no spectrum attached");
    if (blocksize < 1 || blocksize > (1 << 16)) return fail(H, CS_ERR_UNSUPPORTED, "blocksize must be 1..65536");
    CS_CUDA(cudaSetDevice(H->device), "set device");
    // the band's trial grid, as search_core
    const double T = (double)H->N * H->dt;
    const double lodr = H->p.hidr / (double)H->p.nharms;
    double r_lo = lofreq * T;
    if (lobin != 100) r_lo = (double)lobin;
    const double span = std::floor((hifreq * T - r_lo) / lodr);
    if (!(span == span) || span > 4.0e15) return fail(H, CS_ERR_INVALID_ARGUMENT, "band is not finite");
    const int64_t total = std::max<int64_t>(0, (int64_t)span + 1);
    const int64_t nb = (total + blocksize - 1) / blocksize;
    *nblocks_out = nb;
    if (nb > cap_blocks) return fail(H, CS_ERR_CAPACITY, "feature array too small");
    if (nb == 0) return CS_OK;
    CS_CUDA(spec_ready(H), "wait for the spectrum");
    const cudaError_t e = launch_features(H->amps, H->namps, r_lo, lodr, blocksize, total,
                                          H->d_levels.as<DevLevel>(), (int)H->dlev.size(), nfeat, d_out, H->stream);
    if (e == cudaErrorInvalidValue) return fail(H, CS_ERR_UNSUPPORTED, "more than 512 features per block");
    CS_CUDA(e, "features launch");
    CS_CUDA(cudaStreamSynchronize(H->stream), "features");
    return CS_OK;
}

cs_status cs_search_range(cs_handle* H, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                          double threshold, int32_t exact_all, int64_t block_begin, int64_t block_end,
                          cs_candidate* out, int64_t cap, int64_t* n_out) {
    if (!H || !n_out || (cap > 0 && !out) || cap < 0 || block_begin < 0) return CS_ERR_INVALID_ARGUMENT;
    *n_out = 0;
    std::vector<cs_candidate> v;
    cs_status st = search_core(H, lofreq, hifreq, lobin, blocksize, threshold, exact_all, block_begin, block_end,
                               &v);
    if (st != CS_OK) return st;
    const int64_t n = (int64_t)v.size();
    std::copy_n(v.begin(), std::min(n, cap), out);
    *n_out = n;
    if (n > cap) return fail(H, CS_ERR_CAPACITY, "candidate array too small");
    return CS_OK;
}

cs_status cs_search_batch(cs_handle* H, const cs_spectrum* files, int32_t nfiles, int32_t on_device,
                          double lofreq, double hifreq, int64_t lobin, int64_t blocksize, double threshold,
                          cs_candidate* out, int32_t* file_of, int64_t cap, int64_t* n_out) {
    if (!H || !files || nfiles < 0 || !n_out || (cap > 0 && (!out || !file_of)) || cap < 0)
        return CS_ERR_INVALID_ARGUMENT;
    *n_out = 0;
    for (int i = 0; i < nfiles; ++i) {
        const cs_spectrum& f = files[i];
        if (!f.amps || f.namps < 1 || f.N < 2 || !(f.dt > 0))
            return fail(H, CS_ERR_INVALID_ARGUMENT, "every spectrum needs namps >= 1, N >= 2, dt > 0");
        if (on_device && (reinterpret_cast<uintptr_t>(f.amps) & 7u) != 0)
            return fail(H, CS_ERR_INVALID_ARGUMENT, "device spectra must be 8-byte aligned");
    }
    CS_CUDA(cudaSetDevice(H->device), "set device");
    // Host spectra: file i+1 is copied on the copy stream into the other of two
    // device buffers while file i is searched; the search stream waits on the
    // copy's event.  A buffer is refilled only after the search that read it
    // returned (each search ends with a stream synchronisation).
    int64_t maxa = 0;
    for (int i = 0; i < nfiles; ++i) maxa = std::max(maxa, files[i].namps);
    if (!on_device && nfiles > 0) {
        if (!H->copy_stream) CS_CUDA(cudaStreamCreateWithFlags(&H->copy_stream, cudaStreamNonBlocking), "copy stream");
        for (int b = 0; b < 2; ++b) {
            if (!H->copy_ev[b]) CS_CUDA(cudaEventCreateWithFlags(&H->copy_ev[b], cudaEventDisableTiming), "copy event");
            CS_CUDA(H->d_batch[b].ensure((size_t)maxa * sizeof(float2)), "alloc spectrum buffer");
        }
    }
    auto issue_copy = [&](int i) -> cudaError_t {
        const int b = i & 1;
        cudaError_t e = cudaMemcpyAsync(H->d_batch[b].p, files[i].amps, (size_t)files[i].namps * sizeof(float2),
                                        cudaMemcpyHostToDevice, H->copy_stream);
        if (e == cudaSuccess) e = cudaEventRecord(H->copy_ev[b], H->copy_stream);
        return e;
    };
    if (!on_device && nfiles > 0) CS_CUDA(issue_copy(0), "copy spectrum");
    std::vector<cs_candidate> all;
    std::vector<int32_t> owner;
    cs_stats tot{};
    // a replayable graph: device spectra, or host spectra that are all page-locked
    // (the graph's copies read them in place at every replay)
    bool host_pinned = !on_device && nfiles > 0;
    for (int i = 0; i < nfiles && host_pinned; ++i) {
        cudaPointerAttributes at{};
        host_pinned = cudaPointerGetAttributes(&at, files[i].amps) == cudaSuccess && at.type == cudaMemoryTypeHost;
    }
    cudaGetLastError();   // (an unregistered pointer is an answer, not an error)
    const bool want_graph = (on_device || host_pinned) && H->batch_graph && nfiles > 0;
    auto same_key = [&]() {
        if ((int)H->gkey.size() != nfiles) return false;
        if (H->gkey_d[0] != lofreq || H->gkey_d[1] != hifreq || H->gkey_d[2] != threshold ||
            H->gkey_i[0] != lobin || H->gkey_i[1] != blocksize || H->gkey_i[2] != on_device)
            return false;
        for (int i = 0; i < nfiles; ++i)
            if (H->gkey[i].amps != files[i].amps || H->gkey[i].namps != files[i].namps || H->gkey[i].N != files[i].N ||
                H->gkey[i].dt != files[i].dt)
                return false;
        return true;
    };
    const bool key_match = want_graph && same_key();
    if (key_match && H->graph_valid) {
        // replay: one launch for the whole batch, one synchronisation
        CS_CUDA(cudaGraphLaunch(H->gexec, H->stream), "batch graph launch");
        CS_CUDA(cudaStreamSynchronize(H->stream), "batch graph");
        for (int i = 0; i < nfiles; ++i) {
            const cs_spectrum& f = files[i];
            H->amps = on_device ? reinterpret_cast<const float2*>(f.amps) : H->d_batch[i & 1].as<float2>();
            H->namps = f.namps;
            H->N = f.N;
            H->dt = f.dt;
            H->has_spec = true;
            RunSpec R{};
            bool empty = true;
            cs_status st = setup_run(H, lofreq, hifreq, lobin, blocksize, threshold, 0, 0, -1, nullptr, 0, R, &empty);
            if (st != CS_OK) return st;
            const size_t before = all.size();
            if (!empty) {
                const int32_t* counts = H->gslots[i].io.as<int32_t>();
                if (counts[2] != 0) return fail(H, CS_ERR_TIMEOUT, "a device wait ran out in the batch graph");
                const int n_c = counts[1];
                if (n_c > kGraphPrefix) {
                    // more candidates than the captured prefix: search this one
                    // again the ordinary way (the graph is dropped and rebuilt);
                    // a host spectrum is copied to the batch buffer first
                    if (!on_device) {
                        CS_CUDA(cudaMemcpyAsync(H->d_batch[0].p, f.amps, (size_t)f.namps * sizeof(float2),
                                                cudaMemcpyHostToDevice, H->stream),
                                "copy spectrum");
                        H->amps = H->d_batch[0].as<float2>();
                    }
                    st = search_core(H, lofreq, hifreq, lobin, blocksize, threshold, 0, 0, -1, &all);
                    if (st != CS_OK) return st;
                    // the re-search's own launches and copies count too
                    tot.launches += H->stats.launches;
                    tot.h2d_bytes += H->stats.h2d_bytes;
                    tot.d2h_bytes += H->stats.d2h_bytes;
                } else {
                    const DevCand* pre = reinterpret_cast<const DevCand*>(H->gslots[i].io.as<uint8_t>() + 64);
                    std::vector<DevCand> raw(pre, pre + n_c);
                    emit_candidates(H, R, raw, &all);
                }
                tot.trials += R.t_end - R.t_base;
                tot.blocks += R.nblocks;
                tot.rescued += counts[0];
                tot.candidates += n_c;
                tot.waves += 1;
                tot.launches += H->gslots[i].launches;
                tot.d2h_bytes += 64 + (int64_t)std::min(n_c, kGraphPrefix) * (int64_t)sizeof(DevCand);
                if (!on_device) tot.h2d_bytes += f.namps * (int64_t)sizeof(float2);
            }
            owner.insert(owner.end(), all.size() - before, i);
        }
        H->stats = tot;
        H->has_spec = false;
        const int64_t n = (int64_t)all.size();
        std::copy_n(all.begin(), std::min(n, cap), out);
        std::copy_n(owner.begin(), std::min(n, cap), file_of);
        *n_out = n;
        if (n > cap) return fail(H, CS_ERR_CAPACITY, "candidate array too small");
        return CS_OK;
    }
    for (int i = 0; i < nfiles; ++i) {
        if (!on_device) {
            if (i + 1 < nfiles) CS_CUDA(issue_copy(i + 1), "copy spectrum");
            CS_CUDA(cudaStreamWaitEvent(H->stream, H->copy_ev[i & 1], 0), "wait spectrum");
            H->amps = H->d_batch[i & 1].as<float2>();
        } else {
            H->amps = reinterpret_cast<const float2*>(files[i].amps);
        }
        H->namps = files[i].namps;
        H->N = files[i].N;
        H->dt = files[i].dt;
        H->has_spec = true;
        H->spec_h2d_bytes = on_device ? 0 : files[i].namps * (int64_t)sizeof(float2);
        const size_t before = all.size();
        cs_status st = search_core(H, lofreq, hifreq, lobin, blocksize, threshold, 0, 0, -1, &all);
        if (st != CS_OK) return st;
        owner.insert(owner.end(), all.size() - before, i);
        const cs_stats& S = H->stats;
        tot.trials += S.trials;
        tot.blocks += S.blocks;
        tot.profiles += S.profiles;
        tot.rescued += S.rescued;
        tot.candidates += S.candidates;
        tot.waves += S.waves;
        tot.launches += S.launches;
        tot.ms_interp += S.ms_interp;
        tot.ms_synth += S.ms_synth;
        tot.ms_sigma += S.ms_sigma;
        tot.ms_rescue += S.ms_rescue;
        tot.ms_total += S.ms_total;
        tot.h2d_bytes += S.h2d_bytes;
        tot.d2h_bytes += S.d2h_bytes;
    }
    H->stats = tot;
    if (want_graph && !(key_match && H->graph_failed))
        capture_batch(H, files, nfiles, on_device, lofreq, hifreq, lobin, blocksize, threshold);
    H->has_spec = false;   // the batch buffers are not a spectrum of the handle's
    const int64_t n = (int64_t)all.size();
    std::copy_n(all.begin(), std::min(n, cap), out);
    std::copy_n(owner.begin(), std::min(n, cap), file_of);
    *n_out = n;
    if (n > cap) return fail(H, CS_ERR_CAPACITY, "candidate array too small");
    return CS_OK;
}


cs_status cs_search(cs_handle* H, double lofreq, double hifreq, int64_t lobin, int64_t blocksize,
                    double threshold, int32_t exact_all, cs_candidate* out, int64_t cap, int64_t* n_out) {
    return cs_search_range(H, lofreq, hifreq, lobin, blocksize, threshold, exact_all, 0, -1, out, cap, n_out);
}

cs_status cs_set_metricstats(cs_handle* H, int32_t enable, double hist_lo, double hist_hi, int32_t hist_nb,
                             int32_t nwin) {
    if (!H) return CS_ERR_INVALID_ARGUMENT;
    if (enable) {
        // MetricHistogram's checks (src/search.jl:1397-1398) plus a bounded size
        if (!(hist_hi > hist_lo)) return fail(H, CS_ERR_INVALID_ARGUMENT, "histogram hi must exceed lo");
        if (hist_nb < 1 || hist_nb > (1 << 20)) return fail(H, CS_ERR_INVALID_ARGUMENT, "histogram bin count must be >= 1");
        if (nwin < 1 || nwin > 4096) return fail(H, CS_ERR_INVALID_ARGUMENT, "window count must be 1..4096");
        H->ms_lo = hist_lo;
        H->ms_hi = hist_hi;
        H->ms_nb = hist_nb;
        H->ms_nwin = nwin;
    }
    H->ms_on = enable != 0;
    return CS_OK;
}

cs_status cs_get_block_stats(const cs_handle* H, cs_block_stats* out, int64_t cap, int64_t* n_out) {
    if (!H || !n_out) return CS_ERR_INVALID_ARGUMENT;
    const int64_t n = (int64_t)H->ms_blocks.size();
    *n_out = n;
    if (cap < n) return CS_ERR_CAPACITY;
    if (out) std::copy(H->ms_blocks.begin(), H->ms_blocks.end(), out);
    return CS_OK;
}

cs_status cs_get_metric_hists(const cs_handle* H, int32_t* nlev, int32_t* nwin, int32_t* nb, int32_t* ks,
                              double* edges, int64_t* counts, double* moments) {
    if (!H || !nlev || !nwin || !nb) return CS_ERR_INVALID_ARGUMENT;
    const int L = H->ms_nlev, W = H->ms_nwin, B = H->ms_nb;
    *nlev = L;
    *nwin = W;
    *nb = B;
    if (H->ms_counts.size() != (size_t)L * W * B) {   // no statistics collected yet
        *nlev = 0;
        return CS_OK;
    }
    // levels in ascending k (the reference sorts its histograms by k)
    std::vector<int> order(L);
    for (int l = 0; l < L; ++l) order[l] = l;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return H->dlev[x].k < H->dlev[y].k; });
    for (int i = 0; i < L; ++i) {
        const int l = order[i];
        if (ks) ks[i] = H->dlev[l].k;
        if (edges) std::copy_n(&H->ms_edges[(size_t)l * (W + 1)], W + 1, edges + (size_t)i * (W + 1));
        if (counts) std::copy_n(&H->ms_counts[(size_t)l * W * B], (size_t)W * B, counts + (size_t)i * W * B);
        if (moments) std::copy_n(&H->ms_mom[(size_t)l * W * 7], (size_t)W * 7, moments + (size_t)i * W * 7);
    }
    return CS_OK;
}

cs_status cs_set_metricnorm(cs_handle* H, int32_t nlev, int32_t nwin, const int32_t* ks, const double* edges,
                            const double* loc, const double* scale) {
    if (!H) return CS_ERR_INVALID_ARGUMENT;
    if (nlev == 0) {
        H->norm_on = false;
        return CS_OK;
    }
    if (nlev < 0 || nwin < 1 || !ks || !edges || !loc || !scale)
        return fail(H, CS_ERR_INVALID_ARGUMENT, "normalisation needs ks, edges, loc and scale");
    const int L = (int)H->dlev.size();
    std::vector<double> e((size_t)L * (nwin + 1)), lc((size_t)L * nwin), sc((size_t)L * nwin);
    for (int l = 0; l < L; ++l) {
        int src = -1;
        for (int i = 0; i < nlev; ++i)
            if (ks[i] == H->dlev[l].k) src = i;
        if (src < 0) return fail(H, CS_ERR_INVALID_ARGUMENT, "normalisation lacks a decimation factor of the search");
        std::copy_n(edges + (size_t)src * (nwin + 1), nwin + 1, &e[(size_t)l * (nwin + 1)]);
        std::copy_n(loc + (size_t)src * nwin, nwin, &lc[(size_t)l * nwin]);
        std::copy_n(scale + (size_t)src * nwin, nwin, &sc[(size_t)l * nwin]);
    }
    H->norm_edges.swap(e);
    H->norm_loc.swap(lc);
    H->norm_scale.swap(sc);
    H->norm_nwin = nwin;
    H->norm_on = true;
    return CS_OK;
}

cs_status cs_search_stats(const cs_handle* H, cs_stats* out) {
    if (!H || !out) return CS_ERR_INVALID_ARGUMENT;
    *out = H->stats;
    return CS_OK;
}

cs_status cs_chunk_metrics(cs_handle* H, double rstart, int64_t n, double* out) {
    if (!H || !out || n < 1 || n > (1 << 16)) return CS_ERR_INVALID_ARGUMENT;
    // a NaN, infinite or negative start has no bin (floor() of it is undefined as an integer)
    if (!(rstart >= 0.0 && std::isfinite(rstart))) return fail(H, CS_ERR_INVALID_ARGUMENT, "rstart must be finite and >= 0");
    if (!H->has_spec) return fail(H, CS_ERR_NO_SPECTRUM, "no spectrum attached");
    CS_CUDA(cudaSetDevice(H->device), "set device");
    RunSpec R{};
    R.r_lo = rstart;
    R.lodr = H->p.hidr / (double)H->p.nharms;
    R.Nprof = (int)n;
    R.nblocks = 1;
    R.t_base = 0;
    R.t_end = n;
    R.nlev = 1;
    R.exact_all = true;
    R.threshold = INFINITY;
    R.medcut = -INFINITY;
    R.keep_diag = true;
    cs_status st = run_blocks(H, R, nullptr, nullptr);
    if (st != CS_OK) return st;
    for (int64_t j = 0; j < n; ++j) out[j] = (double)H->last_tmetric[j];
    return CS_OK;
}

cs_status cs_block_metrics(cs_handle* H, const double* rfund, int64_t L, int32_t kernel, const int32_t* widths,
                           int32_t nw, double* out) {
    if (!H || !rfund || !out || L < 1 || L > (1 << 22)) return CS_ERR_INVALID_ARGUMENT;
    if (kernel != 0 && kernel != 1) return fail(H, CS_ERR_INVALID_ARGUMENT, "kernel must be :fft (0) or :direct (1)");
    if (!H->has_spec) return fail(H, CS_ERR_NO_SPECTRUM, "no spectrum attached");
    const cs_params& p = H->p;
    const int nh = p.nharms, m = p.m, m2 = p.m / 2, nb = p.numbetween, nbins = 2 * p.nharms;
    if (nb < 1) return fail(H, CS_ERR_INVALID_ARGUMENT, "numbetween must be >= 1");
    if (nbins > kMaxBins) return fail(H, CS_ERR_UNSUPPORTED, "nharms > 128 is not built");
    for (int64_t j = 0; j < L; ++j)
        if (!(rfund[j] >= 0.0)) return fail(H, CS_ERR_INVALID_ARGUMENT, "r must be non-negative");
    std::vector<int> ws;
    if (widths && nw > 0) {
        ws.assign(widths, widths + nw);
        for (int i = 0; i < nw; ++i)
            if (ws[i] < 1 || ws[i] > kMaxBins || (i > 0 && ws[i] <= ws[i - 1]))
                return fail(H, CS_ERR_INVALID_ARGUMENT, "widths must ascend within 1..256");
    } else {
        ws = ladder_widths(nbins, 1, p);   // the base pass's bank (src/search.jl:1069-1070)
    }
    // reference_profiles' per-harmonic grid and guard (src/search.jl:1024-1034)
    std::vector<BmHarm> hm(nh);
    const int64_t Nhalf = H->N / 2;
    for (int h = 1; h <= nh; ++h) {
        const double rmin = rfund[0] * h, rmax = rfund[L - 1] * h;
        const int64_t lobin = (int64_t)std::floor(rmin);
        const int64_t hibin = (int64_t)std::ceil(rmax) + 1;
        const int64_t numbins = hibin - lobin;
        BmHarm& b = hm[h - 1];
        b.lobin = lobin;
        b.K = numbins * nb;
        b.ok = (lobin >= m2 && lobin + numbins + m2 <= H->namps && hibin < Nhalf) ? 1 : 0;
        b.pad = 0;
    }
    CS_CUDA(cudaSetDevice(H->device), "set device");
    CS_CUDA(H->d_bm_r.ensure((size_t)L * sizeof(double)), "alloc trials");
    CS_CUDA(H->d_bm_st.ensure((size_t)L * nh * sizeof(double2)), "alloc amplitudes");
    CS_CUDA(H->d_bm_prof.ensure((size_t)L * nbins * sizeof(double)), "alloc profiles");
    CS_CUDA(H->d_bm_out.ensure((size_t)L * sizeof(double)), "alloc metrics");
    CS_CUDA(H->d_bm_sig.ensure(sizeof(double)), "alloc sigma");
    CS_CUDA(cudaMemcpyAsync(H->d_bm_r.p, rfund, (size_t)L * sizeof(double), cudaMemcpyHostToDevice, H->stream),
            "copy trials");
    CS_CUDA(upload(H->d_bm_h, hm, H->stream), "copy harmonic grid");
    CS_CUDA(spec_ready(H), "wait for the spectrum");
    CS_CUDA(upload(H->d_bm_w, ws, H->stream), "copy widths");
    CS_CUDA(run_block_metrics(H->d_bm_r.as<double>(), (int)L, H->d_bm_h.as<BmHarm>(), nh, m, nb, kernel, H->amps,
                              H->namps, H->d_bm_st.as<double2>(), H->d_bm_prof.as<double>(), H->d_bm_w.as<int>(),
                              (int)ws.size(), H->d_bm_sig.as<double>(), H->d_bm_out.as<double>(), H->stream),
            "block metrics launch");
    CS_CUDA(cudaMemcpyAsync(out, H->d_bm_out.p, (size_t)L * sizeof(double), cudaMemcpyDeviceToHost, H->stream),
            "read metrics");
    CS_CUDA(cudaStreamSynchronize(H->stream), "block metrics");
    return CS_OK;
}

cs_status cs_refold(cs_handle* H, const double* r, const int32_t* nharm, int64_t n, int32_t m, int32_t* Hout,
                    double* profiles, double* ducy) {
    if (!H || !r || !nharm || !Hout || !ducy || n < 0 || n > (1 << 24)) return CS_ERR_INVALID_ARGUMENT;
    if (m < 2 || (m % 2) != 0) return fail(H, CS_ERR_INVALID_ARGUMENT, "m must be even");
    if (!H->has_spec) return fail(H, CS_ERR_NO_SPECTRUM, "no spectrum attached");
    const int maxh = 512;   // the kernel's kRefoldMaxH
    for (int64_t i = 0; i < n; ++i)
        if (nharm[i] > maxh) return fail(H, CS_ERR_UNSUPPORTED, "nharm above 512 is not built");
    if (n == 0) return CS_OK;
    CS_CUDA(cudaSetDevice(H->device), "set device");
    CS_CUDA(H->d_bm_r.ensure((size_t)n * sizeof(double)), "alloc candidates");
    CS_CUDA(H->d_bm_w.ensure((size_t)n * sizeof(int32_t) * 2), "alloc harmonics");
    CS_CUDA(H->d_bm_out.ensure((size_t)n * sizeof(double)), "alloc duty cycles");
    if (profiles) CS_CUDA(H->d_bm_prof.ensure((size_t)n * 2 * maxh * sizeof(double)), "alloc profiles");
    int32_t* d_nh = H->d_bm_w.as<int32_t>();
    int32_t* d_H = d_nh + n;
    CS_CUDA(cudaMemcpyAsync(H->d_bm_r.p, r, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, H->stream), "copy r");
    CS_CUDA(cudaMemcpyAsync(d_nh, nharm, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice, H->stream),
            "copy nharm");
    CS_CUDA(spec_ready(H), "wait for the spectrum");
    CS_CUDA(run_refold(H->d_bm_r.as<double>(), d_nh, (int)n, m, H->p.boxcar_fsp, H->p.boxcar_maxfrac, H->amps,
                       H->namps, H->N / 2, maxh, profiles ? H->d_bm_prof.as<double>() : nullptr, d_H,
                       H->d_bm_out.as<double>(), H->stream),
            "refold launch");
    CS_CUDA(cudaMemcpyAsync(Hout, d_H, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, H->stream), "read H");
    CS_CUDA(cudaMemcpyAsync(ducy, H->d_bm_out.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, H->stream),
            "read duty cycles");
    if (profiles)
        CS_CUDA(cudaMemcpyAsync(profiles, H->d_bm_prof.p, (size_t)n * 2 * maxh * sizeof(double),
                                cudaMemcpyDeviceToHost, H->stream),
                "read profiles");
    CS_CUDA(cudaStreamSynchronize(H->stream), "refold");
    return CS_OK;
}

cs_status cs_interp_chunk(cs_handle* H, double r_lo, int64_t t0, int64_t n, float* out) {
    if (!H || !out || n < 1 || n > (1 << 16) || t0 < 0) return CS_ERR_INVALID_ARGUMENT;
    if (!(r_lo >= 0.0 && std::isfinite(r_lo))) return fail(H, CS_ERR_INVALID_ARGUMENT, "r_lo must be finite and >= 0");
    if (!H->has_spec) return fail(H, CS_ERR_NO_SPECTRUM, "no spectrum attached");
    CS_CUDA(cudaSetDevice(H->device), "set device");
    RunSpec R{};
    R.r_lo = r_lo;
    R.lodr = H->p.hidr / (double)H->p.nharms;
    R.Nprof = (int)n;
    R.nblocks = 1;
    R.t_base = t0;
    R.t_end = t0 + n;
    R.nlev = 1;
    R.interp_only = true;
    return run_blocks(H, R, nullptr, reinterpret_cast<float2*>(out));
}

cs_status cs_search_block_values(const cs_handle* H, float* sigma, int32_t* nvalid, int64_t cap,
                                 int64_t* n_out) {
    if (!H || !n_out) return CS_ERR_INVALID_ARGUMENT;
    const int64_t n = (int64_t)H->last_sigma.size();
    *n_out = n;
    if (cap < n) return CS_ERR_CAPACITY;
    if (sigma) std::copy(H->last_sigma.begin(), H->last_sigma.end(), sigma);
    if (nvalid) std::copy(H->last_nvalid.begin(), H->last_nvalid.end(), nvalid);
    return CS_OK;
}

cs_status cs_autotune(cs_handle* H, double lofreq, double hifreq, int64_t lobin, int64_t blocksize, int64_t nsample,
                      cs_tune_report* out) {
    if (!H || nsample < 1 || blocksize < 1) return CS_ERR_INVALID_ARGUMENT;
    if (!H->has_spec) return fail(H, CS_ERR_NO_SPECTRUM, "no spectrum attached");
    CS_CUDA(cudaSetDevice(H->device), "set device");
    RunSpec R{};
    bool empty = true;
    cs_status st = setup_run(H, lofreq, hifreq, lobin, blocksize, H->p.threshold, 0, 0, -1, nullptr, 0, R, &empty);
    if (st != CS_OK) return st;
    if (empty) return fail(H, CS_ERR_INVALID_ARGUMENT, "the band holds no trials");
    const int64_t ns = std::min(nsample, R.nblocks);
    const int64_t b0 = (R.nblocks - ns) / 2;
    // the sample is searched plainly: no statistics, normalisation or diagnostics
    const bool ms_on = H->ms_on, norm_on = H->norm_on;
    const int diag = H->diag;
    H->ms_on = H->norm_on = false;
    H->diag = 0;
    // stage times of one configuration: the least of 3 runs after a warm-up
    auto timed = [&](double* ms_i, double* ms_s) -> cs_status {
        std::vector<cs_candidate> c;
        double bi = 1e300, bs = 1e300, bg = 1e300;
        for (int r = 0; r < 4; ++r) {
            c.clear();
            const cs_status e = search_core(H, lofreq, hifreq, lobin, blocksize, H->p.threshold, 0, b0, b0 + ns, &c);
            if (e != CS_OK) return e;
            if (r > 0) {
                bi = std::min(bi, H->stats.ms_interp);
                bs = std::min(bs, H->stats.ms_synth);
                bg = std::min(bg, H->stats.ms_sigma);
            }
        }
        H->stats_sigma_min = bg;
        *ms_i = bi;
        *ms_s = bs;
        return CS_OK;
    };
    cs_tune_report rep{};
    rep.sample_blocks = ns;
    rep.ms_interp[0] = rep.ms_interp[1] = -1.0;
    const bool tensor = H->p.synth != CS_SYNTH_FP32;
    double msi = 0.0, mss = 0.0;
    // 1. the interpolation kernel
    H->tune_interp = 1;
    H->tune_div[0] = H->tune_div[1] = 0;
    H->tune_dbuf = 1;
    if (tensor) st = build_tc(H);
    if (st == CS_OK) st = timed(&msi, &mss);
    if (st == CS_OK && H->interp2_ok) rep.ms_interp[1] = msi;
    double ms_model = mss;
    if (st == CS_OK) {
        H->tune_interp = 0;
        st = timed(&msi, &mss);
        rep.ms_interp[0] = msi;
    }
    if (st == CS_OK) H->tune_interp = (rep.ms_interp[1] >= 0.0 && rep.ms_interp[1] < rep.ms_interp[0]) ? 1 : 0;
    // 2. the block-sigma kernel
    rep.ms_sigma[0] = rep.ms_sigma[1] = -1.0;
    for (int v = 0; v < 2 && st == CS_OK; ++v) {
        H->tune_sigma = v;
        double a_ = 0.0, b_ = 0.0;
        st = timed(&a_, &b_);
        rep.ms_sigma[v] = H->stats_sigma_min;
    }
    if (st == CS_OK) H->tune_sigma = rep.ms_sigma[1] < rep.ms_sigma[0] ? 1 : 0;
    // 3. tensor epilogue: the form (one slot, phased double buffer, split) and
    // each phase's segment divisor
    if (st == CS_OK && tensor) {
        int best[3] = {0, 0, 1};   // div0, div1, dbuf
        double best_ms = ms_model;
        auto trial = [&](int d0, int d1, int db, double* ms) -> cs_status {
            if (ms) *ms = 1e300;
            H->tune_div[0] = d0;
            H->tune_div[1] = d1;
            H->tune_dbuf = db;
            if (build_tc(H) != CS_OK) return CS_OK;   // this shape does not fit: skip it
            double a = 0.0, b = 0.0;
            const cs_status e = timed(&a, &b);
            if (e != CS_OK) return e;
            if (ms) *ms = b;
            if (b < best_ms) {
                best_ms = b;
                best[0] = d0;
                best[1] = d1;
                best[2] = db;
            }
            return CS_OK;
        };
        // Per epilogue form (one slot; base level double-buffered and scanned
        // after the decimated levels; split between warpgroup pairs): the
        // divisor of phase 0 first, then, with the base level in a phase of
        // its own, the divisor of phase 1 (each form weighs its segments
        // differently, so none borrows another's).
        const int divs[] = {2, 3, 4, 5, 6, 8, 10, 12, 16};
        for (int db = 0; db < 3 && st == CS_OK; ++db) {
            int bd0 = 2;
            double bms = 1e300;
            if (db == 0 || H->dlev.size() > 1)
                for (int d : divs) {
                    double ms = 0.0;
                    if (st == CS_OK) st = trial(d, 2, db, &ms);
                    if (ms < bms) {
                        bms = ms;
                        bd0 = d;
                    }
                }
            if (db > 0)
                for (int d : divs)
                    if (st == CS_OK) st = trial(bd0, d, db, nullptr);
        }
        H->tune_div[0] = best[0];
        H->tune_div[1] = best[1];
        H->tune_dbuf = best[2];
        const cs_status e = build_tc(H);
        if (st == CS_OK) st = e;
        rep.ms_synth_model = ms_model;
        rep.ms_synth_tuned = best_ms;
    } else {
        rep.ms_synth_model = rep.ms_synth_tuned = mss;
    }
    H->ms_on = ms_on;
    H->norm_on = norm_on;
    H->diag = diag;
    if (st != CS_OK) return st;
    rep.interp_kernel = H->tune_interp;
    rep.sigma_kernel = H->tune_sigma;
    rep.tc_double_buffer = tensor ? H->tc.args.dbuf : 0;
    rep.tc_div[0] = tensor ? H->tune_div[0] : 0;
    rep.tc_div[1] = tensor ? H->tune_div[1] : 0;
    rep.nlev = (int32_t)H->dlev.size();
    for (int l = 0; l < rep.nlev && l < CS_MAX_DECIM; ++l) {
        rep.nbins[l] = H->dlev[l].nbins;
        rep.units[l] = tensor ? H->tc.args.lev[l].nunits : 0;
    }
    tune_store({H->device, H->p, H->tune_interp, H->tune_div[0], H->tune_div[1], H->tune_dbuf, H->tune_sigma});
    if (out) *out = rep;
    return CS_OK;
}

cs_status cs_set_launch_shapes(cs_handle* H, const cs_tune_report* sh) {
    if (!H || !sh) return CS_ERR_INVALID_ARGUMENT;
    auto div_ok = [](int d) { return d == 0 || d == 2 || d == 3 || d == 4 || d == 5 || d == 6 || d == 8 || d == 10 ||
                                     d == 12 || d == 16; };
    if ((sh->interp_kernel != 0 && sh->interp_kernel != 1) || (sh->sigma_kernel != 0 && sh->sigma_kernel != 1) ||
        sh->tc_double_buffer < 0 || sh->tc_double_buffer > 2 || !div_ok(sh->tc_div[0]) || !div_ok(sh->tc_div[1]))
        return fail(H, CS_ERR_INVALID_ARGUMENT, "launch shapes out of range");
    CS_CUDA(cudaSetDevice(H->device), "set device");
    H->tune_interp = sh->interp_kernel;
    H->tune_sigma = sh->sigma_kernel;
    H->tune_dbuf = sh->tc_double_buffer;
    H->tune_div[0] = sh->tc_div[0];
    H->tune_div[1] = sh->tc_div[1];
    H->graph_valid = false;
    return H->p.synth != CS_SYNTH_FP32 ? build_tc(H) : CS_OK;
}

cs_status cs_set_memory_limit(cs_handle* H, int64_t bytes) {
    if (!H || bytes < 0) return CS_ERR_INVALID_ARGUMENT;
    CS_CUDA(cudaSetDevice(H->device), "set device");
    CS_CUDA(cudaStreamSynchronize(H->stream), "drain");
    H->mem_limit = (size_t)bytes;
    // the wave buffers come back at the size the cap allows
    for (DBuf* b : {&H->d_X, &H->d_A, &H->d_samp, &H->d_Q0, &H->d_items, &H->d_cands, &H->d_tmetric, &H->d_sigma,
                    &H->d_nvalid})
        b->release();
    H->graph_valid = false;
    return CS_OK;
}

cs_status cs_set_wait_test(cs_handle* H, int64_t wait_ns) {
    if (!H || wait_ns < 0) return CS_ERR_INVALID_ARGUMENT;
    H->stall_ns = wait_ns;
    H->graph_valid = false;   // a captured graph holds the old kernel arguments
    return CS_OK;
}

cs_status cs_set_diagnostics(cs_handle* H, int32_t level) {
    if (!H || level < 0 || level > 2) return CS_ERR_INVALID_ARGUMENT;
    H->diag = level;
    return CS_OK;
}

cs_status cs_search_gate_values(const cs_handle* H, float* out, int64_t cap, int64_t* n_out) {
    if (!H || !n_out) return CS_ERR_INVALID_ARGUMENT;
    const int64_t n = (int64_t)H->last_gate.size();
    *n_out = n;
    if (cap < n) return CS_ERR_CAPACITY;
    if (out) std::copy(H->last_gate.begin(), H->last_gate.end(), out);
    return CS_OK;
}

cs_status cs_search_trial_metrics(const cs_handle* H, float* out, int64_t cap, int64_t* n_out) {
    if (!H || !n_out) return CS_ERR_INVALID_ARGUMENT;
    const int64_t n = (int64_t)H->last_tmetric.size();
    *n_out = n;
    if (cap < n) return CS_ERR_CAPACITY;
    if (out) std::copy(H->last_tmetric.begin(), H->last_tmetric.end(), out);
    return CS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Chunk metrics without device allocation (cs_chunk_metrics_static).
//
// Some callers are not allowed to call cudaMalloc or cudaFree: a plugin loaded
// into a host pipeline that reserved the device memory for itself at start-up
// and hands out only fixed buffers, or a runtime whose own pooling allocator
// must see every allocation.  cudaFree also synchronises the device, which a
// latency-bound caller cannot afford.  For them the chunk-metrics path keeps
// its scratch -- counters, the level and plan tables and the sigma samples --
// in one file-scope device array of fixed size.
// The caller passes its spectrum and the output as device pointers.

namespace {
constexpr size_t kStaticScratchBytes = (size_t)4 << 20;  // 4 MiB on every device
constexpr int kStaticMaxDevices = 64;
}  // namespace

// Loaded with the library on every GPU it is used on and held until the
// process exits.  In host code this name is a stand-in for the symbol, not a
// device address: the address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

namespace {

std::mutex g_static_mu[kStaticMaxDevices];
void* g_static_base[kStaticMaxDevices];  // device address of g_static_scratch, per device

cs_status static_fail(char* err, int64_t cap, cs_status st, const char* fmt, ...) {
    if (err && cap > 0) {
        va_list ap;
        va_start(ap, fmt);
        std::vsnprintf(err, (size_t)cap, fmt, ap);
        va_end(ap);
    }
    return st;
}

size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" cs_status cs_chunk_metrics_static(const cs_params* params, const float* d_amps, int64_t namps,
                                             int64_t N, double rstart, int64_t n, float* d_out, void* stream,
                                             char* err, int64_t err_cap) {
    if (err && err_cap > 0) err[0] = '\0';
    if (validate(params) != CS_OK)
        return static_fail(err, err_cap, CS_ERR_INVALID_ARGUMENT, "invalid search parameters");
    if (!d_amps || !d_out || namps < 1 || N < 2 || n < 1 || n > (1 << 16))
        return static_fail(err, err_cap, CS_ERR_INVALID_ARGUMENT,
                           "needs device spectrum and output, namps >= 1, N >= 2 and 1 <= n <= 65536");
    if ((reinterpret_cast<uintptr_t>(d_amps) & 7u) != 0 || (reinterpret_cast<uintptr_t>(d_out) & 3u) != 0)
        return static_fail(err, err_cap, CS_ERR_INVALID_ARGUMENT,
                           "spectrum must be 8-byte and output 4-byte aligned");
    if (!(rstart >= 0.0 && std::isfinite(rstart)))
        return static_fail(err, err_cap, CS_ERR_INVALID_ARGUMENT, "rstart must be finite and >= 0");
    const cs_params& p = *params;

    // The base fold (k = 1) only, as cs_chunk_metrics evaluates it.
    DevLevel L{};
    L.k = 1;
    L.Hk = p.nharms;
    L.nbins = 2 * p.nharms;
    const std::vector<int> widths = ladder_widths(L.nbins, 1, p);
    if (L.nbins > kMaxBins || (int)widths.size() > kMaxWidths || widths.back() > kMaxBins)
        return static_fail(err, err_cap, CS_ERR_UNSUPPORTED,
                           "needs nharms <= 128, <= 64 boxcar widths, widths <= 256 bins");
    L.nw = (int)widths.size();
    L.wmax = widths.back();
    L.np = ((L.Hk + 1) + 7) / 8 * 8;
    L.tw_off = 0;
    for (int i = 0; i < L.nw; ++i) {
        L.widths[i] = widths[i];
        L.rsqrtw[i] = (float)(1.0 / std::sqrt((double)widths[i]));
    }
    std::vector<float> tw(2 * (size_t)L.Hk * L.np, 0.0f);
    for (int j = 1; j < L.Hk; ++j)
        for (int k = 0; k <= L.Hk; ++k) {
            const double ang = 2.0 * M_PI * (double)(((int64_t)j * k) % L.nbins) / (double)L.nbins;
            tw[(size_t)j * L.np + k] = (float)(2.0 * std::cos(ang));
            tw[((size_t)L.Hk + j) * L.np + k] = (float)(-2.0 * std::sin(ang));
        }
    HostPlans plans;
    build_plans(p, rstart, plans);
    for (const DevHarm& d : plans.harms)
        if ((double)n * (double)d.h * (double)d.pnum > 4.6e18)
            return static_fail(err, err_cap, CS_ERR_UNSUPPORTED,
                               "trial index times harmonic overflows 64-bit phase state");
    const int Nprof = (int)n;
    const int win_max = (int)std::ceil((double)(Nprof - 1 + 64) * p.hidr) + p.m + 4;
    if (interp_smem(win_max, Nprof) > 200 * 1024)
        return static_fail(err, err_cap, CS_ERR_UNSUPPORTED,
                           "chunk too long for the shared-memory interpolation row");
    if (sigma_smem(L.Hk, L.np) + 16 * 1024 > 227 * 1024)
        return static_fail(err, err_cap, CS_ERR_UNSUPPORTED, "sigma working set exceeds shared memory");

    // Scratch layout, every piece on a 256-byte boundary.
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = up256(off + bytes);
        return o;
    };
    const size_t o_cnt = take(4 * sizeof(int32_t));
    const size_t o_lev = take(sizeof(DevLevel));
    const size_t o_tw = take(tw.size() * sizeof(float));
    const size_t o_harms = take(plans.harms.size() * sizeof(DevHarm));
    const size_t o_w = take(plans.w.size() * sizeof(float));
    const size_t o_a = take(plans.a.size() * sizeof(float2));
    const size_t o_c = take(plans.c.size());
    const size_t o_nv = take(sizeof(int32_t));
    const size_t o_sig = take(sizeof(float));
    const size_t o_samp = take((size_t)kSampStride * sizeof(float2));
    if (off > kStaticScratchBytes)
        return static_fail(err, err_cap, CS_ERR_CAPACITY,
                           "plan tables need %zu bytes of scratch; the static scratch holds %zu (4 MiB): "
                           "lower nharms or m, or use a trial grid with a smaller denominator",
                           off, kStaticScratchBytes);

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return static_fail(err, err_cap, CS_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kStaticMaxDevices)
        return static_fail(err, err_cap, CS_ERR_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_static_mu[dev]);
    if (!g_static_base[dev]) {
        // Once per device, with that device current.
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr)
            return static_fail(err, err_cap, CS_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_static_base[dev] = ptr;
    }
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
    uint8_t* base = static_cast<uint8_t*>(g_static_base[dev]);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int32_t nvalid = Nprof;
    // Every failed step waits for the stream before the lock is released: work
    // already queued must not run on the shared array under the next caller.
#define CS_STATIC_CUDA(call, where)                                                                  \
    do {                                                                                             \
        const cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                                     \
            (void)cudaStreamSynchronize(st);                                                         \
            return static_fail(err, err_cap, CS_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e_)); \
        }                                                                                            \
    } while (0)
    auto put = [&](size_t o, const void* src, size_t bytes) {
        return bytes ? cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, st) : cudaSuccess;
    };
    // The counters must start at zero; every other region is fully rewritten.
    CS_STATIC_CUDA(cudaMemsetAsync(base + o_cnt, 0, 4 * sizeof(int32_t), st), "clear counters");
    CS_STATIC_CUDA(put(o_lev, &L, sizeof(DevLevel)), "copy level");
    CS_STATIC_CUDA(put(o_tw, tw.data(), tw.size() * sizeof(float)), "copy twiddles");
    CS_STATIC_CUDA(put(o_harms, plans.harms.data(), plans.harms.size() * sizeof(DevHarm)), "copy plans");
    CS_STATIC_CUDA(put(o_w, plans.w.data(), plans.w.size() * sizeof(float)), "copy weights");
    CS_STATIC_CUDA(put(o_a, plans.a.data(), plans.a.size() * sizeof(float2)), "copy phases");
    CS_STATIC_CUDA(put(o_c, plans.c.data(), plans.c.size()), "copy carries");
    CS_STATIC_CUDA(put(o_nv, &nvalid, sizeof(int32_t)), "copy valid count");

    int32_t* cnt = reinterpret_cast<int32_t*>(base + o_cnt);
    WaveArgs a{};
    a.amps = reinterpret_cast<const float2*>(d_amps);
    a.namps = namps;
    a.Nhalf = N / 2;
    a.nharms = p.nharms;
    a.m = p.m;
    a.nlev = 1;
    a.Nprof = Nprof;
    a.t_first = 0;
    a.total = n;
    a.nblk = 1;
    a.blk_base = 0;
    a.harms = reinterpret_cast<const DevHarm*>(base + o_harms);
    a.wtab = reinterpret_cast<const float*>(base + o_w);
    a.atab = reinterpret_cast<const float2*>(base + o_a);
    a.ctab = base + o_c;
    a.levels = reinterpret_cast<const DevLevel*>(base + o_lev);
    a.tw = reinterpret_cast<const float*>(base + o_tw);
    a.nvalid = reinterpret_cast<int32_t*>(base + o_nv);
    a.X = nullptr;  // the amplitude rows are not kept: sigma reads the samples,
    a.Atile = nullptr;  // the metric kernel recomputes each trial's amplitudes
    a.tiles_per_blk = (Nprof + 127) / 128;
    a.fp16 = 0;
    a.samp = reinterpret_cast<float2*>(base + o_samp);
    a.Q0 = nullptr;  // no gate: every trial gets the exact metric
    a.sigma = reinterpret_cast<float*>(base + o_sig);
    a.tmetric = d_out;
    a.items = nullptr;
    a.n_items = cnt;
    a.cap_items = 0;
    a.cands = nullptr;
    a.n_cands = cnt + 1;
    a.cap_cands = 0;
    a.threshold = INFINITY;
    a.medcut = -INFINITY;
    a.medcut_gate = -INFINITY;
    a.verify_gate = 0;
    a.exact_all = 1;
    CS_STATIC_CUDA(launch_interp(a, st, win_max, cnt + 2), "interp launch");
    CS_STATIC_CUDA(launch_sigma(a, st, L.Hk, L.np, cnt + 2), "sigma launch");
    CS_STATIC_CUDA(launch_rescue(a, st, sms), "metric launch");
    int32_t counts[4] = {0, 0, 0, 0};
    CS_STATIC_CUDA(cudaMemcpyAsync(counts, cnt, sizeof(counts), cudaMemcpyDeviceToHost, st), "read counters");
    CS_STATIC_CUDA(cudaStreamSynchronize(st), "chunk");
#undef CS_STATIC_CUDA
    if (counts[2] == 1) return static_fail(err, err_cap, CS_ERR_CUDA, "interpolation window exceeded its bound");
    if (counts[2] == 3) return static_fail(err, err_cap, CS_ERR_TIMEOUT, "sigma sample copy wait ran out");
    return CS_OK;
}
