/*
 * cs_cpu.c -- CPU oracle of the coherent-search hot path.  TEST
 * INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg as the checker and the timed CPU restatement; the product
 * never links it.
 *
 * A C restatement of CoherentSearch.jl's production search path with the
 * reference's arithmetic:
 *   - build_direct_plans with Float32 weights (src/directinterp.jl:342-405):
 *     FP64 tables rounded once;
 *   - fill_harmonic_row_direct! (src/directinterp.jl:470-572): residue state
 *     by exact 128-bit divrem (direct_chunk_state, :414-418), phase row lookup,
 *     range guard on the true trial range, sequential FP32 fmaf over the m taps,
 *     unfused Complex{Float32} product;
 *   - _fill_row_direct_slow! (:623-661) for a non-rational trial step.
 * Built with -ffp-contract=off so only the explicit fma calls fuse.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int h, m, P;
    int64_t q, s, base_adv, pnum, rfloor0;
    double dr0;
    int32_t* row;   /* q entries: residue -> phase row */
    float* W;       /* P x m, row-major [p][i] as the reference's (m, P) column-major */
    float* A;       /* P complex (re, im) */
    uint8_t* carry; /* P */
} plan_t;

static int64_t gcd64(int64_t a, int64_t b) {
    while (b) { int64_t t = a % b; a = b; b = t; }
    return a < 0 ? -a : a;
}

/* sin(pi x), cos(pi x) for x in [0, 1). */
static double sinpi_d(double x) {
    if (x <= 0.25) return sin(M_PI * x);
    if (x <= 0.75) return cos(M_PI * (x - 0.5));
    return sin(M_PI * (1.0 - x));
}
static double cospi_d(double x) {
    if (x <= 0.25) return cos(M_PI * x);
    if (x <= 0.75) return -sin(M_PI * (x - 0.5));
    return -cos(M_PI * (1.0 - x));
}

/* trial_grid_rational (src/directinterp.jl:217-225). */
static int trial_grid_rational(double lodr, int64_t* pnum, int64_t* q) {
    if (!(lodr > 0)) return 0;
    double eps8 = 8.0 * (nextafter(lodr, INFINITY) - lodr);
    for (int64_t qq = 1; qq <= 65536; ++qq) {
        double pp = nearbyint(lodr * (double)qq);
        if (pp >= 1 && fabs(pp / (double)qq - lodr) <= eps8) {
            int64_t g = gcd64((int64_t)pp, qq);
            *pnum = (int64_t)pp / g;
            *q = qq / g;
            return 1;
        }
    }
    return 0;
}

static void free_plans(plan_t* pl, int n) {
    for (int i = 0; i < n; ++i) {
        free(pl[i].row); free(pl[i].W); free(pl[i].A); free(pl[i].carry);
    }
    free(pl);
}

static plan_t* build_plans(int nharms, int m, double hidr, double r_lo) {
    double lodr = hidr / (double)nharms;
    int64_t pnum = 1, q = 1;
    int rq = trial_grid_rational(lodr, &pnum, &q);
    int m2 = m / 2;
    plan_t* pl = (plan_t*)calloc((size_t)nharms, sizeof(plan_t));
    for (int h = 1; h <= nharms; ++h) {
        plan_t* d = &pl[h - 1];
        double hr = (double)h * r_lo;
        d->h = h;
        d->m = m;
        d->rfloor0 = (int64_t)floor(hr);
        d->dr0 = hr - floor(hr);
        if (!rq) { d->P = 0; d->q = 1; d->pnum = 1; continue; }
        int64_t step = (int64_t)h * pnum;
        d->pnum = pnum;
        d->q = q;
        d->s = step % q;
        d->base_adv = step / q;
        d->P = (int)(q / gcd64(step, q));
        d->row = (int32_t*)malloc(sizeof(int32_t) * (size_t)q);
        for (int64_t i = 0; i < q; ++i) d->row[i] = -1;
        d->W = (float*)malloc(sizeof(float) * (size_t)d->P * m);
        d->A = (float*)malloc(sizeof(float) * 2 * (size_t)d->P);
        d->carry = (uint8_t*)malloc((size_t)d->P);
        int64_t res = 0;
        for (int p = 0; p < d->P; ++p) {
            d->row[res] = p;
            double u = d->dr0 + (double)res / (double)q;
            int c = u >= 1.0;
            double dr = c ? u - 1.0 : u;
            d->carry[p] = (uint8_t)c;
            if (dr == 0.0) {
                d->A[2 * p] = 1.0f; d->A[2 * p + 1] = 0.0f;
                for (int i = 0; i < m; ++i) d->W[(size_t)p * m + i] = (i == m2 - 1) ? 1.0f : 0.0f;
            } else {
                double sn = sinpi_d(dr), cs = cospi_d(dr);
                d->A[2 * p] = (float)((sn * cs) / M_PI);
                d->A[2 * p + 1] = (float)(-((sn * sn) / M_PI));
                for (int i = 0; i < m; ++i) d->W[(size_t)p * m + i] = (float)(1.0 / (dr - (double)(i + 1 - m2)));
            }
            res += d->s;
            if (res >= q) res -= q;
        }
    }
    return pl;
}

/* direct_chunk_state: (res, qint) = divrem(t*h*pnum, q), exact. */
static void chunk_state(const plan_t* d, int64_t t, int64_t* res, int64_t* qint) {
    __int128 T = (__int128)t * (__int128)(d->h * d->pnum);
    *res = (int64_t)(T % d->q);
    *qint = (int64_t)(T / d->q);
}

/* One harmonic row, trials t0 .. t0+n-1; out is n complex64 (zeros if guarded). */
static void fill_row(const plan_t* d, const float* amps, int64_t namps, int64_t N, double hidr,
                     int nharms, int64_t t0, int64_t n, float* out) {
    int m = d->m, m2 = m / 2;
    int64_t Nhalf = N / 2;
    memset(out, 0, sizeof(float) * 2 * (size_t)n);
    if (n < 1) return;
    if (d->P == 0) {
        /* _fill_row_direct_slow! */
        double lodr = hidr / (double)nharms;
        double hr_lo = (double)d->rfloor0 + d->dr0;
        double dh = (double)d->h * lodr;
        double rfirst = hr_lo + (double)t0 * dh;
        double rlast = hr_lo + (double)(t0 + n - 1) * dh;
        int64_t lo = (int64_t)floor(rfirst + 1e-15) + 2 - m2;
        int64_t hi = (int64_t)floor(rlast + 1e-15) + 1 + m2;
        if (!(lo >= 1 && hi <= namps && (int64_t)floor(rlast) < Nhalf)) return;
        for (int64_t k = 0; k < n; ++k) {
            double r = hr_lo + (double)(t0 + k) * dh;
            int64_t rint = (int64_t)floor(r + 1e-15) + 1;
            double dr = fmod(r, 1.0);
            int64_t base = rint - m2;
            if (dr == 0.0) {
                out[2 * k] = amps[2 * (base + m2 - 1)];
                out[2 * k + 1] = amps[2 * (base + m2 - 1) + 1];
                continue;
            }
            double sre = 0.0, sim = 0.0;
            for (int i = 0; i < m; ++i) {
                double w = 1.0 / (dr - (double)(i + 1 - m2));
                sre = fma(w, (double)amps[2 * (base + i)], sre);
                sim = fma(w, (double)amps[2 * (base + i) + 1], sim);
            }
            double sn = sinpi_d(dr), cs = cospi_d(dr);
            double ar = (sn * cs) / M_PI, ai = -((sn * sn) / M_PI);
            out[2 * k] = (float)(ar * sre - ai * sim);
            out[2 * k + 1] = (float)(ar * sim + ai * sre);
        }
        return;
    }
    int64_t res, qint, resl, qintl;
    chunk_state(d, t0, &res, &qint);
    chunk_state(d, t0 + n - 1, &resl, &qintl);
    int64_t lo_trial = d->rfloor0 + qint + d->carry[d->row[res]] + 2 - m2;          /* 1-based */
    int64_t hi_trial = d->rfloor0 + qintl + d->carry[d->row[resl]] + 1 + m2;
    if (!(lo_trial >= 1 && hi_trial <= namps && (d->rfloor0 + qintl) < Nhalf)) return;
    for (int64_t k = 0; k < n; ++k) {
        int64_t r_, qi;
        chunk_state(d, t0 + k, &r_, &qi);
        int p = d->row[r_];
        int64_t base = d->rfloor0 + qi + d->carry[p] + 1 - m2;  /* 0-based first tap */
        const float* w = d->W + (size_t)p * m;
        float sre = 0.0f, sim = 0.0f;
        for (int i = 0; i < m; ++i) {
            sre = fmaf(w[i], amps[2 * (base + i)], sre);
            sim = fmaf(w[i], amps[2 * (base + i) + 1], sim);
        }
        float ar = d->A[2 * p], ai = d->A[2 * p + 1];
        float pr0 = ar * sre, pr1 = ai * sim, pi0 = ar * sim, pi1 = ai * sre;
        out[2 * k] = pr0 - pr1;
        out[2 * k + 1] = pi0 + pi1;
    }
}

/* Amplitude stack of trials t0 .. t0+n-1 of a search anchored at r_lo:
 * out is (nharms, n) complex64, harmonic-major.  Returns 0. */
int csref_interp_chunk(const float* amps, int64_t namps, int64_t N, int nharms, int m, double hidr,
                       double r_lo, int64_t t0, int64_t n, float* out) {
    if (m < 2 || (m & 1) || nharms < 1 || n < 1) return -1;
    plan_t* pl = build_plans(nharms, m, hidr, r_lo);
    for (int h = 0; h < nharms; ++h)
        fill_row(&pl[h], amps, namps, N, hidr, nharms, t0, n, out + 2 * (size_t)h * n);
    free_plans(pl, nharms);
    return 0;
}

/* The phase-table values of harmonic h (1-based): W (P x m), A (P complex),
 * carry (P), for cross-checking table construction.  Returns P (0 for the
 * per-trial path) or -1; copies at most cap phases. */
int csref_plan_tables(int nharms, int m, double hidr, double r_lo, int h, float* W, float* A,
                      uint8_t* carry, int cap) {
    if (h < 1 || h > nharms) return -1;
    plan_t* pl = build_plans(nharms, m, hidr, r_lo);
    plan_t* d = &pl[h - 1];
    int P = d->P;
    int np = P < cap ? P : cap;
    if (W) memcpy(W, d->W, sizeof(float) * (size_t)np * m);
    if (A) memcpy(A, d->A, sizeof(float) * 2 * (size_t)np);
    if (carry) memcpy(carry, d->carry, (size_t)np);
    free_plans(pl, nharms);
    return P;
}

/* ------------------------------------------------------------------------
 * Full production search over a range of blocks, multithreaded: the timed
 * CPU restatement of `_search_region!` (src/search.jl:1768-1894) with the
 * default profile precision :f64.  Per block: Float32-weight interpolation
 * (fill_row above), the FP64 c2r transform of every level (direct symmetric
 * DFT, vectorised across the block's profiles), the block sigma
 * (src/search.jl:490-566), the batched Float32 zero-baseline gate over
 * 128-profile tiles and the FP64 scalar gate for the tail (:784-807), the
 * exact median rescan of trials reaching medcut (:893-904), and candidate
 * emission (:1827-1838, :1695-1708).  Blocks go to threads round-robin, as
 * the reference's tasks take chunks (src/search.jl:1808-1859).
 * ------------------------------------------------------------------------ */
#include <pthread.h>
#include <time.h>

#define CS_MAXLEV 16
#define CS_MAXW 64
#define CS_BATCH 128
#define CS_SIGCAP 8192

typedef struct { int32_t blk, k, j; float pad; double metric; } cpu_cand_t;

typedef struct {
    const float* amps;
    int64_t namps, N;
    int nharms, m;
    double hidr, lodr, r_lo;
    int nlev, ks[CS_MAXLEV], Hk[CS_MAXLEV], nw[CS_MAXLEV], widths[CS_MAXLEV][CS_MAXW];
    double* C2[CS_MAXLEV];   /* (Hk) x (Hk+1): 2cos(2 pi j n / N) */
    double* S2[CS_MAXLEV];   /* -2 sin */
    int64_t total;
    int Nprof;
    int64_t first_block, nblocks;
    const int64_t* blist;   /* block indices to search (NULL: first_block ..) */
    double* sig_out;        /* [idx][level] block sigma, or NULL */
    int32_t* nv_out;        /* [idx][level] valid trials, or NULL */
    double threshold, medcut;
    plan_t* plans;
    int nthreads;
    cpu_cand_t* cands;
    int64_t cap;
    int64_t ncand;
    int64_t rescued;
    pthread_mutex_t mu;
} job_t;

typedef struct { job_t* job; int tid; } warg_t;

static void sel_swap(double* v, int a, int b) { double t = v[a]; v[a] = v[b]; v[b] = t; }

/* k-th smallest (0-based) of v[lo..hi] into v[k] (Lomuto quickselect). */
static void qselect(double* v, int lo, int hi, int k) {
    while (lo < hi) {
        int mid = lo + (hi - lo) / 2;
        if (v[mid] < v[lo]) sel_swap(v, mid, lo);
        if (v[hi] < v[lo]) sel_swap(v, hi, lo);
        if (v[mid] < v[hi]) sel_swap(v, mid, hi);
        double pivot = v[hi];
        int i = lo;
        for (int j = lo; j < hi; ++j)
            if (v[j] <= pivot) { sel_swap(v, i, j); ++i; }
        sel_swap(v, i, hi);
        if (i == k) return;
        if (i < k) lo = i + 1; else hi = i - 1;
    }
}

/* _median! (src/search.jl:295-305). */
static double median_d(double* v, int n) {
    int half = n >> 1;
    qselect(v, 0, n - 1, half);
    if (n & 1) return v[half];
    double upper = v[half], lower = v[0];
    for (int i = 1; i < half; ++i) if (v[i] > lower) lower = v[i];
    return 0.5 * (lower + upper);
}

static double exact_metric_d(const double* prof, int stride, int nbins, const int* ws, int nw,
                             double invsig, double* tmp, double* ps) {
    for (int i = 0; i < nbins; ++i) tmp[i] = prof[(size_t)i * stride];
    double med = median_d(tmp, nbins);
    int wmax = ws[nw - 1];
    ps[0] = 0.0;
    for (int i = 0; i < nbins + wmax; ++i) {
        int idx = i >= nbins ? i - nbins : i;
        ps[i + 1] = ps[i] + (prof[(size_t)idx * stride] - med);
    }
    double best = -INFINITY;
    for (int a = 0; a < nw; ++a) {
        int w = ws[a];
        double invsw = invsig / sqrt((double)w);
        double mm = ps[w] - ps[0];
        for (int p = 1; p < nbins; ++p) { double d = ps[p + w] - ps[p]; if (d > mm) mm = d; }
        double cand = mm * invsw;
        if (cand > best) best = cand;
    }
    return best;
}

static void* worker(void* arg) {
    warg_t* wa = (warg_t*)arg;
    job_t* J = wa->job;
    const int Np = J->Nprof, nh = J->nharms;
    int maxbins = 0;
    for (int l = 0; l < J->nlev; ++l) if (2 * J->Hk[l] > maxbins) maxbins = 2 * J->Hk[l];
    double* re = (double*)calloc((size_t)(nh + 1) * Np, sizeof(double));
    double* im = (double*)calloc((size_t)(nh + 1) * Np, sizeof(double));
    float* row = (float*)malloc(sizeof(float) * 2 * (size_t)Np);
    double* prof = (double*)malloc(sizeof(double) * (size_t)maxbins * Np);   /* [bin][b] */
    double* E = (double*)malloc(sizeof(double) * (size_t)Np);
    double* O = (double*)malloc(sizeof(double) * (size_t)Np);
    double* sig = (double*)malloc(sizeof(double) * CS_SIGCAP);
    double* mv = (double*)malloc(sizeof(double) * (size_t)Np);
    float* psT = (float*)malloc(sizeof(float) * (size_t)CS_BATCH * (2 * maxbins + 2));
    float mb[CS_BATCH], rs[CS_BATCH];
    double tmp[512], ps[1024];
    for (int64_t idx = wa->tid; idx < J->nblocks; idx += J->nthreads) {
        int64_t c = J->blist ? J->blist[idx] : J->first_block + idx;
        int64_t i0 = c * (int64_t)Np;
        int n = (int)((J->total - i0) < Np ? (J->total - i0) : Np);
        if (n <= 0) {
            if (J->blist) continue;
            break;
        }
        double rstart = J->r_lo + (double)i0 * J->lodr;
        for (int h = 1; h <= nh; ++h) {
            fill_row(&J->plans[h - 1], J->amps, J->namps, J->N, J->hidr, nh, i0, n, row);
            double* rr = re + (size_t)h * Np;
            double* ii = im + (size_t)h * Np;
            for (int b = 0; b < n; ++b) { rr[b] = (double)row[2 * b]; ii[b] = (double)row[2 * b + 1]; }
        }
        double nyq = (double)J->N / 2.0;
        for (int l = 0; l < J->nlev; ++l) {
            int k = J->ks[l], Hk = J->Hk[l], nb = 2 * Hk;
            int nvalid = n;
            if (k > 1) {
                nvalid = 0;
                while (nvalid < n && (double)k * (rstart + (double)nvalid * J->lodr) < nyq) ++nvalid;
            }
            /* c2r of the stride-k stack: prof[n] = E + O, prof[N-n] = E - O */
            const double* C2 = J->C2[l];
            const double* S2 = J->S2[l];
            const double* ny = re + (size_t)(Hk * k) * Np;
            for (int q = 0; q <= Hk; ++q) {
                double sgn = (q & 1) ? -1.0 : 1.0;
                for (int b = 0; b < n; ++b) { E[b] = sgn * ny[b]; O[b] = 0.0; }
                for (int jh = 1; jh < Hk; ++jh) {
                    const double c2 = C2[(size_t)jh * (Hk + 1) + q], s2 = S2[(size_t)jh * (Hk + 1) + q];
                    const double* rr = re + (size_t)(jh * k) * Np;
                    const double* ii = im + (size_t)(jh * k) * Np;
                    for (int b = 0; b < n; ++b) { E[b] += rr[b] * c2; O[b] += ii[b] * s2; }
                }
                double* p0 = prof + (size_t)q * Np;
                for (int b = 0; b < n; ++b) p0[b] = E[b] + O[b];
                if (q >= 1 && q < Hk) {
                    double* p1 = prof + (size_t)(nb - q) * Np;
                    for (int b = 0; b < n; ++b) p1[b] = E[b] - O[b];
                }
            }
            /* block sigma over the valid prefix */
            int64_t Ntot = (int64_t)nb * nvalid;
            int ns = 0;
            if (Ntot <= CS_SIGCAP) {
                for (int b = 0; b < nvalid; ++b)
                    for (int i = 0; i < nb; ++i) sig[ns++] = fabs(prof[(size_t)i * Np + b]);
            } else {
                int ncol = nvalid < CS_SIGCAP / nb ? nvalid : CS_SIGCAP / nb;
                if (ncol < 1) ncol = 1;
                for (int cc = 1; cc <= ncol; ++cc) {
                    int j = ((cc - 1) * nvalid) / ncol;
                    for (int i = 0; i < nb && ns < CS_SIGCAP; ++i) sig[ns++] = fabs(prof[(size_t)i * Np + j]);
                }
            }
            double sg = ns ? 1.4826 * median_d(sig, ns) : 0.0;
            if (J->sig_out) J->sig_out[idx * J->nlev + l] = sg;
            if (J->nv_out) J->nv_out[idx * J->nlev + l] = nvalid;
            double invsig = sg > 0 ? 1.0 / sg : 0.0;
            const int* ws = J->widths[l];
            int nw = J->nw[l], wmax = ws[nw - 1];
            int64_t resc = 0;
            if (J->medcut == -INFINITY || !(invsig > 0)) {
                for (int j = 0; j < nvalid; ++j)
                    mv[j] = invsig > 0 ? exact_metric_d(prof + j, Np, nb, ws, nw, invsig, tmp, ps) : 0.0;
            } else {
                int full = (nvalid / CS_BATCH) * CS_BATCH;
                float inv32 = (float)invsig;
                for (int j0 = 0; j0 < full; j0 += CS_BATCH) {
                    for (int b = 0; b < CS_BATCH; ++b) psT[b] = 0.0f;
                    for (int i = 0; i < nb + wmax; ++i) {
                        int idx = i >= nb ? i - nb : i;
                        const double* src = prof + (size_t)idx * Np + j0;
                        float* o = psT + (size_t)i * CS_BATCH;
                        for (int b = 0; b < CS_BATCH; ++b) o[CS_BATCH + b] = o[b] + (float)src[b];
                    }
                    for (int b = 0; b < CS_BATCH; ++b) rs[b] = -INFINITY;
                    for (int a = 0; a < nw; ++a) {
                        int w = ws[a];
                        float invsw = inv32 / sqrtf((float)w);
                        for (int b = 0; b < CS_BATCH; ++b) mb[b] = psT[(size_t)w * CS_BATCH + b] - psT[b];
                        for (int p = 1; p < nb; ++p) {
                            const float* hi = psT + (size_t)(p + w) * CS_BATCH;
                            const float* lo = psT + (size_t)p * CS_BATCH;
                            for (int b = 0; b < CS_BATCH; ++b) { float d = hi[b] - lo[b]; mb[b] = d > mb[b] ? d : mb[b]; }
                        }
                        for (int b = 0; b < CS_BATCH; ++b) { float cv = mb[b] * invsw; rs[b] = cv > rs[b] ? cv : rs[b]; }
                    }
                    for (int b = 0; b < CS_BATCH; ++b) mv[j0 + b] = (double)rs[b];
                }
                for (int j = full; j < nvalid; ++j) {
                    /* scalar zero-baseline gate in the profile precision */
                    ps[0] = 0.0;
                    for (int i = 0; i < nb + wmax; ++i) {
                        int idx = i >= nb ? i - nb : i;
                        ps[i + 1] = ps[i] + prof[(size_t)idx * Np + j];
                    }
                    double best = -INFINITY;
                    for (int a = 0; a < nw; ++a) {
                        int w = ws[a];
                        double invsw = invsig / sqrt((double)w);
                        double mm = ps[w] - ps[0];
                        for (int p = 1; p < nb; ++p) { double d = ps[p + w] - ps[p]; if (d > mm) mm = d; }
                        double cv = mm * invsw;
                        if (cv > best) best = cv;
                    }
                    mv[j] = best;
                }
                for (int j = 0; j < nvalid; ++j)
                    if (mv[j] >= J->medcut) {
                        mv[j] = exact_metric_d(prof + j, Np, nb, ws, nw, invsig, tmp, ps);
                        ++resc;
                    }
            }
            for (int j = 0; j < nvalid; ++j) {
                if (mv[j] > J->threshold) {
                    pthread_mutex_lock(&J->mu);
                    if (J->ncand < J->cap) {
                        cpu_cand_t* o = &J->cands[J->ncand];
                        o->blk = (int32_t)c; o->k = k; o->j = j; o->pad = 0; o->metric = mv[j];
                    }
                    J->ncand++;
                    pthread_mutex_unlock(&J->mu);
                }
            }
            pthread_mutex_lock(&J->mu);
            J->rescued += resc;
            pthread_mutex_unlock(&J->mu);
        }
    }
    free(re); free(im); free(row); free(prof); free(E); free(O); free(sig); free(mv); free(psT);
    return NULL;
}

static int boxcar_bank(int nbins, double fsp, double maxfrac, int* out) {
    int64_t wmax = (int64_t)floor(maxfrac * (double)nbins);
    if (wmax < 1) wmax = 1;
    int n = 0;
    int64_t w = 1;
    while (w <= wmax && n < CS_MAXW) {
        out[n++] = (int)w;
        int64_t nx = (int64_t)floor(fsp * (double)w);
        w = nx > w + 1 ? nx : w + 1;
    }
    return n;
}

/* Search blocks [first_block, first_block+nblocks) of a search over `total`
 * trials anchored at r_lo; decimations ks (base fold k=1 is always searched
 * first).  Writes up to cap candidates (block, k, j, metric) and returns the
 * number found; *seconds = wall time of the call, *rescued = exact rescans.
 * Default boxcar parameters (fsp 1.5, maxfrac 0.3, medmargin 2.0). */
int64_t csref_search_blocks_ex(const float* amps, int64_t namps, int64_t N, int nharms, int m, double hidr,
                               const int* decims, int ndecim, double r_lo, int64_t total, int Nprof,
                               int64_t first_block, int64_t nblocks, const int64_t* blist, double threshold,
                               int exact_all, int nthreads, cpu_cand_t* cands, int64_t cap, double* seconds,
                               int64_t* rescued, double* sig_out, int32_t* nv_out);

int64_t csref_search_blocks(const float* amps, int64_t namps, int64_t N, int nharms, int m, double hidr,
                            const int* decims, int ndecim, double r_lo, int64_t total, int Nprof,
                            int64_t first_block, int64_t nblocks, double threshold, int exact_all,
                            int nthreads, cpu_cand_t* cands, int64_t cap, double* seconds, int64_t* rescued) {
    return csref_search_blocks_ex(amps, namps, N, nharms, m, hidr, decims, ndecim, r_lo, total, Nprof,
                                  first_block, nblocks, NULL, threshold, exact_all, nthreads, cands, cap, seconds,
                                  rescued, NULL, NULL);
}

/* As csref_search_blocks, over the listed blocks blist[0 .. nblocks) when blist
 * is not NULL, with each searched block's per-level sigma and valid-trial
 * count (levels in search order) written to sig_out / nv_out
 * [idx * nlevels + l] when those are not NULL. */
int64_t csref_search_blocks_ex(const float* amps, int64_t namps, int64_t N, int nharms, int m, double hidr,
                               const int* decims, int ndecim, double r_lo, int64_t total, int Nprof,
                               int64_t first_block, int64_t nblocks, const int64_t* blist, double threshold,
                               int exact_all, int nthreads, cpu_cand_t* cands, int64_t cap, double* seconds,
                               int64_t* rescued, double* sig_out, int32_t* nv_out) {
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    job_t J;
    memset(&J, 0, sizeof(J));
    J.amps = amps; J.namps = namps; J.N = N; J.nharms = nharms; J.m = m; J.hidr = hidr;
    J.lodr = hidr / (double)nharms; J.r_lo = r_lo; J.total = total; J.Nprof = Nprof;
    J.first_block = first_block; J.nblocks = nblocks; J.threshold = threshold;
    J.blist = blist; J.sig_out = sig_out; J.nv_out = nv_out;
    J.medcut = exact_all ? -INFINITY : threshold - 2.0;
    J.nthreads = nthreads < 1 ? 1 : nthreads;
    J.cands = cands; J.cap = cap;
    pthread_mutex_init(&J.mu, NULL);
    /* levels: k = 1, then every k > 1 in order; ladder pruning (src/search.jl:443-459) */
    int ks[CS_MAXLEV], nl = 0;
    ks[nl++] = 1;
    for (int i = 0; i < ndecim && nl < CS_MAXLEV; ++i) if (decims[i] > 1) ks[nl++] = decims[i];
    int sorted[CS_MAXLEV], ns = ndecim < CS_MAXLEV ? ndecim : CS_MAXLEV;
    for (int i = 0; i < ns; ++i) sorted[i] = decims[i];
    for (int i = 1; i < ns; ++i) for (int j = i; j > 0 && sorted[j - 1] > sorted[j]; --j) {
        int t = sorted[j]; sorted[j] = sorted[j - 1]; sorted[j - 1] = t; }
    int ladder = ns > 1;
    for (int i = 0; i + 1 < ns; ++i) if (!(sorted[i + 1] <= 3 * sorted[i])) ladder = 0;
    J.nlev = nl;
    for (int l = 0; l < nl; ++l) {
        int k = ks[l], Hk = nharms / k, nb = 2 * Hk;
        J.ks[l] = k; J.Hk[l] = Hk;
        int full[CS_MAXW];
        int nf = boxcar_bank(nb, 1.5, 0.3, full), np_ = 0;
        if (ladder) {
            for (int a = 0; a < nf; ++a)
                if ((full[a] >= 2 || k == sorted[0]) && (full[a] <= 6 || k == sorted[ns - 1]))
                    J.widths[l][np_++] = full[a];
        }
        if (np_ == 0) { memcpy(J.widths[l], full, sizeof(int) * nf); np_ = nf; }
        J.nw[l] = np_;
        J.C2[l] = (double*)calloc((size_t)Hk * (Hk + 1), sizeof(double));
        J.S2[l] = (double*)calloc((size_t)Hk * (Hk + 1), sizeof(double));
        for (int j = 1; j < Hk; ++j)
            for (int q = 0; q <= Hk; ++q) {
                double ang = 2.0 * M_PI * (double)(((int64_t)j * q) % nb) / (double)nb;
                J.C2[l][(size_t)j * (Hk + 1) + q] = 2.0 * cos(ang);
                J.S2[l][(size_t)j * (Hk + 1) + q] = -2.0 * sin(ang);
            }
    }
    J.plans = build_plans(nharms, m, hidr, r_lo);
    pthread_t th[256];
    warg_t wa[256];
    int nt = J.nthreads > 256 ? 256 : J.nthreads;
    J.nthreads = nt;
    for (int t = 0; t < nt; ++t) { wa[t].job = &J; wa[t].tid = t; pthread_create(&th[t], NULL, worker, &wa[t]); }
    for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
    free_plans(J.plans, nharms);
    for (int l = 0; l < nl; ++l) { free(J.C2[l]); free(J.S2[l]); }
    pthread_mutex_destroy(&J.mu);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (seconds) *seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    if (rescued) *rescued = J.rescued;
    return J.ncand;
}
