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
 *     by exact 128-bit divrem at the row's first trial (direct_chunk_state,
 *     :414-418) and exact integer steps after it, phase row lookup,
 *     range guard on the true trial range, sequential FP32 fmaf over the m taps,
 *     unfused Complex{Float32} product;
 *   - _fill_row_direct_slow! (:623-661) for a non-rational trial step;
 *   - the profile stage's brfft as a mixed-radix FFT (ft_c2r).
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
    /* Trials in groups of FR_V.  The state steps exactly from trial to trial,
     * as the reference advances it (src/directinterp.jl:563-567): one trial
     * adds base_adv to qint and s to res, with a carry of one bin when res
     * passes q.  Each trial keeps its own sequential fmaf chain over the taps;
     * the group's FR_V chains are independent, so they overlap. */
    enum { FR_V = 8 };
    int64_t r_ = res, qi = qint;
    for (int64_t k0 = 0; k0 < n; k0 += FR_V) {
        const int nv = (n - k0) < FR_V ? (int)(n - k0) : FR_V;
        int64_t ao[FR_V];
        int pv[FR_V];
        for (int v = 0; v < FR_V; ++v) {
            if (v >= nv) { pv[v] = pv[0]; ao[v] = ao[0]; continue; }   /* padding lanes, discarded */
            const int p = d->row[r_];
            pv[v] = p;
            ao[v] = 2 * (d->rfloor0 + qi + d->carry[p] + 1 - m2);      /* 0-based first tap */
            qi += d->base_adv;
            r_ += d->s;
            if (r_ >= d->q) { r_ -= d->q; ++qi; }
        }
        float sre[FR_V], sim[FR_V];
        for (int v = 0; v < FR_V; ++v) { sre[v] = 0.0f; sim[v] = 0.0f; }
        for (int i = 0; i < m; ++i)
            for (int v = 0; v < FR_V; ++v) {
                const float w = d->W[(size_t)pv[v] * m + i];
                sre[v] = fmaf(w, amps[ao[v] + 2 * i], sre[v]);
                sim[v] = fmaf(w, amps[ao[v] + 2 * i + 1], sim[v]);
            }
        for (int v = 0; v < nv; ++v) {
            const int p = pv[v];
            float ar = d->A[2 * p], ai = d->A[2 * p + 1];
            float pr0 = ar * sre[v], pr1 = ai * sim[v], pi0 = ar * sim[v], pi1 = ai * sre[v];
            out[2 * (k0 + v)] = pr0 - pr1;
            out[2 * (k0 + v) + 1] = pi0 + pi1;
        }
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
 * The profile stage's c2r transform in FP64, vectorised across trials: the
 * unnormalised brfft the reference applies to each trial's stacked harmonics
 * (src/search.jl:1291, :1675),
 *     prof[t] = X[H] (-1)^t + 2 sum_{j=1}^{H-1} Re(X[j] e^{+2 pi i j t / 2H}),
 * t = 0 .. 2H-1 (the DC term is zero on this path, and brfft drops the
 * imaginary parts of DC and Nyquist).
 *
 * Computed as one complex FFT of length H: with the even/odd split of a real
 * sequence, z[n] = prof[2n] + i prof[2n+1] is the inverse DFT of
 *     Z[j] = E[j] + i O[j],  E[j] = X[j] + conj(X[H-j]),
 *                            O[j] = (X[j] - conj(X[H-j])) e^{+i pi j / H}
 * (Z[0] = X[H] (1 - i)).  The length-H transform is a mixed-radix
 * (4, 2, 3, 5) self-sorting Stockham decimation in frequency: a stage of
 * radix p over sequences of length n = p m at stride s maps
 *     y[q + s (p u + j)] = w_n^{j u} sum_k x[q + s (u + k m)] w_p^{j k}
 * (w_r = e^{+2 pi i / r}), then the next stage takes length m at stride p s;
 * after the last the output is in natural order.  Each element is a vector of
 * up to FT_LANES trials, so every loop runs over contiguous lanes.  Lengths
 * with another prime factor keep the direct symmetric DFT.
 * ------------------------------------------------------------------------ */
#define FT_LANES 64
#define FT_MAXST 24

typedef struct {
    int H, nst, rad[FT_MAXST];
    double* tw[FT_MAXST];   /* stage s: m x (p-1) complex w_n^{j u}, [u][j-1] */
    double* pre;            /* H complex e^{+i pi j / H} */
    double* C2;             /* direct DFT (other lengths): (H) x (H+1) 2 cos(2 pi j t / 2H) */
    double* S2;             /* and -2 sin */
} ft_plan_t;

static void ft_free(ft_plan_t* P) {
    for (int s = 0; s < P->nst; ++s) free(P->tw[s]);
    free(P->pre);
    free(P->C2);
    free(P->S2);
    memset(P, 0, sizeof(*P));
}

static void ft_init(ft_plan_t* P, int H) {
    memset(P, 0, sizeof(*P));
    P->H = H;
    const int nb = 2 * H;
    int n = H, ok = 1;
    while (n > 1 && ok) {
        const int p = n % 4 == 0 ? 4 : n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n % 5 == 0 ? 5 : 0;
        if (!p || P->nst == FT_MAXST) ok = 0;
        else { P->rad[P->nst++] = p; n /= p; }
    }
    if (!ok) {
        P->nst = 0;
        P->C2 = (double*)calloc((size_t)H * (H + 1), sizeof(double));
        P->S2 = (double*)calloc((size_t)H * (H + 1), sizeof(double));
        for (int j = 1; j < H; ++j)
            for (int q = 0; q <= H; ++q) {
                double ang = 2.0 * M_PI * (double)(((int64_t)j * q) % nb) / (double)nb;
                P->C2[(size_t)j * (H + 1) + q] = 2.0 * cos(ang);
                P->S2[(size_t)j * (H + 1) + q] = -2.0 * sin(ang);
            }
        return;
    }
    n = H;
    for (int s = 0; s < P->nst; ++s) {
        const int p = P->rad[s], m = n / p;
        P->tw[s] = (double*)malloc(sizeof(double) * 2 * (size_t)m * (p - 1));
        for (int u = 0; u < m; ++u)
            for (int j = 1; j < p; ++j) {
                double ang = 2.0 * M_PI * (double)(((int64_t)j * u) % n) / (double)n;
                P->tw[s][2 * ((size_t)u * (p - 1) + j - 1)] = cos(ang);
                P->tw[s][2 * ((size_t)u * (p - 1) + j - 1) + 1] = sin(ang);
            }
        n = m;
    }
    P->pre = (double*)malloc(sizeof(double) * 2 * (size_t)H);
    for (int j = 0; j < H; ++j) {
        P->pre[2 * j] = cos(M_PI * (double)j / (double)H);
        P->pre[2 * j + 1] = sin(M_PI * (double)j / (double)H);
    }
}

/* The butterflies of one (u, q) of a stage: inputs a_k at x + k istep,
 * outputs y_j = w_j * (sum_k a_k w_p^{jk}) at y + j ostep (w_0 = 1), for L
 * lanes.  One function per radix, restrict-qualified, so each lane loop
 * vectorises. */
#define FT_ROT(r, i, wr, wi, outr, outi)  do { (outr) = (r) * (wr) - (i) * (wi); (outi) = (r) * (wi) + (i) * (wr); } while (0)

static void ft_bf2(const double* __restrict xr, const double* __restrict xi, size_t is, double* __restrict yr,
                   double* __restrict yi, size_t os, const double* w, int L) {
    const double w1r = w[0], w1i = w[1];
#pragma omp simd
    for (int b = 0; b < L; ++b) {
        const double ar = xr[b], ai = xi[b], br = xr[is + b], bi = xi[is + b];
        yr[b] = ar + br; yi[b] = ai + bi;
        FT_ROT(ar - br, ai - bi, w1r, w1i, yr[os + b], yi[os + b]);
    }
}

static void ft_bf3(const double* __restrict xr, const double* __restrict xi, size_t is, double* __restrict yr,
                   double* __restrict yi, size_t os, const double* w, int L) {
    const double S3 = 0.86602540378443864676;   /* sin(2 pi / 3) */
    const double w1r = w[0], w1i = w[1], w2r = w[2], w2i = w[3];
#pragma omp simd
    for (int b = 0; b < L; ++b) {
        const double a0r = xr[b], a0i = xi[b], a1r = xr[is + b], a1i = xi[is + b];
        const double a2r = xr[2 * is + b], a2i = xi[2 * is + b];
        const double t1r = a1r + a2r, t1i = a1i + a2i;
        const double t2r = a0r - 0.5 * t1r, t2i = a0i - 0.5 * t1i;
        const double t3r = S3 * (a1r - a2r), t3i = S3 * (a1i - a2i);
        yr[b] = a0r + t1r; yi[b] = a0i + t1i;
        FT_ROT(t2r - t3i, t2i + t3r, w1r, w1i, yr[os + b], yi[os + b]);
        FT_ROT(t2r + t3i, t2i - t3r, w2r, w2i, yr[2 * os + b], yi[2 * os + b]);
    }
}

static void ft_bf4(const double* __restrict xr, const double* __restrict xi, size_t is, double* __restrict yr,
                   double* __restrict yi, size_t os, const double* w, int L) {
    const double w1r = w[0], w1i = w[1], w2r = w[2], w2i = w[3], w3r = w[4], w3i = w[5];
#pragma omp simd
    for (int b = 0; b < L; ++b) {
        const double a0r = xr[b], a0i = xi[b], a1r = xr[is + b], a1i = xi[is + b];
        const double a2r = xr[2 * is + b], a2i = xi[2 * is + b], a3r = xr[3 * is + b], a3i = xi[3 * is + b];
        const double t0r = a0r + a2r, t0i = a0i + a2i;
        const double t1r = a0r - a2r, t1i = a0i - a2i;
        const double t2r = a1r + a3r, t2i = a1i + a3i;
        const double t3r = -(a1i - a3i), t3i = a1r - a3r;   /* i (a1 - a3) */
        yr[b] = t0r + t2r; yi[b] = t0i + t2i;
        FT_ROT(t1r + t3r, t1i + t3i, w1r, w1i, yr[os + b], yi[os + b]);
        FT_ROT(t0r - t2r, t0i - t2i, w2r, w2i, yr[2 * os + b], yi[2 * os + b]);
        FT_ROT(t1r - t3r, t1i - t3i, w3r, w3i, yr[3 * os + b], yi[3 * os + b]);
    }
}

static void ft_bf5(const double* __restrict xr, const double* __restrict xi, size_t is, double* __restrict yr,
                   double* __restrict yi, size_t os, const double* w, int L) {
    const double C51 = 0.30901699437494742410, C52 = -0.80901699437494742410;   /* cos(2 pi/5), cos(4 pi/5) */
    const double S51 = 0.95105651629515357212, S52 = 0.58778525229247312917;    /* sin(2 pi/5), sin(4 pi/5) */
    const double w1r = w[0], w1i = w[1], w2r = w[2], w2i = w[3], w3r = w[4], w3i = w[5], w4r = w[6], w4i = w[7];
#pragma omp simd
    for (int b = 0; b < L; ++b) {
        const double a0r = xr[b], a0i = xi[b];
        const double a1r = xr[is + b], a1i = xi[is + b], a2r = xr[2 * is + b], a2i = xi[2 * is + b];
        const double a3r = xr[3 * is + b], a3i = xi[3 * is + b], a4r = xr[4 * is + b], a4i = xi[4 * is + b];
        const double s1r = a1r + a4r, s1i = a1i + a4i, d1r = a1r - a4r, d1i = a1i - a4i;
        const double s2r = a2r + a3r, s2i = a2i + a3i, d2r = a2r - a3r, d2i = a2i - a3i;
        const double c1r = a0r + C51 * s1r + C52 * s2r, c1i = a0i + C51 * s1i + C52 * s2i;
        const double c2r = a0r + C52 * s1r + C51 * s2r, c2i = a0i + C52 * s1i + C51 * s2i;
        const double e1r = S51 * d1r + S52 * d2r, e1i = S51 * d1i + S52 * d2i;
        const double e2r = S52 * d1r - S51 * d2r, e2i = S52 * d1i - S51 * d2i;
        yr[b] = a0r + s1r + s2r; yi[b] = a0i + s1i + s2i;
        FT_ROT(c1r - e1i, c1i + e1r, w1r, w1i, yr[os + b], yi[os + b]);           /* c1 + i e1 */
        FT_ROT(c2r - e2i, c2i + e2r, w2r, w2i, yr[2 * os + b], yi[2 * os + b]);   /* c2 + i e2 */
        FT_ROT(c2r + e2i, c2i - e2r, w3r, w3i, yr[3 * os + b], yi[3 * os + b]);   /* c2 - i e2 */
        FT_ROT(c1r + e1i, c1i - e1r, w4r, w4i, yr[4 * os + b], yi[4 * os + b]);   /* c1 - i e1 */
    }
}

/* One stage of radix p over sequences of length n at stride s (L lanes per
 * element): y[q + s (p u + j)] = w_n^{j u} sum_k x[q + s (u + k m)] w_p^{jk}. */
static void ft_stage(int p, int n, int s, const double* tw, const double* xr, const double* xi, double* yr,
                     double* yi, int L) {
    const int m = n / p;
    const size_t istep = (size_t)s * m * L, ostep = (size_t)s * L;
    for (int u = 0; u < m; ++u) {
        const double* w = tw + 2 * (size_t)u * (p - 1);
        for (int q = 0; q < s; ++q) {
            const size_t i0 = (size_t)(q + s * u) * L, o0 = (size_t)(q + s * p * u) * L;
            switch (p) {
            case 2: ft_bf2(xr + i0, xi + i0, istep, yr + o0, yi + o0, ostep, w, L); break;
            case 3: ft_bf3(xr + i0, xi + i0, istep, yr + o0, yi + o0, ostep, w, L); break;
            case 4: ft_bf4(xr + i0, xi + i0, istep, yr + o0, yi + o0, ostep, w, L); break;
            default: ft_bf5(xr + i0, xi + i0, istep, yr + o0, yi + o0, ostep, w, L); break;
            }
        }
    }
}

/* prof[t * pstride + b] for t < 2H, b < n, from the harmonics
 * X[j] = (re, im)[j * rstride + b], j = 1..H (row 0 is not read).  scratch:
 * 4 H FT_LANES doubles (FFT) or 2 n doubles (direct DFT). */
static void ft_c2r(const ft_plan_t* P, const double* re, const double* im, size_t rstride, double* prof,
                   size_t pstride, int n, double* scratch) {
    const int H = P->H, nb = 2 * H;
    if (P->C2) {
        double* E = scratch;
        double* O = scratch + n;
        const double* ny = re + (size_t)H * rstride;
        for (int q = 0; q <= H; ++q) {
            double sgn = (q & 1) ? -1.0 : 1.0;
            for (int b = 0; b < n; ++b) { E[b] = sgn * ny[b]; O[b] = 0.0; }
            for (int jh = 1; jh < H; ++jh) {
                const double c2 = P->C2[(size_t)jh * (H + 1) + q], s2 = P->S2[(size_t)jh * (H + 1) + q];
                const double* rr = re + (size_t)jh * rstride;
                const double* ii = im + (size_t)jh * rstride;
                for (int b = 0; b < n; ++b) { E[b] += rr[b] * c2; O[b] += ii[b] * s2; }
            }
            double* p0 = prof + (size_t)q * pstride;
            for (int b = 0; b < n; ++b) p0[b] = E[b] + O[b];
            if (q >= 1 && q < H) {
                double* p1 = prof + (size_t)(nb - q) * pstride;
                for (int b = 0; b < n; ++b) p1[b] = E[b] - O[b];
            }
        }
        return;
    }
    const size_t V = (size_t)H * FT_LANES;
    for (int b0 = 0; b0 < n; b0 += FT_LANES) {
        const int L = n - b0 < FT_LANES ? n - b0 : FT_LANES;
        double *xr = scratch, *xi = scratch + V, *yr = scratch + 2 * V, *yi = scratch + 3 * V;
        const double* nr = re + (size_t)H * rstride + b0;
        for (int b = 0; b < L; ++b) { xr[b] = nr[b]; xi[b] = -nr[b]; }
        for (int j = 1; j < H; ++j) {
            const double *ar = re + (size_t)j * rstride + b0, *ai = im + (size_t)j * rstride + b0;
            const double *br = re + (size_t)(H - j) * rstride + b0, *bi = im + (size_t)(H - j) * rstride + b0;
            const double c = P->pre[2 * j], s = P->pre[2 * j + 1];
            double *zr = xr + (size_t)j * L, *zi = xi + (size_t)j * L;
            for (int b = 0; b < L; ++b) {
                const double er = ar[b] + br[b], ei = ai[b] - bi[b];   /* X[j] + conj(X[H-j]) */
                const double dr = ar[b] - br[b], di = ai[b] + bi[b];   /* X[j] - conj(X[H-j]) */
                const double orr = dr * c - di * s, oi = dr * s + di * c;
                zr[b] = er - oi;
                zi[b] = ei + orr;
            }
        }
        int len = H, st = 1;
        for (int k = 0; k < P->nst; ++k) {
            ft_stage(P->rad[k], len, st, P->tw[k], xr, xi, yr, yi, L);
            double* t = xr; xr = yr; yr = t;
            t = xi; xi = yi; yi = t;
            len /= P->rad[k];
            st *= P->rad[k];
        }
        for (int t = 0; t < H; ++t) {
            double* pe = prof + (size_t)(2 * t) * pstride + b0;
            double* po = pe + pstride;
            const double *zr = xr + (size_t)t * L, *zi = xi + (size_t)t * L;
            for (int b = 0; b < L; ++b) { pe[b] = zr[b]; po[b] = zi[b]; }
        }
    }
}

static size_t ft_scratch(int Hmax, int n) {
    size_t a = 4 * (size_t)Hmax * FT_LANES, b = 2 * (size_t)n;
    return a > b ? a : b;
}

/* The profile stage's transform on n profiles, for the tests: X = (re, im)
 * [H+1][n] (harmonic j's lanes at j * n; row 0 ignored), prof [2H][n].
 * Returns the number of FFT stages (0 for the direct DFT of lengths with a
 * prime factor above 5, or for H = 1), or -1 for bad arguments. */
int csref_c2r(const double* re, const double* im, int H, int n, double* prof) {
    if (H < 1 || n < 1 || !re || !im || !prof) return -1;
    ft_plan_t P;
    ft_init(&P, H);
    double* scratch = (double*)malloc(sizeof(double) * ft_scratch(H, n));
    ft_c2r(&P, re, im, (size_t)n, prof, (size_t)n, n, scratch);
    const int nst = P.C2 ? 0 : P.nst;
    free(scratch);
    ft_free(&P);
    return nst;
}

/* ------------------------------------------------------------------------
 * Full production search over a range of blocks, multithreaded: the timed
 * CPU restatement of `_search_region!` (src/search.jl:1768-1894) with the
 * default profile precision :f64.  Per block: Float32-weight interpolation
 * (fill_row above), the FP64 c2r transform of every level (ft_c2r above: a
 * mixed-radix FFT across the block's profiles), the block sigma
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
    ft_plan_t ft[CS_MAXLEV]; /* each level's c2r transform (length Hk) */
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
    int maxH = 1;
    for (int l = 0; l < J->nlev; ++l) if (J->Hk[l] > maxH) maxH = J->Hk[l];
    double* fts = (double*)malloc(sizeof(double) * ft_scratch(maxH, Np));
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
            /* c2r of the stride-k stack (harmonics k, 2k, .., Hk k) */
            ft_c2r(&J->ft[l], re, im, (size_t)k * Np, prof, (size_t)Np, n, fts);
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
    free(re); free(im); free(row); free(prof); free(fts); free(sig); free(mv); free(psT);
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
        ft_init(&J.ft[l], Hk);
    }
    J.plans = build_plans(nharms, m, hidr, r_lo);
    pthread_t th[256];
    warg_t wa[256];
    int nt = J.nthreads > 256 ? 256 : J.nthreads;
    J.nthreads = nt;
    for (int t = 0; t < nt; ++t) { wa[t].job = &J; wa[t].tid = t; pthread_create(&th[t], NULL, worker, &wa[t]); }
    for (int t = 0; t < nt; ++t) pthread_join(th[t], NULL);
    free_plans(J.plans, nharms);
    for (int l = 0; l < nl; ++l) ft_free(&J.ft[l]);
    pthread_mutex_destroy(&J.mu);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (seconds) *seconds = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
    if (rescued) *rescued = J.rescued;
    return J.ncand;
}
