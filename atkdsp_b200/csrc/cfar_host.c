/* Host side of the CFAR detector and burst tracker, in C99 (reference
 * src/cfar.c, include/atkdsp.h:1730-1924).
 *
 * The per-cell work of a call runs on the GPU (cfar.cu): every frame's
 * conversion to linear power, the k-frame average and each bin's test, in
 * one pass over all the call's frames. What stays here:
 *   - the threshold solver: Pfa(alpha) = integral of Q(K, K alpha t) against
 *     the density of the reference statistic T, by Simpson's rule in ln t,
 *     solved by regula falsi (Illinois) in ln alpha (src/cfar.c:25-253);
 *   - the reference-cell tables with the borrowing walk (src/cfar.c:344-372);
 *   - the tracker, a serial state machine over the hit rows in frame order:
 *     blobs, association, OPEN / UPDATE / CLOSE (src/cfar.c:594-742).
 * The solver's grid, tolerances and evaluation order are the reference's, so
 * alpha is the same number; the tracker takes the same steps in the same
 * order, so the events are the same events.
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "host_internal.h"

#define CF_MAX_GRID 131072
#define CF_PI 3.14159265358979323846
#define CF_LN10 2.302585092994045684
/* frames per device pass: at most this many cells, and at most 4096 frames */
#define CF_PASS_CELLS ((size_t)1 << 20)
#define CF_PASS_FRAMES 4096
/* host buffers up to this size are pinned */
#define CF_PINNED_MAX ((size_t)256 << 20)

/* ================================================= special functions
 * Regularised incomplete gammas in log space: the power series of P below
 * x = a + 1 and the modified-Lentz continued fraction of Q above it (Press et
 * al., Numerical Recipes 2nd ed., 6.2), each finite far into its own tail,
 * the other by log1p. Both converge in O(sqrt(a)) terms near x = a; the
 * bound is 1000 + 10 sqrt(a) (src/stat.c:14). */
static int igam_bound(double a) { return 1000 + (int)(10.0 * sqrt(a > 0.0 ? a : 0.0)); }

static void log_igam(double a, double x, double *lnp, double *lnq) {
    if (!(x > 0.0)) {
        *lnp = -INFINITY;
        *lnq = 0.0;
        return;
    }
    const double lg = lgamma(a);
    const int it = igam_bound(a);
    if (x < a + 1.0) {
        double den = a, term = 1.0 / a, sum = term;
        for (int i = 0; i < it; ++i) {
            den += 1.0;
            term *= x / den;
            sum += term;
            if (fabs(term) < fabs(sum) * 1e-16) break;
        }
        *lnp = log(sum) - x + a * log(x) - lg;
        const double p = exp(*lnp);
        *lnq = p < 1.0 ? log1p(-p) : -INFINITY;
        return;
    }
    const double tiny = 1e-300;
    double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < it; ++i) {
        const double an = -(double)i * ((double)i - a);
        b += 2.0;
        d = an * d + b;
        if (fabs(d) < tiny) d = tiny;
        c = b + an / c;
        if (fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double step = d * c;
        h *= step;
        if (fabs(step - 1.0) < 1e-16) break;
    }
    *lnq = -x + a * log(x) - lg + log(h);
    const double q = exp(*lnq);
    *lnp = q < 1.0 ? log1p(-q) : -INFINITY;
}

/* log10 P(Binomial(n, q) >= c), q = exp(ln_q): the terms from c upward,
 * summed relative to the first until they fall 40 e-folds below it; 0 at or
 * below the mean (src/stat.c:89-107). */
static double binom_term(double n, double k, double ln_q, double ln_1mq) {
    return lgamma(n + 1.0) - lgamma(k + 1.0) - lgamma(n - k + 1.0) + k * ln_q + (n - k) * ln_1mq;
}

static double log10_binom_tail(double n, double c, double ln_q) {
    if (c <= 0.0) return 0.0;
    if (c > n) return -INFINITY;
    const double q = exp(ln_q);
    if (c <= n * q) return 0.0;
    const double ln_1mq = log1p(-q);
    const double first = binom_term(n, c, ln_q, ln_1mq);
    double s = 1.0;
    for (double k = c + 1.0; k <= n; k += 1.0) {
        const double d = binom_term(n, k, ln_q, ln_1mq) - first;
        if (d < -40.0) break;
        s += exp(d);
    }
    const double r = (first + log(s)) / CF_LN10;
    return r > 0.0 ? 0.0 : r;
}

/* ================================================= the threshold solver */

/* ln of the Gamma(s, scale 1/s) density (unit mean) at t */
static double ln_unit_gamma(double s, double t) { return s * log(s) + (s - 1.0) * log(t) - s * t - lgamma(s); }

/* ln density of T at t for unit-mean K-look cells; N cells, ne of them
 * effectively independent; OS rank k. CA: the mean of ne cells (shape ne K);
 * GO / SO: the max / min of two side means (shape ne K / 2 each); OS: the
 * k-th order statistic of N single cells. */
static double t_log_density(int mode, double t, int N, double ne, double K, int k) {
    double lp, lq;
    if (mode == ATKDSP_CFAR_CA) return ln_unit_gamma(ne * K, t);
    if (mode == ATKDSP_CFAR_GO || mode == ATKDSP_CFAR_SO) {
        const double s = 0.5 * ne * K;
        log_igam(s, s * t, &lp, &lq);
        return log(2.0) + (mode == ATKDSP_CFAR_GO ? lp : lq) + ln_unit_gamma(s, t);
    }
    log_igam(K, K * t, &lp, &lq);
    double r = log((double)N) + lgamma((double)N) - lgamma((double)k) - lgamma((double)(N - k + 1)) +
               ln_unit_gamma(K, t);
    if (k > 1) r = r + (k - 1) * lp;
    if (N > k) r = r + (N - k) * lq;
    return r;
}

/* ln P(T <= t) and ln P(T > t) */
static void t_log_cdf_sf(int mode, double t, int N, double ne, double K, int k, double *cdf, double *sf) {
    double lp, lq;
    if (mode == ATKDSP_CFAR_CA) {
        log_igam(ne * K, ne * K * t, cdf, sf);
        return;
    }
    if (mode == ATKDSP_CFAR_GO || mode == ATKDSP_CFAR_SO) {
        const double s = 0.5 * ne * K;
        log_igam(s, s * t, &lp, &lq);
        if (mode == ATKDSP_CFAR_GO) {
            *cdf = 2.0 * lp;
            *sf = lq + log1p(exp(lp));
        } else {
            *cdf = lp + log1p(exp(lq));
            *sf = 2.0 * lq;
        }
        return;
    }
    log_igam(K, K * t, &lp, &lq);
    *cdf = lp == -INFINITY ? -INFINITY : log10_binom_tail(N, k, lp) * CF_LN10;
    *sf = lq == -INFINITY ? -INFINITY : log10_binom_tail(N, N - k + 1, lq) * CF_LN10;
}

/* Simpson nodes in u = ln t over the range outside which each tail of T
 * holds less than 1e-9 pfa: t[j] and G[j] = weight x density x t (the
 * Jacobian of u), and E[T] from the same nodes. */
typedef struct {
    double *t, *G;
    int M;
    double et;
} t_grid;

static int grid_build(int mode, int N, double ne, double K, int k, double pfa, t_grid *g) {
    const double ln_eps = log(1e-9 * pfa);
    const double lo = -700.0, hi = 7.0;
    double cdf, sf, u_lo, u_hi;
    t_log_cdf_sf(mode, exp(lo), N, ne, K, k, &cdf, &sf);
    if (cdf >= ln_eps) {
        u_lo = lo;
    } else {
        double a = lo, b = hi;
        for (int i = 0; i < 60; ++i) {
            const double mid = 0.5 * (a + b);
            t_log_cdf_sf(mode, exp(mid), N, ne, K, k, &cdf, &sf);
            if (cdf < ln_eps) a = mid;
            else b = mid;
        }
        u_lo = a;
    }
    t_log_cdf_sf(mode, exp(hi), N, ne, K, k, &cdf, &sf);
    if (sf > ln_eps) {
        u_hi = hi;
    } else {
        double a = u_lo, b = hi;
        for (int i = 0; i < 60; ++i) {
            const double mid = 0.5 * (a + b);
            t_log_cdf_sf(mode, exp(mid), N, ne, K, k, &cdf, &sf);
            if (sf > ln_eps) a = mid;
            else b = mid;
        }
        u_hi = b;
    }
    const double shape = (mode == ATKDSP_CFAR_GO || mode == ATKDSP_CFAR_SO) ? 0.5 * ne * K : ne * K;
    double h0 = 0.2 / sqrt(shape);
    if (h0 > 0.01) h0 = 0.01;
    const double span = u_hi - u_lo;
    long M = 2 * (long)ceil(span / (2.0 * h0));
    if (M < 512) M = 512;
    if (M > CF_MAX_GRID) M = CF_MAX_GRID;
    const double h = span / (double)M;
    g->M = (int)M;
    g->t = (double *)malloc((size_t)(M + 1) * sizeof(double));
    g->G = (double *)malloc((size_t)(M + 1) * sizeof(double));
    if (!g->t || !g->G) {
        free(g->t);
        free(g->G);
        g->t = g->G = NULL;
        return ATKDSP_E_NOMEM;
    }
    for (long j = 0; j <= M; ++j) {
        const double u = u_lo + h * (double)j;
        const double t = exp(u);
        double w = (j == 0 || j == M) ? 1.0 : ((j & 1) ? 4.0 : 2.0);
        w *= h / 3.0;
        const double lg = t_log_density(mode, t, N, ne, K, k) + u;
        g->t[j] = t;
        g->G[j] = isfinite(lg) ? exp(lg) * w : 0.0;
    }
    double et = 0.0;
    for (long j = 0; j <= M; ++j) et += g->G[j] * g->t[j];
    g->et = et;
    return ATKDSP_OK;
}

static void grid_free(t_grid *g) {
    free(g->t);
    free(g->G);
}

/* Pfa at alpha: the integral of Q(K, K alpha t) over T's density */
static double grid_pfa(const t_grid *g, double K, double alpha) {
    double s = 0.0;
    for (int j = 0; j <= g->M; ++j) {
        double lp, lq;
        log_igam(K, K * alpha * g->t[j], &lp, &lq);
        s += g->G[j] * exp(lq);
    }
    return s;
}

static double pfa_gap(const t_grid *g, double K, double v, double ln_pfa) {
    double p = grid_pfa(g, K, exp(v));
    if (p < 1e-300) p = 1e-300;
    return log(p) - ln_pfa;
}

/* regula falsi (Illinois) in v = ln alpha over [ln 1e-3, ln 1e18] */
static int solve_alpha(int mode, int N, double ne, double K, int k, double pfa, double *alpha, double *et) {
    t_grid g;
    const int rc = grid_build(mode, N, ne, K, k, pfa, &g);
    if (rc) return rc;
    const double ln_pfa = log(pfa);
    double a = log(1e-3), b = log(1e18);
    double fa = pfa_gap(&g, K, a, ln_pfa), fb = pfa_gap(&g, K, b, ln_pfa);
    if (!(fa > 0.0 && fb < 0.0)) {
        grid_free(&g);
        return ATKDSP_E_ARG;
    }
    int side = 0, have_prev = 0;
    double c = a, prev = 0.0;
    for (int it = 0; it < 300; ++it) {
        c = (a * fb - b * fa) / (fb - fa);
        const double fc = pfa_gap(&g, K, c, ln_pfa);
        if (fc == 0.0) break;
        if (fc > 0.0) {
            a = c;
            fa = fc;
            if (side == 1) fb *= 0.5;
            side = 1;
        } else {
            b = c;
            fb = fc;
            if (side == -1) fa *= 0.5;
            side = -1;
        }
        if (have_prev && fabs(c - prev) <= 1e-14 * (fabs(c) > 1.0 ? fabs(c) : 1.0)) break;
        prev = c;
        have_prev = 1;
    }
    *alpha = exp(c);
    if (et) *et = g.et;
    grid_free(&g);
    return ATKDSP_OK;
}

static int rho2_valid(const double *rho2) {
    if (!rho2) return 1;
    for (int m = 0; m < ATKDSP_CFAR_RHO_MAX; ++m)
        if (!(rho2[m] >= 0.0 && rho2[m] < 1.0)) return 0;
    return 1;
}

ATKDSP_API double atkdsp_cfar_n_eff(int n_ref, const double *rho2) {
    const double N = 2.0 * (double)n_ref;
    if (n_ref < 1) return 0.0;
    if (!rho2) return N;
    double pairs = 0.0;
    for (int m = 1; m <= ATKDSP_CFAR_RHO_MAX && m < n_ref; ++m) pairs += 2.0 * (double)(n_ref - m) * rho2[m - 1];
    return N / (1.0 + 2.0 * pairs / N);
}

ATKDSP_API int atkdsp_cfar_window_rho2(const float *window, size_t n, double *rho2) {
    if (!window || !rho2 || n < 2) return ATKDSP_E_ARG;
    double s2 = 0.0;
    for (size_t i = 0; i < n; ++i) s2 += (double)window[i] * (double)window[i];
    if (!(s2 > 0.0)) return ATKDSP_E_ARG;
    for (int m = 1; m <= ATKDSP_CFAR_RHO_MAX; ++m) {
        double re = 0.0, im = 0.0;
        for (size_t i = 0; i < n; ++i) {
            const double w2 = (double)window[i] * (double)window[i];
            const double ph = -2.0 * CF_PI * (double)m * (double)i / (double)n;
            re += w2 * cos(ph);
            im += w2 * sin(ph);
        }
        rho2[m - 1] = (re * re + im * im) / (s2 * s2);
    }
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_cfar_alpha(int mode, int n_ref, double pfa, double looks, int os_k, const double *rho2,
                                 double *alpha, double *et) {
    if (mode < 0 || mode > 3 || n_ref < 1 || n_ref > 256 || !(pfa >= 1e-15 && pfa <= 0.5) ||
        !(looks >= 0.25 && looks <= 64e6) || !alpha || !rho2_valid(rho2))
        return ATKDSP_E_ARG;
    const int N = 2 * n_ref;
    const int k = os_k ? os_k : (3 * N + 3) / 4;
    if (mode == ATKDSP_CFAR_OS && (k < 1 || k > N)) return ATKDSP_E_ARG;
    const double ne = atkdsp_cfar_n_eff(n_ref, rho2);
    if (mode != ATKDSP_CFAR_OS || ne == (double)N) return solve_alpha(mode, N, ne, looks, k, pfa, alpha, et);
    /* OS with correlated cells: solve CA at the effective count, take the rate
     * the independent-cell CA test has at that alpha, and solve the order
     * statistic (integer N and rank) at that rate */
    double a_eff, rate;
    int rc = solve_alpha(ATKDSP_CFAR_CA, N, ne, looks, 0, pfa, &a_eff, NULL);
    if (rc) return rc;
    t_grid g;
    rc = grid_build(ATKDSP_CFAR_CA, N, (double)N, looks, 0, pfa, &g);
    if (rc) return rc;
    rate = grid_pfa(&g, looks, a_eff);
    grid_free(&g);
    if (!(rate > 0.0)) rate = 1e-300;
    return solve_alpha(mode, N, (double)N, looks, k, rate, alpha, et);
}

/* beta with P(Gamma(s) / s > beta) = ATKDSP_CFAR_EDGE_PFA for the equivalent
 * independent count among nb contiguous bins (the single-frame band test) */
static double edge_beta(int nb, double looks, const double *rho2) {
    double pairs = 0.0;
    for (int m = 1; m <= ATKDSP_CFAR_RHO_MAX && m < nb; ++m) pairs += (double)(nb - m) * rho2[m - 1];
    const double s = (double)nb / (1.0 + 2.0 * pairs / (double)nb) * looks;
    const double target = log(ATKDSP_CFAR_EDGE_PFA);
    double a = log(1e-6), b = log(1e6);
    for (int i = 0; i < 100; ++i) {
        const double mid = 0.5 * (a + b);
        double lp, lq;
        log_igam(s, s * exp(mid), &lp, &lq);
        if (lq > target) a = mid;
        else b = mid;
    }
    return exp(b);
}

/* ================================================= the handle */

typedef struct {
    uint32_t id;
    int state;                    /* 0 pending, 1 open */
    uint64_t hist;                /* hit frames, newest in bit 0 */
    int misses, is_new;
    int32_t n_hits, cur_lo, cur_hi, ulo, uhi;
    double sbe, se, px, pn, band;
    uint32_t flags;
    double t0;
    int64_t last_hit, last_raw;
    double t_hit_end, dt_hit, t_raw_end;
    int has_obs;                  /* this frame's observation */
    int32_t olo, ohi;
    double fsx, fsn;
} cf_track;

typedef struct {
    int32_t lo, hi;
    double sbe, se, sx, sn, px, pn;
    int track;
} cf_blob;


struct atkdsp_cfar {
    atkdsp_cfar_config cfg;
    size_t nbins;
    int N;
    double n_eff, K, alpha, alpha_ca, et;
    uint8_t *mask, *ok, *sided;
    size_t n_ok, n_untestable;    /* per tested frame */
    double *beta;                 /* edge test thresholds by band width, NaN until used */
    cf_track *tracks;
    int ntracks;
    uint32_t next_id;
    cf_blob *blobs;
    atkdsp_cfar_counters st;
    int64_t seen, frame;
    int has_last;
    double *last_X, *last_thr;
    uint8_t *last_hits;
    /* device: tables; the raw ring (frame F in row F % ring); two sets of a
     * pass's rows (hits, X, noise, thr); a pass's rows at its columns */
    int fc, ring;
    void *stream, *gstream, *ev_in, *ev_pass[2];
    uint8_t *d_ok, *d_sided, *d_hits;
    uint32_t *d_bits;             /* hit rows as bits, `words` per row */
    size_t words;
    int32_t *d_idx, *d_cols;
    double *d_raw, *d_X, *d_noise, *d_thr;
    double *d_Xc, *d_Nc, *d_Rc;
    float *d_frames;
    /* host (pinned when small): two sets of hit bit rows; the gathered rows of
     * the pass being tracked: X and noise of its tested frames, raw of those
     * frames and the k - 1 before them, all at the pass's columns */
    int pinned;
    uint32_t *h_bits;
    double *h_Xc, *h_Nc, *h_Rc;
    int32_t *h_cols, *colmap;     /* colmap[bin]: its column, -1 outside */
    int ncol;
    int64_t rc_f0;                /* the frame of h_Rc's row 0 */
    uint32_t *orm;                /* a pass's hit rows and live spans, OR-ed */
    double *ht, *hd;              /* frame start and duration by ring row */
};

ATKDSP_API void atkdsp_cfar_defaults(atkdsp_cfar_config *c) {
    if (!c) return;
    memset(c, 0, sizeof *c);
    c->mode = ATKDSP_CFAR_CA;
    c->n_ref = 16;
    c->n_guard = 4;
    c->k_frames = 1;
    c->pfa = 1e-6;
    c->looks = 1.0;
    c->open_m = 2;
    c->open_n = 3;
    c->close_k = 3;
    c->merge_gap = 1;
    c->min_bins = 1;
    c->max_tracks = 256;
}

/* the reference's ranges (src/cfar.c:324-340) */
static int config_valid(size_t nbins, const atkdsp_cfar_config *c) {
    const long N = 2L * c->n_ref;
    if (c->mode < 0 || c->mode > 3) return 0;
    if (c->n_ref < 1 || c->n_ref > 256 || c->n_guard < 0 || c->n_guard > 256) return 0;
    if (nbins < (size_t)(N + 2L * c->n_guard + 1) || nbins > ((size_t)1 << 24) ||
        (double)nbins * (double)N > (double)((size_t)1 << 26))
        return 0;
    if (c->k_frames < 1 || c->k_frames > 64 || !(c->looks >= 0.25 && c->looks <= 1e4)) return 0;
    if (!(c->pfa >= 1e-15 && c->pfa <= 0.5)) return 0;
    if (c->mode == ATKDSP_CFAR_OS && (c->os_k < 0 || c->os_k > N)) return 0;
    if (c->open_n < 1 || c->open_n > 64 || c->open_m < 1 || c->open_m > c->open_n) return 0;
    if (c->close_k < 1 || c->close_k > 1000 || c->merge_gap < 0 || (size_t)c->merge_gap > nbins) return 0;
    if (c->min_bins < 1 || (size_t)c->min_bins > nbins || c->max_tracks < 1 || c->max_tracks > 65536) return 0;
    return rho2_valid(c->rho2);
}

/* Every bin's reference cells, cell-major for the device (idx[q * nbins +
 * i]): the nearest unmasked cells beyond the guard on the left, then on the
 * right, then what a short side borrows from beyond the other side's far
 * end (first the right's, then the left's). A bin that cannot gather N cells
 * is untestable; `sided` marks bins that borrowed nothing. */
static int tables_build(atkdsp_cfar *c) {
    const long nb = (long)c->nbins, nr = c->cfg.n_ref, ng = c->cfg.n_guard, N = c->N;
    const uint8_t *m = c->mask;
    int32_t *idx = (int32_t *)malloc((size_t)nb * (size_t)N * sizeof(int32_t));
    int32_t *cells = (int32_t *)malloc((size_t)(2 * N) * sizeof(int32_t));
    if (!idx || !cells) {
        free(idx);
        free(cells);
        return ATKB_E_NOMEM;
    }
    c->n_ok = c->n_untestable = 0;
    for (long i = 0; i < nb; ++i) {
        c->ok[i] = 0;
        c->sided[i] = 0;
        for (long q = 0; q < N; ++q) idx[q * nb + i] = (int32_t)i;   /* untestable: never read */
        if (m[i]) continue;
        long nl = 0, nrt = 0, nx = 0;
        int32_t *left = cells, *right = cells + nr, *ext = cells + N;
        long j = i - ng - 1;
        while (j >= 0 && nl < nr) {
            if (!m[j]) left[nl++] = (int32_t)j;
            --j;
        }
        const long jl = j;
        j = i + ng + 1;
        while (j < nb && nrt < nr) {
            if (!m[j]) right[nrt++] = (int32_t)j;
            ++j;
        }
        const long jr = j;
        long short_l = nr - nl, short_r = nr - nrt;
        for (j = jr; short_l > 0 && j < nb; ++j)
            if (!m[j]) {
                ext[nx++] = (int32_t)j;
                --short_l;
            }
        for (j = jl; short_r > 0 && j >= 0; --j)
            if (!m[j]) {
                ext[nx++] = (int32_t)j;
                --short_r;
            }
        if (nl + nrt + nx < N) {
            ++c->n_untestable;
            continue;
        }
        long o = 0;
        for (long q = 0; q < nl; ++q) idx[(o++) * nb + i] = left[q];
        for (long q = 0; q < nrt; ++q) idx[(o++) * nb + i] = right[q];
        for (long q = 0; q < nx; ++q) idx[(o++) * nb + i] = ext[q];
        c->ok[i] = 1;
        c->sided[i] = nx == 0;
        ++c->n_ok;
    }
    free(cells);
    int rc = atkb_h2d(c->d_idx, idx, (size_t)nb * (size_t)N * sizeof(int32_t), c->stream);
    if (rc == ATKB_OK) rc = atkb_h2d(c->d_ok, c->ok, (size_t)nb, c->stream);
    if (rc == ATKB_OK) rc = atkb_h2d(c->d_sided, c->sided, (size_t)nb, c->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(c->stream);
    free(idx);
    return rc;
}

static void *host_buf(atkdsp_cfar *c, size_t bytes) {
    if (c->pinned) {
        void *p = NULL;
        return atkb_host_alloc(&p, bytes) == ATKB_OK ? p : NULL;
    }
    return malloc(bytes);
}

static void host_buf_free(const atkdsp_cfar *c, void *p) {
    if (!p) return;
    if (c->pinned) atkb_host_free(p);
    else free(p);
}

ATKDSP_API void atkdsp_cfar_destroy(atkdsp_cfar *c) {
    if (!c) return;
    if (c->stream) atkb_stream_sync(c->stream);
    free(c->mask);
    free(c->ok);
    free(c->sided);
    free(c->beta);
    free(c->tracks);
    free(c->blobs);
    free(c->last_X);
    free(c->last_thr);
    free(c->last_hits);
    free(c->ht);
    free(c->hd);
    host_buf_free(c, c->h_bits);
    host_buf_free(c, c->h_Xc);
    host_buf_free(c, c->h_Nc);
    host_buf_free(c, c->h_Rc);
    host_buf_free(c, c->h_cols);
    free(c->colmap);
    free(c->orm);
    atkb_free(c->d_ok);
    atkb_free(c->d_sided);
    atkb_free(c->d_idx);
    atkb_free(c->d_hits);
    atkb_free(c->d_bits);
    atkb_free(c->d_raw);
    atkb_free(c->d_X);
    atkb_free(c->d_noise);
    atkb_free(c->d_thr);
    atkb_free(c->d_cols);
    atkb_free(c->d_Xc);
    atkb_free(c->d_Nc);
    atkb_free(c->d_Rc);
    atkb_free(c->d_frames);
    if (c->ev_in) atkb_event_destroy(c->ev_in);
    if (c->ev_pass[0]) atkb_event_destroy(c->ev_pass[0]);
    if (c->ev_pass[1]) atkb_event_destroy(c->ev_pass[1]);
    if (c->stream) atkb_stream_destroy(c->stream);
    if (c->gstream) atkb_stream_destroy(c->gstream);
    free(c);
}

ATKDSP_API atkdsp_cfar *atkdsp_cfar_create(size_t nbins, const atkdsp_cfar_config *cfg) {
    if (!cfg || !config_valid(nbins, cfg)) return NULL;
    atkdsp_cfar *c = (atkdsp_cfar *)calloc(1, sizeof *c);
    if (!c) return NULL;
    c->cfg = *cfg;
    c->nbins = nbins;
    c->N = 2 * cfg->n_ref;
    if (c->cfg.mode == ATKDSP_CFAR_OS && c->cfg.os_k == 0) c->cfg.os_k = (3 * c->N + 3) / 4;
    c->K = c->cfg.looks * (double)c->cfg.k_frames;
    c->n_eff = atkdsp_cfar_n_eff(c->cfg.n_ref, c->cfg.rho2);
    if (atkdsp_cfar_alpha(c->cfg.mode, c->cfg.n_ref, c->cfg.pfa, c->K, c->cfg.os_k, c->cfg.rho2, &c->alpha,
                          &c->et) != ATKDSP_OK) {
        free(c);
        return NULL;
    }
    if (c->cfg.mode == ATKDSP_CFAR_GO || c->cfg.mode == ATKDSP_CFAR_SO) {
        if (atkdsp_cfar_alpha(ATKDSP_CFAR_CA, c->cfg.n_ref, c->cfg.pfa, c->K, 0, c->cfg.rho2, &c->alpha_ca,
                              NULL) != ATKDSP_OK) {
            free(c);
            return NULL;
        }
    } else {
        c->alpha_ca = c->alpha;
    }
    const int k = c->cfg.k_frames;
    size_t fc = CF_PASS_CELLS / nbins;
    if (fc < 1) fc = 1;
    if (fc > CF_PASS_FRAMES) fc = CF_PASS_FRAMES;
    c->fc = (int)fc;
    c->ring = 2 * c->fc + k - 1;
    const size_t nb = nbins, rows = (size_t)c->fc, ring = (size_t)c->ring;
    const size_t rrows = rows + (size_t)k - 1;     /* raw rows a pass's tracker reads */
    c->words = (nb + 31) / 32;
    const size_t W = c->words;
    c->pinned = (2 * rows * W * 4 + 2 * rows * nb * 8 + (k > 1 ? rrows * nb * 8 : 0) + nb * 4) <= CF_PINNED_MAX;
    c->next_id = 1;
    c->mask = (uint8_t *)calloc(nb, 1);
    c->ok = (uint8_t *)calloc(nb, 1);
    c->sided = (uint8_t *)calloc(nb, 1);
    c->beta = (double *)malloc((nb + 1) * sizeof(double));
    c->tracks = (cf_track *)calloc((size_t)c->cfg.max_tracks, sizeof(cf_track));
    c->blobs = (cf_blob *)calloc(nb, sizeof(cf_blob));
    c->last_X = (double *)calloc(nb, sizeof(double));
    c->last_thr = (double *)calloc(nb, sizeof(double));
    c->last_hits = (uint8_t *)calloc(nb, 1);
    c->ht = (double *)calloc(ring, sizeof(double));
    c->hd = (double *)calloc(ring, sizeof(double));
    c->colmap = (int32_t *)malloc(nb * sizeof(int32_t));
    c->orm = (uint32_t *)malloc(((nb + 31) / 32) * sizeof(uint32_t));
    int rc = (c->mask && c->ok && c->sided && c->beta && c->tracks && c->blobs && c->last_X && c->last_thr &&
              c->last_hits && c->ht && c->hd && c->colmap && c->orm)
                 ? ATKB_OK
                 : ATKB_E_NOMEM;
    if (rc == ATKB_OK) {
        for (size_t i = 0; i < nb; ++i) c->colmap[i] = -1;
        c->h_bits = (uint32_t *)host_buf(c, 2 * rows * W * sizeof(uint32_t));
        c->h_Xc = (double *)host_buf(c, rows * nb * sizeof(double));
        c->h_Nc = (double *)host_buf(c, rows * nb * sizeof(double));
        if (k > 1) c->h_Rc = (double *)host_buf(c, rrows * nb * sizeof(double));
        c->h_cols = (int32_t *)host_buf(c, nb * sizeof(int32_t));
        if (!c->h_bits || !c->h_Xc || !c->h_Nc || (k > 1 && !c->h_Rc) || !c->h_cols) rc = ATKB_E_NOMEM;
    }
    if (rc == ATKB_OK) rc = atkb_stream_create(&c->stream);
    if (rc == ATKB_OK) rc = atkb_stream_create(&c->gstream);
    if (rc == ATKB_OK) rc = atkb_event_create(&c->ev_in);
    if (rc == ATKB_OK) rc = atkb_event_create(&c->ev_pass[0]);
    if (rc == ATKB_OK) rc = atkb_event_create(&c->ev_pass[1]);
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_ok, nb);
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_sided, nb);
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_idx, nb * (size_t)c->N * sizeof(int32_t));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_raw, ring * nb * sizeof(double));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_X, 2 * rows * nb * sizeof(double));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_noise, 2 * rows * nb * sizeof(double));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_thr, 2 * rows * nb * sizeof(double));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_hits, 2 * rows * nb);
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_bits, 2 * rows * W * sizeof(uint32_t));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_cols, nb * sizeof(int32_t));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_Xc, rows * nb * sizeof(double));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_Nc, rows * nb * sizeof(double));
    if (rc == ATKB_OK && k > 1) rc = atkb_malloc((void **)&c->d_Rc, rrows * nb * sizeof(double));
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&c->d_frames, rows * nb * sizeof(float));
    if (rc == ATKB_OK) rc = tables_build(c);
    if (rc != ATKB_OK) {
        atkdsp_cfar_destroy(c);
        return NULL;
    }
    for (size_t i = 0; i <= nb; ++i) c->beta[i] = NAN;
    return c;
}

ATKDSP_API void atkdsp_cfar_reset(atkdsp_cfar *c) {
    if (!c) return;
    c->ntracks = 0;
    c->seen = 0;
    c->frame = 0;
    c->has_last = 0;
    c->st.resets++;
}

ATKDSP_API int atkdsp_cfar_set_mask(atkdsp_cfar *c, const uint8_t *mask) {
    if (!c) return ATKDSP_E_ARG;
    for (size_t i = 0; i < c->nbins; ++i) c->mask[i] = mask ? (mask[i] != 0) : 0;
    return atkb_map_rc(tables_build(c));
}

ATKDSP_API size_t atkdsp_cfar_events_max(const atkdsp_cfar *c, size_t nframes) {
    return c ? nframes * (size_t)c->cfg.max_tracks : 0;
}

/* ================================================= the tracker */

static double band_beta(atkdsp_cfar *c, int nb) {
    if (isnan(c->beta[nb])) c->beta[nb] = edge_beta(nb, c->cfg.looks, c->cfg.rho2);
    return c->beta[nb];
}

/* the single-frame band test: the raw power over the testable bins of
 * [lo, hi] against beta x their noise (this frame's estimate); raw and
 * noise are rows at the pass's columns */
static int band_pass(atkdsp_cfar *c, const double *raw, const double *noise, int32_t lo, int32_t hi) {
    const int32_t *cm = c->colmap;
    double sr = 0.0, sz = 0.0;
    int nb = 0;
    for (int32_t b = lo; b <= hi; ++b) {
        if (c->ok[b]) {
            sr += raw[cm[b]];
            sz += noise[cm[b]];
            ++nb;
        }
    }
    return nb > 0 && sr > band_beta(c, nb) * sz;
}

static uint32_t track_flags(const atkdsp_cfar *c, const cf_track *t) {
    uint32_t f = t->flags;
    for (int32_t b = t->ulo; b <= t->uhi; ++b)
        if (!c->sided[b] || !c->ok[b]) {
            f |= ATKDSP_CFAR_EDGE;
            break;
        }
    const long m = c->cfg.merge_gap + 1;
    long a = (long)t->ulo - m, z = (long)t->uhi + m + 1;
    if (a < 0) a = 0;
    if (z > (long)c->nbins) z = (long)c->nbins;
    for (long b = a; b < z; ++b)
        if (c->mask[b]) {
            f |= ATKDSP_CFAR_MASK_ADJ;
            break;
        }
    return f;
}

static void emit(const atkdsp_cfar *c, const cf_track *t, int type, double t1, uint32_t extra, atkdsp_cfar_event *e) {
    memset(e, 0, sizeof *e);
    e->type = type;
    e->id = t->id;
    e->flags = track_flags(c, t) | extra;
    e->lo_bin = t->ulo;
    e->hi_bin = t->uhi;
    e->n_hits = t->n_hits;
    e->t0 = t->t0;
    e->t1 = t1;
    e->fc_bin = t->se > 0.0 ? t->sbe / t->se : 0.5 * ((double)t->ulo + (double)t->uhi);
    e->level_db = t->px > 0.0 ? (float)(10.0 * log10(t->px)) : -INFINITY;
    e->noise_db = t->pn > 0.0 ? (float)(10.0 * log10(t->pn)) : -INFINITY;
    e->snr_db = t->pn > 0.0 ? e->level_db - e->noise_db : INFINITY;
    e->band_snr_db = t->band > 0.0 ? (float)(10.0 * log10(t->band)) : -INFINITY;
}

static void emit_close(atkdsp_cfar *c, cf_track *t, uint32_t extra, atkdsp_cfar_event *e) {
    const int k = c->cfg.k_frames;
    double t1;
    if (k == 1) {
        t1 = t->t_hit_end;
    } else if (t->last_raw >= t->last_hit - (k - 1)) {
        t1 = t->t_raw_end;
    } else {
        t1 = t->t_hit_end - 0.5 * (double)(k - 1) * t->dt_hit;
        t->flags |= ATKDSP_CFAR_T1_COARSE;
    }
    c->st.closed++;
    emit(c, t, ATKDSP_CFAR_CLOSE, t1, extra, e);
}

static int popcount64(uint64_t x) {
    int n = 0;
    while (x) {
        x &= x - 1;
        ++n;
    }
    return n;
}

/* hit rows are bitmasks: bin b is bit b % 32 of word b / 32 */
static int bit_at(const uint32_t *w, long b) { return (int)((w[b >> 5] >> (b & 31)) & 1u); }

/* the first hit at or after i (nb if none), 32 bins a word */
static long next_hit(const uint32_t *w, long i, long nb) {
    if (i >= nb) return nb;
    const long nw = (nb + 31) >> 5;
    long q = i >> 5;
    uint32_t m = w[q] & (0xffffffffu << (i & 31));
    while (!m) {
        if (++q >= nw) return nb;
        m = w[q];
    }
    const long r = (q << 5) + __builtin_ctz(m);
    return r < nb ? r : nb;
}

/* One tested frame F (absolute): its hit row (every bin) and its X and noise
 * rows at the pass's columns (colmap), the raw rows at the same columns
 * from h_Rc. Every bin the tracker reads is a column: the pass's blobs and
 * every span a track can take during the pass lie in them (pass_columns).
 * Returns the events written. */
static size_t track_frame(atkdsp_cfar *c, int64_t F, const double *X, const double *noise, const uint32_t *hits,
                          double tf, double dt, atkdsp_cfar_event *ev) {
    const long nb = (long)c->nbins;
    const int k = c->cfg.k_frames;
    const int32_t *cm = c->colmap;
    const double *raw = k > 1 ? c->h_Rc + (size_t)(F - c->rc_f0) * (size_t)c->ncol : NULL;
    c->st.cells_tested += c->n_ok;
    c->st.untestable += c->n_untestable;

    /* blobs: hit runs with gaps of at most merge_gap non-hit bins */
    const long g = c->cfg.merge_gap;
    size_t nblob = 0;
    uint64_t nhit = 0;
    long i = 0;
    while ((i = next_hit(hits, i, nb)) < nb) {
        long lo = i, hi = i, prev = i;
        for (long j; (j = next_hit(hits, prev + 1, nb)) < nb && j - prev - 1 <= g;) {
            hi = j;
            prev = j;
        }
        for (long b = lo; b <= hi; ++b) nhit += (uint64_t)bit_at(hits, b);
        i = hi + 1;
        if (hi - lo + 1 < c->cfg.min_bins) continue;
        cf_blob *o = &c->blobs[nblob++];
        o->lo = (int32_t)lo;
        o->hi = (int32_t)hi;
        o->sbe = o->se = o->sx = o->sn = 0.0;
        long pk = -1;
        for (long b = lo; b <= hi; ++b) {
            if (!bit_at(hits, b)) continue;
            const double xb = X[cm[b]], nz = noise[cm[b]];
            double e = xb - nz;
            if (e < 0.0) e = 0.0;
            o->sbe += (double)b * e;
            o->se += e;
            o->sx += xb;
            o->sn += nz;
            if (pk < 0 || xb > X[cm[pk]]) pk = b;
        }
        o->px = X[cm[pk]];
        o->pn = noise[cm[pk]];
        o->track = -1;
    }
    c->st.cell_hits += nhit;

    /* association: each blob to the existing track it overlaps most (within
     * merge_gap + 1 bins; ties keep the older track) */
    const int nexist = c->ntracks;
    for (int t = 0; t < nexist; ++t) c->tracks[t].has_obs = 0;
    const long reach = g + 1;
    for (size_t q = 0; q < nblob; ++q) {
        cf_blob *o = &c->blobs[q];
        int best = -1;
        long bov = 0;
        for (int t = 0; t < nexist; ++t) {
            const cf_track *tr = &c->tracks[t];
            if ((long)o->lo <= (long)tr->cur_hi + reach && (long)o->hi >= (long)tr->cur_lo - reach) {
                const long ov = (long)(o->hi < tr->cur_hi ? o->hi : tr->cur_hi) -
                                (long)(o->lo > tr->cur_lo ? o->lo : tr->cur_lo) + 1;
                if (best < 0 || ov > bov) {
                    best = t;
                    bov = ov;
                }
            }
        }
        o->track = best;
    }
    /* unclaimed blobs start pending tracks, up to max_tracks */
    for (size_t q = 0; q < nblob; ++q) {
        cf_blob *o = &c->blobs[q];
        if (o->track >= 0) continue;
        if (c->ntracks >= c->cfg.max_tracks) {
            c->st.dropped++;
            continue;
        }
        cf_track *tr = &c->tracks[c->ntracks];
        memset(tr, 0, sizeof *tr);
        tr->id = c->next_id;
        c->next_id = c->next_id + 1 ? c->next_id + 1 : 1;
        tr->cur_lo = tr->ulo = o->lo;
        tr->cur_hi = tr->uhi = o->hi;
        tr->px = -1.0;
        tr->last_hit = -1;
        tr->last_raw = -1;
        tr->dt_hit = dt;
        tr->is_new = 1;
        o->track = c->ntracks++;
    }
    /* each track's observation: its blobs in blob order */
    for (size_t q = 0; q < nblob; ++q) {
        const cf_blob *o = &c->blobs[q];
        if (o->track < 0) continue;
        cf_track *tr = &c->tracks[o->track];
        if (!tr->has_obs) {
            tr->has_obs = 1;
            tr->olo = o->lo;
            tr->ohi = o->hi;
            tr->fsx = 0.0;
            tr->fsn = 0.0;
        } else {
            if (o->lo < tr->olo) tr->olo = o->lo;
            if (o->hi > tr->ohi) tr->ohi = o->hi;
        }
        tr->sbe += o->sbe;
        tr->se += o->se;
        tr->fsx += o->sx;
        tr->fsn += o->sn;
        if (o->px > tr->px) {
            tr->px = o->px;
            tr->pn = o->pn;
        }
    }

    /* update in id order, compacting */
    const uint64_t window = (c->cfg.open_n >= 64) ? ~(uint64_t)0 : (((uint64_t)1 << c->cfg.open_n) - 1);
    size_t nev = 0;
    int keep = 0;
    for (int t = 0; t < c->ntracks; ++t) {
        cf_track *tr = &c->tracks[t];
        int grew = 0;
        if (tr->has_obs) {
            const int32_t lo = tr->olo, hi = tr->ohi;
            tr->hist = ((tr->hist << 1) | 1u) & window;
            tr->misses = 0;
            tr->n_hits++;
            tr->cur_lo = lo;
            tr->cur_hi = hi;
            if (!tr->is_new) grew = lo < tr->ulo || hi > tr->uhi;
            if (lo < tr->ulo) tr->ulo = lo;
            if (hi > tr->uhi) tr->uhi = hi;
            if (tr->fsn > 0.0 && tr->fsx / tr->fsn > tr->band) tr->band = tr->fsx / tr->fsn;
            tr->last_hit = F;
            tr->t_hit_end = tf + dt;
            tr->dt_hit = dt;
            if (tr->is_new) {
                tr->is_new = 0;
                if (k == 1) {
                    tr->t0 = tf;
                } else {
                    /* the earliest of the k raw frames up to this one whose band passes */
                    int found = 0;
                    for (int r = 0; r < k; ++r) {
                        const int64_t Fr = F - k + 1 + r;
                        const size_t row = (size_t)(Fr % c->ring);
                        if (band_pass(c, c->h_Rc + (size_t)(Fr - c->rc_f0) * (size_t)c->ncol, noise, lo, hi)) {
                            tr->t0 = c->ht[row];
                            found = 1;
                            break;
                        }
                    }
                    if (!found) {
                        tr->t0 = tf - 0.5 * (double)(k - 1) * dt;
                        tr->flags |= ATKDSP_CFAR_T0_COARSE;
                    }
                }
            }
        } else {
            tr->hist = (tr->hist << 1) & window;
            tr->misses++;
        }
        tr->has_obs = 0;
        if (k > 1 && band_pass(c, raw, noise, tr->cur_lo, tr->cur_hi)) {
            tr->last_raw = F;
            tr->t_raw_end = tf + dt;
        }
        if (tr->state == 0) {
            if (popcount64(tr->hist) >= c->cfg.open_m) {
                tr->state = 1;
                c->st.opened++;
                emit(c, tr, ATKDSP_CFAR_OPEN, NAN, 0, &ev[nev++]);
            } else if (tr->hist == 0) {
                continue;
            }
        } else if (tr->misses >= c->cfg.close_k) {
            emit_close(c, tr, 0, &ev[nev++]);
            continue;
        } else if (grew) {
            c->st.updates++;
            emit(c, tr, ATKDSP_CFAR_UPDATE, NAN, 0, &ev[nev++]);
        }
        if (keep != t) c->tracks[keep] = *tr;
        ++keep;
    }
    c->ntracks = keep;
    return nev;
}

/* ================================================= a call */

/* One pass: frames [done, done + nf) of a call; F0 the absolute frame of its
 * first, j0 its first tested frame (earlier ones are warm-up). */
typedef struct {
    size_t done;
    int nf;
    int64_t F0, j0;
} cf_pass;

/* Enqueue a pass on the handle's stream: conversion into the raw ring, the
 * test into device row set `set`, the hit rows into host set `set`, the
 * caller's device hit masks. Nothing waits. */
static int pass_enqueue(atkdsp_cfar *c, const cf_pass *ps, const float *frames, int on_device, int units, int set,
                        uint8_t *d_hits_out) {
    const size_t nb = c->nbins, hs = (size_t)set * (size_t)c->fc * nb, W = c->words;
    const size_t bs = (size_t)set * (size_t)c->fc * W;
    const int k = c->cfg.k_frames, nf = ps->nf;
    const int64_t F0 = ps->F0, j0 = ps->j0;
    const float *src = frames + ps->done * nb;
    int rc = ATKB_OK;
    if (!on_device) {
        rc = atkb_h2d(c->d_frames, src, (size_t)nf * nb * sizeof(float), c->stream);
        src = c->d_frames;
    }
    if (rc == ATKB_OK) rc = atkb_cfar_raw(src, units, F0, nf, (long long)nb, c->d_raw, c->ring, c->stream);
    if (rc == ATKB_OK && j0 < nf)
        rc = atkb_cfar_test(c->d_raw, c->ring, F0, F0 + j0, nf, (long long)nb, k, c->cfg.mode, c->cfg.n_ref, c->N,
                            c->cfg.os_k, c->alpha, c->alpha_ca, c->et, c->d_ok, c->d_sided, c->d_idx, c->d_X + hs,
                            c->d_noise + hs, c->d_thr + hs, c->d_hits + hs, c->d_bits + bs, (long long)W,
                            c->stream);
    if (rc == ATKB_OK && j0 < nf) {
        const size_t off = (size_t)j0 * nb, rows = (size_t)(nf - j0) * nb;
        rc = atkb_d2h(c->h_bits + bs + (size_t)j0 * W, c->d_bits + bs + (size_t)j0 * W,
                      (size_t)(nf - j0) * W * sizeof(uint32_t), c->stream);
        if (rc == ATKB_OK && d_hits_out)
            rc = atkb_d2d(d_hits_out + (ps->done + (size_t)j0) * nb, c->d_hits + hs + off, rows, c->stream);
    }
    if (rc == ATKB_OK && d_hits_out && j0 > 0)
        rc = atkb_memset(d_hits_out + ps->done * nb, 0, (size_t)(j0 < nf ? j0 : nf) * nb, c->stream);
    if (rc == ATKB_OK) rc = atkb_event_record(c->ev_pass[set], c->stream);
    return rc;
}

/* The bins the tracker can read while it walks a pass, as columns (h_cols,
 * colmap): the runs of hits of the pass's tested frames (bit rows j0..nf-1
 * of `hits`) and the spans of the tracks alive before it, joined whenever two
 * lie within merge_gap + 1 bins of each other. A blob joins a track only
 * within that reach of the track's span, and the track's next span is the
 * hull of its blobs, so by induction every span a track takes during the
 * pass stays inside one joined interval; so do the blobs and their hits.
 * The intervals come from the OR of the hit rows and the spans: a run's hits
 * lie at most merge_gap apart, so joining set bins within the reach gives
 * the same intervals as joining the runs. */
static int pass_columns(atkdsp_cfar *c, const uint32_t *hits, int j0, int nf) {
    const long nb = (long)c->nbins, reach = c->cfg.merge_gap + 1;
    const size_t W = c->words;
    uint32_t *m = c->orm;
    memset(m, 0, W * sizeof(uint32_t));
    for (int j = j0; j < nf; ++j) {
        const uint32_t *row = hits + (size_t)j * W;
        for (size_t w = 0; w < W; ++w) m[w] |= row[w];
    }
    for (int t = 0; t < c->ntracks; ++t)
        for (long b = c->tracks[t].cur_lo; b <= c->tracks[t].cur_hi; ++b) m[b >> 5] |= 1u << (b & 31);
    int ncol = 0;
    for (long i = next_hit(m, 0, nb); i < nb; i = next_hit(m, i, nb)) {
        long hi = i, q;
        while ((q = next_hit(m, hi + 1, nb)) < nb && q <= hi + reach) hi = q;
        for (long b = i; b <= hi; ++b) {
            c->colmap[b] = ncol;
            c->h_cols[ncol++] = (int32_t)b;
        }
        i = hi + 1;
    }
    c->ncol = ncol;
    return ATKB_OK;
}

static void columns_clear(atkdsp_cfar *c) {
    for (int q = 0; q < c->ncol; ++q) c->colmap[c->h_cols[q]] = -1;
    c->ncol = 0;
}

/* frames: host (on_device 0) or device floats, nframes x nbins; d_hits_out:
 * device, nframes x nbins, or NULL. The call runs in passes of at most fc
 * frames. While the host tracks pass i, the GPU converts and tests pass
 * i + 1 into the other row set and copies its hit rows. For the pass it
 * tracks, the host then fetches X, noise and raw at that pass's columns
 * only (a gather on a second stream), not the whole rows. */
static ptrdiff_t cfar_run(atkdsp_cfar *c, const float *frames, int on_device, int units, size_t nframes,
                          double frame_t0, double frame_dt, atkdsp_cfar_event *ev, size_t cap, uint8_t *d_hits_out,
                          void *stream) {
    if (!c || (!frames && nframes) || (!ev && nframes)) return ATKDSP_E_ARG;
    if (units < 0 || units > 1) return ATKDSP_E_ARG;
    if (cap < atkdsp_cfar_events_max(c, nframes)) return ATKDSP_E_CAP;
    if (nframes == 0) return 0;
    const size_t nb = c->nbins;
    const int k = c->cfg.k_frames;
    int rc = ATKB_OK;
    if (on_device) {
        /* the frames' producer: `stream`, NULL being the legacy default stream */
        rc = atkb_event_record(c->ev_in, stream);
        if (rc == ATKB_OK) rc = atkb_stream_wait(c->stream, c->ev_in);
        if (rc != ATKB_OK) return atkb_map_rc(rc);
    }
    const int64_t F_start = c->frame, seen_start = c->seen;
    cf_pass cur, next;
    size_t nev = 0;
    int last_set = -1, last_row = -1;
    for (size_t at = 0, i = 0; at < nframes; ++i) {
        cur.done = at;
        cur.nf = (int)((nframes - at) < (size_t)c->fc ? (nframes - at) : (size_t)c->fc);
        cur.F0 = F_start + (int64_t)at;
        cur.j0 = (int64_t)k - 1 - (seen_start + (int64_t)at);
        if (cur.j0 < 0) cur.j0 = 0;
        if (i == 0) rc = pass_enqueue(c, &cur, frames, on_device, units, 0, d_hits_out);
        at += (size_t)cur.nf;
        if (rc == ATKB_OK && at < nframes) {
            next.done = at;
            next.nf = (int)((nframes - at) < (size_t)c->fc ? (nframes - at) : (size_t)c->fc);
            next.F0 = F_start + (int64_t)at;
            next.j0 = (int64_t)k - 1 - (seen_start + (int64_t)at);
            if (next.j0 < 0) next.j0 = 0;
            rc = pass_enqueue(c, &next, frames, on_device, units, (int)((i + 1) & 1), d_hits_out);
        }
        const int set = (int)(i & 1);
        const size_t hs = (size_t)set * (size_t)c->fc * nb, bs = (size_t)set * (size_t)c->fc * c->words;
        if (rc == ATKB_OK) rc = atkb_event_sync(c->ev_pass[set]);
        const int j0 = (int)cur.j0;
        if (rc == ATKB_OK && j0 < cur.nf) {
            rc = pass_columns(c, c->h_bits + bs, j0, cur.nf);
            c->rc_f0 = cur.F0 + j0 - (k - 1);
            if (rc == ATKB_OK && c->ncol > 0) {
                const int rows = cur.nf - j0, nraw = k > 1 ? rows + k - 1 : 0;
                const size_t nc = (size_t)c->ncol;
                rc = atkb_h2d(c->d_cols, c->h_cols, nc * sizeof(int32_t), c->gstream);
                if (rc == ATKB_OK)
                    rc = atkb_cfar_gather(c->d_X + hs + (size_t)j0 * nb, c->d_noise + hs + (size_t)j0 * nb,
                                          (long long)nb, rows, c->d_raw, c->ring, c->rc_f0, nraw, c->d_cols,
                                          c->ncol, c->d_Xc, c->d_Nc, c->d_Rc, c->gstream);
                if (rc == ATKB_OK) rc = atkb_d2h(c->h_Xc, c->d_Xc, (size_t)rows * nc * sizeof(double), c->gstream);
                if (rc == ATKB_OK) rc = atkb_d2h(c->h_Nc, c->d_Nc, (size_t)rows * nc * sizeof(double), c->gstream);
                if (rc == ATKB_OK && nraw)
                    rc = atkb_d2h(c->h_Rc, c->d_Rc, (size_t)nraw * nc * sizeof(double), c->gstream);
                if (rc == ATKB_OK) rc = atkb_stream_sync(c->gstream);
            }
        }
        if (rc != ATKB_OK) {
            columns_clear(c);
            atkb_stream_sync(c->stream);
            atkb_stream_sync(c->gstream);
            return atkb_map_rc(rc);
        }
        for (int j = 0; j < cur.nf; ++j) {
            const int64_t F = cur.F0 + j;
            const double tf = frame_t0 + (double)(cur.done + (size_t)j) * frame_dt;
            const size_t row = (size_t)(F % c->ring);
            c->st.frames++;
            c->ht[row] = tf;
            c->hd[row] = frame_dt;
            c->seen++;
            c->frame++;
            if (c->seen < k) {
                c->st.warmup++;
                continue;
            }
            const size_t oc = (size_t)(j - j0) * (size_t)c->ncol;
            nev += track_frame(c, F, c->h_Xc + oc, c->h_Nc + oc, c->h_bits + bs + (size_t)j * c->words, tf,
                               frame_dt, ev + nev);
            last_set = set;
            last_row = j;
        }
        columns_clear(c);
    }
    if (last_row >= 0) {
        /* the last tested frame is in the last pass, whose rows nothing overwrote */
        const size_t o = (size_t)last_set * (size_t)c->fc * nb + (size_t)last_row * nb;
        const uint32_t *lb = c->h_bits + ((size_t)last_set * (size_t)c->fc + (size_t)last_row) * c->words;
        for (size_t b = 0; b < nb; ++b) c->last_hits[b] = (uint8_t)bit_at(lb, (long)b);
        rc = atkb_d2h(c->last_X, c->d_X + o, nb * sizeof(double), c->stream);
        if (rc == ATKB_OK) rc = atkb_d2h(c->last_thr, c->d_thr + o, nb * sizeof(double), c->stream);
        if (rc == ATKB_OK) rc = atkb_stream_sync(c->stream);
        if (rc != ATKB_OK) return atkb_map_rc(rc);
        c->has_last = 1;
    } else {
        rc = atkb_stream_sync(c->stream);
        if (rc != ATKB_OK) return atkb_map_rc(rc);
    }
    return (ptrdiff_t)nev;
}

ATKDSP_API ptrdiff_t atkdsp_cfar_process(atkdsp_cfar *c, const float *frames_db, size_t nframes, double frame_t0,
                                         double frame_dt, atkdsp_cfar_event *ev, size_t cap) {
    return cfar_run(c, frames_db, 0, 0, nframes, frame_t0, frame_dt, ev, cap, NULL, NULL);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_cfar_process(atkdsp_cfar *c, const float *d_frames, int units, size_t nframes,
                                             double frame_t0, double frame_dt, atkdsp_cfar_event *ev, size_t cap,
                                             uint8_t *d_hits, void *stream) {
    return cfar_run(c, d_frames, 1, units, nframes, frame_t0, frame_dt, ev, cap, d_hits, stream);
}

ATKDSP_API ptrdiff_t atkdsp_cfar_flush(atkdsp_cfar *c, atkdsp_cfar_event *ev, size_t cap) {
    if (!c) return ATKDSP_E_ARG;
    size_t open = 0;
    for (int t = 0; t < c->ntracks; ++t) open += c->tracks[t].state == 1;
    if (open && (!ev || cap < open)) return ATKDSP_E_CAP;
    size_t nev = 0;
    for (int t = 0; t < c->ntracks; ++t)
        if (c->tracks[t].state == 1) emit_close(c, &c->tracks[t], ATKDSP_CFAR_FLUSHED, &ev[nev++]);
    c->ntracks = 0;
    return (ptrdiff_t)nev;
}

ATKDSP_API int atkdsp_cfar_last(const atkdsp_cfar *c, float *avg_db, float *thr_db, uint8_t *hits) {
    if (!c) return ATKDSP_E_ARG;
    if (!c->has_last) return ATKDSP_E_EMPTY;
    for (size_t i = 0; i < c->nbins; ++i) {
        if (avg_db) avg_db[i] = (float)(10.0 * log10(c->last_X[i]));
        if (thr_db) thr_db[i] = (float)(10.0 * log10(c->last_thr[i]));
        if (hits) hits[i] = c->last_hits[i];
    }
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_cfar_info(const atkdsp_cfar *c, double *alpha, double *alpha_ca, double *et,
                                atkdsp_cfar_config *cfg) {
    if (!c) return ATKDSP_E_ARG;
    if (alpha) *alpha = c->alpha;
    if (alpha_ca) *alpha_ca = c->alpha_ca;
    if (et) *et = c->et;
    if (cfg) *cfg = c->cfg;
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_cfar_describe(const atkdsp_cfar *c, char *buf, size_t cap) {
    if (!c || !buf || !cap) return ATKDSP_E_ARG;
    static const char *const names[4] = {"CA", "OS", "GO", "SO"};
    char os_txt[48] = "", eff_txt[64] = "";
    if (c->cfg.mode == ATKDSP_CFAR_OS) snprintf(os_txt, sizeof os_txt, " (rank %d of %d)", c->cfg.os_k, c->N);
    if (c->n_eff != (double)c->N)
        snprintf(eff_txt, sizeof eff_txt, " (%.1f effective, window-correlated)", c->n_eff);
    size_t masked = 0;
    for (size_t i = 0; i < c->nbins; ++i) masked += c->mask[i] != 0;
    snprintf(buf, cap,
             "CFAR %s%s: %d+%d reference cells%s, %d guard each side, Pfa %.3g per cell per "
             "frame, K = %g look(s) x %d frame(s), alpha %.4g (%.2f dB); open %d of %d, "
             "close after %d misses, merge gap %d, min %d bin(s); %zu bins, %zu masked, "
             "tracks %d/%d",
             names[c->cfg.mode], os_txt, c->cfg.n_ref, c->cfg.n_ref, eff_txt, c->cfg.n_guard, c->cfg.pfa,
             c->cfg.looks, c->cfg.k_frames, c->alpha, 10.0 * log10(c->alpha), c->cfg.open_m, c->cfg.open_n,
             c->cfg.close_k, c->cfg.merge_gap, c->cfg.min_bins, c->nbins, masked, c->ntracks, c->cfg.max_tracks);
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_cfar_stats(const atkdsp_cfar *c, atkdsp_cfar_counters *st) {
    if (!c || !st) return ATKDSP_E_ARG;
    *st = c->st;
    st->tracks = (uint64_t)c->ntracks;
    return ATKDSP_OK;
}
