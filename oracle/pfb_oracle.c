/* CPU oracle for the channelizer hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C99, the algorithm of the reference's
 * polyphase filterbank, its W1/W2 accumulators and its unpack front end, so
 * that the CUDA product can be checked against it on the same inputs. It is
 * never linked into the product; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it (as liboracle.so).
 *
 * Pinning: tests/test_oracle_pinned.py checks every entry point here against
 * the reference library built from its own sources (oracle/_ref) and against
 * the committed golden fixtures in tests/golden/ (made by
 * tests/golden/make_golden.py from the reference build and its numpy twin).
 *
 * Numerics follow the reference exactly where it is deterministic:
 *   - prototype taps in double, same expression order as
 *     src/channelizer.c:79-99 (+ src/design.c:18-22, src/channelizer.c:33-43);
 *   - the fold in float, k ascending, one rounded multiply then one rounded
 *     add per tap (src/channelizer.c:258-266; built with -ffp-contract=off);
 *   - FFT in double (the reference uses pocketfft, src/fft.c:114-117; this file
 *     has its own mixed-radix transform, so results agree to ~1e-16 and round
 *     to the same float except on rare ties);
 *   - bin rotation with the reference's double twiddle table and stepped
 *     index (src/channelizer.c:270-292), cal in double, one rounding to float.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846

typedef struct { float re, im; } orc_cf32;

/* Kaiser beta from stopband attenuation (src/design.c:18-22). */
double orc_kaiser_beta(double atten_db) {
    if (atten_db > 50.0) return 0.1102 * (atten_db - 8.7);
    if (atten_db >= 21.0) return 0.5842 * pow(atten_db - 21.0, 0.4) + 0.07886 * (atten_db - 21.0);
    return 0.0;
}

/* Modified Bessel I0 by its power series; stops once a squared term falls
 * under 1e-17 of the running sum (src/channelizer.c:33-43). */
static double orc_i0(double x) {
    const double half = x * 0.5;
    double acc = 1.0, term = 1.0;
    int k;
    for (k = 1; k < 500; ++k) {
        term *= (half / (double)k);
        const double sq = term * term;
        acc += sq;
        if (sq < acc * 1e-17) break;
    }
    return acc;
}

/* Kaiser-windowed sinc prototype, cutoff 1/(2 nchan), unit DC gain times
 * nchan (src/channelizer.c:79-99). h has nchan*K doubles. */
void orc_pfb_prototype(unsigned nchan, unsigned K, double atten_db, double *h) {
    const size_t L = (size_t)nchan * K;
    const double fc = 1.0 / (2.0 * (double)nchan);
    const double mid = (double)(L - 1) * 0.5;
    if (atten_db < 20.0) atten_db = 20.0;
    const double beta = orc_kaiser_beta(atten_db);
    const double i0b = orc_i0(beta);
    double total = 0.0;
    size_t n;
    for (n = 0; n < L; ++n) {                      /* pass 1: the DC sum */
        const double t = (double)n - mid;
        const double x = 2.0 * fc * t;
        const double sinc = (t == 0.0) ? 1.0 : sin(ORC_PI * x) / (ORC_PI * x);
        const double r = (mid > 0.0) ? t / mid : 0.0;
        const double w = orc_i0(beta * sqrt(r * r < 1.0 ? 1.0 - r * r : 0.0)) / i0b;
        total += 2.0 * fc * sinc * w;
    }
    if (total == 0.0) total = 1.0;
    for (n = 0; n < L; ++n) {                      /* pass 2: normalised */
        const double t = (double)n - mid;
        const double x = 2.0 * fc * t;
        const double sinc = (t == 0.0) ? 1.0 : sin(ORC_PI * x) / (ORC_PI * x);
        const double r = (mid > 0.0) ? t / mid : 0.0;
        const double w = orc_i0(beta * sqrt(r * r < 1.0 ? 1.0 - r * r : 0.0)) / i0b;
        const double v = 2.0 * fc * sinc * w;
        h[n] = (v / total) * (double)nchan;
    }
}

/* ---- a plain double-precision mixed-radix DFT (decimation in time) -------
 * tw[2j], tw[2j+1] = cos, -sin of 2 pi j / N for the top-level N. A length-n
 * sub-transform uses W_n^j = W_N^(j N/n). */
static size_t orc_smallest_factor(size_t n) {
    size_t p;
    if (n % 4 == 0 && n > 4) return 4;
    for (p = 2; p * p <= n; ++p) if (n % p == 0) return p;
    return n;
}

/* the p-point DFT of t[0..p) (interleaved), written to out at stride ostr:
 * exact butterflies for 2 and 4 (no multiply by a rounded +-1 or +-i), the
 * usual closed form for 3, a direct sum otherwise. */
static void orc_small_dft(const double *t, size_t p, double *out, size_t ostr,
                          const double *tw, size_t pstep) {
    size_t o, r;
    if (p == 2) {
        out[0] = t[0] + t[2]; out[1] = t[1] + t[3];
        out[2 * ostr] = t[0] - t[2]; out[2 * ostr + 1] = t[1] - t[3];
        return;
    }
    if (p == 4) {
        const double ar = t[0] + t[4], ai = t[1] + t[5], br = t[0] - t[4], bi = t[1] - t[5];
        const double cr = t[2] + t[6], ci = t[3] + t[7], dr = t[3] - t[7], di = -(t[2] - t[6]);
        out[0] = ar + cr; out[1] = ai + ci;
        out[2 * ostr] = br + dr; out[2 * ostr + 1] = bi + di;
        out[4 * ostr] = ar - cr; out[4 * ostr + 1] = ai - ci;
        out[6 * ostr] = br - dr; out[6 * ostr + 1] = bi - di;
        return;
    }
    if (p == 3) {
        const double s3 = 0.86602540378443864676;
        const double sr = t[2] + t[4], si = t[3] + t[5], dr = t[2] - t[4], di = t[3] - t[5];
        const double mr = t[0] - 0.5 * sr, mi = t[1] - 0.5 * si;
        out[0] = t[0] + sr; out[1] = t[1] + si;
        out[2 * ostr] = mr + s3 * di; out[2 * ostr + 1] = mi - s3 * dr;
        out[4 * ostr] = mr - s3 * di; out[4 * ostr + 1] = mi + s3 * dr;
        return;
    }
    for (o = 0; o < p; ++o) {
        double accr = 0.0, acci = 0.0;
        for (r = 0; r < p; ++r) {
            const size_t j = (r * o) % p * pstep;
            accr += t[2 * r] * tw[2 * j] - t[2 * r + 1] * tw[2 * j + 1];
            acci += t[2 * r] * tw[2 * j + 1] + t[2 * r + 1] * tw[2 * j];
        }
        out[2 * o * ostr] = accr; out[2 * o * ostr + 1] = acci;
    }
}

static void orc_dft(const double *in, size_t stride, size_t n, double *out,
                    const double *tw, size_t N, double *work) {
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }
    const size_t p = orc_smallest_factor(n);
    const size_t step = N / n;                     /* W_n^j = tw[j*step] */
    size_t k, r;
    double t[2 * 64] = {0};
    double *tt = p <= 64 ? t : (double *)malloc(2 * p * sizeof(double));
    if (p == n) {                                  /* a prime (or 4) length */
        for (r = 0; r < n; ++r) { tt[2 * r] = in[2 * r * stride]; tt[2 * r + 1] = in[2 * r * stride + 1]; }
        orc_small_dft(tt, n, out, 1, tw, step);
        if (tt != t) free(tt);
        return;
    }
    const size_t m = n / p;
    /* sub-transform r takes inputs r, r+p, r+2p, ... into work[r*m ...] */
    for (r = 0; r < p; ++r)
        orc_dft(in + 2 * r * stride, stride * p, m, work + 2 * r * m, tw, N, out);
    for (k = 0; k < m; ++k) {
        /* twiddle W_n^(r k), then a p-point DFT across r: X[k + q m] */
        for (r = 0; r < p; ++r) {
            const double yr = work[2 * (r * m + k)], yi = work[2 * (r * m + k) + 1];
            if (r == 0 || k == 0) { tt[2 * r] = yr; tt[2 * r + 1] = yi; continue; }
            const size_t j = (r * k) * step;
            tt[2 * r] = yr * tw[2 * j] - yi * tw[2 * j + 1];
            tt[2 * r + 1] = yr * tw[2 * j + 1] + yi * tw[2 * j];
        }
        orc_small_dft(tt, p, out + 2 * k, m, tw, N / p);
    }
    if (tt != t) free(tt);
}

/* Forward DFT in double, in place on 2N interleaved values. */
static void orc_fft(double *buf, size_t N, const double *tw, double *a, double *b) {
    memcpy(a, buf, 2 * N * sizeof(double));
    orc_dft(a, 1, N, buf, tw, N, b);
}

/* ---- the filterbank --------------------------------------------------------
 * State (src/channelizer.c:48-77): every element keeps the last ov + lc input
 * samples; hop i of a call reads s[i*hop, i*hop + L) of s = carry ++ in. */
typedef struct {
    unsigned nchan, os, K, max_nel, hop;
    size_t L, ov;
    double *h;          /* L prototype taps */
    float *hf;          /* L taps rounded to float */
    double *twd;        /* 2 nchan: cos, sin of 2 pi j / nchan (rotation) */
    double *tw;         /* 2 nchan: cos, -sin (the DFT's table) */
    orc_cf32 *carry;    /* max_nel * (ov + hop) */
    unsigned lc;
    int64_t b;
    orc_cf32 *cal;
    unsigned cal_nel;
} orc_pfb;

void orc_pfb_destroy(orc_pfb *p) {
    if (!p) return;
    free(p->h); free(p->hf); free(p->twd); free(p->tw); free(p->carry); free(p->cal);
    free(p);
}

orc_pfb *orc_pfb_create(double fs, unsigned nchan, unsigned os, unsigned K, double atten_db,
                        unsigned max_nel) {
    if (!(fs > 0.0) || nchan < 2 || os < 1 || nchan % os != 0 || K < 2 || max_nel < 1) return NULL;
    orc_pfb *p = (orc_pfb *)calloc(1, sizeof *p);
    if (!p) return NULL;
    p->nchan = nchan; p->os = os; p->K = K; p->max_nel = max_nel;
    p->hop = nchan / os;
    p->L = (size_t)nchan * K;
    p->ov = p->L - p->hop;
    p->h = (double *)malloc(p->L * sizeof(double));
    p->hf = (float *)malloc(p->L * sizeof(float));
    p->twd = (double *)malloc(2 * (size_t)nchan * sizeof(double));
    p->tw = (double *)malloc(2 * (size_t)nchan * sizeof(double));
    p->carry = (orc_cf32 *)calloc((size_t)max_nel * (p->ov + p->hop), sizeof(orc_cf32));
    if (!p->h || !p->hf || !p->twd || !p->tw || !p->carry) { orc_pfb_destroy(p); return NULL; }
    orc_pfb_prototype(nchan, K, atten_db, p->h);
    for (size_t q = 0; q < p->L; ++q) p->hf[q] = (float)p->h[q];
    for (unsigned j = 0; j < nchan; ++j) {
        const double a = 2.0 * ORC_PI * (double)j / (double)nchan;
        p->twd[2 * j] = cos(a); p->twd[2 * j + 1] = sin(a);
        p->tw[2 * j] = cos(a); p->tw[2 * j + 1] = -sin(a);
    }
    return p;
}

void orc_pfb_reset(orc_pfb *p) {
    if (!p) return;
    memset(p->carry, 0, (size_t)p->max_nel * (p->ov + p->hop) * sizeof(orc_cf32));
    p->lc = 0; p->b = 0;
}

size_t orc_pfb_out_hops(const orc_pfb *p, size_t n) { return p ? ((size_t)p->lc + n) / p->hop : 0; }
const double *orc_pfb_taps(const orc_pfb *p) { return p ? p->h : NULL; }

int orc_pfb_set_cal(orc_pfb *p, const orc_cf32 *table, unsigned nel) {
    if (!p) return -1;
    if (!table) { free(p->cal); p->cal = NULL; p->cal_nel = 0; return 0; }
    if (nel < 1 || nel > p->max_nel) return -1;
    orc_cf32 *t = (orc_cf32 *)malloc((size_t)nel * p->nchan * sizeof(orc_cf32));
    if (!t) return -2;
    memcpy(t, table, (size_t)nel * p->nchan * sizeof(orc_cf32));
    free(p->cal); p->cal = t; p->cal_nel = nel;
    return 0;
}

/* one hop of one element: window w (L samples) -> row (nchan cf32) */
static void orc_one_hop(const orc_pfb *p, const orc_cf32 *w, int64_t b, const orc_cf32 *cal,
                        float *fold, double *acc, double *wa, double *wb, orc_cf32 *row) {
    const unsigned N = p->nchan;
    const size_t N2 = 2 * (size_t)N;
    const float *wf = (const float *)w;
    size_t q, k;
    /* fold: taps duplicated over re/im, k ascending, rounded mul then add */
    for (q = 0; q < N2; ++q) {
        const float hq = p->hf[q >> 1];
        fold[q] = hq * wf[q];
    }
    for (k = 1; k < p->K; ++k) {
        const float *hk = p->hf + k * N;
        const float *wk = wf + k * N2;
        for (q = 0; q < N2; ++q) {
            const float prod = hk[q >> 1] * wk[q];
            fold[q] = fold[q] + prod;
        }
    }
    for (q = 0; q < N2; ++q) acc[q] = (double)fold[q];
    orc_fft(acc, N, p->tw, wa, wb);
    /* rotation to input sample 0: exp(-2 pi i k shift / N), stepped index */
    const unsigned shift = (unsigned)((((b + 1) * (int64_t)p->hop) % (int64_t)N + N) % N);
    unsigned idx = 0;
    for (unsigned c = 0; c < N; ++c) {
        const double xr = acc[2 * c], xi = acc[2 * c + 1];
        const double wr = p->twd[2 * idx], wi = p->twd[2 * idx + 1];
        double yr = xr * wr - xi * wi;
        double yi = xr * wi + xi * wr;
        if (cal) {
            const double cr = cal[c].re, ci = cal[c].im;
            const double zr = yr * cr - yi * ci, zi = yr * ci + yi * cr;
            yr = zr; yi = zi;
        }
        row[c].re = (float)yr;
        row[c].im = (float)yi;
        idx = (idx >= shift) ? idx - shift : idx + N - shift;
    }
}

/* Returns m, -1 (bad argument) or -3 (cap too small; state untouched). */
ptrdiff_t orc_pfb_process_n(orc_pfb *p, const orc_cf32 *const *ins, unsigned nel, size_t n,
                            orc_cf32 *out, size_t cap) {
    if (!p || !ins || nel < 1 || nel > p->max_nel) return -1;
    const unsigned N = p->nchan, hop = p->hop;
    const size_t ov = p->ov, L = p->L;
    const size_t head = ov + p->lc;
    const size_t m = (p->lc + n) / hop;
    const size_t keep = ov + hop;
    if (m == 0) {
        for (unsigned e = 0; e < nel; ++e)
            if (n) memcpy(p->carry + (size_t)e * keep + head, ins[e], n * sizeof(orc_cf32));
        p->lc += (unsigned)n;
        return 0;
    }
    if (!out || cap < (size_t)nel * N * m) return -3;
    const size_t total = head + n;
    for (unsigned e = 0; e < nel; ++e) {
        orc_cf32 *s = (orc_cf32 *)malloc(total * sizeof(orc_cf32));
        if (!s) return -2;
        memcpy(s, p->carry + (size_t)e * keep, head * sizeof(orc_cf32));
        memcpy(s + head, ins[e], n * sizeof(orc_cf32));
        const orc_cf32 *cal = (p->cal && e < p->cal_nel) ? p->cal + (size_t)e * N : NULL;
        orc_cf32 *dst = out + (size_t)e * N * m;
        long long i;
#pragma omp parallel for schedule(static)
        for (i = 0; i < (long long)m; ++i) {
            float *fold = (float *)malloc(2 * (size_t)N * sizeof(float));
            double *acc = (double *)malloc(2 * (size_t)N * sizeof(double));
            double *wa = (double *)malloc(2 * (size_t)N * sizeof(double));
            double *wb = (double *)malloc(2 * (size_t)N * sizeof(double));
            orc_cf32 *row = (orc_cf32 *)malloc((size_t)N * sizeof(orc_cf32));
            orc_one_hop(p, s + (size_t)i * hop, p->b + i, cal, fold, acc, wa, wb, row);
            for (unsigned c = 0; c < N; ++c) dst[(size_t)c * m + (size_t)i] = row[c];
            free(fold); free(acc); free(wa); free(wb); free(row);
        }
        /* carry = s[m*hop, total): ov history samples then the leftover */
        memcpy(p->carry + (size_t)e * keep, s + m * hop, (total - m * hop) * sizeof(orc_cf32));
        free(s);
    }
    (void)L;
    p->lc = (unsigned)(total - m * hop - ov);
    p->b += (int64_t)m;
    return (ptrdiff_t)m;
}

/* ---- W1 / W2 (src/channelizer.c:420-471) ---------------------------------- */
void orc_cov_accumulate(const orc_cf32 *out, unsigned nel, unsigned nchan, size_t m,
                        const uint8_t *gate, orc_cf32 *R, uint32_t *counts) {
    if (!out || !R || !counts || nel < 1 || nchan < 1) return;
    for (unsigned k = 0; k < nchan; ++k) {
        if (gate && !gate[k]) continue;
        orc_cf32 *Rk = R + (size_t)k * nel * nel;
        for (size_t i = 0; i < m; ++i)
            for (unsigned a = 0; a < nel; ++a) {
                const orc_cf32 ya = out[((size_t)a * nchan + k) * m + i];
                for (unsigned c = 0; c < nel; ++c) {
                    const orc_cf32 yb = out[((size_t)c * nchan + k) * m + i];
                    orc_cf32 *r = Rk + (size_t)a * nel + c;
                    const float pr = ya.re * yb.re + ya.im * yb.im;
                    const float pi = ya.im * yb.re - ya.re * yb.im;
                    r->re += pr;
                    r->im += pi;
                }
            }
        counts[k] += (uint32_t)m;
    }
}

void orc_cov_reset(orc_cf32 *R, uint32_t *counts, unsigned nel, unsigned nchan, const uint8_t *gate) {
    if (!R || !counts) return;
    for (unsigned k = 0; k < nchan; ++k) {
        if (gate && !gate[k]) continue;
        memset(R + (size_t)k * nel * nel, 0, (size_t)nel * nel * sizeof(orc_cf32));
        counts[k] = 0;
    }
}

void orc_channel_power(const orc_cf32 *out, unsigned nel, unsigned nchan, size_t m,
                       float *pwr, float *mean_pwr) {
    if (!out || nel < 1 || nchan < 1) return;
    const double inv = m ? 1.0 / (double)m : 0.0;
    for (unsigned k = 0; k < nchan; ++k) {
        double across = 0.0;
        for (unsigned a = 0; a < nel; ++a) {
            double s = 0.0;
            for (size_t i = 0; i < m; ++i) {
                const orc_cf32 y = out[((size_t)a * nchan + k) * m + i];
                s += (double)y.re * y.re + (double)y.im * y.im;
            }
            if (pwr) pwr[(size_t)a * nchan + k] = (float)(s * inv);
            across += s * inv;
        }
        if (mean_pwr) mean_pwr[k] = (float)(across / (double)nel);
    }
}

/* ---- unpack (src/convert.c:33-128, src/atkdsp.c:51-60) -------------------- */
int orc_bytes_per_sample(int fmt) {
    switch (fmt) {
    case 0: case 1: return 2;      /* cu8, ci8 */
    case 2: case 3: return 4;      /* ci16, ci16q11 */
    case 4: return 8;              /* cf32 */
    default: return 0;
    }
}

static ptrdiff_t orc_unpack_core(const void *raw, size_t nbytes, int fmt, orc_cf32 *out,
                                 size_t cap, float off_re, float off_im,
                                 double *mean_re, double *mean_im) {
    if (!raw || !out) return -1;
    const int bps = orc_bytes_per_sample(fmt);
    if (!bps) return -1;
    size_t n = nbytes / (size_t)bps, i;
    if (n > cap) n = cap;
    if (fmt == 0 || fmt == 1 || fmt == 2 || fmt == 3) {
        float k, cre, cim;
        if (fmt == 0) { k = 1.0f / 127.5f; cre = 127.5f + off_re / k; cim = 127.5f + off_im / k; }
        else {
            k = fmt == 1 ? 1.0f / 128.0f : fmt == 2 ? 1.0f / 32768.0f : 1.0f / 2048.0f;
            cre = off_re / k; cim = off_im / k;
        }
        for (i = 0; i < n; ++i) {
            float a, b;
            if (fmt == 0) { a = ((const uint8_t *)raw)[2 * i]; b = ((const uint8_t *)raw)[2 * i + 1]; }
            else if (fmt == 1) { a = ((const int8_t *)raw)[2 * i]; b = ((const int8_t *)raw)[2 * i + 1]; }
            else { a = ((const int16_t *)raw)[2 * i]; b = ((const int16_t *)raw)[2 * i + 1]; }
            out[i].re = (a - cre) * k;
            out[i].im = (b - cim) * k;
        }
    } else {
        const orc_cf32 *src = (const orc_cf32 *)raw;
        if (off_re == 0.0f && off_im == 0.0f) {
            if ((const void *)out != raw) memmove(out, src, n * sizeof(orc_cf32));
        } else {
            for (i = 0; i < n; ++i) { out[i].re = src[i].re - off_re; out[i].im = src[i].im - off_im; }
        }
    }
    if (mean_re || mean_im) {
        /* eight interleaved double partial sums, then the tail, as the reference */
        double pr[8], pi[8], sr = 0.0, si = 0.0;
        int l;
        for (l = 0; l < 8; ++l) { pr[l] = 0.0; pi[l] = 0.0; }
        const size_t whole = n & ~(size_t)7;
        for (i = 0; i < whole; i += 8)
            for (l = 0; l < 8; ++l) { pr[l] += (double)out[i + l].re; pi[l] += (double)out[i + l].im; }
        for (; i < n; ++i) { pr[0] += (double)out[i].re; pi[0] += (double)out[i].im; }
        for (l = 0; l < 8; ++l) { sr += pr[l]; si += pi[l]; }
        const double inv = n ? 1.0 / (double)n : 0.0;
        if (mean_re) *mean_re = sr * inv + (double)off_re;
        if (mean_im) *mean_im = si * inv + (double)off_im;
    }
    return (ptrdiff_t)n;
}

ptrdiff_t orc_unpack(const void *raw, size_t nbytes, int fmt, orc_cf32 *out, size_t cap,
                     float dc_alpha, orc_cf32 *dc_state) {
    const ptrdiff_t n = orc_unpack_core(raw, nbytes, fmt, out, cap, 0.0f, 0.0f, NULL, NULL);
    if (n > 0 && dc_alpha > 0.0f && dc_state) {
        /* one-pole DC block, serial: s += a (x - s); y = x - s (src/convert.c:7-17) */
        float sr = dc_state->re, si = dc_state->im;
        for (ptrdiff_t i = 0; i < n; ++i) {
            const float dr = out[i].re - sr, di = out[i].im - si;
            const float gr = dc_alpha * dr, gi = dc_alpha * di;
            sr = sr + gr; si = si + gi;
            out[i].re = out[i].re - sr;
            out[i].im = out[i].im - si;
        }
        dc_state->re = sr; dc_state->im = si;
    }
    return n;
}

ptrdiff_t orc_unpack_dc(const void *raw, size_t nbytes, int fmt, orc_cf32 *out, size_t cap,
                        float off_re, float off_im, double *mean_re, double *mean_im) {
    return orc_unpack_core(raw, nbytes, fmt, out, cap, off_re, off_im, mean_re, mean_im);
}
