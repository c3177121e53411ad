/* CPU oracle for the overlap-save extractor -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C99 restatement of the reference's atkdsp_osx_* (src/channelizer.c:
 * 473-788), the Kaiser low-pass design it uses (src/design.c:24-64) and the
 * arbitrary resampler that lands each channel on its out_rate
 * (src/resample.c:110-260). It is linked into liboracle.so beside
 * pfb_oracle.c and is never part of the product; only tests/, smoke() and
 * bench.py's CPU leg load it.
 *
 * Pinning: tests/test_oracle_pinned.py checks it against the reference
 * library built from its own sources (oracle/_ref) and against the committed
 * fixtures of tests/golden/osx.npz (made from that build by
 * tests/golden/make_golden.py).
 *
 * Numerics follow the reference where it is deterministic: taps in double
 * with one rounding to float; the resampler's coefficient, position and FIR
 * arithmetic in its types and order (float FIR, q ascending, one rounded
 * multiply then one rounded add; built with -ffp-contract=off); the per-bin
 * fold in float with the reference's expression order; the roll taken to
 * absolute time with double cos/sin. The FFTs are double (the reference
 * uses pocketfft, src/fft.c:114-135, float in, double transform, float out);
 * this file has its own radix-2 transform, so spectra agree to ~1e-16 before
 * the rounding to float.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define OX_PI 3.14159265358979323846
#define OX_E_ARG -1
#define OX_E_NOMEM -2
#define OX_E_CAP -3

typedef struct { float re, im; } ox_cf32;

double orc_kaiser_beta(double atten_db);          /* pfb_oracle.c */

/* ---- Kaiser low-pass design (src/design.c:5-64) --------------------------- */
static double ox_i0(double x) {
    const double y = x * 0.5;
    double s = 1.0, t = 1.0;
    for (int k = 1; k < 500; ++k) {
        t *= (y / (double)k);
        const double t2 = t * t;
        s += t2;
        if (t2 < s * 1e-17) break;
    }
    return s;
}

/* taps for `atten_db` over a transition of `tr_hz` at `rate`: odd, >= 3 */
static size_t ox_kaiser_length(double atten_db, double tr_hz, double rate) {
    if (tr_hz <= 0.0 || rate <= 0.0) return 0;
    const double dw = 2.0 * OX_PI * tr_hz / rate;
    const double n = (atten_db > 8.0 ? (atten_db - 8.0) : 1.0) / (2.285 * dw);
    size_t N = (size_t)ceil(n) + 1;
    if (N < 3) N = 3;
    if ((N & 1) == 0) ++N;
    return N;
}

static double ox_lp_tap(size_t n, double fc, double mid, double beta, double i0b) {
    const double t = (double)n - mid;
    const double x = 2.0 * fc * t;
    const double sinc = (t == 0.0) ? 1.0 : sin(OX_PI * x) / (OX_PI * x);
    const double r = t / mid;
    const double w = ox_i0(beta * sqrt(r * r < 1.0 ? 1.0 - r * r : 0.0)) / i0b;
    return 2.0 * fc * sinc * w;
}

/* the tap count with out == NULL, else the taps (unit DC gain, one rounding) */
ptrdiff_t orc_design_lowpass(double fp_hz, double fs_hz, double atten_db, double rate, float *out,
                             size_t cap) {
    if (rate <= 0.0 || fp_hz < 0.0 || fs_hz <= fp_hz || fs_hz > rate * 0.5 + 1e-9) return OX_E_ARG;
    const size_t N = ox_kaiser_length(atten_db, fs_hz - fp_hz, rate);
    if (!out) return (ptrdiff_t)N;
    if (cap < N) return OX_E_CAP;
    const double beta = orc_kaiser_beta(atten_db), i0b = ox_i0(beta);
    const double fc = 0.5 * (fp_hz + fs_hz) / rate;
    const double mid = (double)(N - 1) * 0.5;
    double sum = 0.0;
    for (size_t n = 0; n < N; ++n) sum += ox_lp_tap(n, fc, mid, beta, i0b);
    if (sum == 0.0) sum = 1.0;
    for (size_t n = 0; n < N; ++n) out[n] = (float)(ox_lp_tap(n, fc, mid, beta, i0b) / sum);
    return (ptrdiff_t)N;
}

/* ---- the arbitrary resampler (src/resample.c:110-260) ----------------------
 * P phases of Q taps; p is the prototype times P, d its forward difference
 * (d[j] = p[j+1] - p[j], p[PQ] = 0). Output K sits at input position
 * base + K*step past the anchor; hist keeps the last Q inputs. */
typedef struct {
    float *p, *d;
    ox_cf32 *hist;
    size_t P, Q;
    double in_rate, out_rate, step, base;
    uint64_t K, in_off;
} orc_arb;

void orc_arb_destroy(orc_arb *r) {
    if (!r) return;
    free(r->p); free(r->d); free(r->hist); free(r);
}

void orc_arb_reset(orc_arb *r) {
    if (!r) return;
    memset(r->hist, 0, r->Q * sizeof(ox_cf32));
    r->base = 0.0; r->K = 0; r->in_off = 0;
}

orc_arb *orc_arb_create(double in_rate, double out_rate, double atten_db, unsigned nphase) {
    if (in_rate <= 0.0 || out_rate <= 0.0) return NULL;
    if (atten_db <= 0.0) atten_db = 60.0;
    const size_t P = nphase ? nphase : 64u;
    const double fsp = in_rate * (double)P;
    const double nyq = 0.5 * (in_rate < out_rate ? in_rate : out_rate);
    const double fp = 0.8 * nyq, fst = nyq;
    const ptrdiff_t nt = orc_design_lowpass(fp, fst, atten_db, fsp, NULL, 0);
    if (nt <= 0) return NULL;
    orc_arb *r = (orc_arb *)calloc(1, sizeof *r);
    if (!r) return NULL;
    r->P = P;
    r->Q = ((size_t)nt + P - 1) / P;
    const size_t PQ = P * r->Q;
    r->p = (float *)calloc(PQ, sizeof(float));
    r->d = (float *)calloc(PQ, sizeof(float));
    r->hist = (ox_cf32 *)calloc(r->Q, sizeof(ox_cf32));
    if (!r->p || !r->d || !r->hist || orc_design_lowpass(fp, fst, atten_db, fsp, r->p, (size_t)nt) != nt) {
        orc_arb_destroy(r);
        return NULL;
    }
    for (size_t j = 0; j < PQ; ++j) r->p[j] *= (float)P;
    for (size_t j = 0; j + 1 < PQ; ++j) r->d[j] = r->p[j + 1] - r->p[j];
    r->d[PQ - 1] = -r->p[PQ - 1];
    r->in_rate = in_rate; r->out_rate = out_rate;
    r->step = in_rate / out_rate;
    orc_arb_reset(r);
    return r;
}

size_t orc_arb_taps(const orc_arb *r) { return r ? r->Q : 0; }

ptrdiff_t orc_arb_process(orc_arb *r, const ox_cf32 *in, size_t n, ox_cf32 *out, size_t cap) {
    if (!r || (!in && n) || !out) return OX_E_ARG;
    const size_t P = r->P, Q = r->Q;
    const double inoff = (double)r->in_off;
    size_t k = 0;
    uint64_t K = r->K;
    double local = r->base + (double)K * r->step - inoff;
    while (local < (double)n) {
        const ptrdiff_t i = (ptrdiff_t)floor(local);
        const double frac = local - (double)i;
        const double ph = frac * (double)P;
        size_t b = (size_t)ph;
        if (b >= P) b = P - 1;
        const float mu = (float)(ph - (double)b);
        float ar = 0.0f, ai = 0.0f;
        for (size_t q = 0; q < Q; ++q) {
            const ptrdiff_t m = i - (ptrdiff_t)q;
            ox_cf32 x;
            if (m >= 0) {
                x = in[m];
            } else {
                const ptrdiff_t hb = (ptrdiff_t)Q + m;
                if (hb < 0) continue;
                x = r->hist[hb];
            }
            const float c = r->p[b + q * P] + mu * r->d[b + q * P];
            ar += c * x.re;
            ai += c * x.im;
        }
        if (k >= cap) return OX_E_CAP;
        out[k].re = ar; out[k].im = ai;
        ++k; ++K;
        local = r->base + (double)K * r->step - inoff;
    }
    r->K = K;
    r->in_off += n;
    if (n >= Q) {
        memcpy(r->hist, in + n - Q, Q * sizeof(ox_cf32));
    } else if (n) {
        memmove(r->hist, r->hist + n, (Q - n) * sizeof(ox_cf32));
        memcpy(r->hist + Q - n, in, n * sizeof(ox_cf32));
    }
    return (ptrdiff_t)k;
}

/* ---- radix-2 FFT in double (iterative, bit-reversed input) ----------------
 * tw[2j], tw[2j+1] = cos, sin of -2 pi j / N for j < N/2; a length-n
 * transform with n | N uses every (N/n)-th entry. sign = +1 conjugates the
 * twiddles (the unscaled inverse). */
static void ox_fft(double *a, size_t n, const double *tw, size_t N, int inverse) {
    size_t i, j = 0;
    for (i = 1; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = a[2 * i]; a[2 * i] = a[2 * j]; a[2 * j] = t;
            t = a[2 * i + 1]; a[2 * i + 1] = a[2 * j + 1]; a[2 * j + 1] = t;
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len >> 1, step = N / len;
        for (i = 0; i < n; i += len) {
            for (size_t k = 0; k < half; ++k) {
                const double wr = tw[2 * k * step];
                const double wi = inverse ? -tw[2 * k * step + 1] : tw[2 * k * step + 1];
                double *u = a + 2 * (i + k), *v = a + 2 * (i + k + half);
                const double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] += vr; u[1] += vi;
            }
        }
    }
}

/* ---- the extractor --------------------------------------------------------- */
typedef struct {
    int active;
    double offset, bw, out_rate, chan_rate, delta;
    unsigned decim, shift;
    size_t M, ntaps, ovd;
    ox_cf32 *H;                       /* nfft: the channel filter's spectrum */
    orc_arb **rs;                     /* max_nel, NULL entries: no resampling */
} ox_chan;

typedef struct {
    double fs, atten;
    size_t nfft, ov, hop;
    unsigned max_nel;
    int64_t blk;
    ox_cf32 *state;                   /* per element: hist (ov) ++ leftover (lc) */
    unsigned lc;
    ox_chan *ch;
    int nslots, cap_slots;
    double *tw;                       /* nfft: the forward twiddles */
    double *work;                     /* 2 nfft doubles */
    ox_cf32 *X;                       /* max_nel * nfft */
    ox_cf32 *ys, *valid;              /* nfft each */
} orc_osx;

static void ox_free_chan(ox_chan *c, unsigned max_nel) {
    if (!c->active) return;
    free(c->H);
    if (c->rs) {
        for (unsigned e = 0; e < max_nel; ++e) orc_arb_destroy(c->rs[e]);
        free(c->rs);
    }
    memset(c, 0, sizeof *c);
}

void orc_osx_destroy(orc_osx *x) {
    if (!x) return;
    for (int i = 0; i < x->nslots; ++i) ox_free_chan(&x->ch[i], x->max_nel);
    free(x->ch); free(x->state); free(x->tw); free(x->work); free(x->X); free(x->ys); free(x->valid);
    free(x);
}

orc_osx *orc_osx_create(double fs, size_t nfft, double atten_db, unsigned max_nel) {
    if (!(fs > 0.0) || nfft < 64 || (nfft & (nfft - 1)) || max_nel < 1) return NULL;
    orc_osx *x = (orc_osx *)calloc(1, sizeof *x);
    if (!x) return NULL;
    x->fs = fs;
    x->atten = atten_db < 20.0 ? 20.0 : atten_db;
    x->nfft = nfft; x->ov = nfft / 2; x->hop = nfft - x->ov; x->max_nel = max_nel;
    x->state = (ox_cf32 *)calloc((size_t)max_nel * nfft, sizeof(ox_cf32));
    x->tw = (double *)malloc(nfft * sizeof(double));
    x->work = (double *)malloc(2 * nfft * sizeof(double));
    x->X = (ox_cf32 *)malloc((size_t)max_nel * nfft * sizeof(ox_cf32));
    x->ys = (ox_cf32 *)malloc(nfft * sizeof(ox_cf32));
    x->valid = (ox_cf32 *)malloc(nfft * sizeof(ox_cf32));
    if (!x->state || !x->tw || !x->work || !x->X || !x->ys || !x->valid) {
        orc_osx_destroy(x);
        return NULL;
    }
    for (size_t j = 0; j < nfft / 2; ++j) {
        const double a = -2.0 * OX_PI * (double)j / (double)nfft;
        x->tw[2 * j] = cos(a);
        x->tw[2 * j + 1] = sin(a);
    }
    return x;
}

void orc_osx_reset(orc_osx *x) {
    if (!x) return;
    memset(x->state, 0, (size_t)x->max_nel * x->nfft * sizeof(ox_cf32));
    x->lc = 0; x->blk = 0;
    for (int i = 0; i < x->nslots; ++i)
        if (x->ch[i].active && x->ch[i].rs)
            for (unsigned e = 0; e < x->max_nel; ++e) orc_arb_reset(x->ch[i].rs[e]);
}

/* float in, double transform, float out (src/fft.c:88-135) */
static void ox_fft_f(const orc_osx *x, const ox_cf32 *in, size_t n, ox_cf32 *out, int inverse) {
    double *a = x->work;
    for (size_t i = 0; i < n; ++i) { a[2 * i] = (double)in[i].re; a[2 * i + 1] = (double)in[i].im; }
    ox_fft(a, n, x->tw, x->nfft, inverse);
    const double sc = inverse ? 1.0 / (double)n : 1.0;
    for (size_t i = 0; i < n; ++i) {
        out[i].re = (float)(a[2 * i] * sc);
        out[i].im = (float)(a[2 * i + 1] * sc);
    }
}

/* the largest power-of-two decimation whose rate still covers the target
 * and divides both nfft and the overlap (src/channelizer.c:564-574) */
static unsigned ox_decim(const orc_osx *x, double bw, double out_rate) {
    const double target = out_rate > 1.25 * bw ? out_rate : 1.25 * bw;
    unsigned d = 1;
    while (!(x->fs / (double)(2 * d) < target) && x->ov % (2 * d) == 0 && x->nfft % (2 * d) == 0) d *= 2;
    return d;
}

/* integer roll s = round(offset / bin) and the residual in Hz (:577-584) */
static void ox_tune(const orc_osx *x, ox_chan *c, double offset_hz) {
    const long s = (long)floor(offset_hz / x->fs * (double)x->nfft + 0.5);
    long sh = s % (long)x->nfft;
    if (sh < 0) sh += (long)x->nfft;
    c->offset = offset_hz;
    c->shift = (unsigned)sh;
    c->delta = offset_hz - (double)s * x->fs / (double)x->nfft;
}

int orc_osx_add(orc_osx *x, double offset_hz, double bw_hz, double out_rate) {
    if (!x || !(bw_hz > 0.0) || !(out_rate > 0.0)) return OX_E_ARG;
    const unsigned decim = ox_decim(x, bw_hz, out_rate);
    const double chan_rate = x->fs / (double)decim;
    const double fp = 0.5 * bw_hz;
    double fst = chan_rate - 0.5 * bw_hz;
    if (fst > 0.5 * x->fs) fst = 0.5 * x->fs;
    if (fst <= fp) return OX_E_ARG;
    const ptrdiff_t nt = orc_design_lowpass(fp, fst, x->atten, x->fs, NULL, 0);
    if (nt <= 0) return OX_E_ARG;
    float *taps = (float *)malloc((size_t)nt * sizeof(float));
    if (!taps) return OX_E_NOMEM;
    orc_design_lowpass(fp, fst, x->atten, x->fs, taps, (size_t)nt);
    size_t ntaps = (size_t)nt;
    if (ntaps > x->ov + 1) {          /* cap to the overlap, DC gain back to 1 */
        ntaps = x->ov + 1;
        double s = 0.0;
        for (size_t i = 0; i < ntaps; ++i) s += taps[i];
        if (s == 0.0) s = 1.0;
        for (size_t i = 0; i < ntaps; ++i) taps[i] = (float)(taps[i] / s);
    }
    int slot = -1;
    for (int i = 0; i < x->nslots; ++i)
        if (!x->ch[i].active) { slot = i; break; }
    if (slot < 0) {
        if (x->nslots >= x->cap_slots) {
            const int nc = x->cap_slots ? 2 * x->cap_slots : 8;
            ox_chan *p = (ox_chan *)realloc(x->ch, (size_t)nc * sizeof(ox_chan));
            if (!p) { free(taps); return OX_E_NOMEM; }
            memset(p + x->cap_slots, 0, (size_t)(nc - x->cap_slots) * sizeof(ox_chan));
            x->ch = p; x->cap_slots = nc;
        }
        slot = x->nslots++;
    }
    ox_chan *c = &x->ch[slot];
    memset(c, 0, sizeof *c);
    c->bw = bw_hz; c->out_rate = out_rate; c->decim = decim; c->chan_rate = chan_rate;
    c->ntaps = ntaps; c->M = x->nfft / decim; c->ovd = x->ov / decim;
    ox_tune(x, c, offset_hz);
    c->H = (ox_cf32 *)calloc(x->nfft, sizeof(ox_cf32));
    c->rs = (orc_arb **)calloc(x->max_nel, sizeof(orc_arb *));
    if (!c->H || !c->rs) { free(taps); free(c->H); free(c->rs); memset(c, 0, sizeof *c); return OX_E_NOMEM; }
    for (size_t i = 0; i < ntaps; ++i) c->H[i].re = taps[i];
    free(taps);
    ox_fft_f(x, c->H, x->nfft, c->H, 0);
    c->active = 1;
    if (fabs(chan_rate - out_rate) > 1e-6 * out_rate) {
        for (unsigned e = 0; e < x->max_nel; ++e) {
            c->rs[e] = orc_arb_create(chan_rate, out_rate, x->atten, 64);
            if (!c->rs[e]) { ox_free_chan(c, x->max_nel); return OX_E_NOMEM; }
        }
    }
    return slot;
}

int orc_osx_retune(orc_osx *x, int ch, double offset_hz) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return OX_E_ARG;
    ox_tune(x, &x->ch[ch], offset_hz);
    return 0;
}

int orc_osx_remove(orc_osx *x, int ch) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return OX_E_ARG;
    ox_free_chan(&x->ch[ch], x->max_nel);
    return 0;
}

int orc_osx_channels(const orc_osx *x) { return x ? x->nslots : 0; }

double orc_osx_chan_rate(const orc_osx *x, int ch) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return 0.0;
    return x->ch[ch].out_rate;
}

size_t orc_osx_out_max(const orc_osx *x, int ch, size_t n) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return 0;
    return (size_t)((double)n * x->ch[ch].out_rate / x->fs) + 64;
}

/* the decimating fold of one element's spectrum into M bins (float, the
 * reference's expression order), the M-point inverse, and the roll taken to
 * absolute time with the residual removed per sample (:704-737) */
static void ox_channel_hop(const orc_osx *x, const ox_chan *c, const ox_cf32 *X, int64_t bi) {
    const size_t M = c->M, nvalid = M - c->ovd, nfft = x->nfft;
    ox_cf32 *Yf = x->valid;           /* M bins, then overwritten by the output */
    for (size_t k = 0; k < M; ++k) {
        float ar = 0.0f, ai = 0.0f;
        for (unsigned j = 0; j < c->decim; ++j) {
            const size_t bin = k + (size_t)j * M;
            const ox_cf32 xv = X[(bin + c->shift) & (nfft - 1)], hv = c->H[bin];
            ar += xv.re * hv.re - xv.im * hv.im;
            ai += xv.re * hv.im + xv.im * hv.re;
        }
        Yf[k].re = ar; Yf[k].im = ai;
    }
    ox_fft_f(x, Yf, M, x->ys, 1);
    const double invd = 1.0 / (double)c->decim;
    const int64_t start = bi * (int64_t)x->hop - (int64_t)x->ov;
    int64_t smod = ((int64_t)c->shift * start) % (int64_t)nfft;
    if (smod < 0) smod += (int64_t)nfft;
    const double a0 = (double)smod / (double)nfft;
    for (size_t k = 0; k < nvalid; ++k) {
        const int64_t nabs = bi * (int64_t)x->hop + (int64_t)k * (int64_t)c->decim;
        const double ph = -2.0 * OX_PI * (a0 + c->delta * (double)nabs / x->fs);
        const double cr = cos(ph), si = sin(ph);
        const double yr = x->ys[c->ovd + k].re * invd, yi = x->ys[c->ovd + k].im * invd;
        x->valid[k].re = (float)(yr * cr - yi * si);
        x->valid[k].im = (float)(yr * si + yi * cr);
    }
}

ptrdiff_t orc_osx_process_n(orc_osx *x, const ox_cf32 *const *ins, unsigned nel, size_t n,
                            ox_cf32 *const *outs, size_t *out_counts, size_t cap_each) {
    if (!x || !ins || nel < 1 || nel > x->max_nel || !out_counts) return OX_E_ARG;
    const size_t nfft = x->nfft, ov = x->ov, hop = x->hop;
    const int ns = x->nslots;
    for (int ci = 0; ci < ns; ++ci) out_counts[ci] = 0;
    const size_t avail = (size_t)x->lc + n, m = avail / hop;
    if (m == 0) {
        for (unsigned e = 0; e < nel; ++e)
            if (n) memcpy(x->state + (size_t)e * nfft + ov + x->lc, ins[e], n * sizeof(ox_cf32));
        x->lc = (unsigned)avail;
        return ns;
    }
    /* s = state ++ in; block i is s[i*hop, i*hop + nfft) */
    const size_t have = ov + x->lc;
    for (size_t i = 0; i < m; ++i) {
        for (unsigned e = 0; e < nel; ++e) {
            const ox_cf32 *st = x->state + (size_t)e * nfft;
            ox_cf32 *blk = x->ys;
            for (size_t s = 0; s < nfft; ++s) {
                const size_t g = i * hop + s;
                blk[s] = g < have ? st[g] : ins[e][g - have];
            }
            ox_fft_f(x, blk, nfft, x->X + (size_t)e * nfft, 0);
        }
        for (int ci = 0; ci < ns; ++ci) {
            const ox_chan *c = &x->ch[ci];
            if (!c->active) continue;
            const size_t nvalid = c->M - c->ovd;
            size_t emit = 0;
            for (unsigned e = 0; e < nel; ++e) {
                ox_channel_hop(x, c, x->X + (size_t)e * nfft, x->blk + (int64_t)i);
                ox_cf32 *dst = outs ? outs[(size_t)e * ns + ci] : NULL;
                if (!dst) return OX_E_ARG;
                const size_t wpos = out_counts[ci];
                if (c->rs[e]) {
                    const ptrdiff_t g = orc_arb_process(c->rs[e], x->valid, nvalid, dst + wpos, cap_each - wpos);
                    if (g < 0) return g;
                    emit = (size_t)g;
                } else {
                    if (wpos + nvalid > cap_each) return OX_E_CAP;
                    memcpy(dst + wpos, x->valid, nvalid * sizeof(ox_cf32));
                    emit = nvalid;
                }
            }
            out_counts[ci] += emit;
        }
    }
    /* the new state: s[m*hop, avail + ov), i.e. hist ++ the unconsumed tail */
    const size_t keep = ov + (avail - m * hop);
    for (unsigned e = 0; e < nel; ++e) {
        ox_cf32 *st = x->state + (size_t)e * nfft;
        ox_cf32 *tmp = x->ys;
        for (size_t s = 0; s < keep; ++s) {
            const size_t g = m * hop + s;
            tmp[s] = g < have ? st[g] : ins[e][g - have];
        }
        memcpy(st, tmp, keep * sizeof(ox_cf32));
    }
    x->lc = (unsigned)(avail - m * hop);
    x->blk += (int64_t)m;
    return ns;
}

int orc_osx_describe(const orc_osx *x, char *buf, size_t cap) {
    if (!x || !buf || cap == 0) return OX_E_ARG;
    int active = 0;
    for (int i = 0; i < x->nslots; ++i) active += x->ch[i].active;
    return snprintf(buf, cap, "OSX %.6g MSPS: %zu-pt FFT, ov %zu, %d channel(s), %.0f dB, <=%u el",
                    x->fs / 1e6, x->nfft, x->ov, active, x->atten, x->max_nel);
}
