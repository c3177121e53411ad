/* The overlap-save extractor's host layer, in C99 (reference
 * src/channelizer.c:473-788, with the low-pass design of src/design.c:24-64
 * and the arbitrary resampler's design of src/resample.c:130-167).
 *
 * Argument checks, return codes, channel slots, decimation choice, filter
 * design and the tuning arithmetic are the reference's and run here; the
 * transforms, folds, rolls, resampling and state movement run on the device
 * (osx.cu), on the handle's stream.
 *
 * Device layout per handle (allocated by create; add allocates a channel's):
 *   state     two buffers (ping-pong) of max_nel x nfft samples: each
 *             element's hist (ov) ++ leftover (lc), the reference's
 *             x->hist ++ x->leftover
 *   in        2 x max_nel x chunk_in samples of input staging (host calls),
 *             alternating chunk by chunk: a chunk's upload runs on a copy stream
 *             while the previous chunk's kernels run
 *   tw        nfft double2 (cos, -sin)(2 pi j / nfft), every transform's roots
 *   X, T, Y   a chunk's spectra and the four-step scratch (nfft > 4096 only)
 *   table     the per-call channel table and input pointer array (+ a
 *             pinned mirror)
 *   channel   H (nfft, the filter's spectrum), v (per element the channel's
 *             samples of a chunk; for a resampled channel behind Q samples
 *             of resampler history), the resampler's taps and output staging
 *
 * A call is processed in chunks of at most chunk_hops blocks, each exactly
 * what the reference computes for that sub-block (its output is chunking-
 * invariant, which tests check bit for bit).
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "host_internal.h"

#define OSX_PI 3.14159265358979323846
/* input samples per element per chunk: enough blocks to fill the GPU */
#define OSX_CHUNK_SAMPLES ((size_t)1 << 22)
#define OSX_CHUNK_SAMPLES_BIG ((size_t)1 << 21)  /* nfft > 4096: the spectra go through HBM */
#define OSX_RS_PHASES 64                       /* resampler phases (:635) */

typedef struct {
    int active;
    double offset, bw, out_rate, chan_rate, delta;
    unsigned decim, shift;
    size_t M, ntaps, ovd, nvalid;
    void *d_H;                    /* nfft cf32                                   */
    void *d_v;                    /* [2][max_nel][vstride] cf32: a chunk's samples
                                   * (behind Q of resampler history); two halves
                                   * that alternate chunk by chunk              */
    int tix;                      /* index in the current call's table           */
    size_t vstride;
    /* the arbitrary resampler (when chan_rate != out_rate) */
    int rs;
    size_t P, Q;
    void *d_pd;                   /* P*Q taps (x P) then P*Q forward differences */
    double step;
    double *base;                 /* per element: the anchor, outputs and inputs */
    uint64_t *K, *in_off;         /* since it (src/resample.c:110-128)           */
    void *d_out;                  /* [max_nel][ostride] resampled output staging */
    uint64_t last_got;            /* outputs of the current chunk (per element) */
    size_t ostride;
} osx_chan;

struct atkdsp_osx {
    double fs, atten;
    size_t nfft, ov, hop;
    unsigned max_nel;
    int lognfft;
    int64_t blk;
    unsigned lc;
    int dev;
    void *stream;
    void *d_state;                /* 2 * max_nel * nfft cf32                     */
    int cur;
    void *d_in;                   /* 2 * max_nel * chunk_in cf32: two input stagings
                                   * that alternate chunk by chunk (host calls) */
    int inb;                      /* the staging the next chunk fills            */
    void *cstream;                /* the copy stream: a chunk's upload overlaps the
                                   * previous chunk's kernels                    */
    void *ev_up[2], *ev_done[2];  /* staging b uploaded / read by its kernels     */
    size_t chunk_hops, chunk_in;
    void *d_tw;
    void *d_X, *d_T, *d_Y;
    void *d_tbl, *h_tbl;          /* atkb_osx_chan[cap_slots] | ins[max_nel]     */
    size_t tbl_bytes;
    int nsmall, nmid, nbig;       /* the current call's table: channels by class */
    int npacks;                   /* ... and the small ones' packs               */
    int par;                      /* which half of the channels' staging is current */
    osx_chan *ch;
    size_t *wpos;                 /* cap_slots: a call's samples per slot so far */
    int nslots, cap_slots, tbl_slots;
};

/* ================================================================ design */
static double osx_kaiser_beta(double atten_db) {
    if (atten_db > 50.0) return 0.1102 * (atten_db - 8.7);
    if (atten_db >= 21.0) return 0.5842 * pow(atten_db - 21.0, 0.4) + 0.07886 * (atten_db - 21.0);
    return 0.0;
}

static double osx_i0(double x) {
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

/* Kaiser length for a transition band (src/design.c:24-32): odd, >= 3 */
static size_t osx_kaiser_len(double atten_db, double tr_hz, double rate) {
    if (tr_hz <= 0.0 || rate <= 0.0) return 0;
    const double dw = 2.0 * OSX_PI * tr_hz / rate;
    const double est = (atten_db > 8.0 ? (atten_db - 8.0) : 1.0) / (2.285 * dw);
    size_t N = (size_t)ceil(est) + 1;
    if (N < 3) N = 3;
    if ((N & 1) == 0) ++N;
    return N;
}

static double osx_lp_tap(size_t n, double fc, double mid, double beta, double i0b) {
    const double t = (double)n - mid;
    const double x = 2.0 * fc * t;
    const double sinc = (t == 0.0) ? 1.0 : sin(OSX_PI * x) / (OSX_PI * x);
    const double r = t / mid;
    const double w = osx_i0(beta * sqrt(r * r < 1.0 ? 1.0 - r * r : 0.0)) / i0b;
    return 2.0 * fc * sinc * w;
}

/* atkdsp_design_lowpass (src/design.c:34-64): the tap count (out == NULL) or
 * the taps, each evaluated in double and rounded once after normalising */
static ptrdiff_t osx_lowpass(double fp_hz, double fs_hz, double atten_db, double rate, float *out,
                             size_t cap) {
    if (rate <= 0.0 || fp_hz < 0.0 || fs_hz <= fp_hz || fs_hz > rate * 0.5 + 1e-9) return ATKDSP_E_ARG;
    const size_t N = osx_kaiser_len(atten_db, fs_hz - fp_hz, rate);
    if (!out) return (ptrdiff_t)N;
    if (cap < N) return ATKDSP_E_CAP;
    const double beta = osx_kaiser_beta(atten_db), i0b = osx_i0(beta);
    const double fc = 0.5 * (fp_hz + fs_hz) / rate, mid = (double)(N - 1) * 0.5;
    double sum = 0.0;
    size_t n;
    for (n = 0; n < N; ++n) sum += osx_lp_tap(n, fc, mid, beta, i0b);
    if (sum == 0.0) sum = 1.0;
    for (n = 0; n < N; ++n) out[n] = (float)(osx_lp_tap(n, fc, mid, beta, i0b) / sum);
    return (ptrdiff_t)N;
}

/* forward DFT in double of n = 2^k interleaved values in place (radix 2) */
static void osx_host_fft(double *a, size_t n) {
    size_t i, j = 0, len;
    for (i = 1; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = a[2 * i]; a[2 * i] = a[2 * j]; a[2 * j] = t;
            t = a[2 * i + 1]; a[2 * i + 1] = a[2 * j + 1]; a[2 * j + 1] = t;
        }
    }
    for (len = 2; len <= n; len <<= 1) {
        const size_t half = len >> 1;
        size_t k;
        for (k = 0; k < half; ++k) {
            const double ang = -2.0 * OSX_PI * (double)k / (double)len;
            const double wr = cos(ang), wi = sin(ang);
            for (i = k; i < n; i += len) {
                double *u = a + 2 * i, *v = a + 2 * (i + half);
                const double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] += vr; u[1] += vi;
            }
        }
    }
}

/* ================================================================ handle */
static void osx_chan_free(osx_chan *c) {
    if (!c->active) return;
    atkb_free(c->d_H); atkb_free(c->d_v); atkb_free(c->d_pd); atkb_free(c->d_out);
    free(c->base); free(c->K); free(c->in_off);
    memset(c, 0, sizeof *c);
}

ATKDSP_API void atkdsp_osx_destroy(atkdsp_osx *x) {
    int i;
    if (!x) return;
    if (x->stream) atkb_stream_sync(x->stream);
    for (i = 0; i < x->nslots; ++i) osx_chan_free(&x->ch[i]);
    free(x->ch); free(x->wpos);
    if (x->cstream) atkb_stream_sync(x->cstream);
    for (i = 0; i < 2; ++i) { atkb_event_destroy(x->ev_up[i]); atkb_event_destroy(x->ev_done[i]); }
    atkb_stream_destroy(x->cstream);
    atkb_free(x->d_state); atkb_free(x->d_in); atkb_free(x->d_tw); atkb_free(x->d_X); atkb_free(x->d_T); atkb_free(x->d_Y);
    atkb_free(x->d_tbl); atkb_host_free(x->h_tbl);
    atkb_stream_destroy(x->stream);
    free(x);
}

static int ilog2(size_t v) {
    int l = 0;
    while (((size_t)1 << l) < v) ++l;
    return l;
}

/* the per-call table: channel entries for `slots`, then two sets of max_nel
 * input pointers (one per input staging; device-pointer calls use the
 * first), then per entry max_nel output pointers (device-pointer calls),
 * then slots + 1 pack boundaries */
static size_t tbl_ins_off(const atkdsp_osx *x) { return atkb_align16((size_t)x->tbl_slots * sizeof(atkb_osx_chan)); }
static size_t tbl_outs_off(const atkdsp_osx *x) { return tbl_ins_off(x) + 2 * (size_t)x->max_nel * sizeof(void *); }
static size_t tbl_packs_off(const atkdsp_osx *x) {
    return tbl_outs_off(x) + (size_t)x->tbl_slots * x->max_nel * sizeof(void *);
}

static int osx_table_reserve(atkdsp_osx *x, int slots) {
    if (slots <= x->tbl_slots && x->d_tbl) return ATKB_OK;
    int want = x->tbl_slots ? x->tbl_slots : 8;
    while (want < slots) want *= 2;
    const size_t bytes = atkb_align16((size_t)want * sizeof(atkb_osx_chan)) +
                         (size_t)x->max_nel * sizeof(void *) * (2 + (size_t)want) + (size_t)(want + 1) * sizeof(int);
    void *d = NULL, *h = NULL;
    int rc = atkb_malloc(&d, bytes);
    if (rc == ATKB_OK) rc = atkb_host_alloc(&h, bytes);
    if (rc != ATKB_OK) { atkb_free(d); atkb_host_free(h); return rc; }
    if (x->stream) atkb_stream_sync(x->stream);   /* the old table may still be read */
    atkb_free(x->d_tbl); atkb_host_free(x->h_tbl);
    x->d_tbl = d; x->h_tbl = h; x->tbl_bytes = bytes; x->tbl_slots = want;
    return ATKB_OK;
}

ATKDSP_API atkdsp_osx *atkdsp_osx_create(double fs, size_t nfft, double atten_db, unsigned max_nel) {
    if (!(fs > 0.0) || nfft < 64 || (nfft & (nfft - 1)) || max_nel < 1) return NULL;
    if (nfft > ATKB_OSX_NFFT_MAX || max_nel > 4096) return NULL;
    atkdsp_osx *x = (atkdsp_osx *)calloc(1, sizeof *x);
    if (!x) return NULL;
    x->fs = fs;
    x->atten = atten_db < 20.0 ? 20.0 : atten_db;
    x->nfft = nfft; x->ov = nfft / 2; x->hop = nfft - x->ov; x->max_nel = max_nel;
    x->lognfft = ilog2(nfft);
    x->chunk_hops = (nfft > ATKB_OSX_FUSED_MAX ? OSX_CHUNK_SAMPLES_BIG : OSX_CHUNK_SAMPLES) / x->hop;
    if (x->chunk_hops < 1) x->chunk_hops = 1;
    x->chunk_in = (x->chunk_hops + 1) * x->hop;
    int rc = atkb_get_device(&x->dev);
    if (rc == ATKB_OK) rc = atkb_stream_create(&x->stream);
    if (rc == ATKB_OK) rc = atkb_malloc(&x->d_state, 2 * (size_t)max_nel * nfft * sizeof(atkdsp_cf32));
    if (rc == ATKB_OK) rc = atkb_malloc(&x->d_in, 2 * (size_t)max_nel * x->chunk_in * sizeof(atkdsp_cf32));
    if (rc == ATKB_OK) rc = atkb_stream_create(&x->cstream);
    for (int b = 0; b < 2 && rc == ATKB_OK; ++b) {
        rc = atkb_event_create(&x->ev_up[b]);
        if (rc == ATKB_OK) rc = atkb_event_create(&x->ev_done[b]);
        /* both stagings start free */
        if (rc == ATKB_OK) rc = atkb_event_record(x->ev_done[b], x->stream);
    }
    if (rc == ATKB_OK) rc = atkb_malloc(&x->d_tw, nfft * 2 * sizeof(double));
    if (rc == ATKB_OK && nfft > ATKB_OSX_FUSED_MAX) {
        const size_t pts = (size_t)max_nel * x->chunk_hops * nfft;
        rc = atkb_malloc(&x->d_X, pts * sizeof(atkdsp_cf32));
        if (rc == ATKB_OK) rc = atkb_malloc(&x->d_T, pts * 2 * sizeof(double));
        if (rc == ATKB_OK) rc = atkb_malloc(&x->d_Y, pts * 2 * sizeof(double));
    }
    if (rc == ATKB_OK) rc = osx_table_reserve(x, 8);
    if (rc == ATKB_OK) rc = atkb_memset(x->d_state, 0, 2 * (size_t)max_nel * nfft * sizeof(atkdsp_cf32), x->stream);
    if (rc == ATKB_OK) {
        double *tw = (double *)malloc(nfft * 2 * sizeof(double));
        size_t j;
        if (!tw) {
            rc = ATKB_E_NOMEM;
        } else {
            for (j = 0; j < nfft; ++j) {
                const double a = 2.0 * OSX_PI * (double)j / (double)nfft;
                tw[2 * j] = cos(a);
                tw[2 * j + 1] = -sin(a);
            }
            rc = atkb_h2d(x->d_tw, tw, nfft * 2 * sizeof(double), x->stream);
            if (rc == ATKB_OK) rc = atkb_stream_sync(x->stream);
            free(tw);
        }
    }
    if (rc != ATKB_OK) {
        atkdsp_osx_destroy(x);
        return NULL;
    }
    return x;
}

static void osx_rs_rewind(osx_chan *c, unsigned max_nel) {
    unsigned e;
    for (e = 0; e < max_nel; ++e) { c->base[e] = 0.0; c->K[e] = 0; c->in_off[e] = 0; }
}

ATKDSP_API void atkdsp_osx_reset(atkdsp_osx *x) {
    int i;
    if (!x) return;
    atkb_memset(x->d_state, 0, 2 * (size_t)x->max_nel * x->nfft * sizeof(atkdsp_cf32), x->stream);
    x->lc = 0; x->blk = 0;
    for (i = 0; i < x->nslots; ++i) {
        osx_chan *c = &x->ch[i];
        if (!c->active || !c->rs) continue;
        osx_rs_rewind(c, x->max_nel);
        atkb_memset(c->d_v, 0, 2 * (size_t)x->max_nel * c->vstride * sizeof(atkdsp_cf32), x->stream);
    }
    atkb_stream_sync(x->stream);
}

/* the largest power-of-two decimation whose rate still covers the target
 * and divides both nfft and the overlap (src/channelizer.c:564-574) */
static unsigned osx_pick_decim(const atkdsp_osx *x, double bw, double out_rate) {
    const double target = out_rate > 1.25 * bw ? out_rate : 1.25 * bw;
    unsigned d = 1;
    while (!(x->fs / (double)(2 * d) < target) && x->ov % (2 * d) == 0 && x->nfft % (2 * d) == 0) d *= 2;
    return d;
}

/* the integer roll s = round(offset / bin) and the residual (Hz) (:577-584) */
static void osx_tune(const atkdsp_osx *x, osx_chan *c, double offset_hz) {
    const long s = (long)floor(offset_hz / x->fs * (double)x->nfft + 0.5);
    long sh = s % (long)x->nfft;
    if (sh < 0) sh += (long)x->nfft;
    c->offset = offset_hz;
    c->shift = (unsigned)sh;
    c->delta = offset_hz - (double)s * x->fs / (double)x->nfft;
}

/* the resampler's prototype at in_rate * P, cut at the lower Nyquist, times
 * P, and its forward differences (src/resample.c:130-167) */
static int osx_rs_design(const atkdsp_osx *x, osx_chan *c) {
    const size_t P = OSX_RS_PHASES;
    const double in_rate = c->chan_rate, out_rate = c->out_rate;
    const double fsp = in_rate * (double)P;
    const double nyq = 0.5 * (in_rate < out_rate ? in_rate : out_rate);
    const double fp = 0.8 * nyq, fst = nyq;
    const ptrdiff_t nt = osx_lowpass(fp, fst, x->atten, fsp, NULL, 0);
    if (nt <= 0) return ATKB_E_NOMEM;            /* the reference's create fails: NOMEM */
    c->P = P;
    c->Q = ((size_t)nt + P - 1) / P;
    const size_t PQ = P * c->Q;
    float *pd = (float *)calloc(2 * PQ, sizeof(float));
    if (!pd) return ATKB_E_NOMEM;
    float *p = pd, *d = pd + PQ;
    osx_lowpass(fp, fst, x->atten, fsp, p, (size_t)nt);
    size_t j;
    for (j = 0; j < PQ; ++j) p[j] *= (float)P;
    for (j = 0; j + 1 < PQ; ++j) d[j] = p[j + 1] - p[j];
    d[PQ - 1] = -p[PQ - 1];
    c->step = in_rate / out_rate;
    int rc = atkb_malloc(&c->d_pd, 2 * PQ * sizeof(float));
    if (rc == ATKB_OK) rc = atkb_h2d(c->d_pd, pd, 2 * PQ * sizeof(float), x->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(x->stream);
    free(pd);
    return rc;
}

ATKDSP_API int atkdsp_osx_add(atkdsp_osx *x, double offset_hz, double bw_hz, double out_rate) {
    if (!x || !(bw_hz > 0.0) || !(out_rate > 0.0)) return ATKDSP_E_ARG;
    const unsigned decim = osx_pick_decim(x, bw_hz, out_rate);
    const double chan_rate = x->fs / (double)decim;
    const double fp = 0.5 * bw_hz;
    double fst = chan_rate - 0.5 * bw_hz;
    if (fst > 0.5 * x->fs) fst = 0.5 * x->fs;
    if (fst <= fp) return ATKDSP_E_ARG;
    const ptrdiff_t nt = osx_lowpass(fp, fst, x->atten, x->fs, NULL, 0);
    if (nt <= 0) return ATKDSP_E_ARG;
    float *taps = (float *)malloc((size_t)nt * sizeof(float));
    double *spec = (double *)calloc(2 * x->nfft, sizeof(double));
    float *H = (float *)malloc(2 * x->nfft * sizeof(float));
    if (!taps || !spec || !H) { free(taps); free(spec); free(H); return ATKDSP_E_NOMEM; }
    osx_lowpass(fp, fst, x->atten, x->fs, taps, (size_t)nt);
    size_t ntaps = (size_t)nt, i;
    if (ntaps > x->ov + 1) {          /* cap to the overlap, DC gain back to 1 (:596-601) */
        double s = 0.0;
        ntaps = x->ov + 1;
        for (i = 0; i < ntaps; ++i) s += taps[i];
        if (s == 0.0) s = 1.0;
        for (i = 0; i < ntaps; ++i) taps[i] = (float)(taps[i] / s);
    }
    /* H = the float spectrum of the zero-padded taps (double transform) */
    for (i = 0; i < ntaps; ++i) spec[2 * i] = (double)taps[i];
    free(taps);
    osx_host_fft(spec, x->nfft);
    for (i = 0; i < 2 * x->nfft; ++i) H[i] = (float)spec[i];
    free(spec);
    /* a slot: the first free one, else a new one (:603-615) */
    int slot = -1, k;
    for (k = 0; k < x->nslots; ++k)
        if (!x->ch[k].active) { slot = k; break; }
    if (slot < 0) {
        if (x->nslots >= x->cap_slots) {
            const int nc = x->cap_slots ? 2 * x->cap_slots : 8;
            osx_chan *p = (osx_chan *)realloc(x->ch, (size_t)nc * sizeof(osx_chan));
            if (p) x->ch = p;
            size_t *w = p ? (size_t *)realloc(x->wpos, (size_t)nc * sizeof(size_t)) : NULL;
            if (!w) { free(H); return ATKDSP_E_NOMEM; }
            x->wpos = w;
            memset(p + x->cap_slots, 0, (size_t)(nc - x->cap_slots) * sizeof(osx_chan));
            x->cap_slots = nc;
        }
        slot = x->nslots;
    }
    osx_chan c;
    memset(&c, 0, sizeof c);
    c.bw = bw_hz; c.out_rate = out_rate; c.decim = decim; c.chan_rate = chan_rate; c.ntaps = ntaps;
    c.M = x->nfft / decim; c.ovd = x->ov / decim; c.nvalid = c.M - c.ovd;
    osx_tune(x, &c, offset_hz);
    c.active = 1;
    int rc = osx_table_reserve(x, slot + 1);
    if (rc == ATKB_OK) rc = atkb_malloc(&c.d_H, x->nfft * sizeof(atkdsp_cf32));
    if (rc == ATKB_OK) rc = atkb_h2d(c.d_H, H, x->nfft * sizeof(atkdsp_cf32), x->stream);
    if (rc == ATKB_OK && fabs(chan_rate - out_rate) > 1e-6 * out_rate) {
        c.rs = 1;
        c.base = (double *)calloc(x->max_nel, sizeof(double));
        c.K = (uint64_t *)calloc(x->max_nel, sizeof(uint64_t));
        c.in_off = (uint64_t *)calloc(x->max_nel, sizeof(uint64_t));
        rc = (c.base && c.K && c.in_off) ? osx_rs_design(x, &c) : ATKB_E_NOMEM;
        if (rc == ATKB_OK) {
            c.ostride = (size_t)ceil((double)(x->chunk_hops * c.nvalid) / c.step) + 4;
            rc = atkb_malloc(&c.d_out, (size_t)x->max_nel * c.ostride * sizeof(atkdsp_cf32));
        }
    }
    if (rc == ATKB_OK) {
        c.vstride = c.Q + x->chunk_hops * c.nvalid;
        rc = atkb_malloc(&c.d_v, 2 * (size_t)x->max_nel * c.vstride * sizeof(atkdsp_cf32));
    }
    if (rc == ATKB_OK) rc = atkb_memset(c.d_v, 0, 2 * (size_t)x->max_nel * c.vstride * sizeof(atkdsp_cf32), x->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(x->stream);
    free(H);
    if (rc != ATKB_OK) {
        osx_chan_free(&c);
        return rc == ATKB_E_NOMEM ? ATKDSP_E_NOMEM : atkb_map_rc(rc);
    }
    x->ch[slot] = c;
    if (slot == x->nslots) x->nslots++;
    return slot;
}

ATKDSP_API int atkdsp_osx_retune(atkdsp_osx *x, int ch, double offset_hz) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return ATKDSP_E_ARG;
    osx_tune(x, &x->ch[ch], offset_hz);
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_osx_remove(atkdsp_osx *x, int ch) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return ATKDSP_E_ARG;
    atkb_stream_sync(x->stream);
    osx_chan_free(&x->ch[ch]);
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_osx_channels(const atkdsp_osx *x) { return x ? x->nslots : 0; }

ATKDSP_API double atkdsp_osx_chan_rate(const atkdsp_osx *x, int ch) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return 0.0;
    return x->ch[ch].out_rate;
}

ATKDSP_API size_t atkdsp_osx_out_max(const atkdsp_osx *x, int ch, size_t n) {
    if (!x || ch < 0 || ch >= x->nslots || !x->ch[ch].active) return 0;
    return (size_t)((double)n * x->ch[ch].out_rate / x->fs) + 64;
}

ATKDSP_API int atkdsp_osx_describe(const atkdsp_osx *x, char *buf, size_t cap) {
    int i, active = 0;
    if (!x || !buf || cap == 0) return ATKDSP_E_ARG;
    for (i = 0; i < x->nslots; ++i) active += x->ch[i].active;
    return snprintf(buf, cap, "OSX %.6g MSPS: %zu-pt FFT, ov %zu, %d channel(s), %.0f dB, <=%u el",
                    x->fs / 1e6, x->nfft, x->ov, active, x->atten, x->max_nel);
}

ATKDSP_API void *atkdsp_gpu_osx_stream(atkdsp_osx *x) { return x ? x->stream : NULL; }

ATKDSP_API int atkdsp_gpu_osx_sync(atkdsp_osx *x) {
    if (!x) return ATKDSP_E_ARG;
    return atkb_map_rc(atkb_stream_sync(x->stream));
}

/* ================================================================ process */
/* resampler outputs K >= K0 at input position base + K*step - inoff below n,
 * with the reference's expression (src/resample.c:205, :233) */
static double rs_local(double base, uint64_t K, double step, double inoff) {
    return base + (double)K * step - inoff;
}

static uint64_t rs_count(const osx_chan *c, unsigned e, size_t len) {
    const double inoff = (double)c->in_off[e], n = (double)len;
    const uint64_t K0 = c->K[e];
    double l0 = rs_local(c->base[e], K0, c->step, inoff);
    if (!(l0 < n)) return 0;
    uint64_t K = K0 + (uint64_t)((n - l0) / c->step);
    while (K > K0 && !(rs_local(c->base[e], K - 1, c->step, inoff) < n)) --K;
    while (rs_local(c->base[e], K, c->step, inoff) < n) ++K;
    return K - K0;
}

static int same_rs_state(const osx_chan *c, unsigned a, unsigned b) {
    return c->K[a] == c->K[b] && c->in_off[a] == c->in_off[b] && c->base[a] == c->base[b];
}

typedef struct {
    int dev_in, dev_out;          /* inputs / outputs are device pointers        */
    const atkdsp_cf32 *const *ins;
    atkdsp_cf32 *const *outs;
    unsigned nel;
    size_t *wpos;                 /* per slot: samples written so far this call  */
} osx_io;

/* one chunk: `sub` new samples per element at input offset `off`, completing
 * h = (lc + sub) / hop >= 1 blocks */
static int osx_chunk(atkdsp_osx *x, const osx_io *io, size_t off, size_t sub, size_t hop_base) {
    const unsigned nel = io->nel;
    const size_t avail = x->lc + sub, h = avail / x->hop;
    const int b = io->dev_in ? 0 : x->inb;
    const void *const *d_ins = (const void *const *)((char *)x->d_tbl + tbl_ins_off(x)) + (size_t)b * x->max_nel;
    void *const *d_outs = (void *const *)((char *)x->d_tbl + tbl_outs_off(x));
    unsigned e;
    int rc = ATKB_OK, ci;
    if (!io->dev_in) {
        /* the upload on the copy stream, once the chunk that last read this
         * staging is done; this chunk's kernels wait for the upload */
        atkdsp_cf32 *stage = (atkdsp_cf32 *)x->d_in + (size_t)b * x->max_nel * x->chunk_in;
        rc = atkb_stream_wait(x->cstream, x->ev_done[b]);
        for (e = 0; e < nel && rc == ATKB_OK; ++e)
            if (sub)
                rc = atkb_h2d(stage + (size_t)e * x->chunk_in, io->ins[e] + off, sub * sizeof(atkdsp_cf32),
                              x->cstream);
        if (rc == ATKB_OK) rc = atkb_event_record(x->ev_up[b], x->cstream);
        if (rc == ATKB_OK) rc = atkb_stream_wait(x->stream, x->ev_up[b]);
    }
    if (rc != ATKB_OK) return rc;
    atkdsp_cf32 *st = (atkdsp_cf32 *)x->d_state + (size_t)x->cur * x->max_nel * x->nfft;
    atkdsp_cf32 *st2 = (atkdsp_cf32 *)x->d_state + (size_t)(x->cur ^ 1) * x->max_nel * x->nfft;
    atkb_osx_run R;
    memset(&R, 0, sizeof R);
    R.state = st; R.ins = d_ins;
    R.state_stride = (long long)x->nfft; R.in_off = io->dev_in ? (long long)off : 0;
    R.head = (long long)(x->ov + x->lc); R.blk0 = x->blk;
    R.tw = x->d_tw; R.chans = (const atkb_osx_chan *)x->d_tbl; R.h_chans = (const atkb_osx_chan *)x->h_tbl;
    R.fs = x->fs; R.hop_base = (long long)hop_base; R.par = x->par;
    R.nfft = (int)x->nfft; R.lognfft = x->lognfft; R.hop = (int)x->hop; R.ov = (int)x->ov;
    R.nchans = x->nsmall + x->nmid + x->nbig; R.nsmall = x->nsmall; R.nmid = x->nmid;
    R.packs = (const int *)((char *)x->d_tbl + tbl_packs_off(x)); R.npacks = x->npacks;
    R.X = x->d_X; R.T = x->d_T; R.Y = x->d_Y;
    if (R.nchans > 0) rc = atkb_osx_launch(&R, (int)h, (int)nel, x->stream);   /* no channel: nothing to compute */
    if (rc != ATKB_OK) return rc;
    /* the resampled channels: one launch for every run of the chunk (a run
     * is a channel and a group of elements whose resamplers stand at the
     * same place), then every channel's samples out to the host */
    atkb_osx_rs runs[ATKB_OSX_RS_MAX];
    int nruns = 0;
    for (ci = 0; ci < x->nslots && rc == ATKB_OK; ++ci) {
        osx_chan *c = &x->ch[ci];
        if (!c->active || !c->rs) continue;
        const size_t nv = h * c->nvalid;
        const size_t half = (size_t)x->max_nel * c->vstride;
        atkdsp_cf32 *v = (atkdsp_cf32 *)c->d_v + (size_t)x->par * half;
        atkdsp_cf32 *vn = (atkdsp_cf32 *)c->d_v + (size_t)(x->par ^ 1) * half;
        for (e = 0; e < nel && rc == ATKB_OK;) {
            unsigned e1 = e + 1, u;
            while (e1 < nel && same_rs_state(c, e, e1)) ++e1;
            const uint64_t got = rs_count(c, e, nv);
            atkb_osx_rs *r = &runs[nruns++];
            memset(r, 0, sizeof *r);
            r->v = v + (size_t)e * c->vstride;
            r->v_next = vn + (size_t)e * c->vstride;
            r->v_stride = (long long)c->vstride;
            r->nv = (long long)nv;
            r->pd = (const float *)c->d_pd;
            r->base = c->base[e]; r->step = c->step; r->inoff = (double)c->in_off[e];
            r->K0 = (unsigned long long)c->K[e];
            r->count = (long long)got;
            r->outs = io->dev_out ? d_outs + (size_t)c->tix * x->max_nel + e : NULL;
            r->out_off = (long long)io->wpos[ci];
            r->stage = (atkdsp_cf32 *)c->d_out + (size_t)e * c->ostride;
            r->stage_stride = (long long)c->ostride;
            r->Q = (int)c->Q; r->P = (int)c->P; r->nel = (int)(e1 - e);
            for (u = e; u < e1; ++u) { c->K[u] += got; c->in_off[u] += nv; }
            c->last_got = got;
            if (nruns == ATKB_OSX_RS_MAX) {
                rc = atkb_osx_resample_batch(runs, nruns, x->stream);
                nruns = 0;
            }
            e = e1;
        }
    }
    if (rc == ATKB_OK) rc = atkb_osx_resample_batch(runs, nruns, x->stream);
    for (ci = 0; ci < x->nslots && rc == ATKB_OK; ++ci) {
        osx_chan *c = &x->ch[ci];
        if (!c->active) continue;
        const size_t got = c->rs ? (size_t)c->last_got : h * c->nvalid;
        const atkdsp_cf32 *src = c->rs ? (const atkdsp_cf32 *)c->d_out
                                       : (const atkdsp_cf32 *)c->d_v + (size_t)x->par * x->max_nel * c->vstride;
        const size_t sstride = c->rs ? c->ostride : c->vstride;
        if (!io->dev_out && got)
            for (e = 0; e < nel && rc == ATKB_OK; ++e)
                rc = atkb_d2h(io->outs[(size_t)e * x->nslots + ci] + io->wpos[ci], src + (size_t)e * sstride,
                              got * sizeof(atkdsp_cf32), x->stream);
        io->wpos[ci] += got;
    }
    if (rc != ATKB_OK) return rc;
    /* the new state: s[h*hop, avail + ov) per element; untouched elements keep theirs */
    const size_t keep = x->ov + (avail - h * x->hop);
    rc = atkb_osx_carry(st, (long long)x->nfft, d_ins, io->dev_in ? (long long)off : 0,
                        (long long)(x->ov + x->lc), (long long)(h * x->hop), (long long)keep, st2,
                        (long long)x->nfft, (int)nel, x->stream);
    if (rc == ATKB_OK && nel < x->max_nel)
        rc = atkb_d2d(st2 + (size_t)nel * x->nfft, st + (size_t)nel * x->nfft,
                      (size_t)(x->max_nel - nel) * x->nfft * sizeof(atkdsp_cf32), x->stream);
    if (rc == ATKB_OK && !io->dev_in) {
        rc = atkb_event_record(x->ev_done[b], x->stream);   /* the staging's last reader */
        x->inb ^= 1;
    }
    if (rc != ATKB_OK) return rc;
    x->cur ^= 1;
    x->par ^= 1;
    x->lc = (unsigned)(avail - h * x->hop);
    x->blk += (int64_t)h;
    return ATKB_OK;
}

/* the order of the small channels: costliest first (a fold of decim terms
 * per lane, ceil(4M / 32) rounds of lanes), equal M together */
static int small_before(const atkb_osx_chan *a, const atkb_osx_chan *b) {
    const long ca = (long)a->decim * (long)((ATKB_OSX_G * a->M + 31) / 32);
    const long cb = (long)b->decim * (long)((ATKB_OSX_G * b->M + 31) / 32);
    return ca > cb || (ca == cb && a->M < b->M);
}

static ptrdiff_t osx_process(atkdsp_osx *x, const osx_io *io0, size_t n, size_t *out_counts, size_t cap_each) {
    osx_io io = *io0;
    const unsigned nel = io.nel;
    const int ns = x->nslots;
    int ci;
    unsigned e;
    for (ci = 0; ci < ns; ++ci) out_counts[ci] = 0;
    const size_t avail = (size_t)x->lc + n, m = avail / x->hop;
    for (e = 0; e < nel; ++e)
        if (n && !io.ins[e]) return ATKDSP_E_ARG;
    if (m == 0) {                 /* no block completes: append to the leftover */
        int rc = ATKB_OK;
        atkdsp_cf32 *st = (atkdsp_cf32 *)x->d_state + (size_t)x->cur * x->max_nel * x->nfft;
        for (e = 0; e < nel && rc == ATKB_OK; ++e)
            if (n)
                rc = io.dev_in ? atkb_d2d(st + (size_t)e * x->nfft + x->ov + x->lc, io.ins[e], n * sizeof(atkdsp_cf32), x->stream)
                               : atkb_h2d(st + (size_t)e * x->nfft + x->ov + x->lc, io.ins[e], n * sizeof(atkdsp_cf32), x->stream);
        if (rc == ATKB_OK && !io.dev_in) rc = atkb_stream_sync(x->stream);
        if (rc != ATKB_OK) return atkb_map_rc(rc);
        x->lc = (unsigned)avail;
        return ns;
    }
    /* every check before any state changes */
    for (ci = 0; ci < ns; ++ci) {
        const osx_chan *c = &x->ch[ci];
        if (!c->active) continue;
        for (e = 0; e < nel; ++e)
            if (!io.outs || !io.outs[(size_t)e * ns + ci]) return ATKDSP_E_ARG;
        for (e = 0; e < nel; ++e) {
            const size_t total = c->rs ? (size_t)rs_count(c, e, m * c->nvalid) : m * c->nvalid;
            if (total > cap_each) return ATKDSP_E_CAP;
        }
    }
    int rc = osx_table_reserve(x, ns);
    if (rc != ATKB_OK) return atkb_map_rc(rc);
    rc = atkb_stream_sync(x->stream);            /* the pinned mirror is free again */
    if (rc != ATKB_OK) return atkb_map_rc(rc);
    /* the call's table: channels by class -- M <= ATKB_OSX_SMALL_M (a warp
     * each), M <= 4096 (the CTA), M > 4096 (their own four-step inverse) --
     * in slot order within each; then the input and output pointers */
    atkb_osx_chan *tc = (atkb_osx_chan *)x->h_tbl;
    void **pin = (void **)((char *)x->h_tbl + tbl_ins_off(x));
    void **pout = (void **)((char *)x->h_tbl + tbl_outs_off(x));
    void *const *d_outs = (void *const *)((char *)x->d_tbl + tbl_outs_off(x));
    int j = 0, cls;
    x->nsmall = x->nmid = x->nbig = 0;
    for (cls = 0; cls < 3; ++cls) {
        const int first = j;
        for (ci = 0; ci < ns; ++ci) {
            osx_chan *c = &x->ch[ci];
            if (!c->active) continue;
            const int kind = c->M <= ATKB_OSX_SMALL_M ? 0 : c->M <= ATKB_OSX_FUSED_MAX ? 1 : 2;
            if (kind != cls) continue;
            atkb_osx_chan t;
            memset(&t, 0, sizeof t);
            t.H = c->d_H;
            t.stage = c->d_v;
            t.stage_stride = (long long)c->vstride;
            t.par_stride = (long long)x->max_nel * (long long)c->vstride;
            t.lead = (long long)c->Q;
            t.delta = c->delta;
            t.M = (int)c->M; t.logm = ilog2(c->M); t.ovd = (int)c->ovd; t.nvalid = (int)c->nvalid;
            t.decim = (int)c->decim; t.shift = (int)c->shift;
            t.dsts = (void *const *)(intptr_t)ci;       /* the slot, until the order is final */
            /* small channels, one warp each, costliest first: a fold of decim
             * terms per lane, ceil(4M / 32) rounds of lanes */
            int at = j;
            if (cls == 0) {
                while (at > first && small_before(&t, &tc[at - 1])) {
                    tc[at] = tc[at - 1];
                    --at;
                }
            }
            tc[at] = t;
            ++j;
            x->nsmall += kind == 0;
            x->nmid += kind == 1;
            x->nbig += kind == 2;
        }
    }
    /* packs: runs of small channels of one M, as many as fill the lanes */
    int *pk = (int *)((char *)x->h_tbl + tbl_packs_off(x));
    int np = 0, t0 = 0;
    while (t0 < x->nsmall) {
        const int lim = tc[t0].M * ATKB_OSX_G >= ATKB_OSX_PACK_LANES ? 1 : ATKB_OSX_PACK_LANES / (tc[t0].M * ATKB_OSX_G);
        int t1 = t0 + 1;
        while (t1 < x->nsmall && t1 - t0 < lim && tc[t1].M == tc[t0].M) ++t1;
        pk[np++] = t0;
        t0 = t1;
    }
    pk[np] = x->nsmall;
    x->npacks = np;
    for (int t = 0; t < j; ++t) {                         /* slots -> table entries */
        osx_chan *c = &x->ch[(intptr_t)tc[t].dsts];
        c->tix = t;
        tc[t].dsts = (io.dev_out && !c->rs) ? d_outs + (size_t)t * x->max_nel : NULL;
        if (io.dev_out)
            for (e = 0; e < nel; ++e)
                pout[(size_t)t * x->max_nel + e] = io.outs[(size_t)e * ns + (int)(c - x->ch)];
    }
    for (e = 0; e < nel; ++e) {
        pin[e] = io.dev_in ? (void *)io.ins[e] : (void *)((atkdsp_cf32 *)x->d_in + (size_t)e * x->chunk_in);
        pin[x->max_nel + e] = (void *)((atkdsp_cf32 *)x->d_in + ((size_t)x->max_nel + e) * x->chunk_in);
    }
    rc = atkb_h2d(x->d_tbl, x->h_tbl, x->tbl_bytes, x->stream);
    if (rc != ATKB_OK) return atkb_map_rc(rc);
    size_t *wp = x->wpos;        /* NULL only while no slot exists (ns == 0) */
    for (ci = 0; ci < ns; ++ci) wp[ci] = 0;
    io.wpos = wp;
    size_t off = 0, done = 0;
    while (done < m && rc == ATKB_OK) {
        size_t h = m - done;
        if (h > x->chunk_hops) h = x->chunk_hops;
        const size_t sub = (done + h == m) ? n - off : h * x->hop - x->lc;
        rc = osx_chunk(x, &io, off, sub, done);
        off += sub;
        done += h;
    }
    if (rc == ATKB_OK && !io.dev_out) rc = atkb_stream_sync(x->stream);
    for (ci = 0; ci < ns; ++ci) out_counts[ci] = wp[ci];
    if (rc != ATKB_OK) return atkb_map_rc(rc);
    return ns;
}

ATKDSP_API ptrdiff_t atkdsp_osx_process_n(atkdsp_osx *x, const atkdsp_cf32 *const *ins, unsigned nel, size_t n,
                                          atkdsp_cf32 *const *outs, size_t *out_counts, size_t cap_each) {
    if (!x || !ins || nel < 1 || nel > x->max_nel || !out_counts) return ATKDSP_E_ARG;
    osx_io io = {0, 0, ins, outs, nel, NULL};
    return osx_process(x, &io, n, out_counts, cap_each);
}

ATKDSP_API ptrdiff_t atkdsp_osx_process(atkdsp_osx *x, const atkdsp_cf32 *in, size_t n, atkdsp_cf32 *const *outs,
                                        size_t *out_counts, size_t cap_each) {
    const atkdsp_cf32 *ins[1];
    ins[0] = in;
    return atkdsp_osx_process_n(x, ins, 1, n, outs, out_counts, cap_each);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_osx_process_n(atkdsp_osx *x, const atkdsp_cf32 *const *d_ins, unsigned nel,
                                              size_t n, atkdsp_cf32 *const *d_outs, size_t *out_counts,
                                              size_t cap_each) {
    if (!x || !d_ins || nel < 1 || nel > x->max_nel || !out_counts) return ATKDSP_E_ARG;
    osx_io io = {1, 1, d_ins, d_outs, nel, NULL};
    return osx_process(x, &io, n, out_counts, cap_each);
}
