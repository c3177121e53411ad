/* The host layer of the B200 channelizer, in C99.
 *
 * It implements the reference's atkdsp_pfb_* / atkdsp_unpack* entry points
 * (include/atkdsp.h) with the reference's argument checks, return codes and
 * bookkeeping, designs the prototype filter and the FFT plan on the host,
 * keeps each handle's streaming state in device memory, and drives the
 * device through the thin atkb_* shim (internal.h). It includes no CUDA
 * header and calls no CUDA function directly.
 *
 * Layout per handle (allocated once, by atkdsp_pfb_create):
 *   bank      taps (float, L), rotation table twd (double2, nchan), DFT
 *             table W (double2, nchan), per-pass twiddles, and a device copy
 *             of the atkb_bank that points at them
 *   state     two buffers per element of ov + hop samples (ping-pong): the
 *             samples s[m*hop, ...) that the next call's windows reach back
 *             into -- the reference's hist ++ leftover (channelizer.c:56-60)
 *   staging   per element an input chunk and an output chunk on the device,
 *             used by the host-pointer calls (long inputs are processed in
 *             chunks; the output is split-invariant, so this changes nothing)
 *   tables    job / tile / carry tables (device + pinned host mirror) and
 *             the persistent kernel's two self-resetting counters
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "host_internal.h"

#define ATKB_PI 3.14159265358979323846
/* W1/W2 on device handle arrays up to this many elements (the wide kernel's
 * shared-memory diagonal); the filterbank itself takes any max_nel */
#define MAX_W12_NEL 6144
#define MAX_POW2_NCHAN 4096
#define MAX_GENERIC_NCHAN 6400

/* ===================================================================== identity */
#define STR2(x) #x
#define STR(x) STR2(x)
static const char BUILD_INFO[] =
    ATKDSP_VERSION_STRING " abi " STR(ATKDSP_ABI_VERSION) " b200 cuda sm_100a fp32-fold fp64-fft"
    " built " __DATE__ " " __TIME__;

ATKDSP_API int atkdsp_abi_version(void) { return ATKDSP_ABI_VERSION; }
ATKDSP_API const char *atkdsp_version_string(void) { return ATKDSP_VERSION_STRING; }
ATKDSP_API const char *atkdsp_build_info(void) { return BUILD_INFO; }

/* reference src/atkdsp.c:51-60 */
ATKDSP_API int atkdsp_bytes_per_sample(int fmt) {
    switch (fmt) {
    case ATKDSP_FMT_CU8: return 2;
    case ATKDSP_FMT_CI8: return 2;
    case ATKDSP_FMT_CI16: return 4;
    case ATKDSP_FMT_CI16Q11: return 4;
    case ATKDSP_FMT_CF32: return 8;
    default: return 0;
    }
}

static int g_threads = 0;
/* reference src/atkdsp.c:64-80: the count in force; <= 0 restores the
 * default (the number of online CPUs, what OpenMP would use). */
ATKDSP_API int atkdsp_set_threads(int n) {
    g_threads = n > 0 ? n : 0;
    return atkdsp_get_threads();
}
ATKDSP_API int atkdsp_get_threads(void) {
    if (g_threads > 0) return g_threads;
    const long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

#define map_rc atkb_map_rc
int atkb_map_rc(int rc) {
    switch (rc) {
    case ATKB_OK: return ATKDSP_OK;
    case ATKB_E_ARG: return ATKDSP_E_ARG;
    case ATKB_E_NOMEM: return ATKDSP_E_NOMEM;
    case ATKB_E_CAP: return ATKDSP_E_CAP;
    default: return ATKDSP_E_FFT;
    }
}

/* =========================================================== prototype design
 * Kaiser-windowed sinc, cutoff half a channel, unit DC gain times nchan
 * (reference src/channelizer.c:79-99 with src/design.c:18-22 and the I0
 * series of src/channelizer.c:33-43). The expressions are evaluated in the
 * reference's order so the double taps -- and their float rounding, which
 * the fold multiplies by -- come out bit-identical. */
static double kaiser_beta(double atten_db) {
    if (atten_db > 50.0) return 0.1102 * (atten_db - 8.7);
    if (atten_db >= 21.0) return 0.5842 * pow(atten_db - 21.0, 0.4) + 0.07886 * (atten_db - 21.0);
    return 0.0;
}

static double bessel_i0(double x) {
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

static double proto_tap(size_t n, double fc, double mid, double beta, double i0b) {
    const double t = (double)n - mid;
    const double x = 2.0 * fc * t;
    const double sinc = (t == 0.0) ? 1.0 : sin(ATKB_PI * x) / (ATKB_PI * x);
    const double r = (mid > 0.0) ? t / mid : 0.0;
    const double w = bessel_i0(beta * sqrt(r * r < 1.0 ? 1.0 - r * r : 0.0)) / i0b;
    return 2.0 * fc * sinc * w;
}

static void design_prototype(unsigned nchan, unsigned K, double atten_db, double *h) {
    const size_t L = (size_t)nchan * K;
    const double fc = 1.0 / (2.0 * (double)nchan);
    const double mid = (double)(L - 1) * 0.5;
    const double beta = kaiser_beta(atten_db);
    const double i0b = bessel_i0(beta);
    double total = 0.0;
    size_t n;
    for (n = 0; n < L; ++n) total += proto_tap(n, fc, mid, beta, i0b);
    if (total == 0.0) total = 1.0;
    for (n = 0; n < L; ++n) h[n] = (proto_tap(n, fc, mid, beta, i0b) / total) * (double)nchan;
}

/* ================================================================== FFT plan */
static int is_pow2(unsigned v) { return v && !(v & (v - 1)); }

/* ---- the tile-shape choice -----------------------------------------------
 * Where several exist (can_pair, can_quad), a bank uses the paired fold (two
 * hops per thread over even or odd branches: half the loads, one more FFT
 * pass), one hop and 8 branches per thread, or the quad fold (four hops per
 * thread over two branches). The choice comes from a runtime override
 * (atkdsp_gpu_tune_set), else from the table the autotuner wrote
 * (tune_table.h, measured on B200), else the paired fold. */
typedef struct { unsigned nchan, os, K; int pair; } tune_entry;
#include "tune_table.h"
#define MAX_TUNE_OVERRIDES 256
static tune_entry g_tune_ovr[MAX_TUNE_OVERRIDES];
static unsigned g_tune_novr;
static pthread_mutex_t g_tune_lock = PTHREAD_MUTEX_INITIALIZER;

/* the paired fold: hop b's window is hop a's shifted by 8/os branch slots,
 * so os must divide 4 (M/os a multiple of 2*M/8), and a tile must hold two
 * hops (nchan <= 2048) */
static int can_pair(unsigned M, unsigned os) {
    return ATKB_PTS == 8 && is_pow2(M) && M >= 16 && M <= 2048 && (os == 1 || os == 2 || os == 4);
}

/* the quad fold: four hops per thread over two branches (q, q + M/2), whose
 * class mod M/8 a hop shift of M/os keeps for os 1 and 2; a tile must hold
 * four hops (nchan <= 1024) */
static int can_quad(unsigned M, unsigned os) {
    return ATKB_PTS == 8 && is_pow2(M) && M >= 16 && M <= 1024 && (os == 1 || os == 2);
}

/* a tile-shape choice: the fold in the low two bits (0 one hop per thread,
 * 1 paired, 2 quad), bit 2 set to keep a small nchan's tile window out of
 * shared memory (the fold then reads it through L1) */
#define TUNE_NOSTAGE 4
static int can_nostage(unsigned M, unsigned os) { return can_pair(M, os) && M <= 512; }
static int choice_ok(unsigned M, unsigned os, int choice) {
    const int shape = choice & 3, ns = choice & TUNE_NOSTAGE;
    if (choice < 0 || choice > 6 || shape == 3) return 0;
    if (shape == 2 && (!can_quad(M, os) || ns)) return 0;
    if (ns && !can_nostage(M, os)) return 0;
    return can_pair(M, os);
}

static int tune_choice(unsigned M, unsigned os, unsigned K) {
    unsigned i;
    int c = -1;
    if (!can_pair(M, os)) return 0;
    pthread_mutex_lock(&g_tune_lock);
    for (i = 0; i < g_tune_novr; ++i)
        if (g_tune_ovr[i].nchan == M && g_tune_ovr[i].os == os && g_tune_ovr[i].K == K) c = g_tune_ovr[i].pair;
    pthread_mutex_unlock(&g_tune_lock);
    if (c >= 0) return c;
    for (i = 0; i < sizeof k_tune_table / sizeof k_tune_table[0]; ++i)
        if (k_tune_table[i].nchan == M && k_tune_table[i].os == os && k_tune_table[i].K == K)
            return k_tune_table[i].pair;
    return 1;
}

ATKDSP_API int atkdsp_gpu_tune_set(unsigned nchan, unsigned oversample, unsigned taps_per_poly, int choice) {
    unsigned i;
    int rc = ATKDSP_OK;
    if (!can_pair(nchan, oversample) || (choice != -1 && !choice_ok(nchan, oversample, choice)))
        return ATKDSP_E_ARG;
    pthread_mutex_lock(&g_tune_lock);
    for (i = 0; i < g_tune_novr; ++i)
        if (g_tune_ovr[i].nchan == nchan && g_tune_ovr[i].os == oversample && g_tune_ovr[i].K == taps_per_poly)
            break;
    if (choice < 0) {                                      /* back to the table */
        if (i < g_tune_novr) g_tune_ovr[i] = g_tune_ovr[--g_tune_novr];
    } else if (i < g_tune_novr) {
        g_tune_ovr[i].pair = choice;
    } else if (g_tune_novr < MAX_TUNE_OVERRIDES) {
        tune_entry t = {nchan, oversample, taps_per_poly, choice};
        g_tune_ovr[g_tune_novr++] = t;
    } else {
        rc = ATKDSP_E_NOMEM;
    }
    pthread_mutex_unlock(&g_tune_lock);
    return rc;
}

ATKDSP_API void atkdsp_gpu_fail_alloc_after(long long n) { atkb_fail_alloc_after(n); }

ATKDSP_API int atkdsp_gpu_tune_get(unsigned nchan, unsigned oversample, unsigned taps_per_poly) {
    if (!can_pair(nchan, oversample)) return ATKDSP_E_ARG;
    return tune_choice(nchan, oversample, taps_per_poly);
}

static int plan_fft(unsigned M, unsigned os, int want_pair, atkb_fft_plan *pl) {
    memset(pl, 0, sizeof *pl);
    if (is_pow2(M) && M >= 16 && M <= MAX_POW2_NCHAN) {
        const int quad = (want_pair & 3) == 2 && can_quad(M, os);
        const int pair = !quad && (want_pair & 3) && can_pair(M, os);
        pl->nostage = (want_pair & TUNE_NOSTAGE) && can_nostage(M, os);
        unsigned rem = M / (quad ? 2 : pair ? 4 : ATKB_PTS);
        pl->fast = 1;
        pl->pair = pair;
        pl->quad = quad;
        /* nchan 4096 at oversample 1/2/4: one thread folds both parities of
         * both hops of its two-hop tile (paired loads), then radix-8 first
         * passes: the paired tap layout with the radix-8 plan */
        pl->ptaps = pair || (M == 4096 && (os == 1 || os == 2 || os == 4));
        pl->radix[pl->npass++] = quad ? 2 : pair ? 4 : ATKB_PTS;
        while (rem >= ATKB_PTS) { pl->radix[pl->npass++] = ATKB_PTS; rem /= ATKB_PTS; }
        if (rem > 1) pl->radix[pl->npass++] = (int)rem;
    } else {
        unsigned rem = M, p;
        while (rem % 16 == 0) { pl->radix[pl->npass++] = 16; rem /= 16; }
        if (rem % 8 == 0) { pl->radix[pl->npass++] = 8; rem /= 8; }
        if (rem % 4 == 0) { pl->radix[pl->npass++] = 4; rem /= 4; }
        if (rem % 2 == 0) { pl->radix[pl->npass++] = 2; rem /= 2; }
        for (p = 3; rem > 1; p += 2) {
            while (rem % p == 0) {
                if (pl->npass >= ATKB_MAX_PASS) return -1;
                pl->radix[pl->npass++] = (int)p;
                rem /= p;
            }
            if (p * p > rem && rem > 1) {
                if (pl->npass >= ATKB_MAX_PASS) return -1;
                pl->radix[pl->npass++] = (int)rem;
                rem = 1;
            }
        }
    }
    /* beyond one CTA's shared memory: the separate-kernel path */
    pl->big = !pl->fast && (M > MAX_GENERIC_NCHAN || (is_pow2(M) && M > MAX_POW2_NCHAN));
    /* per-pass twiddles (fast path): pass p >= 1 holds W_{Ns R}^{k} at k,
     * k in [0, Ns); the kernel forms the powers r = 2 .. R-1 by complex
     * multiplication */
    {
        int p, Ns = 1, off = 0;
        for (p = 0; p < pl->npass; ++p) {
            pl->twoff[p] = off;
            if (p > 0) off += Ns;
            Ns *= pl->radix[p];
        }
        pl->twlen = off > 0 ? off : 1;
    }
    return 0;
}

static size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }
size_t atkb_align16(size_t v) { return align16(v); }

static size_t tables_bytes(unsigned n) {
    return align16((size_t)n * sizeof(atkb_job)) + align16((size_t)n * sizeof(atkb_carry)) +
           align16(((size_t)n + 1) * sizeof(int));
}
size_t atkb_tables_bytes(unsigned n) { return tables_bytes(n); }

static atkb_job *tbl_jobs(void *base) { return (atkb_job *)base; }
static atkb_carry *tbl_carry(void *base, unsigned n) {
    return (atkb_carry *)((char *)base + align16((size_t)n * sizeof(atkb_job)));
}
static int *tbl_tiles(void *base, unsigned n) {
    return (int *)((char *)base + align16((size_t)n * sizeof(atkb_job)) +
                   align16((size_t)n * sizeof(atkb_carry)));
}
atkb_job *atkb_tbl_jobs(void *base) { return tbl_jobs(base); }
atkb_carry *atkb_tbl_carry(void *base, unsigned n) { return tbl_carry(base, n); }
int *atkb_tbl_tiles(void *base, unsigned n) { return tbl_tiles(base, n); }

static atkdsp_cf32 *state_buf(const atkdsp_pfb *p, int which, unsigned e) {
    return (atkdsp_cf32 *)p->d_state + ((size_t)which * p->max_nel + e) * p->cap_state;
}
atkdsp_cf32 *atkb_state_buf(const atkdsp_pfb *p, int which, unsigned e) { return state_buf(p, which, e); }

size_t atkb_stream_footprint(unsigned nchan, unsigned oversample, unsigned taps_per_poly) {
    const size_t cap = (size_t)nchan * taps_per_poly;          /* ov + hop = L */
    return 2 * cap * sizeof(atkdsp_cf32) + (size_t)nchan * sizeof(atkdsp_cf32) + 4096;
    (void)oversample;
}

/* ================================================================ bank cache
 * Taps, tables and the device atkb_bank depend only on (device, nchan,
 * oversample, taps/branch, attenuation). Handles with the same parameters
 * share one copy: a batch of many streams then keeps a handful of banks hot in
 * L2 instead of re-reading one copy per stream from HBM. Refcounted. */
struct bank_entry {
    int dev;
    unsigned nchan, os, K;
    double atten;
    int pair;                     /* the tile-shape choice it was built with */
    int refs;
    void *d_const, *d_bank;
    atkb_bank bank;
    bank_entry *next;
};
static bank_entry *g_banks;
static pthread_mutex_t g_bank_lock = PTHREAD_MUTEX_INITIALIZER;

static void bank_release(bank_entry *e);

ATKDSP_API void atkdsp_pfb_destroy(atkdsp_pfb *p) {
    if (!p) return;
    if (p->dev >= 0) atkb_set_device(p->dev);
    if (p->stream) atkb_stream_sync(p->stream);
    bank_release(p->be);
    if (p->pool_stream) atkb_free_async(p->d_state, p->pool_stream);
    else atkb_free(p->d_state);
    atkb_free(p->d_cal);
    atkb_free(p->d_in_stage);
    atkb_free(p->d_out_stage);
    atkb_free(p->d_tables);
    atkb_free(p->d_counters);
    atkb_host_free(p->h_tables);           /* h_small_in lives inside it */
    atkb_host_free(p->h_small_out);
    atkb_host_free(p->h_pend);
    atkb_event_destroy(p->small_ev);
    atkb_event_destroy(p->small_done);
    atkb_event_destroy(p->tbl_event);
    atkb_stream_destroy(p->stream);
    free((void *)p->dins);
    atkb_free(p->d_big);
    free(p);
}

static int bank_build(bank_entry *be, void *stream) {
    const unsigned M = be->nchan;
    const size_t L = (size_t)M * be->K;
    atkb_fft_plan pl;
    if (plan_fft(M, be->os, be->pair, &pl) != 0) return ATKB_E_ARG;
    const size_t taps_b = align16(L * sizeof(float));
    const size_t tab_b = (size_t)M * 2 * sizeof(double);
    const size_t pass_b = (size_t)pl.twlen * 2 * sizeof(double);
    const size_t total = 3 * taps_b + 2 * tab_b + pass_b;
    char *h = (char *)calloc(1, total);
    double *proto = (double *)malloc(L * sizeof(double));
    if (!h || !proto) { free(h); free(proto); return ATKB_E_NOMEM; }
    design_prototype(M, be->K, be->atten, proto);
    float *taps = (float *)h;
    float *tapsP = (float *)(h + taps_b);
    double *twd = (double *)(h + 2 * taps_b);
    double *W = (double *)(h + 2 * taps_b + tab_b);
    double *wp = (double *)(h + 2 * taps_b + 2 * tab_b);
    float *tapsQ = (float *)(h + 2 * taps_b + 2 * tab_b + pass_b);
    size_t q;
    unsigned j;
    for (q = 0; q < L; ++q) taps[q] = (float)proto[q];
    if (pl.fast) {
        /* float4 g = (k*(P/4) + q)*MP + j, component i, holds the tap of
         * branch j + r*MP, r = 4q + i (paired: r = q + 2i), MP = M/P */
        const size_t P = ATKB_PTS, MP = M / ATKB_PTS;
        size_t k2, q2, jj, i;
        for (k2 = 0; k2 < be->K; ++k2)
            for (q2 = 0; q2 < P / 4; ++q2)
                for (jj = 0; jj < MP; ++jj)
                    for (i = 0; i < 4; ++i) {
                        const size_t r = pl.ptaps ? q2 + 2 * i : 4 * q2 + i;
                        tapsP[((k2 * (P / 4) + q2) * MP + jj) * 4 + i] = taps[k2 * M + jj + r * MP];
                    }
    }
    if (pl.quad) {
        /* (c*2K + v)*MP + j holds the tap (4v + c)*MP + j: class c's 2K taps
         * at stride MP, consecutive across a warp's branches j */
        const size_t MP = M / 8, V = 2 * (size_t)be->K;
        size_t c, v, jj;
        for (c = 0; c < 4; ++c)
            for (v = 0; v < V; ++v)
                for (jj = 0; jj < MP; ++jj) tapsQ[(c * V + v) * MP + jj] = taps[(4 * v + c) * MP + jj];
    }
    for (j = 0; j < M; ++j) {
        /* the reference's rotation table, channelizer.c:164-170 */
        const double a = 2.0 * ATKB_PI * (double)j / (double)M;
        twd[2 * j] = cos(a);
        twd[2 * j + 1] = sin(a);
        W[2 * j] = cos(a);
        W[2 * j + 1] = -sin(a);
    }
    {
        int pidx, Ns = 1;
        for (pidx = 0; pidx < pl.npass; ++pidx) {
            const int R = pl.radix[pidx];
            if (pidx > 0 && pl.fast) {
                int k;
                for (k = 0; k < Ns; ++k) {
                    const size_t e = (size_t)pl.twoff[pidx] + (size_t)k;
                    const size_t jj = (size_t)k * (M / ((size_t)Ns * R));
                    wp[2 * e] = W[2 * jj];
                    wp[2 * e + 1] = W[2 * jj + 1];
                }
            }
            Ns *= R;
        }
    }
    free(proto);
    int rc = atkb_malloc(&be->d_const, total);
    if (rc == ATKB_OK) rc = atkb_h2d(be->d_const, h, total, stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(stream);
    free(h);
    if (rc != ATKB_OK) return rc;
    atkb_bank *B = &be->bank;
    memset(B, 0, sizeof *B);
    B->nchan = (int)M;
    B->os = (int)be->os;
    B->K = (int)be->K;
    B->hop = (int)(M / be->os);
    B->L = (long long)L;
    B->ov = (long long)(L - M / be->os);
    B->taps = (const float *)be->d_const;
    B->tapsP = (const float *)((const char *)be->d_const + taps_b);
    B->twd = (const char *)be->d_const + 2 * taps_b;
    B->wfull = (const char *)be->d_const + 2 * taps_b + tab_b;
    B->wpass = (const char *)be->d_const + 2 * taps_b + 2 * tab_b;
    B->tapsQ = (const float *)((const char *)be->d_const + 2 * taps_b + 2 * tab_b + pass_b);
    B->plan = pl;
    B->logm = 0;
    if (pl.fast) {
        unsigned v = M;
        while (v > 1) { v >>= 1; ++B->logm; }
    }
    if (pl.big) {
        B->tile_hops = 1;                /* no tiles: separate kernels per hop chunk */
        B->smem_bytes = 0;
    } else if (pl.fast && M == 4096) {
        /* two hops a tile, computed in turn: the FFT tile plus the first
         * hop's 4096 outputs (so the write covers two hops per channel) */
        B->tile_hops = 2;
        B->smem_bytes = ATKB_FAST_SMEM_MAX;
    } else if (pl.fast) {
        B->tile_hops = 4096 / (int)M;
        B->smem_bytes = 4096 * 16;
    } else {
        int th = (int)(2048 / M);
        if (th < 1) th = 1;
        B->tile_hops = th;
        B->smem_bytes = 2 * th * (int)M * 16;
    }
    rc = atkb_malloc(&be->d_bank, sizeof *B);
    if (rc == ATKB_OK) rc = atkb_h2d(be->d_bank, B, sizeof *B, stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(stream);
    return rc;
}

static bank_entry *bank_acquire(int dev, unsigned M, unsigned os, unsigned K, double atten,
                                void *stream, int *rc) {
    bank_entry *e;
    const int pair = tune_choice(M, os, K);
    pthread_mutex_lock(&g_bank_lock);
    for (e = g_banks; e; e = e->next)
        if (e->dev == dev && e->nchan == M && e->os == os && e->K == K && e->atten == atten && e->pair == pair) {
            ++e->refs;
            pthread_mutex_unlock(&g_bank_lock);
            *rc = ATKB_OK;
            return e;
        }
    e = (bank_entry *)calloc(1, sizeof *e);
    if (!e) {
        pthread_mutex_unlock(&g_bank_lock);
        *rc = ATKB_E_NOMEM;
        return NULL;
    }
    e->dev = dev; e->nchan = M; e->os = os; e->K = K; e->atten = atten; e->pair = pair; e->refs = 1;
    *rc = bank_build(e, stream);
    if (*rc != ATKB_OK) {
        atkb_free(e->d_const);
        atkb_free(e->d_bank);
        free(e);
        pthread_mutex_unlock(&g_bank_lock);
        return NULL;
    }
    e->next = g_banks;
    g_banks = e;
    pthread_mutex_unlock(&g_bank_lock);
    return e;
}

static void bank_release(bank_entry *e) {
    bank_entry **pp;
    if (!e) return;
    pthread_mutex_lock(&g_bank_lock);
    if (--e->refs == 0) {
        for (pp = &g_banks; *pp; pp = &(*pp)->next)
            if (*pp == e) { *pp = e->next; break; }
        atkb_free(e->d_const);
        atkb_free(e->d_bank);
        free(e);
    }
    pthread_mutex_unlock(&g_bank_lock);
}

/* reference src/channelizer.c:138-171 (argument rules and the atten clamp).
 * lean: a single-element stream for the server, without the host-path
 * staging and tables (it is driven only through batch launches). */
atkdsp_pfb *atkb_pfb_create_internal(double fs, unsigned nchan, unsigned oversample,
                                     unsigned taps_per_poly, double atten_db, unsigned max_nel,
                                     int lean) {
    if (!(fs > 0.0) || nchan < 2 || oversample < 1 || nchan % oversample != 0) return NULL;
    if (taps_per_poly < 2 || max_nel < 1) return NULL;
    if (lean && (is_pow2(nchan) ? nchan > MAX_POW2_NCHAN : nchan > MAX_GENERIC_NCHAN)) return NULL;
    if (atten_db < 20.0) atten_db = 20.0;
    atkdsp_pfb *p = (atkdsp_pfb *)calloc(1, sizeof *p);
    if (!p) return NULL;
    p->dev = -1;
    p->fs = fs;
    p->atten = atten_db;
    p->nchan = nchan;
    p->os = oversample;
    p->K = taps_per_poly;
    p->max_nel = max_nel;
    p->hop = nchan / oversample;
    p->L = (size_t)nchan * taps_per_poly;
    p->ov = p->L - p->hop;
    if (atkb_get_device(&p->dev) != ATKB_OK || atkb_set_device(p->dev) != ATKB_OK) {
        p->dev = -1;
        free(p);
        return NULL;
    }
    p->lean = lean;
    int rc = lean ? ATKB_OK : atkb_stream_create(&p->stream);
    if (rc == ATKB_OK && !lean) rc = atkb_event_create(&p->tbl_event);
    if (rc == ATKB_OK) {
        void *st = p->stream;
        if (lean && (rc = atkb_stream_create(&st)) != ATKB_OK) st = NULL;
        if (rc == ATKB_OK) p->be = bank_acquire(p->dev, nchan, oversample, taps_per_poly, atten_db, st, &rc);
        if (lean && st) atkb_stream_destroy(st);
        if (p->be) {
            p->bank = p->be->bank;
            p->d_bank = p->be->d_bank;
        }
    }
    if (rc != ATKB_OK) { atkdsp_pfb_destroy(p); return NULL; }
    /* state: ov history + up to hop - 1 leftover samples, twice per element */
    p->cap_state = p->ov + p->hop;
    rc = atkb_malloc(&p->d_state, 2 * (size_t)max_nel * p->cap_state * sizeof(atkdsp_cf32));
    if (rc == ATKB_OK)
        rc = atkb_memset(p->d_state, 0, 2 * (size_t)max_nel * p->cap_state * sizeof(atkdsp_cf32),
                         p->stream);
    if (rc == ATKB_OK) rc = atkb_malloc(&p->d_cal, (size_t)max_nel * nchan * sizeof(atkdsp_cf32));
    if (rc == ATKB_OK && lean) rc = atkb_stream_sync(NULL);
    if (lean) {
        if (rc != ATKB_OK) { atkdsp_pfb_destroy(p); return NULL; }
        p->lc = 0; p->b = 0; p->cur = 0;
        return p;
    }
    if (rc == ATKB_OK && !(p->dins = (const void **)calloc(max_nel, sizeof *p->dins))) rc = ATKB_E_NOMEM;
    if (rc == ATKB_OK && p->bank.plan.big)          /* two double2 buffers of a hop chunk */
        rc = atkb_malloc(&p->d_big, 2 * (size_t)atkb_pfb_big_hops((int)nchan) * nchan * 16);
    /* host-path staging: about 2^20 samples per element, whole hops */
    if (rc == ATKB_OK) {
        size_t chunk = ((size_t)1 << 21) / max_nel;
        if (chunk < (size_t)p->hop * 8) chunk = (size_t)p->hop * 8;
        chunk = (chunk / p->hop) * p->hop;
        p->chunk = chunk;
        p->out_ld = chunk / p->hop + 1;
        rc = atkb_malloc(&p->d_in_stage, (size_t)max_nel * chunk * sizeof(atkdsp_cf32));
    }
    if (rc == ATKB_OK)
        rc = atkb_malloc(&p->d_out_stage,
                         (size_t)max_nel * nchan * p->out_ld * sizeof(atkdsp_cf32));
    if (rc == ATKB_OK) {
        p->tbl_bytes = tables_bytes(max_nel);
    }
    {
        /* small calls: their blocks travel right after the tables, in the
         * same pinned buffer and the same host->device copy */
        const int small = p->chunk >= ATKB_SMALL_N;
        const size_t in_b = small ? (size_t)max_nel * ATKB_SMALL_N * sizeof(atkdsp_cf32) : 0;
        if (rc == ATKB_OK) rc = atkb_malloc(&p->d_tables, p->tbl_bytes + in_b);
        if (rc == ATKB_OK) rc = atkb_host_alloc(&p->h_tables, p->tbl_bytes + in_b);
        if (rc == ATKB_OK && small) {
            const size_t m_small = (p->hop - 1 + ATKB_SMALL_N) / p->hop;
            p->h_small_in = (char *)p->h_tables + p->tbl_bytes;
            p->d_small_in = (char *)p->d_tables + p->tbl_bytes;
            rc = atkb_host_alloc(&p->h_small_out, (size_t)max_nel * nchan * m_small * sizeof(atkdsp_cf32));
            if (rc == ATKB_OK && atkb_host_dev_ptr(p->h_small_out, &p->dz_small_out) != ATKB_OK)
                p->dz_small_out = NULL;       /* then the outputs come back by copy */
            if (rc == ATKB_OK) rc = atkb_host_alloc(&p->h_pend, (size_t)max_nel * p->hop * sizeof(atkdsp_cf32));
            if (rc == ATKB_OK) rc = atkb_event_create(&p->small_ev);
            if (rc == ATKB_OK) rc = atkb_event_create(&p->small_done);
        }
    }
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&p->d_counters, ATKB_NCOUNTERS * sizeof(int));
    if (rc == ATKB_OK) rc = atkb_memset(p->d_counters, 0, ATKB_NCOUNTERS * sizeof(int), p->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(p->stream);
    if (rc != ATKB_OK) { atkdsp_pfb_destroy(p); return NULL; }
    p->grid = atkb_pfb_grid(p->dev, p->bank.smem_bytes);
    if (p->grid < 1) { atkdsp_pfb_destroy(p); return NULL; }
    p->lc = 0;
    p->b = 0;
    p->cur = 0;
    return p;
}

atkdsp_pfb *atkb_pfb_create_served(double fs, unsigned nchan, unsigned oversample, unsigned taps_per_poly,
                                   double atten_db, void *pool, void *stream) {
    if (!(fs > 0.0) || nchan < 2 || oversample < 1 || nchan % oversample != 0 || taps_per_poly < 2) return NULL;
    if (is_pow2(nchan) ? nchan > MAX_POW2_NCHAN : nchan > MAX_GENERIC_NCHAN) return NULL;
    if (atten_db < 20.0) atten_db = 20.0;
    atkdsp_pfb *p = (atkdsp_pfb *)calloc(1, sizeof *p);
    if (!p) return NULL;
    p->fs = fs;
    p->atten = atten_db;
    p->nchan = nchan;
    p->os = oversample;
    p->K = taps_per_poly;
    p->max_nel = 1;
    p->hop = nchan / oversample;
    p->L = (size_t)nchan * taps_per_poly;
    p->ov = p->L - p->hop;
    p->lean = 1;
    if (atkb_get_device(&p->dev) != ATKB_OK) { free(p); return NULL; }
    int rc = ATKB_OK;
    /* a bank already in the cache costs nothing; a new one is built (and
     * waited for) on the server's stream */
    p->be = bank_acquire(p->dev, nchan, oversample, taps_per_poly, atten_db, stream, &rc);
    if (p->be) {
        p->bank = p->be->bank;
        p->d_bank = p->be->d_bank;
    }
    p->cap_state = p->ov + p->hop;
    const size_t sb = 2 * p->cap_state * sizeof(atkdsp_cf32);
    if (rc == ATKB_OK) rc = atkb_malloc_pool(&p->d_state, sb, pool, stream);
    if (rc == ATKB_OK) p->pool_stream = stream;
    if (rc == ATKB_OK) rc = atkb_memset(p->d_state, 0, sb, stream);
    if (rc != ATKB_OK) { atkdsp_pfb_destroy(p); return NULL; }
    return p;
}

ATKDSP_API atkdsp_pfb *atkdsp_pfb_create(double fs, unsigned nchan, unsigned oversample,
                                         unsigned taps_per_poly, double atten_db,
                                         unsigned max_nel) {
    return atkb_pfb_create_internal(fs, nchan, oversample, taps_per_poly, atten_db, max_nel, 0);
}

ATKDSP_API void atkdsp_pfb_reset(atkdsp_pfb *p) {
    if (!p) return;
    atkb_set_device(p->dev);
    atkb_memset(p->d_state, 0, 2 * (size_t)p->max_nel * p->cap_state * sizeof(atkdsp_cf32),
                p->stream);
    atkb_stream_sync(p->stream);
    p->small_live = 0;
    p->npend = 0;
    p->lc = 0;
    p->b = 0;
    p->cur = 0;
}

ATKDSP_API unsigned atkdsp_pfb_nchan(const atkdsp_pfb *p) { return p ? p->nchan : 0; }
ATKDSP_API double atkdsp_pfb_out_rate(const atkdsp_pfb *p) {
    return p ? (double)p->os * p->fs / (double)p->nchan : 0.0;
}
ATKDSP_API size_t atkdsp_pfb_out_hops(const atkdsp_pfb *p, size_t n) {
    return p ? ((size_t)p->lc + n) / p->hop : 0;
}
ATKDSP_API double atkdsp_pfb_group_delay(const atkdsp_pfb *p) {
    return p ? (double)(p->L - 1) * 0.5 : 0.0;
}
ATKDSP_API int64_t atkdsp_pfb_block_origin(const atkdsp_pfb *p, int64_t hop_index) {
    return p ? hop_index * (int64_t)p->hop - (int64_t)p->ov : 0;
}

/* reference src/channelizer.c:203-212: the table is copied; NULL clears it */
ATKDSP_API int atkdsp_pfb_set_cal(atkdsp_pfb *p, const atkdsp_cf32 *table, unsigned nel) {
    if (!p) return ATKDSP_E_ARG;
    if (!table) { p->cal_nel = 0; return ATKDSP_OK; }
    if (nel < 1 || nel > p->max_nel) return ATKDSP_E_ARG;
    atkb_set_device(p->dev);
    int rc = atkb_stream_sync(p->stream);       /* earlier work may still read the old table */
    if (rc == ATKB_OK) rc = atkb_h2d(p->d_cal, table, (size_t)nel * p->nchan * sizeof(atkdsp_cf32), p->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(p->stream);
    if (rc != ATKB_OK) return map_rc(rc);
    p->cal_nel = nel;
    return ATKDSP_OK;
}

/* reference src/channelizer.c:410-417 (the same description line) */
ATKDSP_API int atkdsp_pfb_describe(const atkdsp_pfb *p, char *buf, size_t cap) {
    if (!p || !buf || cap == 0) return ATKDSP_E_ARG;
    return snprintf(buf, cap,
                    "PFB %.6g MSPS: %u chan x%u oversample, %.6g kHz spacing, %.6g kHz out, "
                    "%zu-tap proto (%u/poly), %.0f dB, <=%u el",
                    p->fs / 1e6, p->nchan, p->os, p->fs / p->nchan / 1e3,
                    atkdsp_pfb_out_rate(p) / 1e3, p->L, p->K, p->atten, p->max_nel);
}

const conv_t ATKB_CONV_CF32 = {0, 0.0f, 0.0f, 1.0f, NULL};
#define CONV_CF32 ATKB_CONV_CF32

void atkb_job_conv(atkb_job *J, atkb_carry *C, const conv_t *cv);
#define job_conv atkb_job_conv
/* int16 input reaches the kernel as fma(float(v), k, -(c*k)): k is a power of
 * two for both int16 formats, so c*k and v*k are exact and the fused form
 * rounds exactly like the reference's (float(v) - c) * k (scaling by 2^-e
 * commutes with rounding; where c*k would be subnormal, c is below half an
 * ulp of every nonzero v and both forms give v*k, or -(c*k) for v = 0) */
void atkb_job_conv(atkb_job *J, atkb_carry *C, const conv_t *cv) {
    J->in_kind = C->in_kind = cv->kind;
    J->kscale = C->kscale = cv->k;
    J->doff = C->doff = cv->kind ? cv->doff : NULL;
    if (cv->kind) {
        J->cre = C->cre = -(cv->cre * cv->k);
        J->cim = C->cim = -(cv->cim * cv->k);
    } else {
        J->cre = C->cre = cv->cre;
        J->cim = C->cim = cv->cim;
    }
}

/* Bounds-check injection (a test hook, host side only): the next step's
 * jobs claim `n` fewer samples than they have, so the kernel's window check
 * must catch the last tiles and the carry and skip them; the buffers still
 * hold every sample, so nothing can be read out of bounds even if the check
 * failed. */
static long long g_short_window;
static pthread_mutex_t g_short_lock = PTHREAD_MUTEX_INITIALIZER;
static long long take_short_window(void) {
    pthread_mutex_lock(&g_short_lock);
    const long long v = g_short_window;
    g_short_window = 0;
    pthread_mutex_unlock(&g_short_lock);
    return v;
}
ATKDSP_API void atkdsp_gpu_inject_short_window(long long n) {
    pthread_mutex_lock(&g_short_lock);
    g_short_window = n > 0 ? n : 0;
    pthread_mutex_unlock(&g_short_lock);
}

/* The fault bits the handle's launches set since the last query (0: none),
 * cleared by the query; the debug build adds its per-thread index checks. */
ATKDSP_API int atkdsp_gpu_pfb_faults(atkdsp_pfb *p) {
    unsigned v = 0;
    const unsigned z = 0;
    if (!p) return ATKDSP_E_ARG;
    if (atkb_set_device(p->dev) != ATKB_OK) return ATKDSP_E_FFT;
    if (p->stream && atkb_stream_sync(p->stream) != ATKB_OK) return ATKDSP_E_FFT;
    if (p->d_counters) {
        if (atkb_d2h(&v, p->d_counters + ATKB_FAULT_WORD, sizeof v, p->stream) != ATKB_OK ||
            atkb_stream_sync(p->stream) != ATKB_OK)
            return ATKDSP_E_FFT;
        if (v && (atkb_h2d(p->d_counters + ATKB_FAULT_WORD, &z, sizeof z, p->stream) != ATKB_OK ||
                  atkb_stream_sync(p->stream) != ATKB_OK))
            return ATKDSP_E_FFT;
    }
    return (int)(v | atkb_pfb_debug_fault());
}

ATKDSP_API int atkdsp_gpu_debug_build(void) { return atkb_pfb_debug_build(); }

/* One step: nel elements, n new samples each at ins[e] (device), m hops
 * written to outs + e * nchan * ldo (device, row stride ldo). Builds the job
 * and carry tables, uploads them, launches the tile kernel and the carry,
 * and advances the host mirror of the state. Asynchronous on `stream`. */
static int run_step_up(atkdsp_pfb *p, unsigned nel, const void *const *ins, size_t n, atkdsp_cf32 *outs,
                       size_t ldo, size_t m, void *stream, const conv_t *cv, size_t up_extra, int per_hop);

static int run_step(atkdsp_pfb *p, unsigned nel, const void *const *ins, size_t n,
                    atkdsp_cf32 *outs, size_t ldo, size_t m, void *stream, const conv_t *cv) {
    return run_step_up(p, nel, ins, n, outs, ldo, m, stream, cv, 0, 0);
}

/* up_extra: bytes after the tables (a small call's block) in the same upload;
 * per_hop: run the hops through the one-CTA-per-hop kernel (small calls) */
static int run_step_up(atkdsp_pfb *p, unsigned nel, const void *const *ins, size_t n, atkdsp_cf32 *outs,
                       size_t ldo, size_t m, void *stream, const conv_t *cv, size_t up_extra, int per_hop) {
    const size_t head = p->ov + p->lc;
    const unsigned nxt = (unsigned)(p->cur ^ 1);
    int rc;
    unsigned e;
    const long long short_window = take_short_window();
    if (p->tbl_event_live) {
        rc = atkb_event_sync(p->tbl_event);
        if (rc != ATKB_OK) return rc;
    }
    atkb_job *J = tbl_jobs(p->h_tables);
    atkb_carry *C = tbl_carry(p->h_tables, p->max_nel);
    int *T = tbl_tiles(p->h_tables, p->max_nel);
    const int big = p->bank.plan.big;
    const int tiles = big ? 0 : (int)((m + (size_t)p->bank.tile_hops - 1) / (size_t)p->bank.tile_hops);
    for (e = 0; e < nel; ++e) {
        memset(&J[e], 0, sizeof J[e]);
        J[e].state = state_buf(p, p->cur, e);
        J[e].in = ins[e];
        J[e].out = outs + (size_t)e * p->nchan * ldo;
        J[e].cal = (p->cal_nel && e < p->cal_nel) ? (const atkdsp_cf32 *)p->d_cal + (size_t)e * p->nchan
                                                  : NULL;
        J[e].head = (long long)head;
        J[e].ldo = (long long)ldo;
        J[e].out_col = 0;
        J[e].b0 = (long long)p->b;
        J[e].hops = (long long)m;
        J[e].bank = (const atkb_bank *)p->d_bank;
        J[e].tiles = tiles;
        T[e] = (int)e * tiles;
        C[e].state = J[e].state;
        C[e].in = ins[e];
        C[e].dst = state_buf(p, (int)nxt, e);
        C[e].head = (long long)head;
        C[e].from = (long long)(m * p->hop);
        C[e].len = (long long)(head + n - m * p->hop);
        J[e].nsrc = C[e].nsrc = (long long)(head + n) - short_window;
        C[e].cap = (long long)p->cap_state;
        J[e].w2 = e == 0 ? p->w2_next : NULL;
        job_conv(&J[e], &C[e], cv);
    }
    T[nel] = (int)nel * tiles;
    void *tb = p->d_tables;
    const int from_params = nel == 1 && !up_extra;
    if (from_params) {
        /* one job: a kernel writes the table from its launch parameters (and
         * derives the int16 constants there when the offset lives on the
         * device): no host->device copy, and the host table is free at once */
        rc = atkb_pfb_job_from_params(&J[0], &C[0], tiles, tbl_jobs(tb), tbl_carry(tb, p->max_nel),
                                      tbl_tiles(tb, p->max_nel), stream);
        if (rc != ATKB_OK) return rc;
    } else {
        /* the tables as laid out for max_nel, uploaded whole (they are small) */
        rc = atkb_h2d(p->d_tables, p->h_tables, p->tbl_bytes + up_extra, stream);
        if (rc == ATKB_OK) rc = atkb_event_record(p->tbl_event, stream);
        if (rc != ATKB_OK) return rc;
        p->tbl_event_live = 1;
        if (cv->doff) {                  /* the int16 offset lives on the device */
            rc = atkb_pfb_conv_from_offset(tbl_jobs(tb), tbl_carry(tb, p->max_nel), (int)nel, stream);
            if (rc != ATKB_OK) return rc;
        }
    }
    if (big) {
        /* the hops through the separate kernels, a chunk at a time; after the
         * upload (which carries a small call's block), before the tile kernel,
         * which then only copies the state carries */
        const long long H = atkb_pfb_big_hops((int)p->nchan);
        long long h0;
        for (e = 0; e < nel; ++e)
            for (h0 = 0; h0 < (long long)m; h0 += H) {
                const int nh = (int)((long long)m - h0 < H ? (long long)m - h0 : H);
                rc = atkb_pfb_big(&J[e], &p->bank, h0, nh, p->d_big, p->grid, stream);
                if (rc != ATKB_OK) return rc;
            }
    }
    {
        /* nel jobs: tile_start[nel] is their total (the kernel reads
         * tile_start[njobs]); the same launch copies the nel carries */
        const int work = (int)nel * tiles + (int)nel;
        if (per_hop && !big)
            rc = atkb_pfb_hops(tbl_jobs(tb), tbl_carry(tb, p->max_nel), (int)nel, (int)m, p->d_counters, stream);
        else if ((from_params || cv->doff) && !big)   /* right after the table kernel */
            rc = atkb_pfb_launch_pdl(tbl_jobs(tb), tbl_tiles(tb, p->max_nel), tbl_carry(tb, p->max_nel),
                                     (int)nel, p->d_counters, p->grid < work ? p->grid : work,
                                     p->bank.smem_bytes, stream);
        else
            rc = atkb_pfb_launch(tbl_jobs(tb), tbl_tiles(tb, p->max_nel),
                                 tbl_carry(tb, p->max_nel), (int)nel, p->d_counters,
                                 p->grid < work ? p->grid : work, p->bank.smem_bytes, stream);
        if (rc != ATKB_OK) return rc;
    }
    p->cur = (int)nxt;
    p->lc = (unsigned)(p->lc + n - m * p->hop);
    p->b += (int64_t)m;
    return ATKB_OK;
}

/* Pending samples (small calls that completed no hop) into the device state,
 * right after the samples it already holds: one copy per element, left in
 * flight and marked by small_ev. Every path other than the small-call path
 * calls this before it reads or writes the state. */
int atkb_pfb_flush_pending(atkdsp_pfb *p) {
    int rc = ATKB_OK;
    unsigned e;
    if (!p->npend) return ATKB_OK;
    if (p->small_live) {                 /* one copy in flight at a time */
        rc = atkb_event_sync(p->small_ev);
        if (rc != ATKB_OK) return rc;
        p->small_live = 0;
    }
    const size_t at = p->ov + p->lc - p->npend;      /* the device state's head */
    for (e = 0; e < p->pend_nel && rc == ATKB_OK; ++e)
        rc = atkb_h2d(state_buf(p, p->cur, e) + at, (atkdsp_cf32 *)p->h_pend + (size_t)e * p->hop,
                      p->npend * sizeof(atkdsp_cf32), p->stream);
    if (rc == ATKB_OK) rc = atkb_event_record(p->small_ev, p->stream);
    if (rc != ATKB_OK) return rc;
    p->small_live = 1;
    p->npend = 0;
    return ATKB_OK;
}

/* A small host call through the handle's pinned staging. A block that
 * completes no hop is only appended to the pending samples on the host (no
 * device work at all); a block that completes hops travels with the pending
 * samples and the job tables in one host->device copy, then one launch, one
 * device->host copy of the outputs and one synchronisation. */
static ptrdiff_t process_small(atkdsp_pfb *p, const atkdsp_cf32 *const *ins, unsigned nel, size_t n,
                               atkdsp_cf32 *out, size_t m) {
    int rc = ATKB_OK;
    unsigned e;
    if (p->npend && (p->pend_nel != nel || (m > 0 && p->npend + n > ATKB_SMALL_N))) {
        rc = atkb_pfb_flush_pending(p);
        if (rc != ATKB_OK) return map_rc(rc);
    }
    if (m == 0) {                        /* lc + n < hop: the pending samples stay < hop */
        for (e = 0; e < nel && n; ++e)
            memcpy((atkdsp_cf32 *)p->h_pend + (size_t)e * p->hop + p->npend, ins[e], n * sizeof(atkdsp_cf32));
        if (n) {
            p->npend += (unsigned)n;
            p->pend_nel = nel;
        }
        p->lc = (unsigned)(p->lc + n);
        return 0;
    }
    if (p->small_live) {                 /* h_small_in may still feed that copy */
        rc = atkb_event_sync(p->small_ev);
        if (rc != ATKB_OK) return map_rc(rc);
        p->small_live = 0;
    }
    if (p->tbl_event_live) {             /* ... or the last table upload */
        rc = atkb_event_sync(p->tbl_event);
        if (rc != ATKB_OK) return map_rc(rc);
    }
    /* each element's pending samples, then its new block */
    const size_t np = p->npend, nt = np + n;
    atkdsp_cf32 *hin = (atkdsp_cf32 *)p->h_small_in;
    for (e = 0; e < nel; ++e) {
        if (np) memcpy(hin + (size_t)e * ATKB_SMALL_N, (atkdsp_cf32 *)p->h_pend + (size_t)e * p->hop,
                       np * sizeof(atkdsp_cf32));
        if (n) memcpy(hin + (size_t)e * ATKB_SMALL_N + np, ins[e], n * sizeof(atkdsp_cf32));
    }
    const void **dins = p->dins;
    for (e = 0; e < nel; ++e) dins[e] = (const atkdsp_cf32 *)p->d_small_in + (size_t)e * ATKB_SMALL_N;
    /* outputs packed with stride m: [nel * nchan][m], the caller's layout */
    const size_t out_n = (size_t)nel * p->nchan * m;
    const size_t up = ((size_t)(nel - 1) * ATKB_SMALL_N + nt) * sizeof(atkdsp_cf32);
    p->lc -= (unsigned)np;               /* the device state holds lc - npend of the leftover */
    p->npend = 0;
    /* a few hops: one CTA each (a tile's latency is ~20 us, a hop's a few) */
    const int per_hop = !p->w2_next && (size_t)nel * m <= ATKB_PER_HOP_MAX && atkb_pfb_hops_ok(&p->bank);
    /* the per-hop kernel writes up to ATKB_DIRECT_OUT outputs straight into
     * the pinned buffer (each an 8-byte write over the bus: beyond that one
     * device->host copy of the packed outputs is faster) */
    const int direct = per_hop && p->dz_small_out != NULL && out_n <= ATKB_DIRECT_OUT;
    rc = run_step_up(p, nel, dins, nt, (atkdsp_cf32 *)(direct ? p->dz_small_out : p->d_out_stage), m, m,
                     p->stream, &CONV_CF32, up, per_hop);
    if (rc == ATKB_OK && !direct)
        rc = atkb_d2h(p->h_small_out, p->d_out_stage, out_n * sizeof(atkdsp_cf32), p->stream);
    if (rc == ATKB_OK) rc = atkb_event_record(p->small_done, p->stream);
    if (rc == ATKB_OK) rc = atkb_event_spin(p->small_done);
    if (rc != ATKB_OK) return map_rc(rc);
    memcpy(out, p->h_small_out, out_n * sizeof(atkdsp_cf32));
    return (ptrdiff_t)m;
}

int atkb_pfb_order_after_small(atkdsp_pfb *p, void *stream) {
    const int rc = atkb_pfb_flush_pending(p);
    if (rc != ATKB_OK) return rc;
    if (!p->small_live) return ATKB_OK;
    if (!stream || stream == p->stream) return ATKB_OK;
    return atkb_stream_wait(stream, p->small_ev);
}

/* reference src/channelizer.c:305-402 */
ATKDSP_API ptrdiff_t atkdsp_pfb_process_n(atkdsp_pfb *p, const atkdsp_cf32 *const *ins, unsigned nel,
                                          size_t n, atkdsp_cf32 *out, size_t cap) {
    if (!p || !ins || nel < 1 || nel > p->max_nel) return ATKDSP_E_ARG;
    unsigned e;
    for (e = 0; e < nel && n; ++e)
        if (!ins[e]) return ATKDSP_E_ARG;
    const size_t m = ((size_t)p->lc + n) / p->hop;
    if (m > 0 && (!out || cap < (size_t)nel * p->nchan * m)) return ATKDSP_E_CAP;
    if (atkb_set_device(p->dev) != ATKB_OK) return ATKDSP_E_FFT;
    if (p->h_small_in && n <= ATKB_SMALL_N) return process_small(p, ins, nel, n, out, m);
    if (p->npend && atkb_pfb_flush_pending(p) != ATKB_OK) return ATKDSP_E_FFT;
    if (p->small_live) {
        const int rs = atkb_event_sync(p->small_ev);
        if (rs != ATKB_OK) return map_rc(rs);
        p->small_live = 0;
    }
    size_t pos = 0, col = 0;
    int rc = ATKB_OK;
    const void **dins = p->dins;
    for (e = 0; e < nel; ++e) dins[e] = (const atkdsp_cf32 *)p->d_in_stage + (size_t)e * p->chunk;
    while (pos < n && rc == ATKB_OK) {
        const size_t nc = (n - pos < p->chunk) ? n - pos : p->chunk;
        const size_t mc = ((size_t)p->lc + nc) / p->hop;
        for (e = 0; e < nel && rc == ATKB_OK; ++e)
            rc = atkb_h2d((void *)dins[e], ins[e] + pos, nc * sizeof(atkdsp_cf32), p->stream);
        if (rc != ATKB_OK) break;
        if (nc == n) {
            /* the whole call in one chunk: the staging takes the caller's row
             * stride (m <= out_ld), so the outputs come back in one contiguous
             * copy instead of one row per channel */
            rc = run_step(p, nel, (const void *const *)dins, nc, (atkdsp_cf32 *)p->d_out_stage, mc ? mc : 1,
                          mc, p->stream, &CONV_CF32);
            if (rc == ATKB_OK && mc > 0)
                rc = atkb_d2h(out, p->d_out_stage, (size_t)nel * p->nchan * mc * sizeof(atkdsp_cf32), p->stream);
            col += mc;
            pos += nc;
            continue;
        }
        rc = run_step(p, nel, (const void *const *)dins, nc, (atkdsp_cf32 *)p->d_out_stage, p->out_ld,
                      mc, p->stream, &CONV_CF32);
        if (rc != ATKB_OK) break;
        if (mc > 0) {
            /* rows e*nchan + k: out + (e*nchan + k)*m + col  <-  stage + (e*nchan + k)*out_ld */
            rc = atkb_d2h_2d(out + col, m * sizeof(atkdsp_cf32), p->d_out_stage,
                             p->out_ld * sizeof(atkdsp_cf32), mc * sizeof(atkdsp_cf32),
                             (size_t)nel * p->nchan, p->stream);
        }
        col += mc;
        pos += nc;
    }
    if (rc == ATKB_OK) rc = atkb_stream_sync(p->stream);
    if (rc != ATKB_OK) return map_rc(rc);
    return (ptrdiff_t)m;
}

ATKDSP_API ptrdiff_t atkdsp_pfb_process(atkdsp_pfb *p, const atkdsp_cf32 *in, size_t n,
                                        atkdsp_cf32 *out, size_t cap) {
    const atkdsp_cf32 *ins[1];
    ins[0] = in;
    return atkdsp_pfb_process_n(p, ins, 1, n, out, cap);
}

/* ================================================================ device API */
ATKDSP_API void *atkdsp_gpu_pfb_stream(atkdsp_pfb *p) { return p ? p->stream : NULL; }

ATKDSP_API int atkdsp_gpu_pfb_sync(atkdsp_pfb *p) {
    if (!p) return ATKDSP_E_ARG;
    atkb_set_device(p->dev);
    return atkb_stream_sync(p->stream) == ATKB_OK ? ATKDSP_OK : ATKDSP_E_FFT;
}

ATKDSP_API ptrdiff_t atkdsp_gpu_pfb_process_n(atkdsp_pfb *p, const atkdsp_cf32 *const *d_ins,
                                              unsigned nel, size_t n, atkdsp_cf32 *d_out,
                                              size_t cap, void *stream) {
    if (!p || !d_ins || nel < 1 || nel > p->max_nel) return ATKDSP_E_ARG;
    unsigned e;
    for (e = 0; e < nel && n; ++e)
        if (!d_ins[e]) return ATKDSP_E_ARG;
    if ((size_t)p->lc + n >= ((size_t)1 << 62)) return ATKDSP_E_ARG;
    const size_t m = ((size_t)p->lc + n) / p->hop;
    if (m > 0 && (!d_out || cap < (size_t)nel * p->nchan * m)) return ATKDSP_E_CAP;
    if (m > (size_t)0x7fffffff / 4 / nel) return ATKDSP_E_ARG;   /* tile indices are int */
    if (atkb_set_device(p->dev) != ATKB_OK) return ATKDSP_E_FFT;
    if (atkb_pfb_order_after_small(p, stream) != ATKB_OK) return ATKDSP_E_FFT;
    const int rc = run_step(p, nel, (const void *const *)d_ins, n, d_out, m, m,
                            stream ? stream : p->stream, &CONV_CF32);
    return rc == ATKB_OK ? (ptrdiff_t)m : map_rc(rc);
}

static int unpack_consts(int fmt, float off_re, float off_im, float *cre, float *cim, float *k);

/* the int16 formats the filterbank reads directly */
#define raw_conv atkb_raw_conv
int atkb_raw_conv(int fmt, float off_re, float off_im, conv_t *cv) {
    if (fmt != ATKDSP_FMT_CI16 && fmt != ATKDSP_FMT_CI16Q11) return 0;
    cv->kind = 1;
    cv->doff = NULL;
    unpack_consts(fmt, off_re, off_im, &cv->cre, &cv->cim, &cv->k);
    return 1;
}

ATKDSP_API ptrdiff_t atkdsp_gpu_pfb_process_n_raw(atkdsp_pfb *p, const void *const *d_raws,
                                                  unsigned nel, size_t n, int fmt, float off_re,
                                                  float off_im, atkdsp_cf32 *d_out, size_t cap,
                                                  void *stream) {
    conv_t cv;
    if (!p || !d_raws || nel < 1 || nel > p->max_nel || !raw_conv(fmt, off_re, off_im, &cv))
        return ATKDSP_E_ARG;
    unsigned e;
    for (e = 0; e < nel && n; ++e)
        if (!d_raws[e] || ((size_t)d_raws[e] & 3)) return ATKDSP_E_ARG;
    if ((size_t)p->lc + n >= ((size_t)1 << 62)) return ATKDSP_E_ARG;
    const size_t m = ((size_t)p->lc + n) / p->hop;
    if (m > 0 && (!d_out || cap < (size_t)nel * p->nchan * m)) return ATKDSP_E_CAP;
    if (m > (size_t)0x7fffffff / 4 / nel) return ATKDSP_E_ARG;
    if (atkb_set_device(p->dev) != ATKB_OK) return ATKDSP_E_FFT;
    if (atkb_pfb_order_after_small(p, stream) != ATKB_OK) return ATKDSP_E_FFT;
    const int rc = run_step(p, nel, d_raws, n, d_out, m, m, stream ? stream : p->stream, &cv);
    return rc == ATKB_OK ? (ptrdiff_t)m : map_rc(rc);
}

/* ---- the filterbank with W1 / W2 fused into its epilogue (one element) ---- */
static int w2_fusable(const atkdsp_pfb *p) {
    return p->bank.plan.fast && p->nchan <= 2048;
}

ATKDSP_API size_t atkdsp_gpu_pfb_w12_scratch_bytes(const atkdsp_pfb *p, size_t n) {
    if (!p) return 0;
    const size_t m = ((size_t)p->lc + n) / p->hop;
    const size_t th = (size_t)p->bank.tile_hops;
    return w2_fusable(p) ? ((m + th - 1) / th) * p->nchan * sizeof(double) : 0;
}

static ptrdiff_t process_w12(atkdsp_pfb *p, const void *d_in, size_t n, int fmt, float off_re, float off_im,
                             const double *d_off, atkdsp_cf32 *d_out, size_t cap, const uint8_t *d_gate,
                             atkdsp_cf32 *d_R, uint32_t *d_counts, float *d_pwr, float *d_mean_pwr,
                             void *d_scratch, size_t scratch_bytes, void *stream) {
    conv_t cv = CONV_CF32;
    if (!p || (n && !d_in)) return ATKDSP_E_ARG;
    if (fmt != ATKDSP_FMT_CF32 && !raw_conv(fmt, off_re, off_im, &cv)) return ATKDSP_E_ARG;
    if (fmt == ATKDSP_FMT_CF32 && (off_re != 0.0f || off_im != 0.0f || d_off)) return ATKDSP_E_ARG;
    if (n && ((size_t)d_in & (fmt == ATKDSP_FMT_CF32 ? 7 : 3))) return ATKDSP_E_ARG;
    if ((d_R == NULL) != (d_counts == NULL)) return ATKDSP_E_ARG;
    if ((size_t)p->lc + n >= ((size_t)1 << 62)) return ATKDSP_E_ARG;
    const size_t m = ((size_t)p->lc + n) / p->hop;
    if (m > 0 && (!d_out || cap < (size_t)p->nchan * m)) return ATKDSP_E_CAP;
    if (m > (size_t)0x7fffffff / 4) return ATKDSP_E_ARG;
    const int fused = w2_fusable(p);
    const size_t need = atkdsp_gpu_pfb_w12_scratch_bytes(p, n);
    if (fused && m > 0 && (!d_scratch || scratch_bytes < need || ((size_t)d_scratch & 7))) return ATKDSP_E_CAP;
    if (atkb_set_device(p->dev) != ATKB_OK) return ATKDSP_E_FFT;
    if (atkb_pfb_order_after_small(p, stream) != ATKB_OK) return ATKDSP_E_FFT;
    void *st = stream ? stream : p->stream;
    const void *ins[1];
    ins[0] = d_in;
    p->w2_next = (fused && m > 0) ? (double *)d_scratch : NULL;
    cv.doff = d_off;
    int rc = run_step(p, 1, ins, n, d_out, m, m, st, &cv);
    p->w2_next = NULL;
    if (rc == ATKB_OK) {
        if (fused) {
            const size_t th = (size_t)p->bank.tile_hops;
            rc = m > 0 ? atkb_w2_finish((const double *)d_scratch, (int)((m + th - 1) / th), (int)p->nchan,
                                        (long long)m, d_gate, d_R, d_counts, d_pwr, d_mean_pwr, st)
                       : atkb_w12(d_out, 1, p->nchan, 0, d_gate, d_R, d_counts, d_pwr, d_mean_pwr, st);
        } else {
            rc = atkb_w12(d_out, 1, p->nchan, m, d_gate, d_R, d_counts, d_pwr, d_mean_pwr, st);
        }
    }
    return rc == ATKB_OK ? (ptrdiff_t)m : map_rc(rc);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_pfb_process_w12(atkdsp_pfb *p, const void *d_in, size_t n, int fmt,
                                                float off_re, float off_im, atkdsp_cf32 *d_out, size_t cap,
                                                const uint8_t *d_gate, atkdsp_cf32 *d_R, uint32_t *d_counts,
                                                float *d_pwr, float *d_mean_pwr, void *d_scratch,
                                                size_t scratch_bytes, void *stream) {
    return process_w12(p, d_in, n, fmt, off_re, off_im, NULL, d_out, cap, d_gate, d_R, d_counts, d_pwr,
                       d_mean_pwr, d_scratch, scratch_bytes, stream);
}

/* the same with the int16 offset in device memory (the previous block's
 * atkdsp_gpu_block_mean output, rounded to float on the device): a running
 * DC estimate that never visits the host */
ATKDSP_API ptrdiff_t atkdsp_gpu_pfb_process_w12_dev(atkdsp_pfb *p, const void *d_in, size_t n, int fmt,
                                                    const double *d_offset, atkdsp_cf32 *d_out, size_t cap,
                                                    const uint8_t *d_gate, atkdsp_cf32 *d_R,
                                                    uint32_t *d_counts, float *d_pwr, float *d_mean_pwr,
                                                    void *d_scratch, size_t scratch_bytes, void *stream) {
    if (!d_offset || ((size_t)d_offset & 7) || fmt == ATKDSP_FMT_CF32) return ATKDSP_E_ARG;
    return process_w12(p, d_in, n, fmt, 0.0f, 0.0f, d_offset, d_out, cap, d_gate, d_R, d_counts, d_pwr,
                       d_mean_pwr, d_scratch, scratch_bytes, stream);
}

/* ============================================ per-thread scratch for host calls
 * W1/W2 and unpack on HOST buffers stage through device memory. Each calling
 * thread has its own staging area and CUDA stream per device, so calls from
 * different threads never wait on each other (the reference's callers run
 * different handles and these stateless calls from several threads at once,
 * src/undertow.c:252-257). A thread's area is allocated by its first such
 * call on a device and grown only when a larger call comes; later calls of
 * the same or a smaller size allocate nothing. A thread that exits releases
 * its areas. The device-pointer unpack_dc / block_mean calls take their mean
 * partials from a separate fixed per-thread buffer (never regrown, never
 * shared with the staging), so host calls can't move memory that queued
 * device work still uses. */
#define MAX_DEV 16
#define GPU_PARTIALS 4096                 /* atkb_unpack_partials bound, doubles x2 */
typedef struct {
    void *d;                              /* staging for host calls */
    size_t cap;
    void *stream;
    double *partials;                     /* device unpack_dc / block_mean */
} scratch_t;
typedef struct { scratch_t dev[MAX_DEV]; } thread_scratch;
static pthread_key_t g_scr_key;
static pthread_once_t g_scr_once = PTHREAD_ONCE_INIT;
static int g_scr_key_ok;

static void scratch_release(void *v) {
    thread_scratch *t = (thread_scratch *)v;
    int cur = -1, d;
    if (!t) return;
    atkb_get_device(&cur);
    for (d = 0; d < MAX_DEV; ++d) {
        scratch_t *s = &t->dev[d];
        if (!s->d && !s->stream && !s->partials) continue;
        atkb_set_device(d);
        if (s->stream) atkb_stream_sync(s->stream);
        atkb_free(s->d);
        atkb_free(s->partials);
        atkb_stream_destroy(s->stream);
    }
    if (cur >= 0) atkb_set_device(cur);
    free(t);
}
static void scratch_key_init(void) { g_scr_key_ok = pthread_key_create(&g_scr_key, scratch_release) == 0; }

/* this thread's scratch on the current device, with at least `bytes` of
 * staging (0: staging untouched) */
static scratch_t *thread_scratch_get(size_t bytes, int *rc) {
    int dev = 0;
    *rc = atkb_get_device(&dev);
    if (*rc != ATKB_OK) return NULL;
    if (dev < 0 || dev >= MAX_DEV) { *rc = ATKB_E_NODEV; return NULL; }
    pthread_once(&g_scr_once, scratch_key_init);
    if (!g_scr_key_ok) { *rc = ATKB_E_NOMEM; return NULL; }
    thread_scratch *t = (thread_scratch *)pthread_getspecific(g_scr_key);
    if (!t) {
        t = (thread_scratch *)calloc(1, sizeof *t);
        if (!t || pthread_setspecific(g_scr_key, t) != 0) { free(t); *rc = ATKB_E_NOMEM; return NULL; }
    }
    scratch_t *s = &t->dev[dev];
    if (!s->stream && (*rc = atkb_stream_create(&s->stream)) != ATKB_OK) {
        s->stream = NULL;
        return NULL;
    }
    if (s->cap < bytes) {
        atkb_stream_sync(s->stream);      /* the old area may still feed a copy */
        atkb_free(s->d);
        s->d = NULL;
        s->cap = 0;
        const size_t want = bytes + bytes / 4 + 4096;
        if ((*rc = atkb_malloc(&s->d, want)) != ATKB_OK) { s->d = NULL; return NULL; }
        s->cap = want;
    }
    *rc = ATKB_OK;
    return s;
}

/* ====================================================================== W1/W2 */
ATKDSP_API void atkdsp_pfb_cov_accumulate(const atkdsp_cf32 *out, unsigned nel, unsigned nchan,
                                          size_t m, const uint8_t *gate, atkdsp_cf32 *R,
                                          uint32_t *counts) {
    if (!out || !R || !counts || nel < 1 || nchan < 1 || nel > MAX_W12_NEL) return;
    const size_t ob = align16((size_t)nel * nchan * m * sizeof(atkdsp_cf32));
    const size_t rb = align16((size_t)nchan * nel * nel * sizeof(atkdsp_cf32));
    const size_t cb = align16((size_t)nchan * sizeof(uint32_t));
    const size_t gb = align16(nchan);
    int rc;
    scratch_t *s = thread_scratch_get(ob + rb + cb + gb, &rc);
    if (!s) return;
    char *d = (char *)s->d;
    rc = atkb_h2d(d, out, (size_t)nel * nchan * m * sizeof(atkdsp_cf32), s->stream);
    if (rc == ATKB_OK) rc = atkb_h2d(d + ob, R, (size_t)nchan * nel * nel * sizeof(atkdsp_cf32), s->stream);
    if (rc == ATKB_OK) rc = atkb_h2d(d + ob + rb, counts, nchan * sizeof(uint32_t), s->stream);
    if (rc == ATKB_OK && gate) rc = atkb_h2d(d + ob + rb + cb, gate, nchan, s->stream);
    if (rc == ATKB_OK)
        rc = atkb_w12(d, nel, nchan, m, gate ? (const uint8_t *)(d + ob + rb + cb) : NULL, d + ob,
                      (uint32_t *)(d + ob + rb), NULL, NULL, s->stream);
    if (rc == ATKB_OK) rc = atkb_d2h(R, d + ob, (size_t)nchan * nel * nel * sizeof(atkdsp_cf32), s->stream);
    if (rc == ATKB_OK) rc = atkb_d2h(counts, d + ob + rb, nchan * sizeof(uint32_t), s->stream);
    atkb_stream_sync(s->stream);
}

ATKDSP_API void atkdsp_pfb_cov_reset(atkdsp_cf32 *R, uint32_t *counts, unsigned nel, unsigned nchan,
                                     const uint8_t *gate) {
    /* reference src/channelizer.c:442-450: plain memory clearing of the
     * caller's HOST arrays; there is nothing to compute, so it stays on the
     * host rather than round-tripping through the device. */
    unsigned k;
    if (!R || !counts) return;
    for (k = 0; k < nchan; ++k) {
        if (gate && !gate[k]) continue;
        memset(R + (size_t)k * nel * nel, 0, (size_t)nel * nel * sizeof(atkdsp_cf32));
        counts[k] = 0;
    }
}

ATKDSP_API void atkdsp_pfb_channel_power(const atkdsp_cf32 *out, unsigned nel, unsigned nchan,
                                         size_t m, float *pwr, float *mean_pwr) {
    if (!out || nel < 1 || nchan < 1 || nel > MAX_W12_NEL) return;
    const size_t ob = align16((size_t)nel * nchan * m * sizeof(atkdsp_cf32));
    const size_t pb = align16((size_t)nel * nchan * sizeof(float));
    const size_t mb = align16((size_t)nchan * sizeof(float));
    int rc;
    scratch_t *s = thread_scratch_get(ob + pb + mb, &rc);
    if (!s) return;
    char *d = (char *)s->d;
    rc = atkb_h2d(d, out, (size_t)nel * nchan * m * sizeof(atkdsp_cf32), s->stream);
    if (rc == ATKB_OK)
        rc = atkb_w12(d, nel, nchan, m, NULL, NULL, NULL, pwr ? (float *)(d + ob) : NULL,
                      mean_pwr ? (float *)(d + ob + pb) : NULL, s->stream);
    if (rc == ATKB_OK && pwr) rc = atkb_d2h(pwr, d + ob, (size_t)nel * nchan * sizeof(float), s->stream);
    if (rc == ATKB_OK && mean_pwr) rc = atkb_d2h(mean_pwr, d + ob + pb, nchan * sizeof(float), s->stream);
    atkb_stream_sync(s->stream);
}

ATKDSP_API int atkdsp_gpu_pfb_cov_accumulate(const atkdsp_cf32 *d_out, unsigned nel, unsigned nchan,
                                             size_t m, const uint8_t *d_gate, atkdsp_cf32 *d_R,
                                             uint32_t *d_counts, void *stream) {
    if (!d_out || !d_R || !d_counts || nel < 1 || nchan < 1 || nel > MAX_W12_NEL) return ATKDSP_E_ARG;
    return map_rc(atkb_w12(d_out, nel, nchan, m, d_gate, d_R, d_counts, NULL, NULL, stream));
}

ATKDSP_API int atkdsp_gpu_pfb_accumulate(const atkdsp_cf32 *d_out, unsigned nel, unsigned nchan,
                                         size_t m, const uint8_t *d_gate, atkdsp_cf32 *d_R,
                                         uint32_t *d_counts, float *d_pwr, float *d_mean_pwr,
                                         void *stream) {
    if (!d_out || nel < 1 || nchan < 1 || nel > MAX_W12_NEL) return ATKDSP_E_ARG;
    if ((d_R == NULL) != (d_counts == NULL)) return ATKDSP_E_ARG;
    return map_rc(atkb_w12(d_out, nel, nchan, m, d_gate, d_R, d_counts, d_pwr, d_mean_pwr, stream));
}

ATKDSP_API int atkdsp_gpu_pfb_cov_reset(atkdsp_cf32 *d_R, uint32_t *d_counts, unsigned nel,
                                        unsigned nchan, const uint8_t *d_gate, void *stream) {
    if (!d_R || !d_counts) return ATKDSP_E_ARG;
    return map_rc(atkb_cov_reset(d_R, d_counts, nel, nchan, d_gate, stream));
}

ATKDSP_API int atkdsp_gpu_pfb_channel_power(const atkdsp_cf32 *d_out, unsigned nel, unsigned nchan,
                                            size_t m, float *d_pwr, float *d_mean_pwr, void *stream) {
    if (!d_out || nel < 1 || nchan < 1 || nel > MAX_W12_NEL) return ATKDSP_E_ARG;
    return map_rc(atkb_w12(d_out, nel, nchan, m, NULL, NULL, NULL, d_pwr, d_mean_pwr, stream));
}

/* ===================================================================== unpack
 * The constants of reference src/convert.c:45-71, computed in float exactly
 * as the reference does so the device conversion is bit-identical. */
static int unpack_consts(int fmt, float off_re, float off_im, float *cre, float *cim, float *k) {
    switch (fmt) {
    case ATKDSP_FMT_CU8:
        *k = 1.0f / 127.5f;
        *cre = 127.5f + off_re / *k;
        *cim = 127.5f + off_im / *k;
        return 1;
    case ATKDSP_FMT_CI8:
        *k = 1.0f / 128.0f;
        break;
    case ATKDSP_FMT_CI16:
        *k = 1.0f / 32768.0f;
        break;
    case ATKDSP_FMT_CI16Q11:
        *k = 1.0f / 2048.0f;
        break;
    case ATKDSP_FMT_CF32:
        *k = 1.0f;
        *cre = off_re;
        *cim = off_im;
        return 1;
    default:
        return 0;
    }
    *cre = off_re / *k;
    *cim = off_im / *k;
    return 1;
}

static ptrdiff_t unpack_host(const void *raw, size_t nbytes, int fmt, atkdsp_cf32 *out, size_t cap,
                             float off_re, float off_im, double *mean_re, double *mean_im,
                             float dc_alpha, atkdsp_cf32 *dc_state) {
    if (!raw || !out) return ATKDSP_E_ARG;
    const int bps = atkdsp_bytes_per_sample(fmt);
    if (!bps) return ATKDSP_E_ARG;
    float cre, cim, k;
    unpack_consts(fmt, off_re, off_im, &cre, &cim, &k);
    size_t n = nbytes / (size_t)bps;
    if (n > cap) n = cap;
    const int want_mean = mean_re || mean_im;
    const int pole = dc_alpha > 0.0f && dc_state != NULL;
    if (n == 0) {
        if (mean_re) *mean_re = (double)off_re;
        if (mean_im) *mean_im = (double)off_im;
        return 0;
    }
    const size_t rb = align16(n * (size_t)bps);
    const size_t ob = align16(n * sizeof(atkdsp_cf32));
    const size_t pb = align16((size_t)atkb_unpack_partials(n) * 2 * sizeof(double));
    int rc;
    scratch_t *s = thread_scratch_get(rb + ob + pb + 64, &rc);
    if (!s) return map_rc(rc);
    char *d = (char *)s->d;
    double *d_mean = (double *)(d + rb + ob + pb);
    double hm[2] = {0.0, 0.0};
    rc = atkb_h2d(d, raw, n * (size_t)bps, s->stream);
    if (rc == ATKB_OK && pole) rc = atkb_h2d(d_mean + 2, dc_state, sizeof(atkdsp_cf32), s->stream);
    if (rc == ATKB_OK)
        rc = atkb_unpack(d, fmt, n, d + rb, cre, cim, k, off_re, off_im, want_mean ? d_mean : NULL,
                         (double *)(d + rb + ob), NULL, NULL, s->stream);
    if (rc == ATKB_OK && pole) rc = atkb_dc_pole(d + rb, n, dc_alpha, d_mean + 2, s->stream);
    if (rc == ATKB_OK) rc = atkb_d2h(out, d + rb, n * sizeof(atkdsp_cf32), s->stream);
    if (rc == ATKB_OK && want_mean) rc = atkb_d2h(hm, d_mean, sizeof hm, s->stream);
    if (rc == ATKB_OK && pole) rc = atkb_d2h(dc_state, d_mean + 2, sizeof(atkdsp_cf32), s->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(s->stream);
    if (rc != ATKB_OK) return map_rc(rc == ATKB_E_NOMEM ? rc : ATKB_E_KERNEL);
    if (mean_re) *mean_re = hm[0];
    if (mean_im) *mean_im = hm[1];
    return (ptrdiff_t)n;
}

/* reference src/convert.c:113-120 */
ATKDSP_API ptrdiff_t atkdsp_unpack(const void *raw, size_t nbytes, int fmt, atkdsp_cf32 *out,
                                   size_t out_cap, float dc_alpha, atkdsp_cf32 *dc_state) {
    return unpack_host(raw, nbytes, fmt, out, out_cap, 0.0f, 0.0f, NULL, NULL, dc_alpha, dc_state);
}

/* reference src/convert.c:122-128 */
ATKDSP_API ptrdiff_t atkdsp_unpack_dc(const void *raw, size_t nbytes, int fmt, atkdsp_cf32 *out,
                                      size_t out_cap, float off_re, float off_im, double *mean_re,
                                      double *mean_im) {
    return unpack_host(raw, nbytes, fmt, out, out_cap, off_re, off_im, mean_re, mean_im, 0.0f, NULL);
}

/* device-pointer unpack: the calling thread's fixed partials buffer on the
 * current device (allocated by its first such call, then reused), and the
 * fused mean's block counter after the partials (zeroed on the caller's
 * stream when allocated; every launch leaves it at 0) */
static int gpu_partials(double **d, unsigned **done, void *stream) {
    int rc;
    scratch_t *s = thread_scratch_get(0, &rc);
    if (!s) return rc;
    if (!s->partials) {
        void *p = NULL;
        if ((rc = atkb_malloc(&p, GPU_PARTIALS * 2 * sizeof(double) + 256)) != ATKB_OK) return rc;
        if ((rc = atkb_memset((char *)p + GPU_PARTIALS * 2 * sizeof(double), 0, 256, stream)) != ATKB_OK) {
            atkb_free(p);
            return rc;
        }
        s->partials = (double *)p;
    }
    *d = s->partials;
    *done = (unsigned *)(s->partials + GPU_PARTIALS * 2);
    return ATKB_OK;
}

static int aligned_for(const void *ptr, int fmt) {
    const size_t a = fmt == ATKDSP_FMT_CF32 ? 8 : fmt >= ATKDSP_FMT_CI16 ? 4 : 2;
    return ((size_t)ptr % a) == 0;
}

ATKDSP_API ptrdiff_t atkdsp_gpu_unpack_dc(const void *d_raw, size_t nbytes, int fmt, atkdsp_cf32 *d_out,
                                          size_t out_cap, float off_re, float off_im, double *d_mean,
                                          void *stream) {
    if (!d_raw || !d_out) return ATKDSP_E_ARG;
    const int bps = atkdsp_bytes_per_sample(fmt);
    if (!bps || !aligned_for(d_raw, fmt) || ((size_t)d_out & 7)) return ATKDSP_E_ARG;
    float cre, cim, k;
    unpack_consts(fmt, off_re, off_im, &cre, &cim, &k);
    size_t n = nbytes / (size_t)bps;
    if (n > out_cap) n = out_cap;
    double *part = NULL;
    unsigned *done = NULL;
    if (d_mean) {
        const int rc = gpu_partials(&part, &done, stream);
        if (rc != ATKB_OK) return map_rc(rc);
    }
    const int rc = atkb_unpack(d_raw, fmt, n, d_out, cre, cim, k, off_re, off_im, d_mean, part, done, NULL,
                               stream);
    return rc == ATKB_OK ? (ptrdiff_t)n : map_rc(rc);
}

/* atkdsp_gpu_unpack_dc for callers that cannot allocate device memory: the
 * mean's scratch is a static device array (unpack.cu), nothing is allocated. */
ATKDSP_API ptrdiff_t atkdsp_gpu_unpack_dc_noalloc(const void *d_raw, size_t nbytes, int fmt,
                                                  atkdsp_cf32 *d_out, size_t out_cap, float off_re,
                                                  float off_im, double *d_mean, void *stream) {
    if (!d_raw || !d_out) return ATKDSP_E_ARG;
    const int bps = atkdsp_bytes_per_sample(fmt);
    if (!bps || !aligned_for(d_raw, fmt) || ((size_t)d_out & 7)) return ATKDSP_E_ARG;
    float cre, cim, k;
    unpack_consts(fmt, off_re, off_im, &cre, &cim, &k);
    size_t n = nbytes / (size_t)bps;
    if (n > out_cap) n = out_cap;
    if (n > atkb_unpack_noalloc_max_samples()) return ATKDSP_E_ARG;
    const int rc = atkb_unpack_noalloc(d_raw, fmt, n, d_out, cre, cim, k, off_re, off_im, d_mean, stream);
    return rc == ATKB_OK ? (ptrdiff_t)n : map_rc(rc);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_block_mean(const void *d_raw, size_t nbytes, int fmt, float off_re,
                                           float off_im, double *d_mean, void *stream) {
    if (!d_raw || !d_mean) return ATKDSP_E_ARG;
    const int bps = atkdsp_bytes_per_sample(fmt);
    if (!bps || !aligned_for(d_raw, fmt)) return ATKDSP_E_ARG;
    float cre, cim, k;
    unpack_consts(fmt, off_re, off_im, &cre, &cim, &k);
    const size_t n = nbytes / (size_t)bps;
    double *part = NULL;
    unsigned *done = NULL;
    int rc = gpu_partials(&part, &done, stream);
    if (rc == ATKB_OK)
        rc = atkb_unpack(d_raw, fmt, n, NULL, cre, cim, k, off_re, off_im, d_mean, part, done, NULL, stream);
    return rc == ATKB_OK ? (ptrdiff_t)n : map_rc(rc);
}

/* atkdsp_gpu_block_mean with the offset in device memory (two doubles,
 * rounded to float on the device; d_offset may equal d_mean) */
ATKDSP_API ptrdiff_t atkdsp_gpu_block_mean_dev(const void *d_raw, size_t nbytes, int fmt, const double *d_offset,
                                               double *d_mean, void *stream) {
    if (!d_raw || !d_mean || !d_offset || ((size_t)d_offset & 7)) return ATKDSP_E_ARG;
    const int bps = atkdsp_bytes_per_sample(fmt);
    if (!bps || !aligned_for(d_raw, fmt)) return ATKDSP_E_ARG;
    float cre, cim, k;
    unpack_consts(fmt, 0.0f, 0.0f, &cre, &cim, &k);
    const size_t n = nbytes / (size_t)bps;
    double *part = NULL;
    unsigned *done = NULL;
    int rc = gpu_partials(&part, &done, stream);
    if (rc == ATKB_OK)
        rc = atkb_unpack(d_raw, fmt, n, NULL, cre, cim, k, 0.0f, 0.0f, d_mean, part, done, d_offset, stream);
    return rc == ATKB_OK ? (ptrdiff_t)n : map_rc(rc);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_unpack(const void *d_raw, size_t nbytes, int fmt, atkdsp_cf32 *d_out,
                                       size_t out_cap, float dc_alpha, atkdsp_cf32 *d_dc_state,
                                       void *stream) {
    if (!d_raw || !d_out) return ATKDSP_E_ARG;
    const int bps = atkdsp_bytes_per_sample(fmt);
    if (!bps || !aligned_for(d_raw, fmt) || ((size_t)d_out & 7)) return ATKDSP_E_ARG;
    float cre, cim, k;
    unpack_consts(fmt, 0.0f, 0.0f, &cre, &cim, &k);
    size_t n = nbytes / (size_t)bps;
    if (n > out_cap) n = out_cap;
    int rc = atkb_unpack(d_raw, fmt, n, d_out, cre, cim, k, 0.0f, 0.0f, NULL, NULL, NULL, NULL, stream);
    if (rc == ATKB_OK && dc_alpha > 0.0f && d_dc_state) rc = atkb_dc_pole(d_out, n, dc_alpha, d_dc_state, stream);
    return rc == ATKB_OK ? (ptrdiff_t)n : map_rc(rc);
}

/* ===================================================================== batches */
struct atkdsp_gpu_batch {
    unsigned count;
    atkdsp_pfb **h;
    int dev;
    void *stream;
    int use_graph;
    size_t tbl_bytes;
    void *d_tables;
    void *h_tables[2];
    void *ev[2];
    int ev_live[2];
    void *graph[2];
    int slot;
    int *d_counters;
    int grid, smem;
    void *tk[2];                  /* timing events around the tile kernel */
};

ATKDSP_API void atkdsp_gpu_batch_destroy(atkdsp_gpu_batch *b) {
    if (!b) return;
    atkb_set_device(b->dev);
    if (b->stream) atkb_stream_sync(b->stream);
    for (int i = 0; i < 2; ++i) {
        atkb_graph_destroy(b->graph[i]);
        atkb_event_destroy(b->ev[i]);
        atkb_event_destroy(b->tk[i]);
        atkb_host_free(b->h_tables[i]);
    }
    atkb_free(b->d_tables);
    atkb_free(b->d_counters);
    atkb_stream_destroy(b->stream);
    free(b->h);
    free(b);
}

ATKDSP_API atkdsp_gpu_batch *atkdsp_gpu_batch_create(atkdsp_pfb *const *handles, unsigned count,
                                                     int use_graph) {
    if (!handles || count < 1) return NULL;
    unsigned i;
    for (i = 0; i < count; ++i)
        if (!handles[i] || handles[i]->dev != handles[0]->dev || handles[i]->bank.plan.big) return NULL;
    atkdsp_gpu_batch *b = (atkdsp_gpu_batch *)calloc(1, sizeof *b);
    if (!b) return NULL;
    b->count = count;
    b->dev = handles[0]->dev;
    b->use_graph = use_graph;
    b->h = (atkdsp_pfb **)malloc(count * sizeof *b->h);
    if (!b->h) { free(b); return NULL; }
    for (i = 0; i < count; ++i) {
        b->h[i] = handles[i];
        if (handles[i]->bank.smem_bytes > b->smem) b->smem = handles[i]->bank.smem_bytes;
    }
    atkb_set_device(b->dev);
    b->tbl_bytes = tables_bytes(count);
    int rc = atkb_stream_create(&b->stream);
    if (rc == ATKB_OK) rc = atkb_malloc(&b->d_tables, b->tbl_bytes);
    for (i = 0; i < 2 && rc == ATKB_OK; ++i) {
        rc = atkb_host_alloc(&b->h_tables[i], b->tbl_bytes);
        if (rc == ATKB_OK) rc = atkb_event_create(&b->ev[i]);
        if (rc == ATKB_OK) rc = atkb_event_create_timed(&b->tk[i]);
    }
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&b->d_counters, ATKB_NCOUNTERS * sizeof(int));
    if (rc == ATKB_OK) rc = atkb_memset(b->d_counters, 0, ATKB_NCOUNTERS * sizeof(int), b->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(b->stream);
    if (rc != ATKB_OK) { atkdsp_gpu_batch_destroy(b); return NULL; }
    b->grid = atkb_pfb_grid(b->dev, b->smem);
    return b;
}

ATKDSP_API void *atkdsp_gpu_batch_stream(atkdsp_gpu_batch *b) { return b ? b->stream : NULL; }

/* the fault bits of the batch's launches since the last query (cleared) */
ATKDSP_API int atkdsp_gpu_batch_faults(atkdsp_gpu_batch *b) {
    unsigned v = 0;
    const unsigned z = 0;
    if (!b) return ATKDSP_E_ARG;
    if (atkb_set_device(b->dev) != ATKB_OK || atkb_stream_sync(b->stream) != ATKB_OK) return ATKDSP_E_FFT;
    if (atkb_d2h(&v, b->d_counters + ATKB_FAULT_WORD, sizeof v, b->stream) != ATKB_OK ||
        atkb_stream_sync(b->stream) != ATKB_OK)
        return ATKDSP_E_FFT;
    if (v && (atkb_h2d(b->d_counters + ATKB_FAULT_WORD, &z, sizeof z, b->stream) != ATKB_OK ||
              atkb_stream_sync(b->stream) != ATKB_OK))
        return ATKDSP_E_FFT;
    return (int)(v | atkb_pfb_debug_fault());
}

ATKDSP_API float atkdsp_gpu_batch_kernel_ms(atkdsp_gpu_batch *b) {
    float ms = -1.0f;
    if (!b) return -1.0f;
    atkb_set_device(b->dev);
    if (atkb_event_elapsed_ms(&ms, b->tk[0], b->tk[1]) != ATKB_OK) return -1.0f;
    return ms;
}

static int batch_enqueue(atkdsp_gpu_batch *b, int slot, void *stream) {
    int rc = atkb_h2d(b->d_tables, b->h_tables[slot], b->tbl_bytes, stream);
    if (rc == ATKB_OK) rc = atkb_event_record_node(b->tk[0], stream);
    if (rc == ATKB_OK)
        rc = atkb_pfb_launch(tbl_jobs(b->d_tables), tbl_tiles(b->d_tables, b->count),
                             tbl_carry(b->d_tables, b->count), (int)b->count, b->d_counters, b->grid,
                             b->smem, stream);
    if (rc == ATKB_OK) rc = atkb_event_record_node(b->tk[1], stream);
    return rc;
}

static ptrdiff_t batch_process(atkdsp_gpu_batch *b, const void *const *d_ins, const size_t *ns,
                               atkdsp_cf32 *const *d_outs, ptrdiff_t *ms, void *stream, int fmt,
                               const float *offs) {
    if (!b || !d_ins || !ns || !d_outs) return ATKDSP_E_ARG;
    if (atkb_set_device(b->dev) != ATKB_OK) return ATKDSP_E_FFT;
    void *st = stream ? stream : b->stream;
    const int slot = b->slot;
    int rc;
    unsigned i;
    if (b->ev_live[slot] && atkb_event_sync(b->ev[slot]) != ATKB_OK) return ATKDSP_E_FFT;
    for (i = 0; i < b->count; ++i) {     /* a handle's pending small-call samples land first */
        atkdsp_pfb *h = b->h[i];
        if (h->npend && atkb_pfb_flush_pending(h) != ATKB_OK) return ATKDSP_E_FFT;
        if (h->small_live) {
            if (atkb_event_sync(h->small_ev) != ATKB_OK) return ATKDSP_E_FFT;
            h->small_live = 0;
        }
    }
    atkb_job *J = tbl_jobs(b->h_tables[slot]);
    atkb_carry *C = tbl_carry(b->h_tables[slot], b->count);
    int *T = tbl_tiles(b->h_tables[slot], b->count);
    long long total = 0, tiles = 0;
    for (i = 0; i < b->count; ++i) {
        atkdsp_pfb *p = b->h[i];
        const size_t n = ns[i];
        const size_t head = p->ov + p->lc;
        const size_t m = ((size_t)p->lc + n) / p->hop;
        if (n && !d_ins[i]) return ATKDSP_E_ARG;
        if (m && !d_outs[i]) return ATKDSP_E_ARG;
        conv_t cv = CONV_CF32;
        if (fmt >= 0) {
            if (!raw_conv(fmt, offs ? offs[2 * i] : 0.0f, offs ? offs[2 * i + 1] : 0.0f, &cv)) return ATKDSP_E_ARG;
            if (n && ((size_t)d_ins[i] & 3)) return ATKDSP_E_ARG;
        }
        const long long t = (long long)((m + (size_t)p->bank.tile_hops - 1) / (size_t)p->bank.tile_hops);
        memset(&J[i], 0, sizeof J[i]);
        J[i].state = state_buf(p, p->cur, 0);
        J[i].in = d_ins[i];
        J[i].out = d_outs[i];
        J[i].cal = p->cal_nel ? p->d_cal : NULL;
        J[i].head = (long long)head;
        J[i].ldo = (long long)m;
        J[i].b0 = (long long)p->b;
        J[i].hops = (long long)m;
        J[i].bank = (const atkb_bank *)p->d_bank;
        J[i].tiles = (int)t;
        T[i] = (int)tiles;
        tiles += t;
        C[i].state = J[i].state;
        C[i].in = d_ins[i];
        C[i].dst = state_buf(p, p->cur ^ 1, 0);
        C[i].head = (long long)head;
        C[i].from = (long long)(m * p->hop);
        C[i].len = (long long)(head + n - m * p->hop);
        J[i].nsrc = C[i].nsrc = (long long)(head + n);
        C[i].cap = (long long)p->cap_state;
        job_conv(&J[i], &C[i], &cv);
        total += (long long)m;
        if (tiles > 0x3fffffff) return ATKDSP_E_ARG;
    }
    T[b->count] = (int)tiles;
    if (b->use_graph && st == b->stream) {
        if (!b->graph[slot]) {
            rc = atkb_graph_begin(st);
            if (rc == ATKB_OK) {
                rc = batch_enqueue(b, slot, st);
                void *g = NULL;
                const int rc2 = atkb_graph_end(st, &g);
                if (rc == ATKB_OK) rc = rc2;
                b->graph[slot] = g;
            }
            if (rc != ATKB_OK) return map_rc(rc);
        }
        rc = atkb_graph_launch(b->graph[slot], st);
    } else {
        rc = batch_enqueue(b, slot, st);
    }
    if (rc == ATKB_OK) rc = atkb_event_record(b->ev[slot], st);
    if (rc != ATKB_OK) return map_rc(rc);
    b->ev_live[slot] = 1;
    b->slot ^= 1;
    for (i = 0; i < b->count; ++i) {
        atkdsp_pfb *p = b->h[i];
        const size_t n = ns[i];
        const size_t m = ((size_t)p->lc + n) / p->hop;
        if (ms) ms[i] = (ptrdiff_t)m;
        p->cur ^= 1;
        p->lc = (unsigned)(p->lc + n - m * p->hop);
        p->b += (int64_t)m;
    }
    return (ptrdiff_t)total;
}

ATKDSP_API ptrdiff_t atkdsp_gpu_batch_process(atkdsp_gpu_batch *b, const atkdsp_cf32 *const *d_ins,
                                              const size_t *ns, atkdsp_cf32 *const *d_outs,
                                              ptrdiff_t *ms, void *stream) {
    return batch_process(b, (const void *const *)d_ins, ns, d_outs, ms, stream, -1, NULL);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_batch_process_raw(atkdsp_gpu_batch *b, const void *const *d_raws,
                                                  const size_t *ns, int fmt, const float *offs,
                                                  atkdsp_cf32 *const *d_outs, ptrdiff_t *ms,
                                                  void *stream) {
    if (fmt != ATKDSP_FMT_CI16 && fmt != ATKDSP_FMT_CI16Q11) return ATKDSP_E_ARG;
    return batch_process(b, d_raws, ns, d_outs, ms, stream, fmt, offs);
}
