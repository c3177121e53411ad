/* The serving loop: continuous batching of many live channelizer streams.
 *
 * Streams open and close at any time; blocks of samples arrive at any time.
 * Each round folds every open stream's oldest pending block into ONE launch
 * of the persistent tile kernel (and one carry launch), whatever mix of
 * nchan / taps / oversample the streams have. Blocks that arrive while a
 * round is on the GPU wait for the next round; the host prepares round k+1
 * (in the second pinned table) while round k runs, so work overlaps on the
 * device. Every stream's filter history stays resident in device memory for
 * its whole life; streams with the same filterbank share one device bank.
 *
 * Admission: a stream is admitted only if its device footprint fits in the
 * device's free memory minus the configured reserve (cudaMemGetInfo);
 * otherwise open returns ATKDSP_E_NOMEM and the denial is counted.
 *
 * Results equal processing each stream alone, bit for bit: the same kernel
 * computes each hop from the same window, only the launch grouping differs.
 *
 * Host code only (C99); the device is driven through the atkb_* shim.
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "host_internal.h"
#include "atkdsp_serve.h"

#define QCAP 64                       /* pending blocks per stream */
#define NROUNDS 4                     /* rounds in flight at most */

typedef struct {
    const void *raw;
    size_t n;
    atkdsp_cf32 *out;
    size_t cap;
    uint64_t tag;
    double t_arrival;
} blk_t;

typedef struct {
    atkdsp_pfb *p;                    /* lean single-element handle */
    int state;                        /* 0 free, 1 open, 2 closing */
    conv_t cv;
    blk_t q[QCAP];
    unsigned qhead, qlen;
    int inflight;
} sstream;

typedef struct {
    void *ev;                     /* the round's end (timed) */
    void *ev0;                    /* the round's start on the stream (timed) */
    int nrec;
    atkdsp_server_done *rec;
} round_t;

struct atkdsp_server {
    int dev;
    unsigned cap;
    size_t reserve;
    int use_graph;
    sstream *st;
    void *stream;
    size_t tbl_bytes;
    void *d_tables;
    void *h_tables[2];
    void *tbl_ev[2];
    int tbl_live[2];
    void *graph[2];
    int slot;
    int *d_counters;
    int grid;
    round_t rounds[NROUNDS];
    int r_head, r_len;
    atkdsp_server_stats stats;
    /* handles of closed streams, kept for the next open with the same filter
     * (nchan, oversample, taps, attenuation): closing and reopening then
     * allocate and free nothing */
    atkdsp_pfb **parked;
    unsigned nparked;
    void *pool;                   /* stream-ordered pool for the streams' state */
    double gpu_ms;                /* device time of the completed rounds */
    uint64_t gpu_rounds;
};

static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* table layout for cap jobs: jobs | carries | tile_start[cap + 1] | njobs */
static int *tbl_count(void *base, unsigned cap) { return atkb_tbl_tiles(base, cap) + cap + 1; }

ATKDSP_API void atkdsp_server_destroy(atkdsp_server *s) {
    unsigned i;
    int r;
    if (!s) return;
    atkb_set_device(s->dev);
    if (s->stream) atkb_stream_sync(s->stream);
    for (i = 0; s->st && i < s->cap; ++i) atkdsp_pfb_destroy(s->st[i].p);
    for (i = 0; i < s->nparked; ++i) atkdsp_pfb_destroy(s->parked[i]);
    free(s->parked);
    if (s->stream) atkb_stream_sync(s->stream);
    atkb_pool_destroy(s->pool);
    for (r = 0; r < NROUNDS; ++r) {
        atkb_event_destroy(s->rounds[r].ev);
        atkb_event_destroy(s->rounds[r].ev0);
        free(s->rounds[r].rec);
    }
    for (r = 0; r < 2; ++r) {
        atkb_graph_destroy(s->graph[r]);
        atkb_event_destroy(s->tbl_ev[r]);
        atkb_host_free(s->h_tables[r]);
    }
    atkb_free(s->d_tables);
    atkb_free(s->d_counters);
    atkb_stream_destroy(s->stream);
    free(s->st);
    free(s);
}

ATKDSP_API atkdsp_server *atkdsp_server_create(unsigned max_streams, size_t hbm_reserve, int use_graph) {
    int r;
    if (max_streams < 1 || max_streams > (1u << 20)) return NULL;
    atkdsp_server *s = (atkdsp_server *)calloc(1, sizeof *s);
    if (!s) return NULL;
    s->cap = max_streams;
    s->reserve = hbm_reserve;
    s->use_graph = use_graph;
    s->st = (sstream *)calloc(max_streams, sizeof *s->st);
    s->parked = (atkdsp_pfb **)calloc(max_streams, sizeof *s->parked);
    int rc = (s->st && s->parked) ? atkb_get_device(&s->dev) : ATKB_E_NOMEM;
    if (rc == ATKB_OK) rc = atkb_set_device(s->dev);
    if (rc == ATKB_OK) rc = atkb_stream_create(&s->stream);
    if (rc == ATKB_OK) rc = atkb_pool_create(s->dev, &s->pool);
    s->tbl_bytes = atkb_tables_bytes(max_streams) + 16;
    if (rc == ATKB_OK) rc = atkb_malloc(&s->d_tables, s->tbl_bytes);
    for (r = 0; r < 2 && rc == ATKB_OK; ++r) {
        rc = atkb_host_alloc(&s->h_tables[r], s->tbl_bytes);
        if (rc == ATKB_OK) rc = atkb_event_create(&s->tbl_ev[r]);
    }
    for (r = 0; r < NROUNDS && rc == ATKB_OK; ++r) {
        rc = atkb_event_create_timed(&s->rounds[r].ev);
        if (rc == ATKB_OK) rc = atkb_event_create_timed(&s->rounds[r].ev0);
        s->rounds[r].rec = (atkdsp_server_done *)malloc(max_streams * sizeof(atkdsp_server_done));
        if (rc == ATKB_OK && !s->rounds[r].rec) rc = ATKB_E_NOMEM;
    }
    if (rc == ATKB_OK) rc = atkb_malloc((void **)&s->d_counters, ATKB_NCOUNTERS * sizeof(int));
    if (rc == ATKB_OK) rc = atkb_memset(s->d_counters, 0, ATKB_NCOUNTERS * sizeof(int), s->stream);
    if (rc == ATKB_OK) rc = atkb_stream_sync(s->stream);
    if (rc != ATKB_OK) { atkdsp_server_destroy(s); return NULL; }
    s->grid = atkb_pfb_grid(s->dev, ATKB_FAST_SMEM_MAX);
    return s;
}

/* a parked handle for this filter, its state cleared on the server's stream
 * (ordered before any round that uses it), or NULL */
static atkdsp_pfb *unpark(atkdsp_server *s, double fs, unsigned nchan, unsigned os, unsigned K, double atten) {
    unsigned k;
    if (atten < 20.0) atten = 20.0;                 /* as create clamps it */
    for (k = 0; k < s->nparked; ++k) {
        atkdsp_pfb *p = s->parked[k];
        if (p->nchan != nchan || p->os != os || p->K != K || p->atten != atten) continue;
        if (atkb_memset(p->d_state, 0, 2 * (size_t)p->max_nel * p->cap_state * sizeof(atkdsp_cf32), s->stream) !=
            ATKB_OK)
            return NULL;
        s->parked[k] = s->parked[--s->nparked];
        p->fs = fs;
        p->lc = 0;
        p->b = 0;
        p->cur = 0;
        return p;
    }
    return NULL;
}

ATKDSP_API int atkdsp_server_open(atkdsp_server *s, double fs, unsigned nchan, unsigned oversample,
                                  unsigned taps_per_poly, double atten_db, int fmt) {
    unsigned i;
    conv_t cv = ATKB_CONV_CF32;
    if (!s) return ATKDSP_E_ARG;
    if (fmt != ATKDSP_FMT_CF32 && !atkb_raw_conv(fmt, 0.0f, 0.0f, &cv)) return ATKDSP_E_ARG;
    for (i = 0; i < s->cap && s->st[i].state != 0; ++i) {}
    if (i == s->cap) { ++s->stats.denied; return ATKDSP_E_CAP; }
    if (nchan < 2 || oversample < 1 || nchan % oversample || taps_per_poly < 2) return ATKDSP_E_ARG;
    /* only power-of-two channel counts up to 4096 fit the server's 64 KB tile */
    if ((nchan & (nchan - 1)) || nchan < 16 || nchan > 4096) return ATKDSP_E_ARG;
    atkb_set_device(s->dev);
    atkdsp_pfb *p = unpark(s, fs, nchan, oversample, taps_per_poly, atten_db);
    if (!p) {
        /* free HBM plus what the pool holds unused must cover the reserve and
         * the stream's footprint */
        size_t fr = 0, tot = 0;
        const size_t need = s->reserve + atkb_stream_footprint(nchan, oversample, taps_per_poly);
        if (atkb_mem_info(&fr, &tot) != ATKB_OK) return ATKDSP_E_FFT;
        fr += atkb_pool_idle_bytes(s->pool);
        if (fr < need && s->nparked) {              /* parked handles of other shapes give way */
            unsigned k;
            for (k = 0; k < s->nparked; ++k) atkdsp_pfb_destroy(s->parked[k]);
            s->nparked = 0;
            if (atkb_mem_info(&fr, &tot) != ATKB_OK) return ATKDSP_E_FFT;
            fr += atkb_pool_idle_bytes(s->pool);
        }
        if (fr < need) {
            ++s->stats.denied;
            return ATKDSP_E_NOMEM;
        }
        p = atkb_pfb_create_served(fs, nchan, oversample, taps_per_poly, atten_db, s->pool, s->stream);
        if (!p) { ++s->stats.denied; return ATKDSP_E_NOMEM; }
    }
    memset(&s->st[i], 0, sizeof s->st[i]);
    s->st[i].p = p;
    s->st[i].state = 1;
    s->st[i].cv = cv;
    ++s->stats.admitted;
    return (int)i;
}

static void stream_free(atkdsp_server *s, unsigned i) {
    s->st[i].state = 0;
    ++s->stats.closed;
}

/* A closed stream's handle is parked at once, rounds in flight or not: every
 * later use of it -- the memset that clears it for a new stream, that
 * stream's rounds, or an asynchronous free -- is queued on the server's
 * stream behind those rounds. */
static void park(atkdsp_server *s, atkdsp_pfb *p) {
    if (!p) return;
    if (s->nparked < s->cap) s->parked[s->nparked++] = p;
    else atkdsp_pfb_destroy(p);
}

ATKDSP_API int atkdsp_server_close(atkdsp_server *s, int id) {
    if (!s || id < 0 || (unsigned)id >= s->cap || s->st[id].state != 1) return ATKDSP_E_ARG;
    s->st[id].state = 2;
    s->st[id].qlen = 0;                      /* blocks not yet launched are dropped */
    park(s, s->st[id].p);
    s->st[id].p = NULL;
    if (!s->st[id].inflight) stream_free(s, (unsigned)id);
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_server_submit(atkdsp_server *s, int id, const void *d_raw, size_t n,
                                    atkdsp_cf32 *d_out, size_t cap, uint64_t tag, double t_arrival) {
    if (!s || id < 0 || (unsigned)id >= s->cap || s->st[id].state != 1) return ATKDSP_E_ARG;
    sstream *t = &s->st[id];
    atkdsp_pfb *p = t->p;
    if (n && !d_raw) return ATKDSP_E_ARG;
    if (n && ((size_t)d_raw & (t->cv.kind ? 3 : 7))) return ATKDSP_E_ARG;
    /* room for the most hops this block can complete, whatever the leftover */
    if ((size_t)p->nchan * ((p->hop - 1 + n) / p->hop) > cap || (cap && !d_out)) return ATKDSP_E_CAP;
    if (t->qlen == QCAP) return ATKDSP_E_CAP;
    blk_t *b = &t->q[(t->qhead + t->qlen) % QCAP];
    b->raw = d_raw;
    b->n = n;
    b->out = d_out;
    b->cap = cap;
    b->tag = tag;
    b->t_arrival = t_arrival > 0.0 ? t_arrival : now_s();
    ++t->qlen;
    return ATKDSP_OK;
}

ATKDSP_API int atkdsp_server_pending(const atkdsp_server *s) {
    unsigned i;
    int c = 0;
    if (!s) return 0;
    for (i = 0; i < s->cap; ++i) c += (int)s->st[i].qlen;
    return c;
}

ATKDSP_API int atkdsp_server_inflight(const atkdsp_server *s) { return s ? s->r_len : 0; }

static int enqueue_round(atkdsp_server *s, int slot) {
    void *st = s->stream;
    int rc = atkb_h2d(s->d_tables, s->h_tables[slot], s->tbl_bytes, st);
    if (rc == ATKB_OK)
        rc = atkb_pfb_launch_n(atkb_tbl_jobs(s->d_tables), atkb_tbl_tiles(s->d_tables, s->cap),
                               atkb_tbl_carry(s->d_tables, s->cap), (int)s->cap, tbl_count(s->d_tables, s->cap),
                               s->d_counters, s->grid, ATKB_FAST_SMEM_MAX, st);
    return rc;
}

ATKDSP_API int atkdsp_server_launch(atkdsp_server *s) {
    unsigned i;
    int n = 0, rc;
    if (!s) return ATKDSP_E_ARG;
    if (s->r_len == NROUNDS) return 0;                     /* too many rounds in flight */
    const int slot = s->slot;
    if (s->tbl_live[slot]) {
        rc = atkb_event_query(s->tbl_ev[slot]);
        if (rc == 1) return 0;                             /* the slot's last upload is pending */
        if (rc != ATKB_OK) return ATKDSP_E_FFT;
    }
    atkb_set_device(s->dev);
    void *base = s->h_tables[slot];
    atkb_job *J = atkb_tbl_jobs(base);
    atkb_carry *C = atkb_tbl_carry(base, s->cap);
    int *T = atkb_tbl_tiles(base, s->cap);
    round_t *R = &s->rounds[(s->r_head + s->r_len) % NROUNDS];
    long long tiles = 0;
    for (i = 0; i < s->cap; ++i) {
        sstream *t = &s->st[i];
        if (t->state != 1 || !t->qlen) continue;
        atkdsp_pfb *p = t->p;
        const blk_t *b = &t->q[t->qhead];
        const size_t head = p->ov + p->lc;
        const size_t m = ((size_t)p->lc + b->n) / p->hop;
        const long long nt = (long long)((m + (size_t)p->bank.tile_hops - 1) / (size_t)p->bank.tile_hops);
        memset(&J[n], 0, sizeof J[n]);
        J[n].state = atkb_state_buf(p, p->cur, 0);
        J[n].in = b->raw;
        J[n].out = b->out;
        J[n].head = (long long)head;
        J[n].ldo = (long long)m;
        J[n].b0 = (long long)p->b;
        J[n].hops = (long long)m;
        J[n].bank = (const atkb_bank *)p->d_bank;
        J[n].tiles = (int)nt;
        T[n] = (int)tiles;
        tiles += nt;
        memset(&C[n], 0, sizeof C[n]);
        C[n].state = J[n].state;
        C[n].in = b->raw;
        C[n].dst = atkb_state_buf(p, p->cur ^ 1, 0);
        C[n].head = (long long)head;
        C[n].from = (long long)(m * p->hop);
        C[n].len = (long long)(head + b->n - m * p->hop);
        J[n].nsrc = C[n].nsrc = (long long)(head + b->n);
        C[n].cap = (long long)p->cap_state;
        atkb_job_conv(&J[n], &C[n], &t->cv);
        R->rec[n].id = (int)i;
        R->rec[n].tag = b->tag;
        R->rec[n].m = (ptrdiff_t)m;
        R->rec[n].n = b->n;
        R->rec[n].t_arrival = b->t_arrival;
        R->rec[n].t_done = 0.0;
        ++n;
    }
    if (n == 0) return 0;
    if (tiles > 0x3fffffff) return ATKDSP_E_ARG;
    T[n] = (int)tiles;
    *tbl_count(base, s->cap) = n;
    rc = atkb_event_record(R->ev0, s->stream);
    if (rc != ATKB_OK) return atkb_map_rc(rc);
    if (s->use_graph) {
        if (!s->graph[slot]) {
            rc = atkb_graph_begin(s->stream);
            if (rc == ATKB_OK) {
                rc = enqueue_round(s, slot);
                void *g = NULL;
                const int rc2 = atkb_graph_end(s->stream, &g);
                if (rc == ATKB_OK) rc = rc2;
                s->graph[slot] = g;
            }
            if (rc != ATKB_OK) return atkb_map_rc(rc);
        }
        rc = atkb_graph_launch(s->graph[slot], s->stream);
    } else {
        rc = enqueue_round(s, slot);
    }
    if (rc == ATKB_OK) rc = atkb_event_record(s->tbl_ev[slot], s->stream);
    if (rc == ATKB_OK) rc = atkb_event_record(R->ev, s->stream);
    if (rc != ATKB_OK) return atkb_map_rc(rc);
    s->tbl_live[slot] = 1;
    s->slot ^= 1;
    R->nrec = n;
    ++s->r_len;
    ++s->stats.rounds;
    /* the launched blocks leave their queues; the host mirrors advance */
    for (i = 0; i < s->cap; ++i) {
        sstream *t = &s->st[i];
        if (t->state != 1 || !t->qlen) continue;
        atkdsp_pfb *p = t->p;
        const blk_t *b = &t->q[t->qhead];
        const size_t m = ((size_t)p->lc + b->n) / p->hop;
        p->cur ^= 1;
        p->lc = (unsigned)(p->lc + b->n - m * p->hop);
        p->b += (int64_t)m;
        t->qhead = (t->qhead + 1) % QCAP;
        --t->qlen;
        ++t->inflight;
        s->stats.blocks_launched += 1;
        s->stats.samples_launched += (uint64_t)b->n;
    }
    return n;
}

ATKDSP_API int atkdsp_server_poll(atkdsp_server *s, atkdsp_server_done *done, int cap, int wait) {
    int got = 0;
    if (!s || (cap > 0 && !done)) return ATKDSP_E_ARG;
    while (s->r_len > 0) {
        round_t *R = &s->rounds[s->r_head];
        if (R->nrec > cap - got) break;                    /* no room for the whole round */
        int rc = wait ? atkb_event_sync(R->ev) : atkb_event_query(R->ev);
        if (rc == 1) break;
        if (rc != ATKB_OK) return ATKDSP_E_FFT;
        const double t = now_s();
        for (int k = 0; k < R->nrec; ++k) {
            atkdsp_server_done *d = &done[got++];
            *d = R->rec[k];
            d->t_done = t;
            sstream *st = &s->st[d->id];
            if (--st->inflight == 0 && st->state == 2) stream_free(s, (unsigned)d->id);
        }
        s->stats.blocks_done += (uint64_t)R->nrec;
        {
            float ms = 0.0f;
            if (atkb_event_elapsed_ms(&ms, R->ev0, R->ev) == ATKB_OK) {
                s->gpu_ms += ms;
                ++s->gpu_rounds;
            }
        }
        s->r_head = (s->r_head + 1) % NROUNDS;
        --s->r_len;
        wait = 0;
    }
    return got;
}

ATKDSP_API void atkdsp_server_get_stats(const atkdsp_server *s, atkdsp_server_stats *out) {
    if (s && out) *out = s->stats;
}

ATKDSP_API double atkdsp_server_now(void) { return now_s(); }

/* ===================================================== synthetic load driver
 * Open-loop load for the serving configuration: streams at rates drawn from
 * cfg->rates, each delivering blocks of block_s seconds of samples with
 * exponential inter-arrival times (mean block_s: Poisson arrivals at the
 * stream's own rate), nchan drawn from cfg->nchans, churn (one close + one
 * open) at a Poisson rate, for cfg->duration_s seconds. Block samples come
 * from a device pool the caller fills (the host link cannot carry this load);
 * outputs go to per-stream regions of a caller-provided device pool. Latency
 * = completion seen by the host - the block's arrival time. */
typedef struct {
    double t;
    int id;
} arrival_t;

static void heap_push(arrival_t *h, int *n, arrival_t v) {
    int i = (*n)++;
    while (i > 0) {
        int p = (i - 1) / 2;
        if (h[p].t <= v.t) break;
        h[i] = h[p];
        i = p;
    }
    h[i] = v;
}

static arrival_t heap_pop(arrival_t *h, int *n) {
    arrival_t top = h[0], v = h[--(*n)];
    int i = 0;
    for (;;) {
        int c = 2 * i + 1;
        if (c >= *n) break;
        if (c + 1 < *n && h[c + 1].t < h[c].t) ++c;
        if (v.t <= h[c].t) break;
        h[i] = h[c];
        i = c;
    }
    if (*n > 0) h[i] = v;
    return top;
}

static uint64_t rng_next(uint64_t *x) {       /* splitmix64 */
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static double rng_unit(uint64_t *x) { return ((double)(rng_next(x) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
static double rng_exp(uint64_t *x, double mean) { return -mean * log(rng_unit(x)); }

static int cmp_double(const void *a, const void *b) {
    const double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : x > y;
}

ATKDSP_API int atkdsp_server_simulate(atkdsp_server *s, const atkdsp_sim_config *cfg,
                                      atkdsp_sim_result *res) {
    if (!s || !cfg || !res || cfg->streams < 1 || cfg->nrates < 1 || cfg->nnchan < 1 || !cfg->d_raw_pool ||
        !cfg->d_out_pool || cfg->block_s <= 0.0 || cfg->oversample < 1)
        return ATKDSP_E_ARG;
    memset(res, 0, sizeof *res);
    const unsigned ns = cfg->streams;
    uint64_t seed = cfg->seed ? cfg->seed : 12345;
    const size_t bps = cfg->fmt == ATKDSP_FMT_CF32 ? 8 : 4;
    const size_t pool_samples = cfg->raw_pool_bytes / bps;
    double *rate = (double *)malloc(ns * sizeof(double));
    unsigned *nch = (unsigned *)malloc(ns * sizeof(unsigned));
    size_t *blk = (size_t *)malloc(ns * sizeof(size_t));
    int *sid = (int *)malloc(ns * sizeof(int));
    size_t *ooff = (size_t *)malloc(ns * sizeof(size_t));
    size_t *ocap = (size_t *)malloc(ns * sizeof(size_t));
    arrival_t *heap = (arrival_t *)malloc((ns + 1) * sizeof(arrival_t));
    const size_t lat_cap = (size_t)1 << 22;
    double *lat = (double *)malloc(lat_cap * sizeof(double));
    const int dcap = (int)(s->cap * NROUNDS);
    atkdsp_server_done *done = (atkdsp_server_done *)malloc((size_t)dcap * sizeof(atkdsp_server_done));
    int rc = ATKDSP_OK;
    size_t nlat = 0, out_used = 0;
    unsigned i;
    double launch_ms = 0.0;
    uint64_t launches = 0;
    s->gpu_ms = 0.0;
    s->gpu_rounds = 0;
    if (!rate || !nch || !blk || !sid || !ooff || !ocap || !heap || !lat || !done) { rc = ATKDSP_E_NOMEM; goto out; }
    for (i = 0; i < ns; ++i) {
        rate[i] = cfg->rates[rng_next(&seed) % (uint64_t)cfg->nrates];
        nch[i] = cfg->nchans[rng_next(&seed) % (uint64_t)cfg->nnchan];
        blk[i] = (size_t)llround(rate[i] * cfg->block_s);
        if (blk[i] < 1 || blk[i] + 2 > pool_samples) { rc = ATKDSP_E_ARG; goto out; }
        const size_t hop = nch[i] / cfg->oversample;
        ocap[i] = (size_t)nch[i] * ((hop - 1 + blk[i]) / hop);
        ooff[i] = out_used;
        out_used += (ocap[i] + 1) & ~(size_t)1;
        res->offered_samples_per_s += rate[i];
    }
    if (out_used * sizeof(atkdsp_cf32) > cfg->out_pool_bytes) { rc = ATKDSP_E_CAP; goto out; }
    for (i = 0; i < ns; ++i) {
        sid[i] = atkdsp_server_open(s, rate[i], nch[i], cfg->oversample, cfg->taps, cfg->atten_db, cfg->fmt);
        if (sid[i] < 0) ++res->denied;
        else ++res->admitted;
    }
    {
        int hn = 0;
        const double t0 = now_s();
        for (i = 0; i < ns; ++i) {
            arrival_t a = {t0 + rng_exp(&seed, cfg->block_s), (int)i};
            heap_push(heap, &hn, a);
        }
        double next_churn = cfg->churn_per_s > 0 ? t0 + rng_exp(&seed, 1.0 / cfg->churn_per_s) : 1e300;
        const double t_end = t0 + cfg->duration_s;
        const double t_warm = t0 + cfg->warmup_s;
        double t_prev = 0.0;
        for (;;) {
            const double t = now_s();
            if (t >= t_end && s->r_len == 0) break;
            if (t < t_end) {
                while (hn > 0 && heap[0].t <= t) {
                    arrival_t a = heap_pop(heap, &hn);
                    const int id = sid[a.id];
                    if (id >= 0) {
                        /* a block of the stream's size from a random place in the pool */
                        const size_t roff = (rng_next(&seed) % (uint64_t)(pool_samples - blk[a.id] - 1)) & ~(size_t)1;
                        const char *raw = (const char *)cfg->d_raw_pool + roff * bps;
                        const int r2 = atkdsp_server_submit(s, id, raw, blk[a.id],
                                                            (atkdsp_cf32 *)cfg->d_out_pool + ooff[a.id], ocap[a.id],
                                                            (uint64_t)a.id, a.t);
                        if (r2 == ATKDSP_OK) res->offered_blocks += 1;
                        else res->dropped_blocks += 1;
                    }
                    a.t += rng_exp(&seed, cfg->block_s);
                    heap_push(heap, &hn, a);
                }
                if (t >= next_churn) {
                    /* one stream leaves and a new one asks to join */
                    const unsigned k = (unsigned)(rng_next(&seed) % ns);
                    double c0 = now_s();
                    if (sid[k] >= 0) atkdsp_server_close(s, sid[k]);
                    double c1 = now_s();
                    sid[k] = atkdsp_server_open(s, rate[k], nch[k], cfg->oversample, cfg->taps, cfg->atten_db,
                                                cfg->fmt);
                    const double c2 = now_s();
                    if ((c1 - c0) * 1e3 > res->max_close_ms) res->max_close_ms = (c1 - c0) * 1e3;
                    if ((c2 - c1) * 1e3 > res->max_open_ms) res->max_open_ms = (c2 - c1) * 1e3;
                    if (sid[k] < 0) ++res->denied;
                    else ++res->admitted;
                    res->churn_events += 1;
                    next_churn += rng_exp(&seed, 1.0 / cfg->churn_per_s);
                }
            }
            /* continuous batching: a new round whenever fewer than two are on the GPU */
            if (s->r_len < 2) {
                const double l0 = now_s();
                const int got = atkdsp_server_launch(s);
                if (got < 0) { rc = got; goto out; }
                const double dl = (now_s() - l0) * 1e3;
                if (dl > res->max_launch_ms) res->max_launch_ms = dl;
                if (got > 0) {
                    launch_ms += dl;
                    ++launches;
                }
            }
            const double p0 = now_s();
            const int nd = atkdsp_server_poll(s, done, dcap, 0);
            if (nd < 0) { rc = nd; goto out; }
            {
                const double p1 = now_s();
                if ((p1 - p0) * 1e3 > res->max_poll_ms) res->max_poll_ms = (p1 - p0) * 1e3;
                if (t_prev > 0.0 && (p1 - t_prev) * 1e3 > res->max_loop_ms) res->max_loop_ms = (p1 - t_prev) * 1e3;
                t_prev = p1;
            }
            for (int k2 = 0; k2 < nd; ++k2) {
                if (done[k2].t_arrival < t_warm) continue;       /* warm-up blocks not counted */
                res->samples_done += (uint64_t)done[k2].n;
                res->blocks_done += 1;
                if (nlat < lat_cap) lat[nlat++] = (done[k2].t_done - done[k2].t_arrival) * 1e3;
            }
        }
        res->wall_s = now_s() - t_warm;
    }
    if (nlat) {
        qsort(lat, nlat, sizeof(double), cmp_double);
        res->lat_p50_ms = lat[nlat / 2];
        res->lat_p90_ms = lat[(size_t)(0.90 * (double)(nlat - 1))];
        res->lat_p99_ms = lat[(size_t)(0.99 * (double)(nlat - 1))];
        res->lat_max_ms = lat[nlat - 1];
    }
    {
        atkdsp_server_stats st;
        atkdsp_server_get_stats(s, &st);
        res->rounds = st.rounds;
        res->blocks_per_round = st.rounds ? (double)st.blocks_launched / (double)st.rounds : 0.0;
        res->mean_launch_ms = launches ? launch_ms / (double)launches : 0.0;
        res->mean_round_gpu_ms = s->gpu_rounds ? s->gpu_ms / (double)s->gpu_rounds : 0.0;
        res->gpu_busy = res->wall_s > 0 ? s->gpu_ms / 1e3 / (res->wall_s + cfg->warmup_s) : 0.0;
    }
    for (i = 0; i < ns; ++i)
        if (sid[i] >= 0) atkdsp_server_close(s, sid[i]);
    while (s->r_len > 0 && atkdsp_server_poll(s, done, dcap, 1) >= 0) {}
out:
    free(rate); free(nch); free(blk); free(sid); free(ooff); free(ocap); free(heap); free(lat); free(done);
    return rc;
}
