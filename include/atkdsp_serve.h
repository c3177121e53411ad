/*
 * atkdsp_serve.h -- the channelizer serving loop (no reference counterpart).
 *
 * The reference channelizes one stream per call on the caller's thread
 * (include/atkdsp.h:3209-3220); its in-library caller runs one handle per
 * thread (src/undertow.c:244-257). This server keeps many live streams on
 * one GPU and channelizes whatever blocks are pending, for all of them, in
 * one kernel launch per round (continuous batching). Streams are admitted
 * while their device footprint fits in free HBM minus a reserve. All sample
 * pointers are device pointers. Each stream's output equals processing that
 * stream alone with atkdsp_pfb_process, bit for bit.
 *
 * Single-threaded use: one thread drives a server (open/submit/launch/poll).
 */
#ifndef ATKDSP_SERVE_H
#define ATKDSP_SERVE_H

#include "atkdsp.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct atkdsp_server atkdsp_server;

typedef struct {
    int id;                 /* stream id from atkdsp_server_open */
    uint64_t tag;           /* the caller's tag from atkdsp_server_submit */
    ptrdiff_t m;            /* hops written ([nchan][m] channel-major at d_out) */
    size_t n;               /* input samples of the block */
    double t_arrival;       /* seconds, atkdsp_server_now() clock */
    double t_done;          /* when the host saw the block complete */
} atkdsp_server_done;

typedef struct {
    uint64_t admitted, denied, closed, rounds, blocks_launched, samples_launched, blocks_done;
} atkdsp_server_stats;

/* max_streams: capacity (streams open at once, and jobs in one round);
 * hbm_reserve: device bytes admission keeps free; use_graph: replay each
 * round's launches from a CUDA graph. */
ATKDSP_API atkdsp_server *atkdsp_server_create(unsigned max_streams, size_t hbm_reserve, int use_graph);
ATKDSP_API void          atkdsp_server_destroy(atkdsp_server *s);
/* Open a stream (a single-element filterbank as atkdsp_pfb_create, blocks in
 * fmt: ATKDSP_FMT_CF32, ATKDSP_FMT_CI16 or ATKDSP_FMT_CI16Q11, the int16
 * formats converted in the kernel's load path). nchan: power of two, 16..4096.
 * Returns the id, or ATKDSP_E_NOMEM (not admitted: free HBM), ATKDSP_E_CAP (no
 * free slot), ATKDSP_E_ARG. */
ATKDSP_API int           atkdsp_server_open(atkdsp_server *s, double fs, unsigned nchan,
                                            unsigned oversample, unsigned taps_per_poly,
                                            double atten_db, int fmt);
/* Close: queued blocks not yet launched are dropped; launched ones complete. */
ATKDSP_API int           atkdsp_server_close(atkdsp_server *s, int id);
/* Queue one block: n samples at d_raw, output to d_out (cap samples, at least
 * nchan * ((hop - 1 + n) / hop)). t_arrival <= 0 means now. */
ATKDSP_API int           atkdsp_server_submit(atkdsp_server *s, int id, const void *d_raw, size_t n,
                                              atkdsp_cf32 *d_out, size_t cap, uint64_t tag,
                                              double t_arrival);
/* One round: every open stream's oldest pending block, one launch. Returns the
 * number of blocks launched (0 when nothing is pending or the GPU is full). */
ATKDSP_API int           atkdsp_server_launch(atkdsp_server *s);
/* Completed blocks, oldest round first (whole rounds only); wait != 0 blocks
 * until at least the oldest round is done. Returns the count. */
ATKDSP_API int           atkdsp_server_poll(atkdsp_server *s, atkdsp_server_done *done, int cap, int wait);
ATKDSP_API int           atkdsp_server_pending(const atkdsp_server *s);
ATKDSP_API int           atkdsp_server_inflight(const atkdsp_server *s);
ATKDSP_API void          atkdsp_server_get_stats(const atkdsp_server *s, atkdsp_server_stats *out);
ATKDSP_API double        atkdsp_server_now(void);

/* ---- synthetic open-loop load (the serving benchmark) ----------------- */
typedef struct {
    unsigned streams;             /* live streams */
    const double *rates;          /* sample rates to draw from */
    unsigned nrates;
    const unsigned *nchans;       /* channel counts to draw from */
    unsigned nnchan;
    unsigned oversample, taps;
    double atten_db;
    int fmt;                      /* block sample format */
    double block_s;               /* seconds of samples per block; mean inter-arrival */
    double churn_per_s;           /* close + open events per second (Poisson) */
    double duration_s, warmup_s;  /* run time; blocks arriving in the warm-up are not counted */
    const void *d_raw_pool;       /* device samples blocks are taken from */
    size_t raw_pool_bytes;
    atkdsp_cf32 *d_out_pool;      /* device space for every stream's output region */
    size_t out_pool_bytes;
    uint64_t seed;
} atkdsp_sim_config;

typedef struct {
    double offered_samples_per_s;
    uint64_t offered_blocks, dropped_blocks, blocks_done, samples_done, churn_events, admitted, denied,
        rounds;
    double blocks_per_round, wall_s;
    double lat_p50_ms, lat_p90_ms, lat_p99_ms, lat_max_ms;
    /* the longest single host call of each kind during the run, and the
     * longest pass of the driver loop (where a stall on the host shows) */
    double max_open_ms, max_close_ms, max_launch_ms, max_poll_ms, max_loop_ms;
    /* where a round's time goes: the host's launch call (tables for every
     * pending block, graph replay) and the round's device time (its events on
     * the server's stream, table upload + tile kernel + carries), both
     * averaged over rounds; gpu_busy: device time / run time */
    double mean_launch_ms, mean_round_gpu_ms, gpu_busy;
} atkdsp_sim_result;

ATKDSP_API int           atkdsp_server_simulate(atkdsp_server *s, const atkdsp_sim_config *cfg,
                                                atkdsp_sim_result *res);

#ifdef __cplusplus
}
#endif
#endif
