/* Host-layer internals shared by atkdsp_host.c and serve.c. Not public. */
#ifndef ATKB_HOST_INTERNAL_H
#define ATKB_HOST_INTERNAL_H

#include "atkdsp.h"
#include "atkdsp_gpu.h"
#include "internal.h"

/* dynamic shared memory of the largest power-of-two (fast path) tile: the
 * 4096-point double FFT tile plus, at nchan 4096, one hop's 4096 outputs. A
 * launch that may meet any fast-path bank (the server's captured rounds)
 * reserves this much. */
#define ATKB_FAST_SMEM_MAX (4096 * 16 + 4096 * 8)

/* a server stream's handle: lean, its state from `pool` on `stream`
 * (stream-ordered, cleared there), no cal table, no synchronisation */
atkdsp_pfb *atkb_pfb_create_served(double fs, unsigned nchan, unsigned oversample, unsigned taps_per_poly,
                                   double atten_db, void *pool, void *stream);

/* host calls of at most this many samples per element stage through pinned
 * memory owned by the handle */
#define ATKB_SMALL_N ((size_t)1 << 15)
/* small calls of at most this many hops (over all elements) run one CTA per
 * hop; beyond it the tile kernel's throughput wins */
#define ATKB_PER_HOP_MAX 1024
/* ... and write at most this many outputs straight into pinned host memory */
#define ATKB_DIRECT_OUT 2048

/* order `stream` (NULL: the handle's) after the handle's pending small-call
 * copy, if any; the device-pointer and batch paths call it first */
int atkb_pfb_order_after_small(atkdsp_pfb *p, void *stream);
int atkb_pfb_flush_pending(atkdsp_pfb *p);

/* a device bank shared by every handle with the same (device, nchan,
 * oversample, taps, attenuation): taps, tables and the device atkb_bank */
typedef struct bank_entry bank_entry;

struct atkdsp_pfb {
    double fs, atten;
    unsigned nchan, os, K, max_nel, hop;
    size_t L, ov;
    int dev;
    int lean;                     /* no host-path staging or tables (server streams) */
    void *pool_stream;            /* server streams: d_state came from the server's
                                   * pool on this stream and is freed on it */
    void *stream;
    void *tbl_event;              /* the last table upload; gates reuse of h_tables */
    int tbl_event_live;
    bank_entry *be;
    atkb_bank bank;               /* host copy (device pointers inside)       */
    void *d_bank;                 /* the shared device copy                   */
    void *d_state;                /* 2 * max_nel * cap_state cf32            */
    size_t cap_state;
    int cur;
    unsigned lc;
    int64_t b;
    void *d_cal;
    unsigned cal_nel;
    size_t chunk, out_ld;         /* host-path chunk (samples) and its output stride */
    void *d_in_stage, *d_out_stage;
    void *d_tables, *h_tables;    /* jobs | carries | tile_start              */
    /* small host calls (n <= ATKB_SMALL_N): pinned staging for the block and
     * its output; `small_ev` marks the last copy out of h_small_in, which a
     * call that completes no hop leaves in flight (small_live) */
    void *h_small_in, *h_small_out;  /* h_small_in: right after the pinned tables */
    void *dz_small_out;               /* h_small_out's device address, or NULL:
                                       * the per-hop kernel writes there */
    void *d_small_in;                 /* right after the device tables: one copy
                                       * carries a small call's tables and block */
    void *small_ev;
    int small_live;
    /* blocks of small calls that completed no hop wait here, in pinned host
     * memory, instead of costing a copy each: h_pend holds npend (< hop)
     * samples per element for the pend_nel elements of those calls, the tail
     * of the stream past the device state's head. They travel with the next
     * call that produces hops, or are uploaded (atkb_pfb_flush_pending)
     * before any other path reads the state. */
    void *h_pend;
    unsigned npend, pend_nel;
    void *small_done;             /* the end of a small call's work (polled) */
    size_t tbl_bytes;
    int *d_counters;
    int grid;
    double *w2_next;              /* the next step's fused W2 partials (element
                                   * 0), set only inside atkdsp_gpu_pfb_process_w12 */
    void *d_big;                  /* large filterbanks: fold / FFT scratch, two
                                   * double2 buffers of atkb_pfb_big_hops hops */
    const void **dins;            /* max_nel staging input pointers (host array,
                                   * filled per call; allocated at create) */
};

/* How a job's new samples are stored: cf32, or int16 I/Q converted in the
 * kernels' load path with the unpack constants. */
typedef struct {
    int kind;                     /* 0 cf32, 1 int16 pairs */
    float cre, cim, k;
    const double *doff;           /* int16: the offset in device memory, or NULL
                                   * (then cre / cim hold it) */
} conv_t;

extern const conv_t ATKB_CONV_CF32;

atkdsp_pfb *atkb_pfb_create_internal(double fs, unsigned nchan, unsigned oversample,
                                     unsigned taps_per_poly, double atten_db, unsigned max_nel,
                                     int lean);
size_t atkb_align16(size_t v);
size_t atkb_tables_bytes(unsigned n);
atkb_job *atkb_tbl_jobs(void *base);
atkb_carry *atkb_tbl_carry(void *base, unsigned n);
int *atkb_tbl_tiles(void *base, unsigned n);
atkdsp_cf32 *atkb_state_buf(const atkdsp_pfb *p, int which, unsigned e);
int atkb_raw_conv(int fmt, float off_re, float off_im, conv_t *cv);
void atkb_job_conv(atkb_job *J, atkb_carry *C, const conv_t *cv);
int atkb_map_rc(int rc);
/* bytes of device memory a lean single-element stream of these parameters
 * needs beyond its (possibly shared) bank */
size_t atkb_stream_footprint(unsigned nchan, unsigned oversample, unsigned taps_per_poly);

#endif
