/*
 * atkdsp.h -- the channelizer slice of atkdsp's C ABI, implemented on B200.
 *
 * This header declares exactly the entry points of the reference's ABI
 * (include/atkdsp.h of atkdsp 0.25.1, ABI 26) that the polyphase-filterbank
 * path uses: identity, threads, the unpack front end, the atkdsp_pfb_* handle
 * API and the W1/W2 accumulators, the channelizer's other tool, the
 * overlap-save extractor (atkdsp_osx_*), and the CFAR detector and burst
 * tracker that gates W1 on W2's powers (atkdsp_cfar_*). Names, types, argument meaning, return
 * codes and the channel-major output layout are the reference's, so a caller
 * of the reference (its ctypes binding, a C program, the in-library survey)
 * links against this library unchanged for this path. Each declaration cites
 * the reference declaration it replaces.
 *
 * What is different underneath: every *_process / *_unpack call runs on the
 * GPU (CUDA, sm_100a). Sample buffers are still the caller's host memory and
 * calls are synchronous on return, as the reference's are. Each handle keeps
 * its streaming state (FIR history, leftover samples, hop counter) in device
 * memory, and owns one CUDA stream and the device buffers it needs, all
 * allocated by *_create; a process call allocates nothing. Device-pointer
 * entry points for callers that keep samples on the GPU are in atkdsp_gpu.h.
 *
 * Threading: one handle is used by one thread at a time; different handles
 * may be used concurrently from different threads (each has its own stream).
 */
#ifndef ATKDSP_H
#define ATKDSP_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32) || defined(__CYGWIN__)
#  define ATKDSP_API __declspec(dllexport)
#else
#  define ATKDSP_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* reference include/atkdsp.h:63-64 */
#define ATKDSP_ABI_VERSION 26
#define ATKDSP_VERSION_STRING "0.25.1"

/* reference include/atkdsp.h:203-207 */
#define ATKDSP_OK            0
#define ATKDSP_E_ARG        -1   /* null pointer, bad size, unknown enum          */
#define ATKDSP_E_NOMEM      -2   /* allocation failed (host or device)            */
#define ATKDSP_E_CAP        -3   /* caller's output buffer too small              */
#define ATKDSP_E_FFT        -4   /* the transform failed: a GPU launch or kernel error */
/* reference include/atkdsp.h:210 */
#define ATKDSP_E_EMPTY      -7   /* nothing there to return (atkdsp_cfar_last)    */

/* reference include/atkdsp.h:213 -- complex float32, numpy complex64 layout */
typedef struct { float re, im; } atkdsp_cf32;

/* reference include/atkdsp.h:216-222 */
enum atkdsp_format {
    ATKDSP_FMT_CU8     = 0,
    ATKDSP_FMT_CI8     = 1,
    ATKDSP_FMT_CI16    = 2,
    ATKDSP_FMT_CI16Q11 = 3,
    ATKDSP_FMT_CF32    = 4
};

/* ---- identity: reference include/atkdsp.h:237-244 ----------------------- */
ATKDSP_API int         atkdsp_abi_version(void);        /* 26 */
ATKDSP_API const char *atkdsp_version_string(void);     /* "0.25.1" */
ATKDSP_API const char *atkdsp_build_info(void);         /* contains "abi 26" */
ATKDSP_API int         atkdsp_bytes_per_sample(int fmt);
/* Accepted for compatibility; the GPU path has no host worker threads, so the
 * count changes nothing but what atkdsp_get_threads reports. */
ATKDSP_API int         atkdsp_set_threads(int n);
ATKDSP_API int         atkdsp_get_threads(void);

/* ---- unpack: reference include/atkdsp.h:247-273 ------------------------- */
ATKDSP_API ptrdiff_t atkdsp_unpack(const void *raw, size_t nbytes, int fmt,
                                   atkdsp_cf32 *out, size_t out_cap,
                                   float dc_alpha, atkdsp_cf32 *dc_state);
ATKDSP_API ptrdiff_t atkdsp_unpack_dc(const void *raw, size_t nbytes, int fmt,
                                      atkdsp_cf32 *out, size_t out_cap,
                                      float off_re, float off_im,
                                      double *mean_re, double *mean_im);

/* ---- the polyphase filterbank: reference include/atkdsp.h:3185-3229 ----- */
typedef struct atkdsp_pfb atkdsp_pfb;
/* reference include/atkdsp.h:3191-3193. NULL on bad arguments (fs <= 0,
 * nchan < 2, nchan % oversample, taps_per_poly < 2, max_nel < 1), when no GPU
 * is usable, or when device memory runs out. Any nchan is accepted: a power of
 * two up to 4096 or any other value up to 6400 runs through the tile kernel,
 * a larger one through the large-filterbank kernels. */
ATKDSP_API atkdsp_pfb *atkdsp_pfb_create(double fs, unsigned nchan, unsigned oversample,
                                         unsigned taps_per_poly, double atten_db,
                                         unsigned max_nel);
ATKDSP_API void        atkdsp_pfb_destroy(atkdsp_pfb *p);                  /* :3194 */
ATKDSP_API void        atkdsp_pfb_reset(atkdsp_pfb *p);                    /* :3195 */
ATKDSP_API unsigned    atkdsp_pfb_nchan(const atkdsp_pfb *p);              /* :3196 */
ATKDSP_API double      atkdsp_pfb_out_rate(const atkdsp_pfb *p);           /* :3197 */
ATKDSP_API size_t      atkdsp_pfb_out_hops(const atkdsp_pfb *p, size_t n); /* :3200 */
/* reference include/atkdsp.h:3209-3210: out is [nchan][m], channel-major */
ATKDSP_API ptrdiff_t   atkdsp_pfb_process(atkdsp_pfb *p, const atkdsp_cf32 *in, size_t n,
                                          atkdsp_cf32 *out, size_t cap);
/* reference include/atkdsp.h:3218-3220: out is [nel][nchan][m] */
ATKDSP_API ptrdiff_t   atkdsp_pfb_process_n(atkdsp_pfb *p, const atkdsp_cf32 *const *ins,
                                            unsigned nel, size_t n,
                                            atkdsp_cf32 *out, size_t cap);
ATKDSP_API int64_t     atkdsp_pfb_block_origin(const atkdsp_pfb *p, int64_t hop_index); /* :3223 */
ATKDSP_API double      atkdsp_pfb_group_delay(const atkdsp_pfb *p);                      /* :3224 */
ATKDSP_API int         atkdsp_pfb_set_cal(atkdsp_pfb *p, const atkdsp_cf32 *table,
                                          unsigned nel);                                 /* :3228 */
ATKDSP_API int         atkdsp_pfb_describe(const atkdsp_pfb *p, char *buf, size_t cap);  /* :3229 */

/* ---- W1 / W2: reference include/atkdsp.h:3239-3251 ---------------------- */
ATKDSP_API void        atkdsp_pfb_cov_accumulate(const atkdsp_cf32 *out, unsigned nel,
                                                 unsigned nchan, size_t m,
                                                 const uint8_t *gate,
                                                 atkdsp_cf32 *R, uint32_t *counts);
ATKDSP_API void        atkdsp_pfb_cov_reset(atkdsp_cf32 *R, uint32_t *counts, unsigned nel,
                                            unsigned nchan, const uint8_t *gate);
ATKDSP_API void        atkdsp_pfb_channel_power(const atkdsp_cf32 *out, unsigned nel,
                                                unsigned nchan, size_t m,
                                                float *pwr, float *mean_pwr);

/* ---- overlap-save extractor: reference include/atkdsp.h:3252-3289 --------
 * One forward FFT of nfft points per block of hop = nfft/2 new samples; each
 * channel folds it to M = nfft/decim bins, inverts them (the integer
 * decimation), rolls to absolute time and is landed on its out_rate by the
 * arbitrary resampler. nfft <= 2^24 in this build (create returns NULL
 * beyond). Capacity and missing output buffers are checked before any state
 * changes (the reference finds them part-way through a call). */
typedef struct atkdsp_osx atkdsp_osx;
ATKDSP_API atkdsp_osx *atkdsp_osx_create(double fs, size_t nfft, double atten_db,
                                         unsigned max_nel);                               /* :3257 */
ATKDSP_API void        atkdsp_osx_destroy(atkdsp_osx *x);                                 /* :3259 */
ATKDSP_API void        atkdsp_osx_reset(atkdsp_osx *x);                                   /* :3260 */
ATKDSP_API int         atkdsp_osx_add(atkdsp_osx *x, double offset_hz, double bw_hz,
                                      double out_rate);                                   /* :3264 */
ATKDSP_API int         atkdsp_osx_retune(atkdsp_osx *x, int ch, double offset_hz);        /* :3265 */
ATKDSP_API int         atkdsp_osx_remove(atkdsp_osx *x, int ch);                          /* :3266 */
ATKDSP_API int         atkdsp_osx_channels(const atkdsp_osx *x);                          /* :3267 */
ATKDSP_API double      atkdsp_osx_chan_rate(const atkdsp_osx *x, int ch);                 /* :3268 */
ATKDSP_API size_t      atkdsp_osx_out_max(const atkdsp_osx *x, int ch, size_t n);         /* :3271 */
ATKDSP_API ptrdiff_t   atkdsp_osx_process(atkdsp_osx *x, const atkdsp_cf32 *in, size_t n,
                                          atkdsp_cf32 *const *outs, size_t *out_counts,
                                          size_t cap_each);                               /* :3280 */
ATKDSP_API ptrdiff_t   atkdsp_osx_process_n(atkdsp_osx *x, const atkdsp_cf32 *const *ins,
                                            unsigned nel, size_t n,
                                            atkdsp_cf32 *const *outs, size_t *out_counts,
                                            size_t cap_each);                             /* :3285 */
ATKDSP_API int         atkdsp_osx_describe(const atkdsp_osx *x, char *buf, size_t cap);  /* :3289 */

/* ---- CFAR across frequency and the burst tracker: reference
 * include/atkdsp.h:1821-1924 ------------------------------------------------
 * Each frame (nbins powers in dB) is converted to linear power, averaged over
 * k_frames frames, and every unmasked bin is tested against alpha x T, T the
 * CA / OS / GO / SO statistic of its 2 n_ref reference cells beyond n_guard
 * guard cells (a side that runs short at an edge or a mask borrows from the
 * other). alpha is solved for the per-cell false-alarm rate. Hit bins merge
 * into blobs, blobs into tracks, tracks report OPEN / UPDATE / CLOSE events.
 * Here the per-cell work of a whole call (conversion, average, statistic,
 * test) runs on the GPU in one pass over all its frames; the tracker walks
 * the hit rows on the host in frame order. The layouts of the three structs
 * are the reference's (96, 64 and 88 bytes as compiled; the reference's
 * own comment on the config says 104). */
#define ATKDSP_CFAR_CA 0
#define ATKDSP_CFAR_OS 1
#define ATKDSP_CFAR_GO 2
#define ATKDSP_CFAR_SO 3
#define ATKDSP_CFAR_OPEN   1
#define ATKDSP_CFAR_UPDATE 2
#define ATKDSP_CFAR_CLOSE  3
#define ATKDSP_CFAR_T0_COARSE 1u
#define ATKDSP_CFAR_T1_COARSE 2u
#define ATKDSP_CFAR_EDGE      4u
#define ATKDSP_CFAR_MASK_ADJ  8u
#define ATKDSP_CFAR_FLUSHED  16u
#define ATKDSP_CFAR_EDGE_PFA 1e-3
#define ATKDSP_CFAR_RHO_MAX  4

typedef struct {                                                                          /* :1836 */
    int32_t mode;        /* ATKDSP_CFAR_CA (default) / OS / GO / SO           */
    int32_t n_ref;       /* reference cells each side, 1..256 (16)            */
    int32_t n_guard;     /* guard cells each side, 0..256 (4)                 */
    int32_t k_frames;    /* frames averaged before testing, 1..64 (1)         */
    double  pfa;         /* per cell per frame, 1e-15..0.5 (1e-6)             */
    double  looks;       /* periodograms averaged into one frame, 0.25..1e4 (1) */
    int32_t os_k;        /* OS rank 1..2 n_ref; 0 = ceil(3N/4)                */
    int32_t open_m;      /* open after open_m hit frames ... (2)              */
    int32_t open_n;      /* ... in the last open_n, 1..64 (3)                 */
    int32_t close_k;     /* close after close_k misses in a row, 1..1000 (3)  */
    int32_t merge_gap;   /* non-hit bins inside one detection (1)             */
    int32_t min_bins;    /* narrower blobs ignored (1)                        */
    int32_t max_tracks;  /* pending + open at once, 1..65536 (256)            */
    int32_t reserved;
    double  rho2[4];     /* power correlation of bins 1..4 apart, [0, 1)      */
} atkdsp_cfar_config;

typedef struct {                                                                          /* :1856 */
    double   t0, t1;     /* seconds; t1 NaN until CLOSE                       */
    double   fc_bin;     /* excess-weighted centroid, fractional bin          */
    int32_t  type;       /* OPEN / UPDATE / CLOSE                             */
    uint32_t id;         /* unique per handle (from 1)                        */
    uint32_t flags;
    int32_t  lo_bin, hi_bin;
    int32_t  n_hits;     /* frames with a hit                                 */
    float    level_db, noise_db, snr_db, band_snr_db;
} atkdsp_cfar_event;

typedef struct {                                                                          /* :1867 */
    uint64_t frames, warmup;
    uint64_t cells_tested, cell_hits, untestable;
    uint64_t opened, closed, updates;
    uint64_t dropped;
    uint64_t resets;
    uint64_t tracks;
} atkdsp_cfar_counters;

typedef struct atkdsp_cfar atkdsp_cfar;
ATKDSP_API void         atkdsp_cfar_defaults(atkdsp_cfar_config *cfg);                  /* :1877 */
ATKDSP_API int          atkdsp_cfar_alpha(int mode, int n_ref, double pfa, double looks,
                                          int os_k, const double *rho2,
                                          double *alpha, double *et);                    /* :1882 */
ATKDSP_API double       atkdsp_cfar_n_eff(int n_ref, const double *rho2);                /* :1888 */
ATKDSP_API int          atkdsp_cfar_window_rho2(const float *window, size_t n,
                                                double *rho2);                           /* :1892 */
ATKDSP_API atkdsp_cfar *atkdsp_cfar_create(size_t nbins, const atkdsp_cfar_config *cfg); /* :1894 */
ATKDSP_API void         atkdsp_cfar_destroy(atkdsp_cfar *c);                             /* :1895 */
ATKDSP_API void         atkdsp_cfar_reset(atkdsp_cfar *c);                               /* :1897 */
ATKDSP_API int          atkdsp_cfar_set_mask(atkdsp_cfar *c, const uint8_t *mask);       /* :1900 */
ATKDSP_API size_t       atkdsp_cfar_events_max(const atkdsp_cfar *c, size_t nframes);    /* :1901 */
ATKDSP_API ptrdiff_t    atkdsp_cfar_process(atkdsp_cfar *c, const float *frames_db,
                                            size_t nframes, double frame_t0,
                                            double frame_dt, atkdsp_cfar_event *ev,
                                            size_t cap);                                 /* :1903 */
ATKDSP_API ptrdiff_t    atkdsp_cfar_flush(atkdsp_cfar *c, atkdsp_cfar_event *ev,
                                          size_t cap);                                   /* :1909 */
ATKDSP_API int          atkdsp_cfar_last(const atkdsp_cfar *c, float *avg_db, float *thr_db,
                                         uint8_t *hits);                                 /* :1913 */
ATKDSP_API int          atkdsp_cfar_info(const atkdsp_cfar *c, double *alpha,
                                         double *alpha_ca, double *et,
                                         atkdsp_cfar_config *cfg);                       /* :1917 */
ATKDSP_API int          atkdsp_cfar_describe(const atkdsp_cfar *c, char *buf, size_t cap); /* :1923 */
ATKDSP_API int          atkdsp_cfar_stats(const atkdsp_cfar *c, atkdsp_cfar_counters *st);  /* :1924 */

#ifdef __cplusplus
}
#endif
#endif
