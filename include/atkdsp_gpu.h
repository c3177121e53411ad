/*
 * atkdsp_gpu.h -- device-pointer entry points of the B200 channelizer.
 *
 * The reference has no device boundary: its atkdsp_pfb_* / atkdsp_unpack*
 * calls take host memory (include/atkdsp.h:3185-3251, :247-273). These entry
 * points are the same operations for callers whose samples already live in
 * GPU memory: every pointer named d_* is a device pointer, work is enqueued
 * on `stream` (a cudaStream_t passed as void*; NULL means the handle's own
 * stream for handle calls, the legacy default stream otherwise) and the call
 * returns without waiting. Results match the host-pointer calls bit for bit.
 *
 * State: a handle's streaming state lives on the device and is advanced in
 * stream order, so successive calls on one handle must be ordered on the
 * GPU (same stream, or events between streams).
 */
#ifndef ATKDSP_GPU_H
#define ATKDSP_GPU_H

#include "atkdsp.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The handle's own CUDA stream (cudaStream_t as void*). */
ATKDSP_API void       *atkdsp_gpu_pfb_stream(atkdsp_pfb *p);
/* Wait for the handle's stream. ATKDSP_OK, or ATKDSP_E_FFT if a kernel failed. */
ATKDSP_API int         atkdsp_gpu_pfb_sync(atkdsp_pfb *p);

/* atkdsp_pfb_process_n (reference include/atkdsp.h:3218) on device buffers:
 * d_ins[el] are nel device pointers of n samples each (the array itself is
 * host memory), d_out is [nel][nchan][m] device memory of cap samples.
 * Returns m (known on the host before the work runs), or ATKDSP_E_ARG /
 * ATKDSP_E_CAP (state untouched) / ATKDSP_E_FFT (launch failure). */
ATKDSP_API ptrdiff_t   atkdsp_gpu_pfb_process_n(atkdsp_pfb *p, const atkdsp_cf32 *const *d_ins,
                                                unsigned nel, size_t n, atkdsp_cf32 *d_out,
                                                size_t cap, void *stream);

/* The front end fused into the filterbank: atkdsp_unpack_dc (reference
 * include/atkdsp.h:270) of int16 I/Q samples (ATKDSP_FMT_CI16 or
 * ATKDSP_FMT_CI16Q11) with the offset (off_re, off_im), followed by
 * atkdsp_pfb_process_n (:3218), in one pass: the filterbank reads the raw
 * samples (4 bytes each instead of 8) and converts them in its load path with
 * the unpack arithmetic, so the result equals unpacking first, bit for bit.
 * d_raws[el]: n samples (2n int16) per element, 4-byte aligned. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_pfb_process_n_raw(atkdsp_pfb *p, const void *const *d_raws,
                                                    unsigned nel, size_t n, int fmt,
                                                    float off_re, float off_im,
                                                    atkdsp_cf32 *d_out, size_t cap, void *stream);

/* atkdsp_unpack_dc (reference include/atkdsp.h:270) on device buffers. When
 * d_mean is not NULL it receives the two means (re, im) as doubles on the
 * device. d_raw must be aligned to the sample's component size. The mean's
 * partial sums and the counter that lets the launch's last block finish the
 * mean live in a scratch area of the calling thread on the current device,
 * allocated by that thread's first such call. One thread's calls with a mean
 * (this and atkdsp_gpu_block_mean / _dev) must not overlap on the GPU: issue
 * them on one stream, or order them with events. Calls from different host
 * threads never share the area. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_unpack_dc(const void *d_raw, size_t nbytes, int fmt,
                                            atkdsp_cf32 *d_out, size_t out_cap,
                                            float off_re, float off_im, double *d_mean,
                                            void *stream);
/* atkdsp_gpu_unpack_dc for callers that cannot allocate GPU memory. It has
 * no counterpart in the reference (whose unpack runs on the CPU and needs no
 * scratch). Some callers must not allocate device memory when they call in:
 * a host application that owns all device memory through its own pool, a
 * real-time thread that cannot block in the CUDA allocator, a plugin given
 * buffers but no allocator. This entry point allocates nothing: the partial
 * sums of the mean live in a 32 KiB static device array that every GPU
 * loading the library holds until exit. Same arguments and results (the same
 * bits) as atkdsp_gpu_unpack_dc, for at most 4,194,304 samples per call;
 * larger calls return ATKDSP_E_ARG. The first call on a device looks up the
 * array's device address, so make it before any stream capture. All calls
 * share the array: calls that overlap on the GPU race. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_unpack_dc_noalloc(const void *d_raw, size_t nbytes, int fmt,
                                                    atkdsp_cf32 *d_out, size_t out_cap,
                                                    float off_re, float off_im, double *d_mean,
                                                    void *stream);
/* One element's block through the filterbank with W2 (per-channel power)
 * and W1 (per-channel covariance, one element: the power sum) fused into the
 * filterbank's epilogue (no reference counterpart as one call: it is
 * atkdsp_pfb_process, then atkdsp_pfb_cov_accumulate and
 * atkdsp_pfb_channel_power of reference include/atkdsp.h:3209, 3239, 3248 on
 * the block's output). Each tile of the filterbank adds up its channels'
 * power in double as it writes them; a small second kernel adds the tiles in
 * order, so the block's outputs are not read again. d_in: n cf32 samples
 * (fmt ATKDSP_FMT_CF32, zero offset) or int16 I/Q (ATKDSP_FMT_CI16 /
 * CI16Q11, converted with the offset as atkdsp_gpu_pfb_process_n_raw does).
 * d_R / d_counts (W1) and d_pwr / d_mean_pwr (W2) may each be NULL, d_gate
 * gates W1 as in atkdsp_pfb_cov_accumulate. d_scratch: device memory of at
 * least atkdsp_gpu_pfb_w12_scratch_bytes(p, n) bytes (0 where the filterbank
 * does not fuse -- nchan 4096 or not a power of two -- and W1/W2 run as a
 * separate pass instead). Returns m, ATKDSP_E_CAP for too small a d_out or
 * scratch, ATKDSP_E_ARG. */
ATKDSP_API size_t      atkdsp_gpu_pfb_w12_scratch_bytes(const atkdsp_pfb *p, size_t n);
ATKDSP_API ptrdiff_t   atkdsp_gpu_pfb_process_w12(atkdsp_pfb *p, const void *d_in, size_t n, int fmt,
                                                  float off_re, float off_im, atkdsp_cf32 *d_out,
                                                  size_t cap, const uint8_t *d_gate, atkdsp_cf32 *d_R,
                                                  uint32_t *d_counts, float *d_pwr, float *d_mean_pwr,
                                                  void *d_scratch, size_t scratch_bytes, void *stream);
/* The mean that atkdsp_unpack_dc (reference include/atkdsp.h:270) returns --
 * of the samples before the offset (off_re, off_im) is taken out -- without
 * writing the samples: for a caller whose filterbank reads the raw samples
 * (atkdsp_gpu_pfb_process_n_raw) and who keeps a running DC estimate. d_mean
 * receives 2 doubles (device). Returns the sample count. Uses the calling
 * thread's scratch as atkdsp_gpu_unpack_dc does (the same ordering rule). */
ATKDSP_API ptrdiff_t   atkdsp_gpu_block_mean(const void *d_raw, size_t nbytes, int fmt, float off_re,
                                             float off_im, double *d_mean, void *stream);
/* The running DC estimate kept on the device: atkdsp_gpu_block_mean and
 * atkdsp_gpu_pfb_process_w12 with the offset read from device memory --
 * d_offset holds two doubles (typically the previous block's d_mean), each
 * rounded to float on the device exactly as a host caller rounds the mean it
 * read back, so the results equal the host-offset calls' bit for bit. No
 * host round trip per block. block_mean_dev accepts d_offset == d_mean;
 * process_w12_dev takes the int16 formats only. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_block_mean_dev(const void *d_raw, size_t nbytes, int fmt,
                                                 const double *d_offset, double *d_mean, void *stream);
ATKDSP_API ptrdiff_t   atkdsp_gpu_pfb_process_w12_dev(atkdsp_pfb *p, const void *d_in, size_t n, int fmt,
                                                      const double *d_offset, atkdsp_cf32 *d_out,
                                                      size_t cap, const uint8_t *d_gate,
                                                      atkdsp_cf32 *d_R, uint32_t *d_counts,
                                                      float *d_pwr, float *d_mean_pwr, void *d_scratch,
                                                      size_t scratch_bytes, void *stream);
/* atkdsp_unpack (reference include/atkdsp.h:252) on device buffers;
 * d_dc_state is one device cf32, read and updated when dc_alpha > 0. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_unpack(const void *d_raw, size_t nbytes, int fmt,
                                         atkdsp_cf32 *d_out, size_t out_cap, float dc_alpha,
                                         atkdsp_cf32 *d_dc_state, void *stream);

/* W1 / W2 (reference include/atkdsp.h:3239-3251) on a device output block. */
ATKDSP_API int         atkdsp_gpu_pfb_cov_accumulate(const atkdsp_cf32 *d_out, unsigned nel,
                                                     unsigned nchan, size_t m,
                                                     const uint8_t *d_gate, atkdsp_cf32 *d_R,
                                                     uint32_t *d_counts, void *stream);
/* W1 and W2 (reference include/atkdsp.h:3239-3251) in ONE pass over the
 * block: R/counts as atkdsp_pfb_cov_accumulate (both NULL to skip W1),
 * pwr/mean_pwr as atkdsp_pfb_channel_power (either may be NULL). */
ATKDSP_API int         atkdsp_gpu_pfb_accumulate(const atkdsp_cf32 *d_out, unsigned nel, unsigned nchan,
                                                 size_t m, const uint8_t *d_gate, atkdsp_cf32 *d_R,
                                                 uint32_t *d_counts, float *d_pwr, float *d_mean_pwr,
                                                 void *stream);
ATKDSP_API int         atkdsp_gpu_pfb_cov_reset(atkdsp_cf32 *d_R, uint32_t *d_counts,
                                                unsigned nel, unsigned nchan,
                                                const uint8_t *d_gate, void *stream);
ATKDSP_API int         atkdsp_gpu_pfb_channel_power(const atkdsp_cf32 *d_out, unsigned nel,
                                                    unsigned nchan, size_t m, float *d_pwr,
                                                    float *d_mean_pwr, void *stream);

/* ---- tile shape (no reference counterpart) ------------------------------
 * For a power-of-two nchan <= 2048 at oversample 1, 2 or 4 the kernel has
 * several tile shapes, i.e. hops per thread in the fold: the paired fold
 * (each thread folds two consecutive hops over the even or odd branches:
 * half the sample and tap loads, one more FFT pass), one hop and 8 branches
 * per thread, and -- at oversample 1 or 2 with nchan <= 1024 -- the quad fold
 * (four hops per thread over two branches, a radix-2 first pass).
 * Filterbanks take the choice for their (nchan, oversample, taps/branch) from
 * the table compiled into the library (written by `python -m
 * atkdsp_b200.autotune --write` from measurements on the device), else the
 * paired fold.
 * atkdsp_gpu_tune_set overrides it for filterbanks created afterwards in this
 * process (choice 1: paired, 0: one hop per thread, 2: quad, -1: back to the
 * table; add 4 to 1 or 0 for nchan <= 512 to have the fold read the tile
 * window through L1 instead of staging it in shared memory); ATKDSP_E_ARG
 * for a shape without that choice.
 * atkdsp_gpu_tune_get returns the choice such a filterbank gets now (0, 1,
 * 2, 4 or 5), or ATKDSP_E_ARG. Every shape meets the same parity bar; they differ
 * only in speed (and, through their FFT plans, in the last bit of a few
 * outputs). */
ATKDSP_API int         atkdsp_gpu_tune_set(unsigned nchan, unsigned oversample,
                                           unsigned taps_per_poly, int choice);
ATKDSP_API int         atkdsp_gpu_tune_get(unsigned nchan, unsigned oversample,
                                           unsigned taps_per_poly);

/* ---- allocation fault injection (no reference counterpart) --------------
 * A test hook for callers' out-of-memory handling, acting on the host only:
 * with n > 0 the n-th device, pool or pinned-host allocation this library
 * makes from now on fails as a real out-of-memory would (create returns
 * NULL, the server's open ATKDSP_E_NOMEM, the host W1/W2/unpack calls leave
 * their outputs untouched), and the hook disarms itself; n <= 0 disarms it.
 * No kernel is involved and no device fault is raised. */
ATKDSP_API void        atkdsp_gpu_fail_alloc_after(long long n);

/* ---- bounds checks (no reference counterpart) ----------------------------
 * The tile kernel checks, before it touches a tile or a state carry, that
 * every window it reads ends within the samples the job has and that its
 * outputs and the carry fit their buffers; a violation sets a fault bit and
 * the tile or carry is skipped -- nothing out of bounds is read or written,
 * and the launch completes. atkdsp_gpu_pfb_faults returns the bits the
 * handle's launches set since the last call (atkdsp_gpu_batch_faults, below,
 * those of a batch's launches) (1 window, 2 output, 4 carry,
 * 8 an index caught by the debug build's per-thread checks; 0: none) and
 * clears them. The library built with ATKB_DEBUG_BOUNDS
 * (lib/libatkdsp_b200_debug.so, `make -C atkdsp_b200 debug`) also checks each
 * shared-memory and output index per thread; atkdsp_gpu_debug_build returns
 * 1 in that build. atkdsp_gpu_inject_short_window(n) is a test hook: the next
 * filterbank step's jobs claim n fewer samples than they hold (the buffers
 * hold them all, so even a missed check could read nothing out of bounds),
 * which the window check must report. */
ATKDSP_API int         atkdsp_gpu_pfb_faults(atkdsp_pfb *p);
ATKDSP_API int         atkdsp_gpu_debug_build(void);
ATKDSP_API void        atkdsp_gpu_inject_short_window(long long n);

/* ---- batches: many independent handles in one persistent launch --------
 * A batch groups handles (each single-element, any nchan / taps / oversample)
 * so that one call channelizes one new block of every handle with a single
 * kernel launch over all their hops (CTAs out of hops then carry every
 * handle's state forward). With use_graph != 0 the launch sequence is
 * captured once in a CUDA graph and replayed; the per-call description of the
 * blocks travels in a pinned table that the graph copies to the device. */
typedef struct atkdsp_gpu_batch atkdsp_gpu_batch;
ATKDSP_API atkdsp_gpu_batch *atkdsp_gpu_batch_create(atkdsp_pfb *const *handles, unsigned count,
                                                     int use_graph);
/* the fault bits of the batch's launches since the last call, cleared (as
 * atkdsp_gpu_pfb_faults) */
ATKDSP_API int         atkdsp_gpu_batch_faults(atkdsp_gpu_batch *b);
ATKDSP_API void        atkdsp_gpu_batch_destroy(atkdsp_gpu_batch *b);
/* d_ins[i]: ns[i] new samples of handle i (device); d_outs[i]: its
 * [nchan][m_i] output (device), at least nchan * out_hops(handle i, ns[i])
 * samples. ms (host, may be NULL) receives each m_i. ns[i] may be 0. Work runs
 * on `stream` (NULL: the batch's own stream). Returns the total number of
 * hops, or ATKDSP_E_*. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_batch_process(atkdsp_gpu_batch *b, const atkdsp_cf32 *const *d_ins,
                                                const size_t *ns, atkdsp_cf32 *const *d_outs,
                                                ptrdiff_t *ms, void *stream);
/* The same with int16 I/Q input converted in the load path (see
 * atkdsp_gpu_pfb_process_n_raw); offs (host, may be NULL) holds each
 * handle's offset (re, im) as 2 floats per handle. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_batch_process_raw(atkdsp_gpu_batch *b, const void *const *d_raws,
                                                    const size_t *ns, int fmt, const float *offs,
                                                    atkdsp_cf32 *const *d_outs, ptrdiff_t *ms,
                                                    void *stream);
ATKDSP_API void       *atkdsp_gpu_batch_stream(atkdsp_gpu_batch *b);
/* Measurement hook: device time in ms of the filterbank kernel of the most
 * recent atkdsp_gpu_batch_process (CUDA events recorded around that launch,
 * also inside a replayed graph); waits for it to finish. -1 on error. Events
 * are shared by all calls on the batch, so read it before the next call. */
ATKDSP_API float       atkdsp_gpu_batch_kernel_ms(atkdsp_gpu_batch *b);

/* ---- the overlap-save extractor on device buffers ----------------------- */
/* atkdsp_osx_process_n (reference include/atkdsp.h:3285) with device buffers:
 * d_ins[el] are nel device pointers of n samples, d_outs[el*nslots + ch]
 * device pointers of cap_each samples (NULL for free slots); both arrays are
 * host memory. The work is enqueued on the handle's stream and the call
 * returns without waiting; out_counts (known on the host before the work
 * runs) are set on return. Returns the slot count, or ATKDSP_E_ARG /
 * ATKDSP_E_CAP (state untouched) / ATKDSP_E_FFT. */
ATKDSP_API ptrdiff_t   atkdsp_gpu_osx_process_n(atkdsp_osx *x, const atkdsp_cf32 *const *d_ins,
                                                unsigned nel, size_t n, atkdsp_cf32 *const *d_outs,
                                                size_t *out_counts, size_t cap_each);
/* The handle's CUDA stream, and a wait for it (ATKDSP_E_FFT if a kernel failed). */
ATKDSP_API void       *atkdsp_gpu_osx_stream(atkdsp_osx *x);
ATKDSP_API int         atkdsp_gpu_osx_sync(atkdsp_osx *x);

/* ---- spectrum reduction on device buffers ------------------------------- */
/* atkdsp_spectrum_reduce / atkdsp_spectrum_stats (reference
 * include/atkdsp.h:400-433, src/fft.c:176-430) on a device block, for the
 * power-of-two lengths 16 <= n <= 4096: every frame of n samples at stride
 * hop (0 or > n means n) of d_in[0, n_samples) windowed by d_window (n device
 * floats, or NULL for rectangular), transformed, and reduced per bin into
 * one fftshifted line of n device floats in dB (detector ATKDSP_DET_MAX 0,
 * MIN 1, AVG 2), or into the four stats lines (peak, mean, floor dB, spectral
 * kurtosis; any may be NULL, not all). Enqueued on `stream` (NULL: the
 * legacy default stream); returns the frame count (0 when n_samples < n) or
 * ATKDSP_E_ARG / ATKDSP_E_FFT. One call at a time per plan: its partial
 * lines live in the plan. */
typedef struct atkdsp_gpu_spectrum atkdsp_gpu_spectrum;
ATKDSP_API atkdsp_gpu_spectrum *atkdsp_gpu_spectrum_create(size_t n);
ATKDSP_API void        atkdsp_gpu_spectrum_destroy(atkdsp_gpu_spectrum *p);
ATKDSP_API ptrdiff_t   atkdsp_gpu_spectrum_reduce(atkdsp_gpu_spectrum *p, const atkdsp_cf32 *d_in,
                                                  size_t n_samples, size_t hop, const float *d_window,
                                                  int detector, float *d_out_line, void *stream);
ATKDSP_API ptrdiff_t   atkdsp_gpu_spectrum_stats(atkdsp_gpu_spectrum *p, const atkdsp_cf32 *d_in,
                                                 size_t n_samples, size_t hop, const float *d_window,
                                                 float *d_max_db, float *d_avg_db, float *d_min_db,
                                                 float *d_sk, void *stream);

/* ---- CFAR on device frames ---------------------------------------------- */
/* atkdsp_cfar_process (reference include/atkdsp.h:1903) on nframes frames of
 * nbins floats in device memory: units 0 = dB, as the reference takes them
 * (a spectrum line from atkdsp_gpu_spectrum_*); units 1 = linear power (W2's
 * channel powers as they come, clamped below at 1e-30, the linear value of
 * the reference's -300 dB floor). The handle's stream first waits for
 * `stream`'s pending work (NULL: the legacy default stream), so the frames'
 * producer needs no host synchronisation. The events go to the caller's host array
 * as from atkdsp_cfar_process; when d_hits is not NULL, every frame's hit
 * mask (nframes x nbins bytes, 1 = hit, 0 for warm-up frames) is also
 * written there in device memory: a row is the gate W1 takes
 * (atkdsp_gpu_pfb_cov_accumulate), with no host round trip. Synchronous on
 * return; returns the event count or ATKDSP_E_ARG / ATKDSP_E_CAP /
 * ATKDSP_E_FFT (a kernel failure). */
ATKDSP_API ptrdiff_t   atkdsp_gpu_cfar_process(atkdsp_cfar *c, const float *d_frames, int units,
                                               size_t nframes, double frame_t0, double frame_dt,
                                               atkdsp_cfar_event *ev, size_t cap, uint8_t *d_hits,
                                               void *stream);

#ifdef __cplusplus
}
#endif
#endif
