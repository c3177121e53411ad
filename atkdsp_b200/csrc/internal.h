/* Internal interface between the C99 host layer (atkdsp_host.c) and the CUDA
 * shim (*.cu). Not part of the public ABI.
 *
 * The host layer owns handles, validation, prototype design and all the
 * bookkeeping the reference keeps on the CPU; it never includes a CUDA
 * header. Everything that touches the device goes through the atkb_* calls
 * below, implemented in shim.cu / pfb.cu / unpack.cu / w12.cu. Device
 * pointers cross this boundary as void*.
 */
#ifndef ATKB_INTERNAL_H
#define ATKB_INTERNAL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes of the shim (mapped onto ATKDSP_E_* by the host) ------ */
#define ATKB_OK        0
#define ATKB_E_ARG    -1
#define ATKB_E_NOMEM  -2
#define ATKB_E_CAP    -3
#define ATKB_E_KERNEL -4   /* a launch or an asynchronous kernel failure */
#define ATKB_E_NODEV  -8   /* no usable CUDA device */

/* ---- FFT plan --------------------------------------------------------------
 * nchan = radix[0] * radix[1] * ... * radix[npass-1], Stockham order. For a
 * power of two >= 16 the fast path is used: radix[0] == ATKB_PTS (4 when
 * `pair` is set, 2 when `quad` is) and every later radix is ATKB_PTS except
 * a smaller last one.
 * `pair`: the paired fold (two consecutive hops per thread, even or odd
 * branches), used for oversample 1, 2 or 4. */
#define ATKB_MAX_PASS 24
/* complex points per thread in the fast path's Stockham passes (8 or 16);
 * the host's plan and permuted taps follow it */
#ifndef ATKB_PTS
#define ATKB_PTS 8
#endif
typedef struct {
    int npass;
    int fast;                     /* 1: power-of-two fast path */
    int pair;                     /* 1: paired fold, first radix 4             */
    int quad;                     /* 1: quad fold (four hops per thread over two
                                   * branches), first radix 2; oversample 1 or
                                   * 2, nchan <= 1024 */
    int nostage;                  /* 1: nchan <= 512 folds read global memory
                                   * even where the tile window would fit in
                                   * shared memory (the autotuner's choice) */
    int big;                      /* 1: nchan beyond one CTA's shared memory:
                                   * separate fold / pass / epilogue kernels */
    int ptaps;                    /* taps in the paired layout (pair, or the
                                   * nchan-4096 two-hop tile's paired fold) */
    int radix[ATKB_MAX_PASS];
    int twoff[ATKB_MAX_PASS];     /* offset of pass p's twiddles in the table */
    int twlen;                    /* total twiddle entries (double2)          */
} atkb_fft_plan;

/* ---- a filterbank's device constants ----------------------------------- */
typedef struct {
    int nchan, os, K, hop;
    long long L, ov;
    const float *taps;            /* device: L floats, (float)h[q]            */
    const float *tapsP;           /* device: fast path, taps permuted for float4
                                   * loads that are contiguous across a warp's
                                   * branches j (MP = nchan/ATKB_PTS):
                                   * float4 (k*(P/4) + q)*MP + j holds the taps
                                   * k*nchan + j + r*MP, r = 4q .. 4q+3; paired:
                                   * float4 (2k + c)*MP + j holds r = c + 2i,
                                   * i = 0..3 */
    const float *tapsQ;           /* device: quad fold, (c*2K + v)*MP + j holds
                                   * the tap (4v + c)*MP + j, c = 0..3 */
    const void *twd;              /* device: nchan double2 (cos, sin)(2 pi j/nchan) */
    const void *wfull;            /* device: nchan double2 W^j = (cos, -sin)  */
    const void *wpass;            /* device: per-pass twiddles (fast path)    */
    atkb_fft_plan plan;
    int logm;                     /* log2(nchan) on the fast path, else 0      */
    int tile_hops;                /* hops per CTA tile                        */
    int smem_bytes;               /* dynamic shared memory a tile needs       */
} atkb_bank;

/* ---- one unit of PFB work: a run of hops of one element stream --------- */
typedef struct {
    const void *state;            /* device cf32: s[0, head)                   */
    const void *in;               /* device cf32: s[head, head + n)            */
    void *out;                    /* device cf32: this element's [nchan][ldo]  */
    const void *cal;              /* device cf32: nchan factors, or NULL       */
    long long head;               /* samples held in state                     */
    long long ldo;                /* output row stride in samples              */
    long long out_col;            /* column of hop 0 in out                    */
    long long b0;                 /* global hop index of this call's hop 0     */
    long long hops;               /* hops in this job                          */
    const atkb_bank *bank;        /* device copy of the bank                   */
    int in_kind;                  /* 0: `in` is cf32; 1: `in` is int16 I/Q     */
    float cre, cim, kscale;       /* int16 input: sample = (float(v) - c) * k,
                                   * held as cre/cim = -(c * k), kscale = k (a
                                   * power of two): fma(float(v), k, cre) */
    int tiles;                    /* ceil(hops / bank->tile_hops)              */
    long long nsrc;               /* samples of s = state ++ in there are (head
                                   * + n): every window must end within them */
    double *w2;                   /* device, or NULL: the fused W2 partials, one
                                   * row of nchan doubles per tile of the job
                                   * (power-of-two nchan <= 2048 banks only) */
    const double *doff;           /* device, or NULL: the int16 offset (two
                                   * doubles, rounded to float); when set,
                                   * cre/cim are derived from it on the device
                                   * as atkb_job_conv does on the host (the
                                   * table by atkb_pfb_conv_from_offset, the
                                   * large-filterbank fold by itself) */
} atkb_job;

/* ---- state carry: dst[0, len) = s[from, from + len) -------------------- */
typedef struct {
    const void *state;
    const void *in;
    void *dst;
    long long head;
    long long from;
    long long len;
    int in_kind;                  /* as atkb_job: int16 input is converted   */
    float cre, cim, kscale;
    long long nsrc;               /* samples of s there are (head + n)       */
    long long cap;                /* capacity of dst in samples              */
    const double *doff;           /* as atkb_job                             */
} atkb_carry;

/* ---- the tile kernel's fault word (counters[ATKB_FAULT_WORD]) -------------
 * Before touching a tile or a carry the kernel checks, uniformly across the
 * CTA, that every window it will read ends within the job's nsrc samples,
 * that its output columns lie within the row stride and that a carry fits its
 * destination; a violation sets a bit here and the tile or carry is skipped
 * (nothing is read or written for it), so the launch completes and the host
 * reports ATKDSP_E_FFT. Built with ATKB_DEBUG_BOUNDS, every thread also checks
 * each shared-memory and output index it computes. */
#define ATKB_FAULT_WORD 3
#define ATKB_FAULT_WINDOW 1u
#define ATKB_FAULT_OUTPUT 2u
#define ATKB_FAULT_CARRY  4u
#define ATKB_FAULT_INDEX  8u

/* device / memory ---------------------------------------------------------- */
int  atkb_get_device(int *dev);
int  atkb_set_device(int dev);
int  atkb_sm_count(int dev);
int  atkb_stream_create(void **stream);
void atkb_stream_destroy(void *stream);
int  atkb_stream_sync(void *stream);
int  atkb_malloc(void **p, size_t bytes);
void atkb_free(void *p);
int  atkb_pool_create(int dev, void **pool);       /* stream-ordered device pool */
void atkb_pool_destroy(void *pool);
size_t atkb_pool_idle_bytes(void *pool);
int  atkb_malloc_pool(void **p, size_t bytes, void *pool, void *stream);
void atkb_free_async(void *p, void *stream);
int  atkb_host_alloc(void **p, size_t bytes);      /* pinned */
/* fault injection: the n-th allocation (device, pool or pinned) from now
 * fails with ATKB_E_NOMEM; 0 disarms */
void atkb_fail_alloc_after(long long n);
void atkb_host_free(void *p);
/* the device address of pinned host memory (kernels write it over the bus) */
int  atkb_host_dev_ptr(void *h, void **d);
int  atkb_h2d(void *dst, const void *src, size_t bytes, void *stream);
int  atkb_d2h(void *dst, const void *src, size_t bytes, void *stream);
int  atkb_d2d(void *dst, const void *src, size_t bytes, void *stream);
int  atkb_d2h_2d(void *dst, size_t dpitch, const void *src, size_t spitch,
                 size_t width, size_t height, void *stream);
int  atkb_memset(void *p, int v, size_t bytes, void *stream);
int  atkb_mem_info(size_t *free_bytes, size_t *total_bytes);
int  atkb_event_create(void **ev);
void atkb_event_destroy(void *ev);
int  atkb_event_record(void *ev, void *stream);
int  atkb_event_sync(void *ev);
int  atkb_stream_wait(void *stream, void *ev);
/* timing events: recorded as graph nodes when the stream is capturing */
int  atkb_event_create_timed(void **ev);
int  atkb_event_record_node(void *ev, void *stream);
int  atkb_event_elapsed_ms(float *ms, void *start, void *stop);
/* graphs: capture the work enqueued on `stream` between begin and end */
int  atkb_graph_begin(void *stream);
int  atkb_graph_end(void *stream, void **exec);
int  atkb_graph_launch(void *exec, void *stream);       /* inside an NVTX range */
/* NVTX ranges on the host timeline (no-ops unless a profiler is attached) */
void atkb_range_push(const char *name);
void atkb_range_pop(void);
void atkb_graph_destroy(void *exec);

/* filterbank --------------------------------------------------------------- */
/* occupancy-derived number of CTAs for the persistent tile kernel */
int  atkb_pfb_grid(int dev, int smem_bytes);
int  atkb_pfb_max_smem(void);
/* jobs / tile_start / carries / counters are DEVICE arrays; tile_start has
 * njobs + 1 entries, the last one the total tile count, read by the kernel
 * (so a captured graph can replay with new work). grid CTAs loop over the
 * tiles, then over the carries (one per job: it writes only the other state
 * buffer, which no tile reads, so it needs no ordering against the tiles).
 * counters: ATKB_NCOUNTERS ints, zero before the first launch; the kernel
 * leaves them zero again. */
#define ATKB_NCOUNTERS 4
int  atkb_pfb_launch(const atkb_job *d_jobs, const int *d_tile_start, const atkb_carry *d_carry,
                     int njobs, int *d_counters, int grid, int smem_bytes, void *stream);
/* the same with the job count read from device memory (at most the given
 * maximum): a launch that serves a different set of streams each time can
 * be captured once */
int  atkb_pfb_launch_n(const atkb_job *d_jobs, const int *d_tile_start, const atkb_carry *d_carry,
                       int njobs_max, const int *d_njobs, int *d_counters, int grid, int smem_bytes,
                       void *stream);
/* atkb_pfb_launch as a programmatic dependent of the kernel before it on the
 * stream (which triggers early; the tile kernel waits for its completion
 * before reading the tables) */
int  atkb_pfb_launch_pdl(const atkb_job *d_jobs, const int *d_tile_start, const atkb_carry *d_carry,
                         int njobs, int *d_counters, int grid, int smem_bytes, void *stream);
int  atkb_event_query(void *ev);        /* ATKB_OK when complete, 1 when pending */
int  atkb_event_spin(void *ev);         /* wait for an event by polling it */
/* large filterbanks (plan.big: nchan beyond one CTA's shared memory): hops
 * [h0, h0 + nh) of job J (a host copy; its pointers are device pointers)
 * through fold, FFT-pass and epilogue kernels in `scratch`, 2 * nh * nchan
 * double2 of device memory. At most atkb_pfb_big_hops(nchan) hops a call
 * with the scratch the host sizes by it. The state carry is left to a
 * tile-kernel launch with no tiles. */
long long atkb_pfb_big_hops(int nchan);
/* the debug build's per-thread index-check word (read and cleared), and
 * whether this library is that build */
unsigned atkb_pfb_debug_fault(void);
int  atkb_pfb_debug_build(void);
/* small calls: one CTA per hop of njobs jobs of m hops each (the bank a
 * power of two 16..1024 on the fast plan, atkb_pfb_hops_ok), then one CTA per
 * carry; the same outputs and fault word as atkb_pfb_launch */
int  atkb_pfb_hops(const atkb_job *d_jobs, const atkb_carry *d_carry, int njobs, int m, int *d_counters,
                   void *stream);
int  atkb_pfb_hops_ok(const atkb_bank *B);
/* the int16 constants of nel device jobs and carries whose doff is set, from
 * that device-held offset (after the table upload, before the tile kernel) */
int  atkb_pfb_conv_from_offset(atkb_job *d_jobs, atkb_carry *d_carry, int nel, void *stream);
/* a one-job table written by a kernel from its launch parameters (the job,
 * its carry, tile_start = {0, tiles}), constants derived as above: no
 * host->device copy; the tile kernel follows as a programmatic dependent */
int  atkb_pfb_job_from_params(const atkb_job *J, const atkb_carry *C, int tiles, atkb_job *d_jobs,
                              atkb_carry *d_carry, int *d_tile_start, void *stream);

int  atkb_pfb_big(const atkb_job *J, const atkb_bank *B, long long h0, int nh, void *scratch, int grid,
                  void *stream);

/* W1 + W2 over a device [nel][nchan][m] block. R, counts, pwr, mean_pwr are
 * device pointers (any may be NULL to skip that output). */
int  atkb_w12(const void *out, unsigned nel, unsigned nchan, size_t m, const uint8_t *gate,
              void *R, uint32_t *counts, float *pwr, float *mean_pwr, void *stream);
/* the fused W2 partials (tiles rows of nchan doubles, tile order) of one
 * single-element block of m hops: W2 power per channel and, for one
 * element, W1 (R[k] += S, counts += m, gated) -- the same sums atkb_w12
 * computes over the block's outputs */
int  atkb_w2_finish(const double *part, int tiles, int nchan, long long m, const uint8_t *gate, void *R,
                    uint32_t *counts, float *pwr, float *mean_pwr, void *stream);
int  atkb_cov_reset(void *R, uint32_t *counts, unsigned nel, unsigned nchan,
                    const uint8_t *gate, void *stream);

/* overlap-save extractor ----------------------------------------------------
 * One run = m consecutive blocks (hops) of nel element streams. Block i of
 * element e is s[i*hop, i*hop + nfft) of s = state[e][0, head) ++
 * ins[e][in_off, ...).
 * Each block is forward-transformed (double, rounded to float like the
 * reference's spectrum), then every channel folds it to M bins, inverts them
 * and writes its nvalid = hop/decim samples of block i, rolled to absolute
 * time: to dsts[e] + (hop_base + i)*nvalid when dsts is set (the caller's
 * device buffers), else to the channel's staging
 * stage + par*par_stride + e*stage_stride + lead + i*nvalid. */
typedef struct {
    const void *H;                /* device cf32, nfft: the channel filter's spectrum */
    void *const *dsts;            /* device array of nel device pointers, or NULL */
    void *stage;                  /* device cf32 [2][max_nel][stage_stride]       */
    long long stage_stride, par_stride, lead;
    double delta;                 /* residual offset (Hz) after the integer roll  */
    int M, logm, ovd, nvalid, decim, shift;
} atkb_osx_chan;

typedef struct {
    const void *state;            /* device cf32 [nel][state_stride]              */
    const void *const *ins;       /* device array of nel device cf32 pointers     */
    long long state_stride, in_off, head;
    long long blk0;               /* absolute index of block 0                    */
    const void *tw;               /* device double2 [nfft]: (cos, -sin)(2 pi j/nfft) */
    const atkb_osx_chan *chans;   /* device, nchans: nsmall channels with
                                   * M <= ATKB_OSX_SMALL_M, then nmid with
                                   * M <= 4096, then those with M > 4096       */
    const atkb_osx_chan *h_chans; /* the same table in host memory (launcher)   */
    const int *packs;             /* device, npacks + 1: the small channels in
                                   * packs [packs[p], packs[p+1]) of equal M, one
                                   * warp each                                 */
    int npacks;
    double fs;
    long long hop_base;           /* blocks of this call before this run          */
    int par;                      /* which half of the channels' staging          */
    int nfft, lognfft, hop, ov, nchans, nsmall, nmid;
    void *X;                      /* device cf32 [nel][m][nfft]: nfft > fused max */
    void *T, *Y;                  /* device double2 scratch, same shape           */
} atkb_osx_run;
/* channels of at most this many bins run one warp each; those with
 * OSX_G * M <= ATKB_OSX_PACK_LANES share a warp with others of their M */
#define ATKB_OSX_SMALL_M 64
#define ATKB_OSX_PACK_LANES 32
#define ATKB_OSX_G 4                  /* blocks per CTA of the fused kernel */
/* dynamic shared memory of the fused kernel for one nfft */
size_t atkb_osx_group_smem(int nfft);

/* the largest nfft whose whole chain runs in one CTA's shared memory */
#define ATKB_OSX_FUSED_MAX 4096
/* the largest nfft at all (two passes of at most 4096 points) */
#define ATKB_OSX_NFFT_MAX (1 << 24)
int  atkb_osx_launch(const atkb_osx_run *run, int m, int nel, void *stream);
/* the arbitrary resampler over one channel's sample stream, per element
 * e < nel: v + e*v_stride holds hist (Q) ++ nv new samples. Outputs K0 + k,
 * k < count, at input position base + K*step - inoff (the reference's
 * formula) go to outs[e] + out_off (outs: a device array of nel device
 * pointers) or, when outs is NULL, to stage + e*stage_stride + k. The new
 * history, the last Q of hist ++ new, goes to v_next + e*v_stride. pd = P*Q
 * prototype taps then P*Q forward differences. blocks: the launcher's
 * 128-thread blocks per element (set by atkb_osx_resample_batch). */
typedef struct {
    const void *v;
    void *v_next;
    long long v_stride, nv;
    const float *pd;
    double base, step, inoff;
    unsigned long long K0;
    long long count;
    void *const *outs;
    long long out_off;
    void *stage;
    long long stage_stride;
    int Q, P, nel, blocks;
} atkb_osx_rs;
#define ATKB_OSX_RS_MAX 128
/* n <= ATKB_OSX_RS_MAX resampler runs in one launch (their descriptors
 * travel as the kernel's parameters) */
int  atkb_osx_resample_batch(const atkb_osx_rs *runs, int n, void *stream);
/* dst[e][0, len) = s[from, from + len) of s = state[e][0, head) ++
 * ins[e][in_off, ...), ins a device array of nel device pointers */
int  atkb_osx_carry(const void *state, long long state_stride, const void *const *ins, long long in_off,
                    long long head, long long from, long long len, void *dst, long long dst_stride,
                    int nel, void *stream);

/* spectrum reduction --------------------------------------------------------
 * frames f < `frames` of n = 2^logn samples at in + f*hop (device cf32),
 * windowed by win (device, n floats, or NULL), transformed with the n-point
 * table tw; nblk CTAs take `per` consecutive frames each into `part`
 * (nblk lines: float for modes 0/1/2, 4 double planes for mode 3), then the
 * merged line goes to o0 (modes 0/1/2: max / min / average detector, dB) or
 * o0..o3 (mode 3: max / avg / min dB and kurtosis; NULL skips one). */
#define ATKB_SPEC_NMAX 4096
int  atkb_spec_launch(int mode, const void *in, long long frames, long long hop, int logn, const float *win,
                      const void *tw, int nblk, int per, void *part, float *o0, float *o1, float *o2,
                      float *o3, void *stream);

/* CFAR cell test ------------------------------------------------------------
 * Frames f0 .. f0+nf-1 (absolute frame numbers since reset) of nbins powers
 * each; raw is a ring of `ring` rows (frame F in row F % ring).
 * atkb_cfar_raw: raw[F] = linear power of frames[f - f0] (units 0: dB, read
 * as exp(v ln10/10) with v clamped at -300; 1: linear, clamped at 1e-30).
 * atkb_cfar_test: for the frames f >= t0 (t0 >= f0 + k - 1), X = the mean of
 * raw rows f-k+1 .. f (oldest first), then each testable bin's statistic over
 * its n_cells reference cells (idx: n_cells x nbins, cell-major) and the
 * test; X, noise, thr (double) and hits (u8) rows go to row f - f0 of the
 * outputs, and the hits as bits (bin i: bit i % 32 of word i / 32, `words`
 * words a row) to row f - f0 of `bits` (frames below t0 are left alone). */
int  atkb_cfar_raw(const float *frames, int units, long long f0, int nf, long long nbins, double *raw, int ring,
                   void *stream);
int  atkb_cfar_test(const double *raw, int ring, long long f0, long long t0, int nf, long long nbins, int k,
                    int mode, int n_ref, int n_cells, int os_k, double alpha, double alpha_ca, double et,
                    const uint8_t *ok, const uint8_t *sided, const int32_t *idx, double *X, double *noise,
                    double *thr, uint8_t *hits, uint32_t *bits, long long words, void *stream);
/* the rows the tracker reads, at the columns `cols` (ncol bins) only: rows
 * 0..rows-1 of X and noise (stride nbins) into Xc / Nc (stride ncol), and
 * raw frames rf0 .. rf0+nraw-1 from the ring into Rc (stride ncol) */
int  atkb_cfar_gather(const double *X, const double *noise, long long nbins, int rows, const double *raw, int ring,
                      long long rf0, int nraw, const int32_t *cols, int ncol, double *Xc, double *Nc, double *Rc,
                      void *stream);

/* unpack ------------------------------------------------------------------- */
/* device raw -> device cf32 (out may be NULL: mean only), (x - c) * k per component; the means (double,
 * BEFORE subtraction of the offset, i.e. sum(out)/n + off) go to d_mean[0..1]
 * when d_mean != NULL, using d_partial (>= 2 * atkb_unpack_partials(n)
 * doubles) as scratch. d_done (may be NULL): a device counter that is 0
 * between calls; with it the unpack launch's last block computes the mean
 * (no second launch) and puts the counter back to 0. d_off (may be NULL): the
 * offset as two doubles in device memory, rounded to float and turned into
 * the constants on the device (cre, cim, off_re, off_im are then unused). */
int  atkb_unpack_partials(size_t n);
int  atkb_unpack(const void *raw, int fmt, size_t n, void *out, float cre, float cim, float k,
                 float off_re, float off_im, double *d_mean, double *d_partial, unsigned *d_done,
                 const double *d_off, void *stream);
/* the same conversion and mean with the partial sums in a static device
 * array instead of caller scratch; at most atkb_unpack_noalloc_max_samples()
 * samples per call (ATKB_E_ARG beyond) */
size_t atkb_unpack_noalloc_max_samples(void);
int  atkb_unpack_noalloc(const void *raw, int fmt, size_t n, void *out, float cre, float cim, float k,
                         float off_re, float off_im, double *d_mean, void *stream);
/* the one-pole DC block over converted samples, serial per component;
 * d_state is one cf32 on the device (read and updated). */
int  atkb_dc_pole(void *out, size_t n, float alpha, void *d_state, void *stream);

#ifdef __cplusplus
}
#endif
#endif
