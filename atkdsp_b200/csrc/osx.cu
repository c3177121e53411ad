/* The overlap-save extractor on sm_100a (reference src/channelizer.c:473-788).
 *
 * One CTA per (block, element). For nfft <= ATKB_OSX_FUSED_MAX the whole chain
 * stays in shared memory: the block's nfft samples are gathered from the
 * element's state and input, transformed in double (Stockham, radix 8 with
 * a radix-4 or radix-2 pass for the bits left), and rounded to a float spectrum X
 * as the reference stores it. Then, per channel: the decimating fold of X
 * against the channel filter's spectrum into M bins (float, the reference's
 * expression order with rounded operations: src/channelizer.c:707-716), the
 * M-point inverse (double, scaled by 1/M and rounded to float like
 * pocketfft's backward transform), and the roll to absolute time with the
 * residual offset removed per sample (double, :721-737), one rounding to
 * float. X never leaves the SM. Larger transforms run as two passes of at
 * most 4096 points over a double scratch in HBM (the four-step form), then
 * the same per-channel code reads X from HBM.
 *
 * The arbitrary resampler (src/resample.c:194-260) computes every output
 * independently: output K sits at input position base + K*step - in_off,
 * which the reference made blocking-invariant, so one thread per output
 * reproduces the reference's per-block loop bit for bit.
 */
#include <cuda_runtime.h>
#include <atomic>
#include <stdint.h>

#include "fft_sm.cuh"
#include "internal.h"

#define OSX_NT 512
#define OSX_WARPS (OSX_NT / 32)
#define OSX_G ATKB_OSX_G                     /* blocks per CTA */
#define OSX_WREG 256                         /* double2 per warp's region */
#define OSX_WORK (OSX_WARPS * OSX_WREG)      /* 4096 double2: the work area */
static_assert(OSX_G * ATKB_OSX_SMALL_M <= OSX_WREG, "a small channel's blocks fit its warp's region");
static_assert(ATKB_OSX_PACK_LANES <= OSX_WREG && OSX_G == ATKB_OSX_G, "a pack's blocks fit its warp's region");
static_assert(OSX_WORK >= ATKB_OSX_FUSED_MAX, "the work area holds one fused transform");
#ifndef OSX_FOLD_UNROLL
#define OSX_FOLD_UNROLL 8                    /* fold iterations in flight per lane */
#endif
#define OSX_PI2 6.283185307179586476925286766559

namespace {

using namespace atkb_fft;

/* one run of the fold: n terms from bin address xa / x and filter h, stride
 * M bins (M = 1 << LOGM, or the runtime m when LOGM < 0) */
template <int LOGM, bool SM>
__device__ __forceinline__ void fold_run(float &ar, float &ai, unsigned xa, const float2 *x, const float2 *h, int n,
                                         int m) {
    constexpr int kUnroll = OSX_FOLD_UNROLL;
    constexpr int XB = SM ? 8 * OSX_G : 8;      /* bytes per bin */
    const int M = LOGM >= 0 ? (1 << (LOGM < 0 ? 0 : LOGM)) : m;
#pragma unroll kUnroll
    for (int j = 0; j < n; ++j) {
        float2 xv;
        if (SM) asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(xv.x), "=f"(xv.y) : "r"(xa + j * M * XB));
        else xv = __ldg(x + j * M);
        const float2 hv = __ldg(h + j * M);
        ar = __fadd_rn(ar, __fsub_rn(__fmul_rn(xv.x, hv.x), __fmul_rn(xv.y, hv.y)));
        ai = __fadd_rn(ai, __fadd_rn(__fmul_rn(xv.x, hv.y), __fmul_rn(xv.y, hv.x)));
    }
}

/* bin k of a channel's decimating fold of one spectrum (float, j ascending,
 * the reference's rounded expression, src/channelizer.c:707-716). The bins
 * k + j*M + shift run up to nfft and then wrap once: two runs of a fixed
 * stride (M a template parameter for M <= 4096, so the unrolled loads carry
 * it in their immediate offsets). SM: the spectrum is the fused kernel's
 * shared one, bin b of this block at shared address xs + b * 8 * OSX_G;
 * else global, bin b at X[b]. */
template <int LOGM, bool SM>
__device__ __forceinline__ double2 fold_bin(const float2 *X, unsigned xs, const float2 *__restrict__ H, int k,
                                            int m, int decim, int shift, int nfft) {
    constexpr int XB = SM ? 8 * OSX_G : 8;
    const int M = LOGM >= 0 ? (1 << (LOGM < 0 ? 0 : LOGM)) : m;
    float ar = 0.0f, ai = 0.0f;
    int start = k + shift;
    if (start >= nfft) start -= nfft;
    const int jw = min(decim, (nfft - start + M - 1) / M);        /* start + j*M < nfft */
    fold_run<LOGM, SM>(ar, ai, xs + start * XB, X + start, H + k, jw, m);
    const int s2 = start + jw * M - nfft;
    fold_run<LOGM, SM>(ar, ai, xs + s2 * XB, X + s2, H + k + jw * M, decim - jw, m);
    return make_double2((double)ar, (double)ai);
}

template <bool SM>
__device__ __forceinline__ double2 fold_any(int logm, const float2 *X, unsigned xs, const float2 *H, int k, int decim,
                                            int shift, int nfft) {
    switch (logm) {
#define OSX_FOLD_CASE(L) case L: return fold_bin<L, SM>(X, xs, H, k, 1 << L, decim, shift, nfft);
        OSX_FOLD_CASE(1) OSX_FOLD_CASE(2) OSX_FOLD_CASE(3) OSX_FOLD_CASE(4) OSX_FOLD_CASE(5)
        OSX_FOLD_CASE(6) OSX_FOLD_CASE(7) OSX_FOLD_CASE(8) OSX_FOLD_CASE(9) OSX_FOLD_CASE(10)
        OSX_FOLD_CASE(11) OSX_FOLD_CASE(12)
#undef OSX_FOLD_CASE
    default: return fold_bin<-1, SM>(X, xs, H, k, 1 << logm, decim, shift, nfft);   /* M > 4096 */
    }
}

/* output k of block bi from the channel's unscaled inverse y (the float
 * output pocketfft's 1/M scaling gives, then the roll to absolute time with
 * the residual removed: src/channelizer.c:721-737, one rounding per step) */
__device__ __forceinline__ float2 roll_out(double2 y, const atkb_osx_chan &C, long long bi, int k, int hop,
                                           int ov, int nfft, double fs) {
    const long long start = bi * hop - ov;
    long long smod = ((long long)C.shift * start) % nfft;
    if (smod < 0) smod += nfft;
    const double a0 = (double)smod / (double)nfft;
    const double invm = 1.0 / (double)C.M, invd = 1.0 / (double)C.decim;
    const float ysr = __double2float_rn(__dmul_rn(y.x, invm));
    const float ysi = __double2float_rn(__dmul_rn(y.y, invm));
    const double yr = __dmul_rn((double)ysr, invd), yi = __dmul_rn((double)ysi, invd);
    const long long nabs = bi * hop + (long long)k * C.decim;
    const double ph = __dmul_rn(-OSX_PI2, __dadd_rn(a0, __ddiv_rn(__dmul_rn(C.delta, (double)nabs), fs)));
    double s, c;
    sincos(ph, &s, &c);
    return make_float2(__double2float_rn(__dsub_rn(__dmul_rn(yr, c), __dmul_rn(yi, s))),
                       __double2float_rn(__dadd_rn(__dmul_rn(yr, s), __dmul_rn(yi, c))));
}

/* where element e's samples of block 0 of this run go */
__device__ __forceinline__ float2 *osx_dst(const atkb_osx_chan &C, const atkb_osx_run &R, int e) {
    if (C.dsts) return (float2 *)C.dsts[e] + R.hop_base * C.nvalid;
    return (float2 *)C.stage + R.par * C.par_stride + e * C.stage_stride + C.lead;
}

/* S channels of equal M (table entries c0 .. c0+S-1) over nb consecutive
 * blocks (block i0 + g's spectrum bin b at X[b*XCOL + g*xrow]) by NTH
 * threads in `buf` (S*nb*M <= 8*NTH double2): folds, one batched inverse,
 * rolled outputs. Items run block-fastest within a channel, so the lanes
 * of a warp share each filter value and, with interleaved spectra (xrow 1),
 * read neighbouring words. Ends with a barrier of the NTH threads. */
template <int NTH, int XCOL>
__device__ void osx_channel(const float2 *X, int xrow, int nb, int c0, int S, double2 *buf, const atkb_osx_run &R,
                            int e, int i0, int tid) {
    const int logm = R.chans[c0].logm;
    const int per = nb << logm;                /* items per channel */
    for (int it = tid; it < S * per; it += NTH) {
        const int sub = it / per, r = it - sub * per;
        const int g = r % nb, k = r / nb;
        const atkb_osx_chan &C = R.chans[c0 + sub];
        buf[((sub * nb + g) << logm) + k] =
            XCOL == OSX_G
                ? fold_any<true>(logm, nullptr, (unsigned)__cvta_generic_to_shared(X) + g * 8, (const float2 *)C.H, k,
                                 C.decim, C.shift, R.nfft)
                : fold_any<false>(logm, X + g * xrow, 0u, (const float2 *)C.H, k, C.decim, C.shift, R.nfft);
    }
    fft_sync<NTH>();
    fft_b<NTH>(buf, logm, S * nb, (const double2 *)R.tw, R.lognfft, true, tid);
    const int lv = logm - 1;                   /* nvalid = M / 2 */
    const int pero = nb << lv;
    for (int it = tid; it < S * pero; it += NTH) {
        const int sub = it / pero, r = it - sub * pero;
        const int g = r >> lv, k = r & ((1 << lv) - 1);
        const int i = i0 + g;
        const atkb_osx_chan C = R.chans[c0 + sub];
        osx_dst(C, R, e)[(long long)i * C.nvalid + k] =
            roll_out(buf[((sub * nb + g) << logm) + C.ovd + k], C, R.blk0 + i, k, R.hop, R.ov, R.nfft, R.fs);
    }
    fft_sync<NTH>();
}

/* the channels of nb blocks (spectra as for osx_channel): the packs of
 * small ones (equal M, at most 32 lanes of items together; the host puts
 * the costliest first) one warp each in its own region of `work`, taken
 * from a shared counter; then the others by the whole CTA in batches of
 * blocks */
template <int XCOL>
__device__ void osx_channels(const float2 *X, int xrow, int nb, double2 *work, const atkb_osx_run &R, int e,
                             int i0, int *next, int slice = 0, int nslices = 1) {
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    for (;;) {
        int p = 0;
        if (lane == 0) p = slice + nslices * atomicAdd(next, 1);
        p = __shfl_sync(0xffffffffu, p, 0);
        if (p >= R.npacks) break;
        const int c0 = R.packs[p], c1 = R.packs[p + 1];
        osx_channel<32, XCOL>(X, xrow, nb, c0, c1 - c0, work + w * OSX_WREG, R, e, i0, lane);
    }
    __syncthreads();
    for (int c = R.nsmall + slice; c < R.nsmall + R.nmid; c += nslices) {
        const int per = ATKB_OSX_FUSED_MAX >> R.chans[c].logm;     /* blocks per batch */
        for (int g0 = 0; g0 < nb; g0 += per) {
            const int cnt = min(per, nb - g0);
            osx_channel<OSX_NT, XCOL>(X + g0 * xrow, xrow, cnt, c, 1, work, R, e, i0 + g0, tid);
        }
    }
}

/* sample g of element e's stream state ++ in (in: the element's input, at
 * the run's offset) */
__device__ __forceinline__ float2 osx_sample(const atkb_osx_run &R, const float2 *in, int e, long long g) {
    if (g < R.head) return __ldg((const float2 *)R.state + e * R.state_stride + g);
    return __ldg(in + (g - R.head));
}
__device__ __forceinline__ const float2 *osx_in(const atkb_osx_run &R, int e) {
    return (const float2 *)R.ins[e] + R.in_off;
}

/* nfft <= ATKB_OSX_FUSED_MAX: grid (ceil(m / OSX_G), nel). Shared memory:
 * the work area (OSX_WORK double2: each forward transform, then the
 * channels' folds and inverses) and the OSX_G blocks' float spectra,
 * interleaved: bin b of block g at X[b * OSX_G + g]. */
__global__ void __launch_bounds__(OSX_NT, 1) osx_group_kernel(const atkb_osx_run R, int m) {
    extern __shared__ double2 smem[];
    __shared__ int s_next;
    double2 *work = smem;
    const int nfft = R.nfft;
    float2 *X = (float2 *)(smem + OSX_WORK);
    if (threadIdx.x == 0) s_next = 0;
    const int i0 = blockIdx.x * OSX_G, e = blockIdx.y, nb = min(OSX_G, m - i0);
    const float2 *in = osx_in(R, e);
    const double2 *tw = (const double2 *)R.tw;
    for (int g = 0; g < nb; ++g) {
        const long long g0 = (long long)(i0 + g) * R.hop;
        for (int p = threadIdx.x; p < nfft; p += OSX_NT) {
            const float2 v = osx_sample(R, in, e, g0 + p);
            work[swz(p)] = make_double2((double)v.x, (double)v.y);
        }
        __syncthreads();
        fft_r8<OSX_NT>(work, R.lognfft, tw, R.lognfft, false, threadIdx.x);
        for (int p = threadIdx.x; p < nfft; p += OSX_NT) {
            const double2 y = work[swz(p)];
            X[p * OSX_G + g] = make_float2(__double2float_rn(y.x), __double2float_rn(y.y));
        }
        __syncthreads();
    }
    osx_channels<OSX_G>(X, 1, nb, work, R, e, i0, &s_next);
}

/* nfft > ATKB_OSX_FUSED_MAX: the channels read the spectra from HBM, so the
 * channels split over gridDim.z slices (packs and CTA-wide channels dealt
 * round-robin) as well as over blocks */
__global__ void __launch_bounds__(OSX_NT, 1) osx_group_chan_kernel(const atkb_osx_run R, int m) {
    extern __shared__ double2 smem[];
    __shared__ int s_next;
    const int i0 = blockIdx.x * OSX_G, e = blockIdx.y, nb = min(OSX_G, m - i0);
    const float2 *X = (const float2 *)R.X + ((long long)e * m + i0) * R.nfft;
    if (threadIdx.x == 0) s_next = 0;
    __syncthreads();
    osx_channels<1>(X, R.nfft, nb, smem, R, e, i0, &s_next, blockIdx.z, gridDim.z);
}

/* Transforms longer than 4096 points: n = n1 * n2 in the four-step form,
 * X[k1 + n1 k2] = sum_q W_n2^(q k2) W_n^(q k1) sum_r x[q + n2 r] W_n1^(r k1).
 * Pass A, grid (n2, m, nel): column q's n1-point transform, times
 * W_n^(q k1), to T[item][k1 n2 + q]. The source is the block of the stream
 * (SRC 0, a forward transform of nfft points) or a double buffer of n-point
 * items (SRC 1). */
template <int SRC>
__global__ void __launch_bounds__(OSX_NT) osx_four_a(const atkb_osx_run R, const double2 *__restrict__ src, int logn1,
                                                     int logn2, bool inv, double2 *__restrict__ T, int m) {
    extern __shared__ double2 sm[];
    const int q = blockIdx.x, i = blockIdx.y, e = blockIdx.z;
    const int n1 = 1 << logn1, logn = logn1 + logn2;
    const double2 *tw = (const double2 *)R.tw;
    const long long item = (long long)e * m + i;
    if (SRC == 0) {
        const float2 *in = osx_in(R, e);
        const long long g0 = (long long)i * R.hop + q;
        for (int r = threadIdx.x; r < n1; r += OSX_NT) {
            const float2 v = osx_sample(R, in, e, g0 + ((long long)r << logn2));
            sm[swz(r)] = make_double2((double)v.x, (double)v.y);
        }
    } else {
        const double2 *s = src + (item << logn) + q;
        for (int r = threadIdx.x; r < n1; r += OSX_NT) sm[swz(r)] = s[(long long)r << logn2];
    }
    __syncthreads();
    fft_r8<OSX_NT>(sm, logn1, tw, R.lognfft, inv, threadIdx.x);
    double2 *t = T + (item << logn);
    const int sh = R.lognfft - logn, mask = (1 << logn) - 1;
    for (int k1 = threadIdx.x; k1 < n1; k1 += OSX_NT) {
        const double2 y = sm[swz(k1)];
        t[((long long)k1 << logn2) + q] = q ? d2mul(y, tw_at(tw, (q * k1) & mask, sh, inv)) : y;
    }
}

/* Pass B, grid (n1, m, nel): row k1's n2-point transform, to a float
 * spectrum (DST 0) or a double buffer (DST 1), natural order */
template <int DST>
__global__ void __launch_bounds__(OSX_NT) osx_four_b(const atkb_osx_run R, const double2 *__restrict__ T, int logn1,
                                                     int logn2, bool inv, void *out, int m) {
    extern __shared__ double2 sm[];
    const int k1 = blockIdx.x, i = blockIdx.y, e = blockIdx.z;
    const int n2 = 1 << logn2, logn = logn1 + logn2;
    const long long item = (long long)e * m + i;
    const double2 *t = T + (item << logn) + ((long long)k1 << logn2);
    for (int q = threadIdx.x; q < n2; q += OSX_NT) sm[swz(q)] = t[q];
    __syncthreads();
    fft_r8<OSX_NT>(sm, logn2, (const double2 *)R.tw, R.lognfft, inv, threadIdx.x);
    for (int k2 = threadIdx.x; k2 < n2; k2 += OSX_NT) {
        const long long o = (item << logn) + k1 + ((long long)k2 << logn1);
        const double2 y = sm[swz(k2)];
        if (DST == 0) ((float2 *)out)[o] = make_float2(__double2float_rn(y.x), __double2float_rn(y.y));
        else ((double2 *)out)[o] = y;
    }
}

/* a channel with M > 4096 (nfft > 4096, small decimation): its folds to a
 * double buffer Y[item][M], grid (ceil(M / 256), m, nel) */
__global__ void osx_fold_big(const atkb_osx_run R, int c, double2 *__restrict__ Y, int m) {
    const atkb_osx_chan C = R.chans[c];
    const int k = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y, e = blockIdx.z;
    if (k >= C.M) return;
    const long long item = (long long)e * m + i;
    Y[(item << C.logm) + k] = fold_any<false>(C.logm, (const float2 *)R.X + item * R.nfft, 0u, (const float2 *)C.H,
                                              k, C.decim, C.shift, R.nfft);
}

/* ... and its rolled outputs from the inverse in Y, grid (ceil(nvalid / 256), m, nel) */
__global__ void osx_roll_big(const atkb_osx_run R, int c, const double2 *__restrict__ Y, int m) {
    const atkb_osx_chan C = R.chans[c];
    const int k = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y, e = blockIdx.z;
    if (k >= C.nvalid) return;
    const long long item = (long long)e * m + i;
    float2 *dst = osx_dst(C, R, e);
    dst[(long long)i * C.nvalid + k] = roll_out(Y[(item << C.logm) + C.ovd + k], C, R.blk0 + i, k, R.hop, R.ov,
                                                R.nfft, R.fs);
}

/* every resampler run of a chunk: run r owns blocks [first[r], first[r+1]),
 * blocks_r per element, one thread per output (and per history sample) */
struct RsBatch {
    int n;
    int first[ATKB_OSX_RS_MAX + 1];
    atkb_osx_rs r[ATKB_OSX_RS_MAX];
};

__global__ void __launch_bounds__(128) osx_resample_batch_kernel(const __grid_constant__ RsBatch B) {
    const int bid = blockIdx.x;
    int lo = 0, hi = B.n - 1;                       /* the run whose blocks hold bid */
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (B.first[mid] <= bid) lo = mid;
        else hi = mid - 1;
    }
    const atkb_osx_rs &D = B.r[lo];
    const int local = bid - B.first[lo];
    const int e = local / D.blocks;
    const long long k = (long long)(local - e * D.blocks) * blockDim.x + threadIdx.x;
    const int Q = D.Q, P = D.P;
    const float2 *x = (const float2 *)D.v + (long long)e * D.v_stride + Q;   /* x[m], m >= -Q */
    if (k < Q) ((float2 *)D.v_next)[(long long)e * D.v_stride + k] = x[D.nv - Q + k];
    if (k >= D.count) return;
    const double local_pos =
        __dsub_rn(__dadd_rn(D.base, __dmul_rn((double)(D.K0 + (unsigned long long)k), D.step)), D.inoff);
    const long long i = (long long)floor(local_pos);
    const double frac = __dsub_rn(local_pos, (double)i);
    const double ph = __dmul_rn(frac, (double)P);
    int b = (int)ph;
    if (b >= P) b = P - 1;
    const float mu = __double2float_rn(__dsub_rn(ph, (double)b));
    const float *pp = D.pd, *dd = D.pd + (size_t)P * Q;
    float ar = 0.0f, ai = 0.0f;
    for (int q = 0; q < Q; ++q) {
        const long long mm = i - q;
        if (mm < -(long long)Q) break;                          /* older than the kept history */
        const float2 xv = __ldg(x + mm);
        const float c = __fadd_rn(__ldg(pp + b + q * P), __fmul_rn(mu, __ldg(dd + b + q * P)));
        ar = __fadd_rn(ar, __fmul_rn(c, xv.x));
        ai = __fadd_rn(ai, __fmul_rn(c, xv.y));
    }
    float2 *o = D.outs ? (float2 *)D.outs[e] + D.out_off : (float2 *)D.stage + (long long)e * D.stage_stride;
    o[k] = make_float2(ar, ai);
}

__global__ void osx_carry_kernel(const float2 *__restrict__ state, long long state_stride,
                                 const void *const *__restrict__ ins, long long in_off, long long head,
                                 long long from, long long len, float2 *__restrict__ dst, long long dst_stride) {
    const int e = blockIdx.y;
    const float2 *in = (const float2 *)ins[e] + in_off;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < len;
         t += (long long)gridDim.x * blockDim.x) {
        const long long g = from + t;
        dst[e * dst_stride + t] = g < head ? state[e * state_stride + g] : in[g - head];
    }
}

/* the attributes are idempotent: concurrent first callers may both set them */
std::atomic<bool> g_configured[64];

int set_smem(const void *fn, int bytes) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
}

}  // namespace

extern "C" size_t atkb_osx_group_smem(int nfft) {
    return (size_t)OSX_WORK * 16 + (size_t)OSX_G * nfft * 8;
}

extern "C" int atkb_osx_launch(const atkb_osx_run *run, int m, int nel, void *stream) {
    if (m <= 0 || nel <= 0) return ATKB_OK;
    const atkb_osx_run &R = *run;
    cudaStream_t s = (cudaStream_t)stream;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ATKB_E_NODEV;
    if (!g_configured[dev].load(std::memory_order_acquire)) {
        const int big = (int)atkb_osx_group_smem(ATKB_OSX_FUSED_MAX);
        if (!set_smem((const void *)osx_group_kernel, big) || !set_smem((const void *)osx_group_chan_kernel, OSX_WORK * 16) ||
            !set_smem((const void *)osx_four_a<0>, 4096 * 16) || !set_smem((const void *)osx_four_a<1>, 4096 * 16) ||
            !set_smem((const void *)osx_four_b<0>, 4096 * 16) || !set_smem((const void *)osx_four_b<1>, 4096 * 16))
            return ATKB_E_KERNEL;
        g_configured[dev].store(true, std::memory_order_release);
    }
    const dim3 groups((m + OSX_G - 1) / OSX_G, nel);
    if (R.nfft <= ATKB_OSX_FUSED_MAX) {
        osx_group_kernel<<<groups, OSX_NT, atkb_osx_group_smem(R.nfft), s>>>(R, m);
        return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
    }
    int logn2 = R.lognfft / 2, logn1 = R.lognfft - logn2;
    if (logn1 > 12) return ATKB_E_ARG;
    osx_four_a<0><<<dim3(1 << logn2, m, nel), OSX_NT, (size_t)16 << logn1, s>>>(R, nullptr, logn1, logn2, false,
                                                                                (double2 *)R.T, m);
    osx_four_b<0><<<dim3(1 << logn1, m, nel), OSX_NT, (size_t)16 << logn2, s>>>(R, (const double2 *)R.T, logn1,
                                                                                logn2, false, R.X, m);
    if (R.nsmall + R.nmid > 0) {
        /* enough channel slices to give every SM two CTAs, no more than
         * there are packs or CTA-wide channels to deal */
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const long long ctas = (long long)groups.x * groups.y;
        int slices = (int)((2LL * sms + ctas - 1) / ctas);
        const int units = R.npacks > R.nmid ? R.npacks : R.nmid;
        if (slices > units) slices = units;
        if (slices < 1) slices = 1;
        osx_group_chan_kernel<<<dim3(groups.x, groups.y, slices), OSX_NT, OSX_WORK * 16, s>>>(R, m);
    }
    for (int c = R.nsmall + R.nmid; c < R.nchans; ++c) {
        /* M > 4096: fold to Y, four-step inverse through T back into Y, roll */
        const int logm = R.h_chans[c].logm;
        const int M = 1 << logm, nv = M >> 1;
        double2 *Y = (double2 *)R.Y, *T = (double2 *)R.T;
        logn2 = logm / 2;
        logn1 = logm - logn2;
        osx_fold_big<<<dim3((M + 255) / 256, m, nel), 256, 0, s>>>(R, c, Y, m);
        osx_four_a<1><<<dim3(1 << logn2, m, nel), OSX_NT, (size_t)16 << logn1, s>>>(R, Y, logn1, logn2, true, T, m);
        osx_four_b<1><<<dim3(1 << logn1, m, nel), OSX_NT, (size_t)16 << logn2, s>>>(R, T, logn1, logn2, true, Y, m);
        osx_roll_big<<<dim3((nv + 255) / 256, m, nel), 256, 0, s>>>(R, c, Y, m);
    }
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" int atkb_osx_resample_batch(const atkb_osx_rs *runs, int n, void *stream) {
    if (n <= 0) return ATKB_OK;
    if (n > ATKB_OSX_RS_MAX) return ATKB_E_ARG;
    RsBatch B;
    B.n = n;
    long long total = 0;
    for (int r = 0; r < n; ++r) {
        B.r[r] = runs[r];
        const long long work = runs[r].count > runs[r].Q ? runs[r].count : runs[r].Q;
        B.r[r].blocks = (int)((work + 127) / 128);
        B.first[r] = (int)total;
        total += (long long)B.r[r].blocks * runs[r].nel;
    }
    B.first[n] = (int)total;
    if (total <= 0) return ATKB_OK;
    if (total > 0x7fffffffLL) return ATKB_E_ARG;
    osx_resample_batch_kernel<<<(unsigned)total, 128, 0, (cudaStream_t)stream>>>(B);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" int atkb_osx_carry(const void *state, long long state_stride, const void *const *ins,
                              long long in_off, long long head, long long from, long long len, void *dst,
                              long long dst_stride, int nel, void *stream) {
    if (len <= 0 || nel <= 0) return ATKB_OK;
    const int nt = 256;
    long long blocks = (len + nt - 1) / nt;
    if (blocks > 1024) blocks = 1024;
    osx_carry_kernel<<<dim3((unsigned)blocks, nel), nt, 0, (cudaStream_t)stream>>>(
        (const float2 *)state, state_stride, ins, in_off, head, from, len, (float2 *)dst, dst_stride);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}
