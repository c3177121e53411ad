/* Device-resident spectrum reduction on sm_100a (reference src/fft.c:154-164,
 * :176-295 atkdsp_spectrum_reduce, :315-430 atkdsp_spectrum_stats).
 *
 * Every frame of n samples (stride hop) of a device cf32 block is windowed
 * and transformed in double in shared memory (the radix-8 Stockham transform
 * of fft_sm.cuh), and its per-bin power folded into per-CTA accumulators held
 * in registers (stats: in shared memory beside the transform): each CTA
 * takes a contiguous run of frames, as the
 * reference's OpenMP threads do, and writes one partial line (reduce: float
 * max / min / sum of |X|^2/n^2 from the float-rounded bin; stats: double
 * max, min, sum P, sum P^2). A second kernel merges the partials in CTA
 * order and converts to dB fftshifted, with the reference's rounded steps.
 * Max and min are exact in any order; the sums differ from a one-thread run
 * only in their rounding sequence.
 */
#include <cuda_runtime.h>
#include <atomic>
#include <stdint.h>

#include "fft_sm.cuh"
#include "internal.h"

#define SP_NT 512
#define SP_BINS (ATKB_SPEC_NMAX / SP_NT)      /* output bins per thread */

namespace {

using namespace atkb_fft;

/* MODE 0 / 1 / 2: reduce with the max / min / average detector; 3: stats */
template <int MODE>
__global__ void __launch_bounds__(SP_NT) spec_frames_kernel(const float2 *__restrict__ in, long long frames,
                                                            long long hop, int logn, const float *__restrict__ win,
                                                            const double2 *__restrict__ tw, int per,
                                                            void *__restrict__ part) {
    extern __shared__ double2 sm[];
    const int n = 1 << logn, half = n >> 1, tid = threadIdx.x;
    const long long f0 = (long long)blockIdx.x * per;
    const long long f1 = min(frames, f0 + per);
    const float inv2f = __fdiv_rn(1.0f, __fmul_rn((float)n, (float)n));
    const double inv2d = 1.0 / ((double)n * (double)n);
    float acc[SP_BINS];
    /* stats: the four accumulator planes in shared memory after the transform */
    double *mx = (double *)(sm + n), *mn = mx + n, *su = mn + n, *s2 = su + n;
    for (long long f = f0; f < f1; ++f) {
        const float2 *x = in + f * hop;
        for (int p = tid; p < n; p += SP_NT) {
            const float2 v = __ldg(x + p);
            if (win) {
                const double g = (double)__ldg(win + p);
                sm[swz(p)] = make_double2(__dmul_rn((double)v.x, g), __dmul_rn((double)v.y, g));
            } else {
                sm[swz(p)] = make_double2((double)v.x, (double)v.y);
            }
        }
        __syncthreads();
        fft_r8<SP_NT>(sm, logn, tw, logn, false, tid);
#pragma unroll
        for (int u = 0; u < SP_BINS; ++u) {
            const int i = tid + u * SP_NT;
            if (i >= n) break;
            const double2 X = sm[swz((i + half) & (n - 1))];
            if (MODE < 3) {
                const float re = __double2float_rn(X.x), im = __double2float_rn(X.y);
                const float pw = __fmul_rn(__fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im)), inv2f);
                if (f == f0) acc[u] = pw;
                else if (MODE == 0) acc[u] = pw > acc[u] ? pw : acc[u];
                else if (MODE == 1) acc[u] = pw < acc[u] ? pw : acc[u];
                else acc[u] = __fadd_rn(acc[u], pw);
            } else {
                const double pw = __dmul_rn(__dadd_rn(__dmul_rn(X.x, X.x), __dmul_rn(X.y, X.y)), inv2d);
                if (f == f0) {
                    mx[i] = mn[i] = su[i] = pw;
                    s2[i] = __dmul_rn(pw, pw);
                } else {
                    if (pw > mx[i]) mx[i] = pw;
                    if (pw < mn[i]) mn[i] = pw;
                    su[i] = __dadd_rn(su[i], pw);
                    s2[i] = __dadd_rn(s2[i], __dmul_rn(pw, pw));
                }
            }
        }
        __syncthreads();                       /* the next frame overwrites sm */
    }
#pragma unroll
    for (int u = 0; u < SP_BINS; ++u) {
        const int i = tid + u * SP_NT;
        if (i >= n) break;
        if (MODE < 3) {
            ((float *)part)[(long long)blockIdx.x * n + i] = acc[u];
        } else {
            double *d = (double *)part + (long long)blockIdx.x * 4 * n;
            d[i] = mx[i];
            d[n + i] = mn[i];
            d[2 * n + i] = su[i];
            d[3 * n + i] = s2[i];
        }
    }
}

/* the partial lines merged in CTA order, then dB (src/fft.c:280-290 and
 * :405-426): reduce -> o0; stats -> o0 max, o1 avg, o2 min, o3 kurtosis
 * (NULL: skipped) */
template <int MODE>
__global__ void spec_final_kernel(const void *__restrict__ part, int nblk, int n, long long frames, float *o0,
                                  float *o1, float *o2, float *o3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (MODE < 3) {
        const float *p = (const float *)part;
        float a = p[i];
        for (int b = 1; b < nblk; ++b) {
            const float v = p[(long long)b * n + i];
            if (MODE == 0) a = v > a ? v : a;
            else if (MODE == 1) a = v < a ? v : a;
            else a = __fadd_rn(a, v);
        }
        const float scale = MODE == 2 ? __fdiv_rn(1.0f, (float)frames) : 1.0f;
        const float mag = __fsqrt_rn(__fmul_rn(a, scale));
        o0[i] = __fmul_rn(20.0f, log10f(__fadd_rn(mag, 1e-12f)));
        return;
    }
    const double *d = (const double *)part;
    double mx = d[i], mn = d[n + i], su = d[2 * n + i], s2 = d[3 * n + i];
    for (int b = 1; b < nblk; ++b) {
        const double *e = d + (long long)b * 4 * n;
        if (e[i] > mx) mx = e[i];
        if (e[n + i] < mn) mn = e[n + i];
        su = __dadd_rn(su, e[2 * n + i]);
        s2 = __dadd_rn(s2, e[3 * n + i]);
    }
    const double M = (double)frames;
    if (o0) o0[i] = __fmul_rn(10.0f, log10f(__fadd_rn(__double2float_rn(mx), 1e-12f)));
    if (o2) o2[i] = __fmul_rn(10.0f, log10f(__fadd_rn(__double2float_rn(mn), 1e-12f)));
    if (o1) o1[i] = __fmul_rn(10.0f, log10f(__fadd_rn(__double2float_rn(__ddiv_rn(su, M)), 1e-12f)));
    if (o3) {
        const double den = __dmul_rn(su, su);
        o3[i] = (frames < 2 || den <= 0.0) ? 1.0f : __double2float_rn(__ddiv_rn(__dmul_rn(M, s2), den));
    }
}

template <int MODE>
int spec_launch(const void *in, long long frames, long long hop, int logn, const float *win, const void *tw,
                int nblk, int per, void *part, float *o0, float *o1, float *o2, float *o3, cudaStream_t s) {
    const int n = 1 << logn;
    spec_frames_kernel<MODE><<<nblk, SP_NT, (size_t)n * (MODE == 3 ? 48 : 16), s>>>((const float2 *)in, frames, hop, logn, win,
                                                                (const double2 *)tw, per, part);
    spec_final_kernel<MODE><<<(n + 255) / 256, 256, 0, s>>>(part, nblk, n, frames, o0, o1, o2, o3);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

/* the attributes are idempotent: concurrent first callers may both set them */
std::atomic<bool> g_configured[64];

}  // namespace

extern "C" int atkb_spec_launch(int mode, const void *in, long long frames, long long hop, int logn, const float *win,
                                const void *tw, int nblk, int per, void *part, float *o0, float *o1, float *o2,
                                float *o3, void *stream) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ATKB_E_NODEV;
    if (!g_configured[dev].load(std::memory_order_acquire)) {
        const int b = ATKB_SPEC_NMAX * 16;
        if (cudaFuncSetAttribute(spec_frames_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) != cudaSuccess ||
            cudaFuncSetAttribute(spec_frames_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) != cudaSuccess ||
            cudaFuncSetAttribute(spec_frames_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b) != cudaSuccess ||
            cudaFuncSetAttribute(spec_frames_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, 3 * b) != cudaSuccess)
            return ATKB_E_KERNEL;
        g_configured[dev].store(true, std::memory_order_release);
    }
    cudaStream_t s = (cudaStream_t)stream;
    switch (mode) {
    case 0: return spec_launch<0>(in, frames, hop, logn, win, tw, nblk, per, part, o0, o1, o2, o3, s);
    case 1: return spec_launch<1>(in, frames, hop, logn, win, tw, nblk, per, part, o0, o1, o2, o3, s);
    case 2: return spec_launch<2>(in, frames, hop, logn, win, tw, nblk, per, part, o0, o1, o2, o3, s);
    case 3: return spec_launch<3>(in, frames, hop, logn, win, tw, nblk, per, part, o0, o1, o2, o3, s);
    default: return ATKB_E_ARG;
    }
}
