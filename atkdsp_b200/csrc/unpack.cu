/* The unpack front end on sm_100a (reference src/convert.c:1-128).
 *
 *   out = (float(raw) - c') * k        (c' = c + off/k, precomputed on the
 *                                       host in float as the reference does)
 *   cf32: out = raw - off (or a copy when off == 0)
 *
 * Subtract and multiply are __fsub_rn / __fmul_rn so nvcc cannot fuse them:
 * the samples are bit-identical to the reference's. With 16-byte aligned
 * buffers every thread converts four samples per step with 16-byte loads and
 * stores (unpack_kernel_v4), four steps in flight, one wave of blocks. The mean of the samples
 * BEFORE the offset came out is sum(double(out)) / n + off; the double sum
 * is a two-stage deterministic reduction (per-block partials, then one
 * block), so it agrees with the reference's eight-way serial sum to ~1e-16.
 *
 * The one-pole DC block (src/convert.c:7-17) is a serial float recurrence;
 * bit-exactness forbids reassociating it, so one thread per component runs
 * it in order with rounded operations.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "internal.h"

#define UNPACK_NT 256
#define UNPACK_PER_THREAD 8
#define UNPACK_MAX_BLOCKS 2048
/* one wave on a B200: 148 SMs x UNPACK_MINB resident blocks of 256 threads (the v4
 * kernel's launch bounds); more blocks would leave a partial second wave */
#ifndef UNPACK_MINB
#define UNPACK_MINB 4
#endif
#ifndef UNPACK_GRID_MAX
#define UNPACK_GRID_MAX (148 * UNPACK_MINB)
#endif
/* 16-byte loads in flight per thread in the v4 kernel */
#ifndef UNPACK_STEPS
#define UNPACK_STEPS 4
#endif

namespace {

__device__ __forceinline__ float2 convert_one(const void *raw, int fmt, size_t i, float cre,
                                              float cim, float k, float offr, float offi) {
    float a, b;
    switch (fmt) {
    case 0: {
        const uchar2 v = ((const uchar2 *)raw)[i];
        a = (float)v.x; b = (float)v.y;
        break;
    }
    case 1: {
        const char2 v = ((const char2 *)raw)[i];
        a = (float)v.x; b = (float)v.y;
        break;
    }
    case 2:
    case 3: {
        const short2 v = ((const short2 *)raw)[i];
        a = (float)v.x; b = (float)v.y;
        break;
    }
    default: {
        const float2 v = ((const float2 *)raw)[i];
        if (offr == 0.0f && offi == 0.0f) return v;       /* the reference copies */
        return make_float2(__fsub_rn(v.x, offr), __fsub_rn(v.y, offi));
    }
    }
    return make_float2(__fmul_rn(__fsub_rn(a, cre), k), __fmul_rn(__fsub_rn(b, cim), k));
}

/* With the offset in device memory (the previous block's mean, rounded to
 * float as a host caller would round it): the same constants unpack_consts
 * computes on the host, by the same IEEE float operations. */
__device__ __forceinline__ void offset_consts(const double *doff, int fmt, float k, float &cre, float &cim,
                                              float &offr, float &offi) {
    offr = __double2float_rn(__ldg(doff));
    offi = __double2float_rn(__ldg(doff + 1));
    if (fmt == 4) {
        cre = offr;
        cim = offi;
    } else if (fmt == 0) {
        cre = __fadd_rn(127.5f, __fdiv_rn(offr, k));
        cim = __fadd_rn(127.5f, __fdiv_rn(offi, k));
    } else {
        cre = __fdiv_rn(offr, k);
        cim = __fdiv_rn(offi, k);
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

/* The mean from the blocks' partial sums, by one block of UNPACK_NT threads:
 * thread t adds partials t, t + UNPACK_NT, ... in order, then the warps and
 * the warp sums reduce in a fixed order. The loads bypass L1: in the fused
 * form the partials were written by other blocks of the same launch. Not
 * inlined: its eight loads in flight would otherwise raise the register
 * count of the whole conversion kernel. */
__device__ __noinline__ void mean_finish(const double *partial, int nblocks, size_t n, float offr, float offi,
                                         double *mean) {
    __shared__ double red[2][UNPACK_NT / 32];
    double sr = 0.0, si = 0.0;
    /* eight partials in flight per thread; past the last block +0.0, which
     * leaves the sums exact (they never hold -0.0) and in the same order */
    for (int b0 = threadIdx.x; b0 < nblocks; b0 += 8 * UNPACK_NT) {
        double2 v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int b = b0 + u * UNPACK_NT;
            v[u] = b < nblocks ? __ldcg((const double2 *)partial + b) : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            sr += v[u].x;
            si += v[u].y;
        }
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = sr; red[1][w] = si; }
    __syncthreads();
    if (w == 0) {
        sr = l < UNPACK_NT / 32 ? red[0][l] : 0.0;
        si = l < UNPACK_NT / 32 ? red[1][l] : 0.0;
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (l == 0) {
            const double inv = n ? 1.0 / (double)n : 0.0;
            mean[0] = sr * inv + (double)offr;
            mean[1] = si * inv + (double)offi;
        }
    }
}

/* This block's partial sums into partial[2 * blockIdx.x]. With done set, the
 * block that finishes last (a ticket on *done after a fence on its partial)
 * also computes the mean, exactly as unpack_mean_kernel would, and puts
 * *done back to 0 for the next launch: one launch instead of two. */
__device__ __forceinline__ void block_partial(double sr, double si, double *partial, double *mean,
                                              unsigned *done, size_t n, float offr, float offi) {
    __shared__ double red[2][UNPACK_NT / 32];
    __shared__ int last;
    sr = warp_sum(sr);
    si = warp_sum(si);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = sr; red[1][w] = si; }
    __syncthreads();
    if (w == 0) {
        sr = l < UNPACK_NT / 32 ? red[0][l] : 0.0;
        si = l < UNPACK_NT / 32 ? red[1][l] : 0.0;
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (l == 0) {
            partial[2 * blockIdx.x] = sr;
            partial[2 * blockIdx.x + 1] = si;
            if (done) {
                __threadfence();
                last = atomicAdd(done, 1u) == gridDim.x - 1;
            }
        }
    }
    if (!done) return;
    __syncthreads();
    if (!last) return;
    __threadfence();
    mean_finish(partial, (int)gridDim.x, n, offr, offi, mean);
    if (threadIdx.x == 0) *done = 0u;
}

__global__ void __launch_bounds__(UNPACK_NT)
unpack_kernel(const void *__restrict__ raw, int fmt, size_t n, float2 *__restrict__ out, float cre,
              float cim, float k, float offr, float offi, double *__restrict__ partial, double *mean,
              unsigned *done, const double *doff) {
    if (doff) offset_consts(doff, fmt, k, cre, cim, offr, offi);
    double sr = 0.0, si = 0.0;
    const size_t stride = (size_t)gridDim.x * UNPACK_NT;
    for (size_t i = (size_t)blockIdx.x * UNPACK_NT + threadIdx.x; i < n; i += stride) {
        const float2 y = convert_one(raw, fmt, i, cre, cim, k, offr, offi);
        if (out) out[i] = y;
        sr += (double)y.x;
        si += (double)y.y;
    }
    if (partial) block_partial(sr, si, partial, mean, done, n, offr, offi);
}

/* The same conversion and partial sums with 16-byte accesses: four samples
 * per thread and step (UNPACK_STEPS steps in flight), for raw and out 16-byte
 * aligned; the last n % 4 samples by the first threads of block 0 after.
 * Each sample is converted exactly as convert_one does; only the order of
 * the per-thread double sums differs from unpack_kernel. */
template <int FMT>
__device__ __forceinline__ void load4(const void *raw, size_t q, float (&a)[4], float (&b)[4]) {
    if (FMT == 0) {
        const uchar4 u = ((const uchar4 *)raw)[2 * q], v = ((const uchar4 *)raw)[2 * q + 1];
        a[0] = u.x; b[0] = u.y; a[1] = u.z; b[1] = u.w; a[2] = v.x; b[2] = v.y; a[3] = v.z; b[3] = v.w;
    } else if (FMT == 1) {
        const char4 u = ((const char4 *)raw)[2 * q], v = ((const char4 *)raw)[2 * q + 1];
        a[0] = u.x; b[0] = u.y; a[1] = u.z; b[1] = u.w; a[2] = v.x; b[2] = v.y; a[3] = v.z; b[3] = v.w;
    } else if (FMT == 2 || FMT == 3) {
        const int4 w = __ldg((const int4 *)raw + q);
        const int ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a[j] = (float)(short)(ws[j] & 0xffff);
            b[j] = (float)(short)(ws[j] >> 16);
        }
    } else {
        const float4 u = __ldg((const float4 *)raw + 2 * q), v = __ldg((const float4 *)raw + 2 * q + 1);
        a[0] = u.x; b[0] = u.y; a[1] = u.z; b[1] = u.w; a[2] = v.x; b[2] = v.y; a[3] = v.z; b[3] = v.w;
    }
}

template <int FMT>
__global__ void __launch_bounds__(UNPACK_NT, UNPACK_MINB)
unpack_kernel_v4(const void *__restrict__ raw, size_t n, float2 *__restrict__ out, float cre, float cim, float k,
                 float offr, float offi, double *__restrict__ partial, double *mean, unsigned *done,
                 const double *doff) {
    if (doff) offset_consts(doff, FMT, k, cre, cim, offr, offi);
    double sr = 0.0, si = 0.0;
    const size_t nq = n >> 2;
    const size_t stride = (size_t)gridDim.x * UNPACK_NT;
    const bool copy = FMT == 4 && offr == 0.0f && offi == 0.0f;
    for (size_t q0 = (size_t)blockIdx.x * UNPACK_NT + threadIdx.x; q0 < nq; q0 += UNPACK_STEPS * stride) {
        float a[UNPACK_STEPS][4], b[UNPACK_STEPS][4];
#pragma unroll
        for (int h = 0; h < UNPACK_STEPS; ++h)
            if (q0 + h * stride < nq) load4<FMT>(raw, q0 + h * stride, a[h], b[h]);
#pragma unroll
        for (int h = 0; h < UNPACK_STEPS; ++h) {
            if (q0 + h * stride >= nq) break;
            float2 y[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (FMT == 4) y[j] = copy ? make_float2(a[h][j], b[h][j])
                                          : make_float2(__fsub_rn(a[h][j], offr), __fsub_rn(b[h][j], offi));
                else y[j] = make_float2(__fmul_rn(__fsub_rn(a[h][j], cre), k), __fmul_rn(__fsub_rn(b[h][j], cim), k));
                sr += (double)y[j].x;
                si += (double)y[j].y;
            }
            if (out) {
                float4 *o = (float4 *)out + 2 * (q0 + h * stride);
                o[0] = make_float4(y[0].x, y[0].y, y[1].x, y[1].y);
                o[1] = make_float4(y[2].x, y[2].y, y[3].x, y[3].y);
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < (n & 3)) {   /* the tail */
        const size_t i = (nq << 2) + threadIdx.x;
        const float2 y = convert_one(raw, FMT, i, cre, cim, k, offr, offi);
        if (out) out[i] = y;
        sr += (double)y.x;
        si += (double)y.y;
    }
    if (partial) block_partial(sr, si, partial, mean, done, n, offr, offi);
}

/* unpack_kernel_v4 when both pointers allow 16-byte accesses, else unpack_kernel.
 * done (with partial and mean) fuses the mean into the launch. */
void launch_unpack(const void *raw, int fmt, size_t n, float2 *out, float cre, float cim, float k, float offr,
                   float offi, double *partial, int nb, cudaStream_t s, double *mean = nullptr,
                   unsigned *done = nullptr, const double *doff = nullptr) {
    const bool v4 = ((uintptr_t)raw & 15) == 0 && ((uintptr_t)out & 15) == 0 && fmt >= 0 && fmt <= 4;
    if (!v4) {
        unpack_kernel<<<nb, UNPACK_NT, 0, s>>>(raw, fmt, n, out, cre, cim, k, offr, offi, partial, mean, done,
                                               doff);
        return;
    }
    switch (fmt) {
    case 0: unpack_kernel_v4<0><<<nb, UNPACK_NT, 0, s>>>(raw, n, out, cre, cim, k, offr, offi, partial, mean, done, doff); break;
    case 1: unpack_kernel_v4<1><<<nb, UNPACK_NT, 0, s>>>(raw, n, out, cre, cim, k, offr, offi, partial, mean, done, doff); break;
    case 2: unpack_kernel_v4<2><<<nb, UNPACK_NT, 0, s>>>(raw, n, out, cre, cim, k, offr, offi, partial, mean, done, doff); break;
    case 3: unpack_kernel_v4<3><<<nb, UNPACK_NT, 0, s>>>(raw, n, out, cre, cim, k, offr, offi, partial, mean, done, doff); break;
    default: unpack_kernel_v4<4><<<nb, UNPACK_NT, 0, s>>>(raw, n, out, cre, cim, k, offr, offi, partial, mean, done, doff); break;
    }
}

__global__ void __launch_bounds__(UNPACK_NT)
unpack_mean_kernel(const double *__restrict__ partial, int nblocks, size_t n, float offr, float offi,
                   double *__restrict__ mean, const double *doff) {
    if (doff) {
        offr = __double2float_rn(__ldg(doff));
        offi = __double2float_rn(__ldg(doff + 1));
    }
    mean_finish(partial, nblocks, n, offr, offi, mean);
}

/* s += alpha (x - s); y = x - s, in order, one thread per component */
__global__ void dc_pole_kernel(float *__restrict__ x, size_t n, float alpha, float *__restrict__ state) {
    const int c = threadIdx.x;
    if (c > 1) return;
    float s = state[c];
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) v[u] = x[2 * (i + u) + c];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            s = __fadd_rn(s, __fmul_rn(alpha, __fsub_rn(v[u], s)));
            v[u] = __fsub_rn(v[u], s);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) x[2 * (i + u) + c] = v[u];
    }
    for (; i < n; ++i) {
        const float v = x[2 * i + c];
        s = __fadd_rn(s, __fmul_rn(alpha, __fsub_rn(v, s)));
        x[2 * i + c] = __fsub_rn(v, s);
    }
    state[c] = s;
}

}  // namespace

extern "C" int atkb_unpack_partials(size_t n) {
    size_t b = (n + (size_t)UNPACK_NT * UNPACK_PER_THREAD - 1) / ((size_t)UNPACK_NT * UNPACK_PER_THREAD);
    if (b < 1) b = 1;
    if (b > UNPACK_GRID_MAX) b = UNPACK_GRID_MAX;
    return (int)b;
}

extern "C" int atkb_unpack(const void *raw, int fmt, size_t n, void *out, float cre, float cim,
                           float k, float off_re, float off_im, double *d_mean, double *d_partial,
                           unsigned *d_done, const double *d_off, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = atkb_unpack_partials(n);
    if (n) {
        if (fmt == 4 && off_re == 0.0f && off_im == 0.0f && !d_mean && !d_off) {
            if (out && out != raw &&
                cudaMemcpyAsync(out, raw, n * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                return ATKB_E_KERNEL;
        } else {
            launch_unpack(raw, fmt, n, (float2 *)out, cre, cim, k, off_re, off_im, d_mean ? d_partial : nullptr,
                          nb, s, d_mean, d_mean ? d_done : nullptr, d_off);
        }
    }
    if (d_mean) {
        if (!n && d_off) {
            /* the mean of nothing is the offset: the kernel reads no partial */
            unpack_mean_kernel<<<1, UNPACK_NT, 0, s>>>(d_partial, 0, 0, off_re, off_im, d_mean, d_off);
        } else if (!n) {
            /* the reference: inv = 0, so the mean is the offset itself */
            const double z[2] = {(double)off_re, (double)off_im};
            if (cudaMemcpyAsync(d_mean, z, sizeof z, cudaMemcpyHostToDevice, s) != cudaSuccess)
                return ATKB_E_KERNEL;
            if (cudaStreamSynchronize(s) != cudaSuccess) return ATKB_E_KERNEL;
        } else if (!d_done) {               /* with d_done the unpack launch computed it */
            unpack_mean_kernel<<<1, UNPACK_NT, 0, s>>>(d_partial, nb, n, off_re, off_im, d_mean, d_off);
        }
    }
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" int atkb_dc_pole(void *out, size_t n, float alpha, void *d_state, void *stream) {
    if (!n) return ATKB_OK;
    dc_pole_kernel<<<1, 32, 0, (cudaStream_t)stream>>>((float *)out, n, alpha, (float *)d_state);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

/* ---- the allocation-free variant of the device unpack_dc ------------------
 * Some callers cannot allocate GPU memory when they call in: a host
 * application that hands the whole device to its own memory pool and forbids
 * other allocations, a real-time thread that must not block in the CUDA
 * allocator, or a plugin whose host gives it buffers but no allocator. For
 * them the mean's scratch -- two doubles of partial sums per reduction block
 * -- lives in this file-scope device array instead of memory the library
 * allocates. It is 32 KiB, on every GPU that loads the library, until the
 * process exits.
 *
 * One block reduces 2048 samples, so the array covers calls of up to
 * ATKB_NOALLOC_MAX_SAMPLES = 2048 * 2048 = 4,194,304 samples; larger calls are
 * refused (split the block and combine the means weighted by their lengths).
 * Up to that size the block count -- and so the order of the double sum --
 * is exactly the allocating entry point's, and the two give the same bits.
 *
 * Every call reuses the same array and leaves its partial sums there. Nothing
 * in it needs to start at zero: each call writes every entry its mean kernel
 * reads before reading it. Two calls that overlap on the GPU (different
 * streams, no ordering between them) race on the array.
 *
 * The array's device address is looked up once per device, by the first call
 * made with that device current; make that first call before any stream
 * capture begins. */
#define ATKB_NOALLOC_BLOCKS UNPACK_MAX_BLOCKS
static __device__ __align__(256) double g_unpack_noalloc_partials[2 * ATKB_NOALLOC_BLOCKS];

static double *g_noalloc_addr[64];
static std::mutex g_noalloc_lock;

static int noalloc_partials(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ATKB_E_NODEV;
    std::lock_guard<std::mutex> guard(g_noalloc_lock);
    if (!g_noalloc_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_unpack_noalloc_partials);
        if (e != cudaSuccess || !p) return ATKB_E_KERNEL;
        g_noalloc_addr[dev] = (double *)p;
    }
    *out = g_noalloc_addr[dev];
    return ATKB_OK;
}

extern "C" size_t atkb_unpack_noalloc_max_samples(void) {
    return (size_t)ATKB_NOALLOC_BLOCKS * UNPACK_NT * UNPACK_PER_THREAD;
}

extern "C" int atkb_unpack_noalloc(const void *raw, int fmt, size_t n, void *out, float cre, float cim,
                                   float k, float off_re, float off_im, double *d_mean, void *stream) {
    if (n > atkb_unpack_noalloc_max_samples()) return ATKB_E_ARG;
    const int nb = atkb_unpack_partials(n);
    if (nb > ATKB_NOALLOC_BLOCKS) return ATKB_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    double *part = nullptr;
    if (d_mean) {
        const int rc = noalloc_partials(&part);
        if (rc != ATKB_OK) return rc;
    }
    if (n) {
        if (fmt == 4 && off_re == 0.0f && off_im == 0.0f && !d_mean) {
            if (out != raw && cudaMemcpyAsync(out, raw, n * 8, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
                return ATKB_E_KERNEL;
        } else {
            launch_unpack(raw, fmt, n, (float2 *)out, cre, cim, k, off_re, off_im, part, nb, s);
        }
    }
    /* with n == 0 the mean kernel reads no partial and writes the offset */
    if (d_mean) unpack_mean_kernel<<<1, UNPACK_NT, 0, s>>>(part, n ? nb : 0, n, off_re, off_im, d_mean, nullptr);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}
