/* The CFAR detector's per-cell work on sm_100a (reference src/cfar.c:524-592,
 * the first half of one_frame): the conversion of each frame to linear power,
 * the average over k_frames frames, and each bin's test against alpha x T.
 *
 * One call covers every frame a process call brings, as a grid of (bins x
 * frames): the per-cell work of different frames is independent once the raw
 * ring holds the k - 1 frames before them. Every sum runs in the reference's
 * order (the k frames oldest first; the reference cells in table order), so
 * X, T and the threshold differ from the reference's only where the device
 * exp rounds the dB conversion differently in the last bit.
 *
 * The reference-cell table is cell-major (idx[q * nbins + i]), so the threads
 * of a warp, one bin each, read one table row with coalesced loads; the
 * frame's X row they index stays in L1 / L2. Each hit row is written twice:
 * as bytes (the W1 gate's layout) and as a bitmask from one warp ballot per
 * 32 bins, which is what the host tracker reads.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <math_constants.h>
#include <stdint.h>

#include "internal.h"

namespace {

constexpr double kLn10Over10 = 0.23025850929940458;   /* ln(10) / 10 */
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) cfar_raw_kernel(const float *__restrict__ frames, int units,
                                                            long long f0, int nf, long long nbins,
                                                            double *__restrict__ raw, int ring) {
    const long long total = (long long)nf * nbins;
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < total;
         e += (long long)gridDim.x * kThreads) {
        const long long j = e / nbins, i = e - j * nbins;
        double v = (double)frames[e];
        if (units == 0) {
            if (v < -300.0) v = -300.0;
            v = exp(v * kLn10Over10);
        } else if (v < 1e-30) {
            v = 1e-30;
        }
        raw[((f0 + j) % ring) * nbins + i] = v;
    }
}

/* X row of frame f: the mean of raw rows f-k+1 .. f, oldest first */
__global__ void __launch_bounds__(kThreads) cfar_mean_kernel(const double *__restrict__ raw, int ring, long long f0,
                                                             long long t0, long long nbins, int k,
                                                             double *__restrict__ X) {
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    const long long f = t0 + blockIdx.y;
    if (i >= nbins) return;
    double s = 0.0;
    for (int r = 0; r < k; ++r) s = __dadd_rn(s, raw[((f - k + 1 + r) % ring) * nbins + i]);
    X[(f - f0) * nbins + i] = __ddiv_rn(s, (double)k);
}

/* the k-th smallest (0-based) of a[0..n), NaN-free: Hoare's selection,
 * partitioning around the middle element; i and j stay inside [lo, hi]
 * because the pivot value stops both scans. The value is unique, whatever
 * order the cells came in. */
__device__ __forceinline__ double select_kth(double *a, int n, int k) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const double pivot = a[(lo + hi) >> 1];
        int i = lo, j = hi;
        while (i <= j) {
            while (a[i] < pivot) ++i;
            while (a[j] > pivot) --j;
            if (i <= j) {
                const double t = a[i];
                a[i] = a[j];
                a[j] = t;
                ++i;
                --j;
            }
        }
        if (k <= j) hi = j;
        else if (k >= i) lo = i;
        else break;
    }
    return a[k];
}

/* a bitonic network over P registers (every index a compile-time constant
 * once unrolled, so v stays in registers): ascending on return */
template <int LOGP>
__device__ __forceinline__ void bitonic_sort(double (&v)[1 << LOGP]) {
    constexpr int P = 1 << LOGP;
#pragma unroll
    for (int kk = 1; kk <= LOGP; ++kk) {
#pragma unroll
        for (int jj = kk - 1; jj >= 0; --jj) {
#pragma unroll
            for (int i = 0; i < P; ++i) {
                const int l = i ^ (1 << jj);
                if (l > i) {
                    const double a = v[i], b = v[l];
                    const bool swap = ((i >> kk) & 1) == 0 ? (a > b) : (a < b);
                    v[i] = swap ? b : a;
                    v[l] = swap ? a : b;
                }
            }
        }
    }
}

/* one testable bin's statistic, threshold and hit. OSMAX > 0: the OS
 * statistic over at most OSMAX cells: up to 32 sorted in registers (padded
 * with +inf, which sorts after every cell), more gathered into a local array
 * and selected. */
template <int OSMAX>
__device__ __forceinline__ bool cell_test(long long i, long long row, long long nbins, int mode, int n_ref, int N,
                                          int os_k, double alpha, double alpha_ca, double et,
                                          const uint8_t *__restrict__ sided, const int32_t *__restrict__ idx,
                                          const double *__restrict__ X, double *__restrict__ noise,
                                          double *__restrict__ thr) {
    const double *Xr = X + row;
    double Z, a = alpha, scale = et;
    if constexpr (OSMAX == 32) {
        /* the os_k-th smallest; a NaN among the cells makes T NaN */
        double v[32];
        bool has_nan = false;
#pragma unroll
        for (int q = 0; q < 32; ++q) {
            v[q] = q < N ? Xr[idx[(long long)q * nbins + i]] : CUDART_INF;
            has_nan |= isnan(v[q]);
        }
        bitonic_sort<5>(v);
        /* v[os_k - 1] by masks, not an index: a runtime index would move v
         * to local memory */
        unsigned long long pick = 0;
#pragma unroll
        for (int q = 0; q < 32; ++q)
            pick |= (unsigned long long)__double_as_longlong(v[q]) & (0ull - (unsigned long long)(q == os_k - 1));
        Z = has_nan ? CUDART_NAN : __longlong_as_double((long long)pick);
    } else if constexpr (OSMAX > 0) {
        double v[OSMAX];
        bool has_nan = false;
        for (int q = 0; q < N; ++q) {
            v[q] = Xr[idx[(long long)q * nbins + i]];
            has_nan |= isnan(v[q]);
        }
        Z = has_nan ? CUDART_NAN : select_kth(v, N, os_k - 1);
    } else if ((mode == 2 || mode == 3) && sided[i]) {
        double L = 0.0, R = 0.0;
        for (int q = 0; q < n_ref; ++q) L = __dadd_rn(L, Xr[idx[(long long)q * nbins + i]]);
        for (int q = n_ref; q < N; ++q) R = __dadd_rn(R, Xr[idx[(long long)q * nbins + i]]);
        L = __ddiv_rn(L, (double)n_ref);
        R = __ddiv_rn(R, (double)n_ref);
        if (isnan(L) || isnan(R)) Z = CUDART_NAN;
        else Z = mode == 2 ? (L > R ? L : R) : (L < R ? L : R);
    } else {
        double s = 0.0;
        for (int q = 0; q < N; ++q) s = __dadd_rn(s, Xr[idx[(long long)q * nbins + i]]);
        Z = __ddiv_rn(s, (double)N);
        if (mode == 2 || mode == 3) {
            a = alpha_ca;
            scale = 1.0;
        }
    }
    const double t = __dmul_rn(a, Z);
    thr[row + i] = t;
    noise[row + i] = __ddiv_rn(Z, scale);
    return Xr[i] > t;
}

template <int OSMAX>
__global__ void __launch_bounds__(kThreads) cfar_cell_kernel(long long f0, long long t0, long long nbins, int mode,
                                                             int n_ref, int N, int os_k, double alpha,
                                                             double alpha_ca, double et,
                                                             const uint8_t *__restrict__ ok,
                                                             const uint8_t *__restrict__ sided,
                                                             const int32_t *__restrict__ idx,
                                                             const double *__restrict__ X,
                                                             double *__restrict__ noise, double *__restrict__ thr,
                                                             uint8_t *__restrict__ hits, uint32_t *__restrict__ bits,
                                                             long long words) {
    const long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
    const long long f = t0 - f0 + blockIdx.y;
    const long long row = f * nbins;
    bool hit = false;
    if (i < nbins && !ok[i]) {
        noise[row + i] = CUDART_NAN;
        thr[row + i] = CUDART_NAN;
        hits[row + i] = 0;
    } else if (i < nbins) {
        hit = cell_test<OSMAX>(i, row, nbins, mode, n_ref, N, os_k, alpha, alpha_ca, et, sided, idx, X, noise, thr);
        hits[row + i] = hit;
    }
    /* the row as a bitmask too: bin i is bit i % 32 of word i / 32 */
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if ((threadIdx.x & 31) == 0 && (i >> 5) < words) bits[f * words + (i >> 5)] = m;
}



/* a pass's rows at its columns: rows of X and noise (row r of X / noise to
 * row r of Xc / Nc), then nraw raw rows from frame rf0 on (to Rc) */
__global__ void __launch_bounds__(kThreads) cfar_gather_kernel(const double *__restrict__ X,
                                                               const double *__restrict__ noise, long long nbins,
                                                               int rows, const double *__restrict__ raw, int ring,
                                                               long long rf0, int nraw,
                                                               const int32_t *__restrict__ cols, int ncol,
                                                               double *__restrict__ Xc, double *__restrict__ Nc,
                                                               double *__restrict__ Rc) {
    const long long total = (long long)(rows + nraw) * ncol;
    for (long long e = (long long)blockIdx.x * kThreads + threadIdx.x; e < total;
         e += (long long)gridDim.x * kThreads) {
        const long long r = e / ncol, q = e - r * ncol;
        const long long b = cols[q];
        if (r < rows) {
            Xc[e] = X[r * nbins + b];
            Nc[e] = noise[r * nbins + b];
        } else {
            const long long rr = r - rows;
            Rc[rr * ncol + q] = raw[((rf0 + rr) % ring) * nbins + b];
        }
    }
}

int grid_for(long long work) {
    long long g = (work + kThreads - 1) / kThreads;
    return (int)(g < 148LL * 16 ? (g < 1 ? 1 : g) : 148LL * 16);
}

}  // namespace

extern "C" int atkb_cfar_raw(const float *frames, int units, long long f0, int nf, long long nbins, double *raw,
                             int ring, void *stream) {
    if (nf <= 0) return ATKB_OK;
    cfar_raw_kernel<<<grid_for((long long)nf * nbins), kThreads, 0, (cudaStream_t)stream>>>(frames, units, f0, nf,
                                                                                             nbins, raw, ring);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" int atkb_cfar_test(const double *raw, int ring, long long f0, long long t0, int nf, long long nbins,
                              int k, int mode, int n_ref, int n_cells, int os_k, double alpha, double alpha_ca,
                              double et, const uint8_t *ok, const uint8_t *sided, const int32_t *idx, double *X,
                              double *noise, double *thr, uint8_t *hits, uint32_t *bits, long long words,
                              void *stream) {
    const long long ntest = f0 + nf - t0;
    if (ntest <= 0) return ATKB_OK;
    if (ntest > 65535 || nbins <= 0) return ATKB_E_ARG;
    const dim3 grid((unsigned)((nbins + kThreads - 1) / kThreads), (unsigned)ntest);
    cudaStream_t s = (cudaStream_t)stream;
    cfar_mean_kernel<<<grid, kThreads, 0, s>>>(raw, ring, f0, t0, nbins, k, X);
    if (mode != 1)
        cfar_cell_kernel<0><<<grid, kThreads, 0, s>>>(f0, t0, nbins, mode, n_ref, n_cells, os_k, alpha, alpha_ca, et,
                                                      ok, sided, idx, X, noise, thr, hits, bits, words);
    else if (n_cells <= 32)
        cfar_cell_kernel<32><<<grid, kThreads, 0, s>>>(f0, t0, nbins, mode, n_ref, n_cells, os_k, alpha, alpha_ca, et,
                                                       ok, sided, idx, X, noise, thr, hits, bits, words);
    else if (n_cells <= 64)
        cfar_cell_kernel<64><<<grid, kThreads, 0, s>>>(f0, t0, nbins, mode, n_ref, n_cells, os_k, alpha, alpha_ca, et,
                                                       ok, sided, idx, X, noise, thr, hits, bits, words);
    else if (n_cells <= 512)
        cfar_cell_kernel<512><<<grid, kThreads, 0, s>>>(f0, t0, nbins, mode, n_ref, n_cells, os_k, alpha, alpha_ca,
                                                        et, ok, sided, idx, X, noise, thr, hits, bits, words);
    else
        return ATKB_E_ARG;
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" int atkb_cfar_gather(const double *X, const double *noise, long long nbins, int rows, const double *raw,
                                int ring, long long rf0, int nraw, const int32_t *cols, int ncol, double *Xc,
                                double *Nc, double *Rc, void *stream) {
    if (ncol <= 0 || rows + nraw <= 0) return ATKB_OK;
    cfar_gather_kernel<<<grid_for((long long)(rows + nraw) * ncol), kThreads, 0, (cudaStream_t)stream>>>(
        X, noise, nbins, rows, raw, ring, rf0, nraw, cols, ncol, Xc, Nc, Rc);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}
