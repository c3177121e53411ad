/* W1 (per-channel covariance) and W2 (per-channel power) on sm_100a,
 * reference src/channelizer.c:419-471.
 *
 * Input: a channel-major element-array block out[nel][nchan][m] in device
 * memory. One CTA per channel k (grid-stride over channels):
 *   S_ab = sum_i y_a(i) conj(y_b(i))   in double, for a <= b
 *   W1:  R[k][a][b] += S_ab, R[k][b][a] += conj(S_ab)   (gated channels only;
 *        each entry is added in double and rounded once to float)
 *        counts[k] += m
 *   W2:  pwr[a][k] = (float)(S_aa / m); mean_pwr[k] = (float)(sum_a S_aa/m / nel)
 * The reference accumulates W1 serially in float and W2 serially in double;
 * here every sum is double, reduced in a fixed order, so the results are
 * deterministic and at least as accurate.
 *
 * Work split inside a CTA: the upper triangle of the nel x nel matrix is cut
 * into TB x TB tiles (TB = 1, 2 or 4 by nel), and the threads into (tile, hop
 * group) pairs: each thread keeps a tile's TB*TB sums in registers over its
 * share of the hops, so one hop's 2*TB loads feed TB*TB products (the old
 * one-pair-per-thread split loaded both operands for every product). The
 * block of hops is staged through shared memory in chunks of CHUNK hops
 * (2048 for one element, 256 otherwise), rows only for the elements present,
 * double-buffered: the next chunk's asynchronous copies (cp.async) fly while
 * the current one is summed. The hop groups' partial sums are then added in
 * group order, so the results are deterministic.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include "internal.h"

#define W_NT 256
/* hops per staged chunk: one element's rows are short, so it takes longer
 * chunks (more hops per thread between barriers) */
template <int TB>
struct chunk_of { static constexpr int value = TB == 1 ? 2048 : 256; };
#define MAX_NEL 32

namespace {

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

template <int TB, int CHUNK = chunk_of<TB>::value>
__global__ void __launch_bounds__(W_NT)
w12_kernel(const float2 *__restrict__ out, int nel, int nchan, long long m,
           const uint8_t *__restrict__ gate, float2 *__restrict__ R, uint32_t *__restrict__ counts,
           float *__restrict__ pwr, float *__restrict__ mean_pwr) {
    __shared__ double diag[MAX_NEL];
    /* dynamic: the groups' partial sums [W_NT][TB*TB][2], then the two
     * staging buffers [2][rows][CHUNK] of the hop chunks */
    extern __shared__ double red[];
    const int nb = (nel + TB - 1) / TB;
    const int rows = nb * TB;
    float2 *ys = (float2 *)(red + (size_t)W_NT * TB * TB * 2);
    const int T = nb * (nb + 1) / 2;           /* tiles of the upper triangle */
    const int groups = T >= W_NT ? 1 : W_NT / T;
    const int tid = threadIdx.x;
    const int tile = tid % T, g = tid / T;
    const bool active = g < groups;
    /* tile -> (A, B), A <= B, row-major over the upper triangle of tiles */
    int A = 0, rem = tile;
    while (rem >= nb - A) { rem -= nb - A; ++A; }
    const int B = A + rem;
    for (int k = blockIdx.x; k < nchan; k += gridDim.x) {
        const bool w1 = R && counts && (!gate || gate[k]);
        const bool w2 = pwr || mean_pwr;
        if (!w1 && !w2) continue;
        double sr[TB][TB], si[TB][TB];
#pragma unroll
        for (int r = 0; r < TB; ++r)
#pragma unroll
            for (int c = 0; c < TB; ++c) sr[r][c] = si[r][c] = 0.0;
        /* chunk c's hops into buffer c & 1: copies for real samples, zeros
         * for the padding rows and the tail */
        auto stage = [&](long long i0, int buf) {
            const int cnt = (int)((m - i0) < CHUNK ? (m - i0) : CHUNK);
            for (int e = tid; e < nb * TB * CHUNK; e += W_NT) {
                const int a = e / CHUNK, i = e - a * CHUNK;
                float2 *dst = ys + ((size_t)buf * rows + a) * CHUNK + i;
                if (a < nel && i < cnt) cp_async8(dst, out + ((long long)a * nchan + k) * m + i0 + i);
                else *dst = make_float2(0.f, 0.f);
            }
            cp_async_commit();
        };
        if (m > 0) stage(0, 0);
        for (long long i0 = 0, c = 0; i0 < m; i0 += CHUNK, ++c) {
            const int cnt = (int)((m - i0) < CHUNK ? (m - i0) : CHUNK);
            const int buf = (int)(c & 1);
            if (i0 + CHUNK < m) {
                stage(i0 + CHUNK, buf ^ 1);
                cp_async_wait<1>();            /* this chunk's group has landed */
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
            if (active && (w1 || A == B)) {
                for (int i = g; i < cnt; i += groups) {
                    float2 ya[TB], yb[TB];
                    const float2 *yc = ys + (size_t)buf * rows * CHUNK;
#pragma unroll
                    for (int r = 0; r < TB; ++r) {
                        ya[r] = yc[(A * TB + r) * CHUNK + i];
                        yb[r] = yc[(B * TB + r) * CHUNK + i];
                    }
#pragma unroll
                    for (int r = 0; r < TB; ++r)
#pragma unroll
                        for (int c = 0; c < TB; ++c) {
                            sr[r][c] += (double)ya[r].x * yb[c].x + (double)ya[r].y * yb[c].y;
                            si[r][c] += (double)ya[r].y * yb[c].x - (double)ya[r].x * yb[c].y;
                        }
                }
            }
            __syncthreads();
        }
        /* the groups' partials, then each tile entry summed over groups in order */
        double *mine = red + (size_t)tid * TB * TB * 2;
#pragma unroll
        for (int r = 0; r < TB; ++r)
#pragma unroll
            for (int c = 0; c < TB; ++c) {
                mine[2 * (r * TB + c)] = active ? sr[r][c] : 0.0;
                mine[2 * (r * TB + c) + 1] = active ? si[r][c] : 0.0;
            }
        __syncthreads();
        for (int idx = tid; idx < T * TB * TB; idx += W_NT) {
            const int t = idx / (TB * TB), e = idx - t * TB * TB;
            const int r = e / TB, c = e - r * TB;
            int tA = 0, trem = t;
            while (trem >= nb - tA) { trem -= nb - tA; ++tA; }
            const int a = tA * TB + r, b = (tA + trem) * TB + c;
            if (a >= nel || b >= nel || a > b) continue;
            double tr = 0.0, ti = 0.0;
            for (int gg = 0; gg < groups; ++gg) {
                const double *p = red + (size_t)(gg * T + t) * TB * TB * 2;
                tr += p[2 * e];
                ti += p[2 * e + 1];
            }
            if (a == b) diag[a] = tr;
            if (w1 && m > 0) {
                float2 *Rk = R + (long long)k * nel * nel;
                float2 v = Rk[a * nel + b];
                Rk[a * nel + b] = make_float2((float)((double)v.x + tr), (float)((double)v.y + ti));
                if (a != b) {
                    v = Rk[b * nel + a];
                    Rk[b * nel + a] = make_float2((float)((double)v.x + tr), (float)((double)v.y - ti));
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            if (w1) counts[k] += (uint32_t)m;
            if (w2) {
                const double inv = m ? 1.0 / (double)m : 0.0;
                double across = 0.0;
                for (int a = 0; a < nel; ++a) {
                    if (pwr) pwr[(long long)a * nchan + k] = (float)(diag[a] * inv);
                    across += diag[a] * inv;
                }
                if (mean_pwr) mean_pwr[k] = (float)(across / (double)nel);
            }
        }
        __syncthreads();
    }
}

/* W1 / W2 for arrays wider than MAX_NEL elements: one CTA per channel, one
 * thread per (a, b) pair of the upper triangle (grid-stride), each summing
 * its pair over the hops in hop order, in double, straight from global
 * memory (a thread's loads of element a and b are strided by nchan*m, so
 * this path trades bandwidth for generality; wide arrays are rare). The
 * diagonal sums land in shared memory (nel doubles, dynamic) for W2. Same
 * results as the tiled kernel's: every sum in double, rounded once. */
__global__ void __launch_bounds__(W_NT)
w12_wide_kernel(const float2 *__restrict__ out, int nel, int nchan, long long m,
                const uint8_t *__restrict__ gate, float2 *__restrict__ R, uint32_t *__restrict__ counts,
                float *__restrict__ pwr, float *__restrict__ mean_pwr) {
    extern __shared__ double wdiag[];
    const long long pairs = (long long)nel * (nel + 1) / 2;
    for (int k = blockIdx.x; k < nchan; k += gridDim.x) {
        const bool w1 = R && counts && (!gate || gate[k]);
        const bool w2 = pwr || mean_pwr;
        if (!w1 && !w2) continue;
        for (long long t = threadIdx.x; t < pairs; t += W_NT) {
            int a = 0;
            long long rem = t;
            while (rem >= nel - a) { rem -= nel - a; ++a; }
            const int b = a + (int)rem;
            if (!w1 && a != b) continue;
            const float2 *ya = out + ((long long)a * nchan + k) * m;
            const float2 *yb = out + ((long long)b * nchan + k) * m;
            double tr = 0.0, ti = 0.0;
            for (long long i = 0; i < m; ++i) {
                const float2 u = __ldg(ya + i), v = __ldg(yb + i);
                tr += (double)u.x * v.x + (double)u.y * v.y;
                ti += (double)u.y * v.x - (double)u.x * v.y;
            }
            if (a == b) wdiag[a] = tr;
            if (w1 && m > 0) {
                float2 *Rk = R + (long long)k * nel * nel;
                float2 q = Rk[(long long)a * nel + b];
                Rk[(long long)a * nel + b] = make_float2((float)((double)q.x + tr), (float)((double)q.y + ti));
                if (a != b) {
                    q = Rk[(long long)b * nel + a];
                    Rk[(long long)b * nel + a] = make_float2((float)((double)q.x + tr), (float)((double)q.y - ti));
                }
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (w1) counts[k] += (uint32_t)m;
            if (w2) {
                const double inv = m ? 1.0 / (double)m : 0.0;
                double across = 0.0;
                for (int a = 0; a < nel; ++a) {
                    if (pwr) pwr[(long long)a * nchan + k] = (float)(wdiag[a] * inv);
                    across += wdiag[a] * inv;
                }
                if (mean_pwr) mean_pwr[k] = (float)(across / (double)nel);
            }
        }
        __syncthreads();
    }
}

__global__ void cov_reset_kernel(float2 *R, uint32_t *counts, int nel, int nchan,
                                 const uint8_t *__restrict__ gate) {
    const long long per = (long long)nel * nel;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < per * nchan;
         e += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(e / per);
        if (gate && !gate[k]) continue;
        R[e] = make_float2(0.f, 0.f);
        if (e % per == 0) counts[k] = 0;
    }
}


template <int TB>
int w12_launch(const void *out, unsigned nel, unsigned nchan, size_t m, const uint8_t *gate, void *R,
               uint32_t *counts, float *pwr, float *mean_pwr, cudaStream_t s) {
    /* the attribute is idempotent: concurrent first callers may both set it */
    static std::atomic<bool> configured[64];
    constexpr int CHUNK = chunk_of<TB>::value;
    const size_t red = (size_t)W_NT * TB * TB * 2 * sizeof(double);
    const size_t rows = ((nel + TB - 1) / TB) * TB;
    const size_t smem = red + 2 * rows * CHUNK * sizeof(float2);
    /* TB 1 and 2 serve one and two elements (atkb_w12), TB 4 up to MAX_NEL */
    constexpr size_t rows_max = TB == 4 ? MAX_NEL : TB;
    constexpr size_t smem_max = (size_t)W_NT * TB * TB * 2 * sizeof(double) + 2 * rows_max * CHUNK * sizeof(float2);
    static_assert(smem_max <= 227 * 1024, "one CTA's shared memory fits an SM");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ATKB_E_NODEV;
    if (!configured[dev].load(std::memory_order_acquire)) {
        if (cudaFuncSetAttribute(w12_kernel<TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max) !=
            cudaSuccess)
            return ATKB_E_KERNEL;
        configured[dev].store(true, std::memory_order_release);
    }
    const int grid = (int)(nchan < 4096 ? nchan : 4096);
    w12_kernel<TB><<<grid, W_NT, smem, s>>>((const float2 *)out, (int)nel, (int)nchan, (long long)m, gate,
                                            (float2 *)R, counts, pwr, mean_pwr);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

}  // namespace

extern "C" int atkb_w12(const void *out, unsigned nel, unsigned nchan, size_t m, const uint8_t *gate,
                        void *R, uint32_t *counts, float *pwr, float *mean_pwr, void *stream) {
    if (nel < 1 || nchan < 1) return ATKB_E_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (nel > MAX_NEL) {
        const size_t smem = (size_t)nel * sizeof(double);
        if (smem > 48 * 1024) return ATKB_E_ARG;          /* 6144 elements */
        const int grid = (int)(nchan < 4096 ? nchan : 4096);
        w12_wide_kernel<<<grid, W_NT, smem, s>>>((const float2 *)out, (int)nel, (int)nchan, (long long)m, gate,
                                                 (float2 *)R, counts, pwr, mean_pwr);
        return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
    }
    if (nel == 1) return w12_launch<1>(out, nel, nchan, m, gate, R, counts, pwr, mean_pwr, s);
    if (nel == 2) return w12_launch<2>(out, nel, nchan, m, gate, R, counts, pwr, mean_pwr, s);
    return w12_launch<4>(out, nel, nchan, m, gate, R, counts, pwr, mean_pwr, s);
}

extern "C" int atkb_cov_reset(void *R, uint32_t *counts, unsigned nel, unsigned nchan,
                              const uint8_t *gate, void *stream) {
    const long long total = (long long)nel * nel * nchan;
    int grid = (int)((total + 255) / 256);
    if (grid > 4096) grid = 4096;
    if (grid < 1) grid = 1;
    cov_reset_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>((float2 *)R, counts, (int)nel, (int)nchan,
                                                             gate);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}
