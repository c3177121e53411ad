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
 * Work split inside a CTA: P = nel(nel+1)/2 pairs; threads are (pair, lane
 * group) so that small arrays still use every thread; the block of hops is
 * staged through shared memory in chunks of CHUNK hops.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "internal.h"

#define W_NT 256
#define CHUNK 64
#define MAX_NEL 32

namespace {

__global__ void __launch_bounds__(W_NT)
w12_kernel(const float2 *__restrict__ out, int nel, int nchan, long long m,
           const uint8_t *__restrict__ gate, float2 *__restrict__ R, uint32_t *__restrict__ counts,
           float *__restrict__ pwr, float *__restrict__ mean_pwr) {
    __shared__ float2 ys[MAX_NEL][CHUNK];
    __shared__ double red[W_NT][2];
    __shared__ double diag[MAX_NEL];
    const int P = nel * (nel + 1) / 2;
    for (int k = blockIdx.x; k < nchan; k += gridDim.x) {
        const bool w1 = R && counts && (!gate || gate[k]);
        const bool w2 = pwr || mean_pwr;
        if (!w1 && !w2) continue;
        /* pairs this thread owns: p = tid % P_eff + j * W_NT ...; lane group g */
        const int groups = P >= W_NT ? 1 : W_NT / P;
        const int tpair = threadIdx.x % (P >= W_NT ? W_NT : P);
        const int g = P >= W_NT ? 0 : threadIdx.x / P;
        const bool active = g < groups && (P >= W_NT || threadIdx.x < groups * P);
        double sr[4] = {0, 0, 0, 0}, si[4] = {0, 0, 0, 0};
        int pa[4], pb[4], np = 0;
        for (int p = tpair; p < P && np < 4; p += (P >= W_NT ? W_NT : P), ++np) {
            /* p -> (a, b), a <= b, row-major over the upper triangle */
            int a = 0, rem = p;
            while (rem >= nel - a) { rem -= nel - a; ++a; }
            pa[np] = a; pb[np] = a + rem;
        }
        for (long long i0 = 0; i0 < m; i0 += CHUNK) {
            const int cnt = (int)((m - i0) < CHUNK ? (m - i0) : CHUNK);
            for (int e = threadIdx.x; e < nel * CHUNK; e += W_NT) {
                const int a = e / CHUNK, i = e - a * CHUNK;
                ys[a][i] = i < cnt ? out[((long long)a * nchan + k) * m + i0 + i] : make_float2(0.f, 0.f);
            }
            __syncthreads();
            if (active) {
                for (int q = 0; q < np; ++q) {
                    const bool need = w1 || pa[q] == pb[q];
                    if (!need) continue;
                    const int a = pa[q], b = pb[q];
                    for (int i = g; i < cnt; i += groups) {
                        const float2 ya = ys[a][i], yb = ys[b][i];
                        sr[q] += (double)ya.x * yb.x + (double)ya.y * yb.y;
                        si[q] += (double)ya.y * yb.x - (double)ya.x * yb.y;
                    }
                }
            }
            __syncthreads();
        }
        /* reduce over lane groups (fixed order), pair by pair */
        for (int q = 0; q < 4; ++q) {
            red[threadIdx.x][0] = (active && q < np) ? sr[q] : 0.0;
            red[threadIdx.x][1] = (active && q < np) ? si[q] : 0.0;
            __syncthreads();
            if (active && q < np && g == 0) {
                double tr = 0.0, ti = 0.0;
                for (int gg = 0; gg < groups; ++gg) {
                    tr += red[gg * (P >= W_NT ? W_NT : P) + tpair][0];
                    ti += red[gg * (P >= W_NT ? W_NT : P) + tpair][1];
                }
                const int a = pa[q], b = pb[q];
                if (a == b) diag[a] = tr;
                if (w1 && m > 0) {
                    float2 *Rk = R + (long long)k * nel * nel;
                    float2 r = Rk[a * nel + b];
                    Rk[a * nel + b] = make_float2((float)((double)r.x + tr), (float)((double)r.y + ti));
                    if (a != b) {
                        r = Rk[b * nel + a];
                        Rk[b * nel + a] = make_float2((float)((double)r.x + tr), (float)((double)r.y - ti));
                    }
                }
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
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

}  // namespace

extern "C" int atkb_w12(const void *out, unsigned nel, unsigned nchan, size_t m, const uint8_t *gate,
                        void *R, uint32_t *counts, float *pwr, float *mean_pwr, void *stream) {
    if (nel < 1 || nel > MAX_NEL || nchan < 1) return ATKB_E_ARG;
    int grid = (int)(nchan < 4096 ? nchan : 4096);
    w12_kernel<<<grid, W_NT, 0, (cudaStream_t)stream>>>((const float2 *)out, (int)nel, (int)nchan,
                                                        (long long)m, gate, (float2 *)R, counts, pwr,
                                                        mean_pwr);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
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
