/* Shared-memory complex FFTs in double for the sm_100a kernels of the
 * overlap-save extractor and the spectrum reduction: batched in-place
 * Stockham transforms of power-of-two lengths by a warp or a whole CTA. */
#ifndef ATKB_FFT_SM_CUH
#define ATKB_FFT_SM_CUH

#include <cuda_runtime.h>

namespace atkb_fft {

__device__ __forceinline__ double2 d2add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 d2sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 d2mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

/* W^j of the nfft-point table, read at stride 2^sh for a shorter transform;
 * conjugated for the inverse */
__device__ __forceinline__ double2 tw_at(const double2 *tw, int j, int sh, bool inv) {
    double2 w = __ldg(tw + ((size_t)j << sh));
    if (inv) w.y = -w.y;
    return w;
}

/* 4-point DFT in place; the inverse swaps the roles of -i and +i */
__device__ __forceinline__ void dft4(double2 *v, bool inv) {
    const double2 s02 = d2add(v[0], v[2]), d02 = d2sub(v[0], v[2]);
    const double2 s13 = d2add(v[1], v[3]), d13 = d2sub(v[1], v[3]);
    const double2 r = inv ? make_double2(-d13.y, d13.x) : make_double2(d13.y, -d13.x);  /* -+i d13 */
    v[0] = d2add(s02, s13);
    v[2] = d2sub(s02, s13);
    v[1] = d2add(d02, r);
    v[3] = d2sub(d02, r);
}

/* a barrier of the NTH threads of a transform: a warp or the CTA */
template <int NTH>
__device__ __forceinline__ void fft_sync() {
    if (NTH == 32) __syncwarp();
    else __syncthreads();
}

/* Batched in-place Stockham transforms by NTH threads (a warp or the CTA):
 * nb transforms of n = 2^logn points at sm + b*n, natural order in and out,
 * nb*n <= 8*NTH. Each pass reads every value a thread needs into registers,
 * then all write after a barrier (radix 4, after one radix-2 pass when
 * log2 n is odd). Twiddles come from the nfft-point table (lognfft) at the
 * stride that gives this length's roots. Ends with a barrier. */
template <int NTH>
__device__ void fft_b(double2 *sm, int logn, int nb, const double2 *__restrict__ tw, int lognfft, bool inv,
                      int tid) {
    const int n = 1 << logn;
    int lg = 0;                                /* log2 of the finished sub-length Ns */
    if (logn & 1) {                            /* radix 2 with Ns = 1: no twiddles */
        const int h = n >> 1, tot = nb * h;
        double2 a[4], c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int T = tid + u * NTH;
            if (T < tot) {
                const int base = (T >> (logn - 1)) << logn, t = T & (h - 1);
                a[u] = sm[base + t];
                c[u] = sm[base + t + h];
            }
        }
        fft_sync<NTH>();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int T = tid + u * NTH;
            if (T < tot) {
                const int base = (T >> (logn - 1)) << logn, t = T & (h - 1);
                sm[base + 2 * t] = d2add(a[u], c[u]);
                sm[base + 2 * t + 1] = d2sub(a[u], c[u]);
            }
        }
        fft_sync<NTH>();
        lg = 1;
    }
    const int q = n >> 2, totq = nb * q;
    for (; lg < logn; lg += 2) {
        const int Ns = 1 << lg;
        const int sh = lognfft - lg - 2;       /* W_{4 Ns}^j = W_nfft^(j << sh) */
        double2 v[2][4];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int T = tid + u * NTH;
            if (T < totq) {
                const int base = (T >> (logn - 2)) << logn, t = T & (q - 1), k = t & (Ns - 1);
#pragma unroll
                for (int r = 0; r < 4; ++r) v[u][r] = sm[base + t + r * q];
                if (lg) {
#pragma unroll
                    for (int r = 1; r < 4; ++r) v[u][r] = d2mul(v[u][r], tw_at(tw, r * k, sh, inv));
                }
                dft4(v[u], inv);
            }
        }
        fft_sync<NTH>();
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int T = tid + u * NTH;
            if (T < totq) {
                const int base = (T >> (logn - 2)) << logn, t = T & (q - 1), k = t & (Ns - 1);
                const int o = base + ((t >> lg) << (lg + 2)) + k;
#pragma unroll
                for (int r = 0; r < 4; ++r) sm[o + r * Ns] = v[u][r];
            }
        }
        fft_sync<NTH>();
    }
}

/* bin k of a channel's decimating fold of one spectrum (float, j ascending,
 * the reference's rounded expression, src/channelizer.c:707-716). The bins
 * k + j*M + shift run up to nfft and then wrap once: two runs, each a
 * fixed stride (M is a template parameter, so the unrolled loads carry it
 * as an immediate offset). SM: the spectrum is the fused kernel's shared
 * one, bin b of this block at shared address xs + b * 8 * OSX_G; else
 * global, bin b at X[b]. */
}  // namespace atkb_fft

#endif
