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

/* ---- radix-8 transforms in a swizzled layout --------------------------------
 * Element p of a transform lives at sm[swz(p)]: the low 3 index bits XORed
 * with the next 3, so the stride-8 stores of a radix-8 pass and the
 * unit-stride loads both spread over distinct 16-byte slots of a wavefront. */
__device__ __forceinline__ int swz(int i) { return i ^ ((i >> 3) & 7); }

__device__ __forceinline__ double2 d2sq(double2 a) { return make_double2(a.x * a.x - a.y * a.y, 2.0 * a.x * a.y); }

/* 8-point DFT in place (two 4-point DFTs and the W8 twiddles); the inverse
 * conjugates every root */
__device__ __forceinline__ void dft8(double2 *v, bool inv) {
    const double h = 0.70710678118654752440;   /* sqrt(1/2) */
    double2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft4(e, inv);
    dft4(o, inv);
    /* W8^1 = (1 -+ i) h, W8^2 = -+ i, W8^3 = (-1 -+ i) h */
    const double s = inv ? 1.0 : -1.0;
    const double2 t1 = make_double2((o[1].x - s * o[1].y) * h, (o[1].y + s * o[1].x) * h);
    const double2 t2 = make_double2(-s * o[2].y, s * o[2].x);
    const double2 t3 = make_double2((-o[3].x - s * o[3].y) * h, (-o[3].y + s * o[3].x) * h);
    v[0] = d2add(e[0], o[0]);
    v[4] = d2sub(e[0], o[0]);
    v[1] = d2add(e[1], t1);
    v[5] = d2sub(e[1], t1);
    v[2] = d2add(e[2], t2);
    v[6] = d2sub(e[2], t2);
    v[3] = d2add(e[3], t3);
    v[7] = d2sub(e[3], t3);
}

/* One transform of n = 2^logn points (8 <= n <= 8*NTH) in the swizzled
 * layout by NTH threads, natural order in and out: radix-8 Stockham passes,
 * then one radix-4 or radix-2 pass for the bits left. A butterfly's
 * twiddles W^(r k), r = 1..7, come from one table entry W^k (the nfft-point
 * table at the stride of this pass) and its powers by multiplication, each
 * at most three roundings from the exact root. Ends with a barrier. */
template <int NTH>
__device__ void fft_r8(double2 *sm, int logn, const double2 *__restrict__ tw, int lognfft, bool inv, int tid) {
    const int n = 1 << logn;
    int lg = 0;
    for (; logn - lg >= 3; lg += 3) {
        const int Ns = 1 << lg, q = n >> 3, sh = lognfft - lg - 3;
        double2 v[8];
        const int t = tid;
        const bool on = t < q;                 /* n <= 8*NTH: one butterfly per thread */
        int k = 0;
        if (on) {
            k = t & (Ns - 1);
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = sm[swz(t + r * q)];
            if (lg) {
                double2 w[8];
                w[1] = tw_at(tw, k, sh, inv);
                w[2] = d2sq(w[1]);
                w[3] = d2mul(w[2], w[1]);
                w[4] = d2sq(w[2]);
                w[5] = d2mul(w[4], w[1]);
                w[6] = d2sq(w[3]);
                w[7] = d2mul(w[4], w[3]);
#pragma unroll
                for (int r = 1; r < 8; ++r) v[r] = d2mul(v[r], w[r]);
            }
            dft8(v, inv);
        }
        __syncthreads();
        if (on) {
            const int o = ((t >> lg) << (lg + 3)) + k;
#pragma unroll
            for (int r = 0; r < 8; ++r) sm[swz(o + r * Ns)] = v[r];
        }
        __syncthreads();
    }
    if (logn - lg == 2) {                      /* a radix-4 pass for the last two bits */
        const int Ns = 1 << lg, q = n >> 2, sh = lognfft - lg - 2;
        double2 v[2][4];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = tid + u * NTH;
            if (t < q) {
                const int k = t & (Ns - 1);
#pragma unroll
                for (int r = 0; r < 4; ++r) v[u][r] = sm[swz(t + r * q)];
                if (lg) {
#pragma unroll
                    for (int r = 1; r < 4; ++r) v[u][r] = d2mul(v[u][r], tw_at(tw, r * k, sh, inv));
                }
                dft4(v[u], inv);
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = tid + u * NTH;
            if (t < q) {
                const int k = t & (Ns - 1), o = ((t >> lg) << (lg + 2)) + k;
#pragma unroll
                for (int r = 0; r < 4; ++r) sm[swz(o + r * Ns)] = v[u][r];
            }
        }
        __syncthreads();
    } else if (logn - lg == 1) {               /* ... or a radix-2 pass for the last bit */
        const int Ns = 1 << lg, q = n >> 1, sh = lognfft - lg - 1;
        double2 a[4], c[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = tid + u * NTH;
            if (t < q) {
                const int k = t & (Ns - 1);
                a[u] = sm[swz(t)];
                c[u] = sm[swz(t + q)];
                if (lg) c[u] = d2mul(c[u], tw_at(tw, k, sh, inv));
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int t = tid + u * NTH;
            if (t < q) {
                const int k = t & (Ns - 1), o = ((t >> lg) << (lg + 1)) + k;
                sm[swz(o)] = d2add(a[u], c[u]);
                sm[swz(o + Ns)] = d2sub(a[u], c[u]);
            }
        }
        __syncthreads();
    }
}

}  // namespace atkb_fft

#endif
