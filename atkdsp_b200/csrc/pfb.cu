/* The polyphase filterbank on sm_100a.
 *
 * What one hop computes (reference src/channelizer.c:235-292):
 *   window   w = s[h*hop, h*hop + L),  s = history ++ leftover ++ input
 *   fold     f[q] = sum_{k ascending} taps[k*M + q] * w[k*M + q]   (float,
 *            one rounded multiply then one rounded add per tap -- the
 *            reference's pinned C99 build does exactly this, so the fold is
 *            bit-identical)
 *   FFT      X = DFT_M(f) in DOUBLE (the reference runs pocketfft in double;
 *            a float FFT misses the 1e-5 per-channel bar at M >= 1024)
 *   rotate   y[k] = X[k] * twd[(-k*shift) mod M], shift = ((b+1)*hop) mod M,
 *            with the reference's own double table (cos, sin)(2 pi j / M)
 *   cal      y[k] *= cal[k] (double), then one rounding to float
 *   out      channel-major: out[k*ldo + h]
 *
 * Kernel layout (B200-first):
 *   - ONE persistent kernel over a device job list. A job is a run of hops of
 *     one element stream (a handle's element, one stream of a batch, or one
 *     served block); a tile is tile_hops consecutive hops of a job. CTAs
 *     (512 threads, 2 per SM) claim tiles from an atomic counter; warp 0
 *     claims and looks up the next tile while the CTA works on the current
 *     one. CTAs out of tiles copy the state carries (each job's tail into
 *     its other state buffer, which no tile reads). The launch shape is
 *     fixed (CUDA graph friendly) and the counters reset themselves when the
 *     last CTA leaves.
 *   - Fast path (M a power of two, 16..4096): a tile is 4096 complex points
 *     (tile_hops = 4096/M), 512 threads x 8 points. For oversample 1/2/4 and
 *     M <= 2048 each thread folds two consecutive hops over the even or odd
 *     branches (the paired fold: every sample and tap load serves both
 *     hops) into a radix-4 first Stockham pass in registers; otherwise one
 *     hop's 8 branches into a radix-8 first pass. Small M stages the tile
 *     window in shared memory with cp.async first. The FFT runs in double,
 *     radix-8 passes in place in shared memory (XOR swizzle, one twiddle
 *     load per butterfly, group barriers), the last pass fused with the
 *     rotation, cal, rounding and the transpose to channel-major; each
 *     channel gets a run of tile_hops consecutive outputs.
 *   - Generic path (any M >= 2): ping-pong shared buffers, mixed radix
 *     (2, 3, 4, 8, 16 butterflies, direct DFT for any other prime factor).
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include "internal.h"

/* the fast path's tile: 4096 complex points, PTS per thread (ATKB_PTS in
 * internal.h: 8 points -> 512 threads at <= 64 registers, 32 warps per SM) */
#define PTS ATKB_PTS
#define LOGP (PTS == 16 ? 4 : 3)
#define TILE_POINTS 4096
#define NT (TILE_POINTS / PTS)

namespace {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
/* multiply by -i */
__device__ __forceinline__ double2 cmi(double2 a) { return make_double2(a.y, -a.x); }

/* the reference's rotation / cal product: one rounding per multiply and add */
__device__ __forceinline__ double2 cmul_rn(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}

#define C16_1 0.92387953251128675613   /* cos(pi/8) */
#define S16_1 0.38268343236508977173   /* sin(pi/8) */
#define SQH   0.70710678118654752440   /* sqrt(1/2) */

/* forward DFTs, e^{-2 pi i nk/R} */
__device__ __forceinline__ void dft2(double2 &a, double2 &b) {
    const double2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

__device__ __forceinline__ void dft4(double2 &v0, double2 &v1, double2 &v2, double2 &v3) {
    const double2 t0 = cadd(v0, v2), t1 = csub(v0, v2);
    const double2 t2 = cadd(v1, v3), t3 = cmi(csub(v1, v3));
    v0 = cadd(t0, t2);
    v2 = csub(t0, t2);
    v1 = cadd(t1, t3);
    v3 = csub(t1, t3);
}

__device__ __forceinline__ void dft8(double2 *v) {
    /* n = 2 n1 + n2, k = k1 + 4 k2 */
    double2 a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
    double2 b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
    dft4(a0, a1, a2, a3);
    dft4(b0, b1, b2, b3);
    b1 = make_double2(SQH * (b1.x + b1.y), SQH * (b1.y - b1.x));      /* W8^1 */
    b2 = cmi(b2);                                                     /* W8^2 */
    b3 = make_double2(SQH * (b3.y - b3.x), -SQH * (b3.x + b3.y));     /* W8^3 */
    v[0] = cadd(a0, b0); v[4] = csub(a0, b0);
    v[1] = cadd(a1, b1); v[5] = csub(a1, b1);
    v[2] = cadd(a2, b2); v[6] = csub(a2, b2);
    v[3] = cadd(a3, b3); v[7] = csub(a3, b3);
}

__device__ __forceinline__ void dft16(double2 *v) {
    /* n = 4 n1 + n2, k = k1 + 4 k2: radix-4 columns, W16^(n2 k1), radix-4
     * rows, all in place; the rows leave y[k1 + 4 k2] at v[4 k1 + k2], and a
     * final renaming (free once unrolled) restores natural order */
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
    v[4 * 1 + 1] = cmul(v[4 * 1 + 1], make_double2(C16_1, -S16_1));
    v[4 * 2 + 1] = cmul(v[4 * 2 + 1], make_double2(SQH, -SQH));
    v[4 * 3 + 1] = cmul(v[4 * 3 + 1], make_double2(S16_1, -C16_1));
    v[4 * 1 + 2] = cmul(v[4 * 1 + 2], make_double2(SQH, -SQH));
    v[4 * 2 + 2] = cmi(v[4 * 2 + 2]);
    v[4 * 3 + 2] = cmul(v[4 * 3 + 2], make_double2(-SQH, -SQH));
    v[4 * 1 + 3] = cmul(v[4 * 1 + 3], make_double2(S16_1, -C16_1));
    v[4 * 2 + 3] = cmul(v[4 * 2 + 3], make_double2(-SQH, -SQH));
    v[4 * 3 + 3] = cmul(v[4 * 3 + 3], make_double2(-C16_1, S16_1));
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    /* transpose the 4x4 index grid */
    double2 t;
    t = v[1]; v[1] = v[4]; v[4] = t;
    t = v[2]; v[2] = v[8]; v[8] = t;
    t = v[3]; v[3] = v[12]; v[12] = t;
    t = v[6]; v[6] = v[9]; v[9] = t;
    t = v[7]; v[7] = v[13]; v[13] = t;
    t = v[11]; v[11] = v[14]; v[14] = t;
}

__device__ __forceinline__ void dft3(double2 &a, double2 &b, double2 &c) {
    const double S3 = 0.86602540378443864676;   /* sin(2 pi / 3) */
    const double2 s = cadd(b, c), d = csub(b, c);
    const double2 m = make_double2(a.x - 0.5 * s.x, a.y - 0.5 * s.y);
    const double2 r = make_double2(S3 * d.y, -S3 * d.x);  /* -i sin(2pi/3) (b - c) */
    a = cadd(a, s);
    b = cadd(m, r);
    c = csub(m, r);
}

template <int R>
__device__ __forceinline__ void dftR(double2 *v) {
    if (R == 2) dft2(v[0], v[1]);
    else if (R == 4) dft4(v[0], v[1], v[2], v[3]);
    else if (R == 8) dft8(v);
    else if (R == 16) dft16(v);
}

/* Per-thread index checks of the debug build (ATKB_DEBUG_BOUNDS): an index
 * outside its buffer sets a bit of g_atkb_debug_fault and the access is
 * skipped; atkb_pfb_debug_fault reads and clears the word. In the normal
 * build IDX_OK is constant true and costs nothing. */
#ifdef ATKB_DEBUG_BOUNDS
__device__ unsigned g_atkb_debug_fault;
__device__ __forceinline__ bool idx_ok(bool ok) {
    if (!ok) atomicOr(&g_atkb_debug_fault, ATKB_FAULT_INDEX);
    return ok;
}
#define IDX_OK(c) idx_ok(c)
#else
#define IDX_OK(c) true
#endif

/* one element of the stream s = state[0, head) ++ in[0, ...) */
/* int16 I/Q -> cf32 exactly as the unpack front end does, (float(v) - c) * k
 * with rounded operations (reference src/convert.c:64-73), in the fused form
 * the host prepares: nc = -(c * k) with k a power of two, one rounding */
__device__ __forceinline__ float2 conv16(short2 v, float ncre, float ncim, float k) {
    return make_float2(__fmaf_rn((float)v.x, k, ncre), __fmaf_rn((float)v.y, k, ncim));
}

/* one element of the stream s = state[0, head) ++ in[0, ...); `in` is cf32 or
 * raw int16 I/Q converted on the fly */
struct Src {
    const float2 *st;
    const void *in;
    long long head;
    int kind;
    float cre, cim, k;
    __device__ __forceinline__ float2 at(long long i) const {
        if (i < head) return __ldg(st + i);
        if (kind) return conv16(__ldg((const short2 *)in + (i - head)), cre, cim, k);
        return __ldg((const float2 *)in + (i - head));
    }
};

/* The int16 constants from an offset held in device memory (a job's or a
 * carry's doff): atkb_job_conv's -((off / k) * k), off the double rounded to
 * float, by the same IEEE float operations as the host. */
__device__ __forceinline__ void doff_consts(const double *doff, float k, float &cre, float &cim) {
    cre = -__fmul_rn(__fdiv_rn(__double2float_rn(__ldg(doff)), k), k);
    cim = -__fmul_rn(__fdiv_rn(__double2float_rn(__ldg(doff + 1)), k), k);
}

/* ---- fast path: nchan = 2^n, 16 <= nchan <= 4096 ------------------------- */
/* Shared-memory index swizzle for the 16-byte complex doubles: the low LOGP
 * index bits are XORed with the next LOGP. The first pass stores at a stride
 * of PTS (or 4) elements across lanes; swizzled, every 8-lane wavefront lands
 * on 8 distinct 16-byte slots, and the unit-stride accesses of later passes
 * stay conflict-free too (a XOR with a per-block constant permutes the
 * slots). */
__device__ __forceinline__ int SW(int i) { return i ^ ((i >> LOGP) & (PTS - 1)); }

/* the twiddles of one butterfly, w[r] = W^(r k) for r = 1 .. R-1, from the
 * one table entry w1 = W^k: squares and products (each power carries at most
 * two double roundings more than a table entry, ~1e-16 relative) instead of
 * R-1 table loads, so a pass reads Ns table entries, not (R-1)*Ns */
__device__ __forceinline__ double2 csq(double2 a) {
    return make_double2(a.x * a.x - a.y * a.y, 2.0 * a.x * a.y);
}
template <int R>
__device__ __forceinline__ void tw_powers(double2 w1, double2 *w) {
    w[1] = w1;
    if constexpr (R > 2) {
        w[2] = csq(w1);
        w[3] = cmul(w[2], w1);
    }
    if constexpr (R > 4) {
        w[4] = csq(w[2]);
        w[5] = cmul(w[4], w1);
        w[6] = csq(w[3]);
        w[7] = cmul(w[4], w[3]);
    }
}

/* Barrier over the G consecutive threads that share a hop group (G a power of
 * two): a warp sync up to 32 threads, a named barrier (ids 1..NT/G) up to
 * the CTA, __syncthreads for the whole CTA. Memory ordering among the
 * participants is that of bar.sync / bar.warp.sync. */
template <int G>
__device__ __forceinline__ void group_sync() {
    static_assert((G & (G - 1)) == 0 && G <= NT, "group size");
    if constexpr (G >= NT) {
        __syncthreads();
    } else if constexpr (G <= 32) {
        __syncwarp();
    } else {
        static_assert(NT / G <= 15, "named barrier ids 1..15");
        asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)threadIdx.x / G), "r"(G) : "memory");
    }
}

/* Butterfly u of this thread in a pass with U butterflies per thread:
 * warp w owns butterflies [32 w U, 32 (w + 1) U), lanes consecutive, so a
 * warp's butterflies are the same hops as its threads' points in a radix-PTS
 * pass (M/PTS consecutive threads per hop) and lanes read consecutive j. */
template <int U>
__device__ __forceinline__ int bfly(int u) {
    return (((int)threadIdx.x & ~31) * U) + u * 32 + ((int)threadIdx.x & 31);
}

/* One in-place Stockham pass over a 4096-point tile (NT threads x PTS
 * points): every index is a compile-time shift or mask. tw holds
 * W_{Ns R}^{k} at k (tw_powers forms the other powers). G is the group whose barrier
 * suffices (a multiple of the M/PTS threads of one hop): with bfly's
 * numbering the pass reads and writes only its group's hops. */
template <int LOGM, int R, int LOGNS, int G = NT>
__device__ __forceinline__ void pass_c(double2 *sm, const double2 *__restrict__ tw) {
    constexpr int M = 1 << LOGM;
    constexpr int NS = 1 << LOGNS;
    constexpr int LOGR = R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1;
    constexpr int LOGMR = LOGM - LOGR;
    constexpr int MR = 1 << LOGMR;
    constexpr int U = PTS / R;
    double2 v[U][R];
    int dst[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int bi = bfly<U>(u);
        const int tt = bi >> LOGMR;
        const int j = bi & (MR - 1);
        const int k = j & (NS - 1);
        const int base = (tt << LOGM) + j;
#pragma unroll
        for (int r = 0; r < R; ++r) v[u][r] = sm[SW(base + r * MR)];
        double2 w[R];
        tw_powers<R>(__ldg(tw + k), w);
#pragma unroll
        for (int r = 1; r < R; ++r) v[u][r] = cmul(v[u][r], w[r]);
        dst[u] = (tt << LOGM) + ((j - k) << LOGR) + k;
    }
    group_sync<G>();
#pragma unroll
    for (int u = 0; u < U; ++u) {
        dftR<R>(v[u]);
#pragma unroll
        for (int r = 0; r < R; ++r) sm[SW(dst[u] + r * NS)] = v[u][r];
    }
    group_sync<G>();
}

/* Rotation to input sample 0 and cal for bin kb of a hop whose (b + 1) mod os
 * is s, then one rounding to float (reference src/channelizer.c:270-292). */
__device__ __forceinline__ float2 finish_bin(double2 X, int kb, int s, int M, int os, int hop,
                                             bool os_pow2, const double2 *twd, const float2 *cal) {
    const int jr = os_pow2 ? ((kb * s) & (os - 1)) : ((kb * s) % os);
    X = cmul_rn(X, __ldg(twd + (jr ? M - jr * hop : 0)));
    if (cal) {
        const float2 c = __ldg(cal + kb);
        X = cmul_rn(X, make_double2((double)c.x, (double)c.y));
    }
    return make_float2(__double2float_rn(X.x), __double2float_rn(X.y));
}

/* The last Stockham pass fused with the epilogue: after the butterflies every
 * output is a final bin (j + r*Ns of hop tt), rotated, calibrated, rounded and
 * written straight into the padded channel-major tile. The loads read only
 * this thread's group's hops (so the previous pass may end on a group
 * barrier); the tile_out stores overlap every group's points, hence the
 * CTA-wide barrier between them. */
template <int LOGM, int R, int LOGNS>
__device__ __forceinline__ void pass_last(double2 *sm, const double2 *__restrict__ tw,
                                          float2 *tile_out, const atkb_bank &B, const atkb_job &J,
                                          long long h0) {
    constexpr int M = 1 << LOGM;
    constexpr int NS = 1 << LOGNS;
    constexpr int LOGR = R == 16 ? 4 : R == 8 ? 3 : R == 4 ? 2 : 1;
    constexpr int LOGMR = LOGM - LOGR;          /* == LOGNS: Ns * R == M */
    constexpr int MR = 1 << LOGMR;
    constexpr int U = PTS / R;
    constexpr int NH = 1 << (12 - LOGM);
    double2 v[U][R];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int bi = bfly<U>(u);
        const int tt = bi >> LOGMR;
        const int j = bi & (MR - 1);
        const int base = (tt << LOGM) + j;
#pragma unroll
        for (int r = 0; r < R; ++r) v[u][r] = sm[SW(base + r * MR)];
        double2 w[R];
        tw_powers<R>(__ldg(tw + j), w);
#pragma unroll
        for (int r = 1; r < R; ++r) v[u][r] = cmul(v[u][r], w[r]);
    }
    __syncthreads();
    const double2 *twd = (const double2 *)B.twd;
    const float2 *cal = (const float2 *)J.cal;
    /* os divides M, a power of two here: every "mod os" is a mask */
    const int osm = B.os - 1, hop = B.hop;
    const int s0 = (int)(J.b0 + h0 + 1) & osm;
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int bi = bfly<U>(u);
        const int tt = bi >> LOGMR;
        const int j = bi & (MR - 1);
        const int s = (s0 + tt) & osm;
        dftR<R>(v[u]);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int kb = j + r * NS;
            tile_out[kb * (NH + 1) + tt] = finish_bin(v[u][r], kb, s, M, osm + 1, hop, true, twd, cal);
        }
    }
    __syncthreads();
}

/* The fold of one hop's PTS branches q = j + r*M/PTS (r < PTS), straight
 * into the registers of the first radix-PTS butterfly. Taps come from the
 * bank's permuted copy: float4 loads whose addresses are consecutive across
 * the lanes (branches j) of a warp.
 * MODE 0: the tile's windows lie wholly in one cf32 buffer, read through
 * `lin` (offset to this thread's first sample); MODE 1: the same in raw int16
 * I/Q converted on the fly; MODE 2: each sample from the state or the input
 * by index. */
template <int LOGM, int MODE>
__device__ __forceinline__ void foldP(double2 *v, const atkb_job &J, const atkb_bank &B,
                                      long long h0, int tt, int j, const void *lin) {
    constexpr int M = 1 << LOGM;
    constexpr int MP = M >> LOGP;
    const float4 *tq = (const float4 *)B.tapsP + j;
    float fr[PTS], fi[PTS];
    const float2 *xk = (const float2 *)lin;
    const short2 *xk16 = (const short2 *)lin;
    const float cre = J.cre, cim = J.cim, ks = J.kscale;
    const Src src{(const float2 *)J.state, J.in, J.head, J.in_kind, J.cre, J.cim, J.kscale};
    const long long base = (h0 + tt) * (long long)B.hop + j;
#pragma unroll
    for (int q = 0; q < PTS / 4; ++q) {
        const float4 h = __ldg(tq + q * MP);
        const float hh[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int r = 4 * q + c;
            const float2 x = MODE == 0 ? __ldg(xk + r * MP)
                           : MODE == 1 ? conv16(__ldg(xk16 + r * MP), cre, cim, ks)
                                       : src.at(base + r * MP);
            fr[r] = __fmul_rn(hh[c], x.x);
            fi[r] = __fmul_rn(hh[c], x.y);
        }
    }
    for (int k = 1; k < B.K; ++k) {
        tq += MP * (PTS / 4);
        xk += M;
        xk16 += M;
#pragma unroll
        for (int q = 0; q < PTS / 4; ++q) {
            const float4 h = __ldg(tq + q * MP);
            const float hh[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int r = 4 * q + c;
                const float2 x = MODE == 0 ? __ldg(xk + r * MP)
                               : MODE == 1 ? conv16(__ldg(xk16 + r * MP), cre, cim, ks)
                                           : src.at(base + (long long)k * M + r * MP);
                fr[r] = __fadd_rn(fr[r], __fmul_rn(hh[c], x.x));
                fi[r] = __fadd_rn(fi[r], __fmul_rn(hh[c], x.y));
            }
        }
    }
#pragma unroll
    for (int r = 0; r < PTS; ++r) v[r] = make_double2((double)fr[r], (double)fi[r]);
}

/* ---- the staged fold for small nchan ----------------------------------------
 * With nchan <= 512 a tile spans many hops whose windows overlap heavily (each
 * staged sample is used 6-20 times). The whole tile window is copied once into
 * shared memory with asynchronous copies (cp.async: no registers held while
 * the copies fly), then folded from there. Layout: logical sample i of the
 * window lives at i + (i / hop) * (M/16), a pad of M/16 samples after every
 * hop-long block, so the lanes of a warp (several hops x M/16 branches) hit
 * distinct banks. */
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

/* physical size (in samples) of a staged window of W samples */
__device__ __forceinline__ int staged_size(int W, int logs, int MR) { return W + ((W - 1) >> logs) * MR + MR; }

template <int LOGM, int LOGOS>
__device__ __forceinline__ void foldP_staged(double2 *v, const atkb_bank &B, int tt, int j,
                                             const float2 *xs) {
    constexpr int M = 1 << LOGM;
    constexpr int MP = M >> LOGP;
    constexpr int OS = 1 << LOGOS;
    constexpr int HOP = M >> LOGOS;
    /* logical tt*hop + k*M + j + r*MP  ->  physical, with (i / hop) = tt + k*os + (r*os)/PTS */
    const float2 *xb = xs + tt * (HOP + MP) + j;
    const float4 *tq = (const float4 *)B.tapsP + j;
    float fr[PTS], fi[PTS];
#pragma unroll
    for (int q = 0; q < PTS / 4; ++q) {
        const float4 h = __ldg(tq + q * MP);
        const float hh[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int r = 4 * q + c;
            const float2 x = xb[r * MP + ((r * OS) >> LOGP) * MP];
            fr[r] = __fmul_rn(hh[c], x.x);
            fi[r] = __fmul_rn(hh[c], x.y);
        }
    }
    for (int k = 1; k < B.K; ++k) {
        tq += MP * (PTS / 4);
        xb += M + OS * MP;
#pragma unroll
        for (int q = 0; q < PTS / 4; ++q) {
            const float4 h = __ldg(tq + q * MP);
            const float hh[4] = {h.x, h.y, h.z, h.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int r = 4 * q + c;
                const float2 x = xb[r * MP + ((r * OS) >> LOGP) * MP];
                fr[r] = __fadd_rn(fr[r], __fmul_rn(hh[c], x.x));
                fi[r] = __fadd_rn(fi[r], __fmul_rn(hh[c], x.y));
            }
        }
    }
#pragma unroll
    for (int r = 0; r < PTS; ++r) v[r] = make_double2((double)fr[r], (double)fi[r]);
}

/* copy the tile window s[h0*hop, h0*hop + W) into the padded shared layout */
__device__ __forceinline__ void stage_window(float2 *xs, const atkb_job &J, long long g0, int W,
                                             int logs, int MR) {
    const float2 *st = (const float2 *)J.state;
    const float2 *in = (const float2 *)J.in;
    for (int i = threadIdx.x; i < W; i += NT) {
        const long long g = g0 + i;
        const float2 *src = g < J.head ? st + g : in + (g - J.head);
        if (IDX_OK(i + (i >> logs) * MR < 8192 && g < J.nsrc)) cp_async8(xs + i + (i >> logs) * MR, src);
    }
    cp_async_wait_all();
    __syncthreads();
}

template <int LOGM>
__device__ __forceinline__ bool fold_tile_staged(double2 *v, const atkb_job &J, const atkb_bank &B,
                                                 long long h0, int nvalid, int tt, int j, double2 *sm) {
    constexpr int M = 1 << LOGM;
    constexpr int MR = M >> LOGP;
    if constexpr (LOGM > 9) {
        return false;
    } else {
        const int os = B.os;
        if (J.in_kind || B.plan.nostage || (os != 1 && os != 2 && os != 4)) return false;
        const int logs = LOGM - (os == 1 ? 0 : os == 2 ? 1 : 2);
        const long long Wl = (long long)(nvalid - 1) * B.hop + B.L;
        if (Wl > 8192) return false;
        const int W = (int)Wl;
        if (staged_size(W, logs, MR) > 8192) return false;     /* sm holds 8192 float2 */
        float2 *xs = (float2 *)sm;
        stage_window(xs, J, h0 * (long long)B.hop, W, logs, MR);
        if (tt < nvalid) {
            if (os == 1) foldP_staged<LOGM, 0>(v, B, tt, j, xs);
            else if (os == 2) foldP_staged<LOGM, 1>(v, B, tt, j, xs);
            else foldP_staged<LOGM, 2>(v, B, tt, j, xs);
        } else {
#pragma unroll
            for (int r = 0; r < PTS; ++r) v[r] = make_double2(0.0, 0.0);
        }
        __syncthreads();              /* the window is dead; sm becomes the FFT tile */
        return true;
    }
}

/* ---- the paired fold: oversample 1, 2 or 4, nchan <= 2048 -------------------
 * Thread (pair p, parity c, branch j) folds hops ta = 2p and tb = 2p + 1 of
 * the tile over the four branches j + r*MP with r = c + 2i, i = 0..3
 * (MP = M/8). Slot u = 8k + r of hop ta's window (sample u*MP + j, tap
 * k*M + r*MP + j) is slot u - 8/os of hop tb's: every sample the thread loads
 * feeds both hops, and each float4 of taps (row k, parity c) serves hop ta in
 * row k and hop tb in rows k and k + 1. Against one hop and eight branches per
 * thread this halves the loads of samples and taps per output. Slots stream in
 * ascending order, so every branch still sums its taps k ascending; the sums
 * start from -0.0f, and -0 + p == p for every p, so the first product enters
 * unchanged as in the reference's loop. */
__device__ __forceinline__ void mac(float2 &a, float h, float2 x) {
    a.x = __fadd_rn(a.x, __fmul_rn(h, x.x));
    a.y = __fadd_rn(a.y, __fmul_rn(h, x.y));
}

/* sample loaders: at(k, i) is slot 8k + c + 2i of hop ta's window */
template <int LOGM>
struct PairLin {                       /* cf32, the tile's windows in one buffer */
    const float2 *p;
    __device__ __forceinline__ float2 at(int k, int i) const {
        return __ldg(p + ((long long)k << LOGM) + 2 * i * (1 << (LOGM - LOGP)));
    }
};
template <int LOGM>
struct PairLin16 {                     /* raw int16 I/Q, converted on the fly */
    const short2 *p;
    float cre, cim, ks;
    __device__ __forceinline__ float2 at(int k, int i) const {
        return conv16(__ldg(p + ((long long)k << LOGM) + 2 * i * (1 << (LOGM - LOGP))), cre, cim, ks);
    }
};
template <int LOGM>
struct PairMixed {                     /* cf32 state / input by index */
    const float2 *st, *in;
    long long g, head;
    __device__ __forceinline__ float2 at(int k, int i) const {
        const long long pos = g + ((long long)k << LOGM) + 2 * i * (1 << (LOGM - LOGP));
        return __ldg(pos < head ? st + pos : in + (pos - head));
    }
};
template <int LOGM>
struct PairMixed16 {                   /* cf32 state / raw int16 input by index */
    const float2 *st;
    const short2 *in;
    long long g, head;
    float cre, cim, ks;
    __device__ __forceinline__ float2 at(int k, int i) const {
        const long long pos = g + ((long long)k << LOGM) + 2 * i * (1 << (LOGM - LOGP));
        return pos < head ? __ldg(st + pos) : conv16(__ldg(in + (pos - head)), cre, cim, ks);
    }
};
template <int LOGM, int LOGOS>
struct PairStaged {                    /* the padded shared-memory window */
    const float2 *p;                   /* at slot c of hop ta, row 0 */
    __device__ __forceinline__ float2 at(int k, int i) const {
        constexpr int MP = 1 << (LOGM - LOGP);
        constexpr int LOGD = 3 - LOGOS;             /* slot shift 8/os = 2^LOGD */
        return p[k * ((1 << LOGM) + (MP << LOGOS)) + (2 * i + (i >> (LOGD - 1))) * MP];
    }
};

template <int LOGM, int LOGOS, class LD>
__device__ __forceinline__ void fold_pair(float2 (&a)[4], float2 (&b)[4], const float4 *tq, int K,
                                          bool tb_ok, const LD &ld) {
    constexpr int MP = 1 << (LOGM - LOGP);
    constexpr int D2 = 4 >> LOGOS;     /* hop tb's taps trail hop ta's by D2 entries */
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        a[i] = make_float2(-0.0f, -0.0f);
        b[i] = make_float2(-0.0f, -0.0f);
    }
    float4 pv = __ldg(tq);
    {
        const float h[4] = {pv.x, pv.y, pv.z, pv.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 x = ld.at(0, i);
            mac(a[i], h[i], x);
            if (i >= D2) mac(b[i - D2], h[i - D2], x);
        }
    }
    for (int k = 1; k < K; ++k) {
        const float4 cv = __ldg(tq + k * 2 * MP);
        const float h[4] = {cv.x, cv.y, cv.z, cv.w};
        const float g[4] = {pv.x, pv.y, pv.z, pv.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 x = ld.at(k, i);
            mac(a[i], h[i], x);
            if (i >= D2) mac(b[i - D2], h[i - D2], x);
            else mac(b[i - D2 + 4], g[i - D2 + 4], x);
        }
        pv = cv;
    }
    if (tb_ok) {                       /* the slots past hop ta's window */
        const float g[4] = {pv.x, pv.y, pv.z, pv.w};
#pragma unroll
        for (int i = 0; i < D2; ++i) mac(b[i - D2 + 4], g[i - D2 + 4], ld.at(K, i));
    }
}

/* radix-4 first pass (Ns = 1) of one hop's four even or odd branches:
 * branch j + (c + 2i)*MP is point jp + i*M/4 of the hop, jp = j + c*MP */
template <int LOGM>
__device__ __forceinline__ void first_pass4(const float2 (&f)[4], double2 *sm, int t, int jp) {
    double2 v[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = make_double2((double)f[i].x, (double)f[i].y);
    dft4(v[0], v[1], v[2], v[3]);
#pragma unroll
    for (int i = 0; i < 4; ++i)
        if (IDX_OK((t << LOGM) + jp * 4 + i < TILE_POINTS)) sm[SW((t << LOGM) + jp * 4 + i)] = v[i];
}

/* the paired fold of hops ta, ta + 1 (parity c, branch j) from global memory;
 * the window source (input, state, or both by index) is chosen per tile */
template <int LOGM, int LOGOS>
__device__ __forceinline__ void fold_pair_global(float2 (&a)[4], float2 (&b)[4], const atkb_job &J,
                                                 const atkb_bank &B, long long h0, int nvalid, int ta,
                                                 int c, int j, bool tb_ok) {
    constexpr int MP = 1 << (LOGM - LOGP);
    constexpr int HOP = (1 << LOGM) >> LOGOS;
    const float4 *tq = (const float4 *)B.tapsP + c * MP + j;
    const long long w0 = h0 * (long long)HOP;
    const long long w1 = (h0 + nvalid - 1) * (long long)HOP + B.L;
    const long long off = (h0 + ta) * (long long)HOP + c * MP + j;
    if (w0 >= J.head) {
        if (J.in_kind) {
            const PairLin16<LOGM> ld{(const short2 *)J.in + (off - J.head), J.cre, J.cim, J.kscale};
            fold_pair<LOGM, LOGOS>(a, b, tq, B.K, tb_ok, ld);
        } else {
            const PairLin<LOGM> ld{(const float2 *)J.in + (off - J.head)};
            fold_pair<LOGM, LOGOS>(a, b, tq, B.K, tb_ok, ld);
        }
    } else if (w1 <= J.head) {
        const PairLin<LOGM> ld{(const float2 *)J.state + off};
        fold_pair<LOGM, LOGOS>(a, b, tq, B.K, tb_ok, ld);
    } else {
        if (J.in_kind) {
            const PairMixed16<LOGM> ld{(const float2 *)J.state, (const short2 *)J.in, off, J.head,
                                       J.cre, J.cim, J.kscale};
            fold_pair<LOGM, LOGOS>(a, b, tq, B.K, tb_ok, ld);
        } else {
            const PairMixed<LOGM> ld{(const float2 *)J.state, (const float2 *)J.in, off, J.head};
            fold_pair<LOGM, LOGOS>(a, b, tq, B.K, tb_ok, ld);
        }
    }
}

template <int LOGM, int LOGOS>
__device__ __forceinline__ void fold_tile_pair(const atkb_job &J, const atkb_bank &B, long long h0,
                                               int nvalid, double2 *sm) {
    constexpr int M = 1 << LOGM;
    constexpr int LOGMP = LOGM - LOGP;
    constexpr int MP = 1 << LOGMP;
    constexpr int HOP = M >> LOGOS;
    const int tid = threadIdx.x;
    const int j = tid & (MP - 1);
    const int c = (tid >> LOGMP) & 1;
    const int ta = (tid >> (LOGMP + 1)) * 2;
    const bool ta_ok = ta < nvalid, tb_ok = ta + 1 < nvalid;
    const float4 *tq = (const float4 *)B.tapsP + c * MP + j;
    float2 a[4], b[4];
    if constexpr (LOGM <= 9) {
        /* small nchan: the whole tile window through shared memory (as in
         * fold_tile_staged; logical sample i at i + (i / hop) * MP) */
        const long long Wl = (long long)(nvalid - 1) * HOP + B.L;
        if (!J.in_kind && !B.plan.nostage && Wl <= 8192 && staged_size((int)Wl, LOGM - LOGOS, MP) <= 8192) {
            float2 *xs = (float2 *)sm;
            stage_window(xs, J, h0 * (long long)HOP, (int)Wl, LOGM - LOGOS, MP);
            if (ta_ok) {
                const PairStaged<LOGM, LOGOS> ld{xs + ta * (HOP + MP) + j + c * MP};
                fold_pair<LOGM, LOGOS>(a, b, tq, B.K, tb_ok, ld);
            } else {
#pragma unroll
                for (int i = 0; i < 4; ++i) a[i] = b[i] = make_float2(0.0f, 0.0f);
            }
            __syncthreads();          /* the window is dead; sm becomes the FFT tile */
            /* the first pass inside this branch: merging the sums of both
             * branches ahead of one first pass cost ~1 KB of spills */
            first_pass4<LOGM>(a, sm, ta, j + c * MP);
            first_pass4<LOGM>(b, sm, ta + 1, j + c * MP);
            return;
        }
    }
    if (ta_ok) fold_pair_global<LOGM, LOGOS>(a, b, J, B, h0, nvalid, ta, c, j, tb_ok);
    if (!ta_ok) {
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = b[i] = make_float2(0.0f, 0.0f);
    }
    first_pass4<LOGM>(a, sm, ta, j + c * MP);
    first_pass4<LOGM>(b, sm, ta + 1, j + c * MP);
}

/* the Stockham passes after the first (which left Ns = 2^LOGNS): radix PTS
 * while more than LOGP index bits remain, then the last pass (radix 2, 4 or
 * 8) fused with the epilogue; P indexes the plan's twiddle offsets */
template <int LOGM, int LOGNS, int P, int G = NT>
__device__ __forceinline__ void fft_rest(double2 *sm, const double2 *wp, const int *twoff,
                                         float2 *tile_out, const atkb_bank &B, const atkb_job &J,
                                         long long h0) {
    if constexpr (LOGM - LOGNS > LOGP) {
        pass_c<LOGM, PTS, LOGNS, G>(sm, wp + twoff[P]);
        fft_rest<LOGM, LOGNS + LOGP, P + 1, G>(sm, wp, twoff, tile_out, B, J, h0);
    } else {
        pass_last<LOGM, (1 << (LOGM - LOGNS)), LOGNS>(sm, wp + twoff[P], tile_out, B, J, h0);
    }
}

/* write a finished tile: thread -> (channel kb0 + u*MP, hop t2), runs of NH
 * consecutive hops per channel */
template <int LOGM>
__device__ __forceinline__ void write_tile(const atkb_job &J, long long h0, int nvalid,
                                           const float2 *tile_out) {
    constexpr int LOGNH = 12 - LOGM;
    constexpr int NH = 1 << LOGNH;
    constexpr int MP = (1 << LOGM) >> LOGP;
    const int tid = threadIdx.x;
    const int t2 = tid & (NH - 1);
    if (t2 < nvalid) {
        const int kb0 = tid >> LOGNH;
        float2 *o = (float2 *)J.out + (J.out_col + h0 + t2) + (long long)kb0 * J.ldo;
        const long long step = (long long)MP * J.ldo;
#pragma unroll 4
        for (int u = 0; u < PTS; ++u) {
            const int row = kb0 + u * MP;
            if (IDX_OK(row < (1 << LOGM) && J.out_col + h0 + t2 < J.ldo &&
                       row * (NH + 1) + t2 < TILE_POINTS * 2))
                *o = tile_out[row * (NH + 1) + t2];
            o += step;
        }
    }
}

/* W2 fused into the epilogue: the tile's power per channel, sum over its
 * valid hops t of |y|^2 in double from the rounded outputs (the reference's
 * W2 sum, src/channelizer.c:459-461, for these hops), written to the job's
 * partial buffer at row h0 / tile_hops. A second kernel adds the tiles' rows
 * in tile order (atkb_w2_finish). tile_out stays intact until the barrier
 * that opens the next tile. */
template <int LOGM>
__device__ __forceinline__ void w2_partial(const atkb_job &J, long long h0, int nvalid, const float2 *tile_out) {
    constexpr int M = 1 << LOGM;
    constexpr int NH = 1 << (12 - LOGM);
    double *row = J.w2 + (h0 / NH) * M;
    for (int kb = threadIdx.x; kb < M; kb += NT) {
        double s = 0.0;
        for (int t = 0; t < nvalid; ++t) {
            const float2 y = tile_out[kb * (NH + 1) + t];
            s += (double)y.x * y.x + (double)y.y * y.y;
        }
        row[kb] = s;
    }
}

/* ---- the quad fold: oversample 1 or 2, nchan <= 1024 --------------------------
 * Thread (quad g, class c, branch j) folds the four hops ta + t (ta = 4g,
 * t = 0..3) of the tile over the two branches q0 = j + c*MP and q1 = q0 + M/2
 * (MP = M/8, c = 0..3). In hop ta's frame its samples are the slots
 * u = 4v + c (sample u*MP + j, tap u*MP + j), v = 0 .. 2K-1; hop ta + t sees
 * the same sample at slot u - t*8/os, i.e. at v - t*D with D = 2/os, which
 * keeps the class c. So every sample the thread loads feeds all four hops,
 * and each tap it loads serves the four hops in turn through a window of
 * W = 4*D taps held in registers: per input sample position one 8-byte
 * sample load, one 4-byte tap load and four complex multiply-adds (against
 * one tap load per two multiply-adds in the paired fold). Branch q_i of hop t
 * sums its taps in slot order -- k ascending, a rounded multiply then a
 * rounded add, from -0.0f -- like every other fold here, so all tile shapes
 * give the reference's bits. The two branches feed a radix-2
 * first Stockham pass (Ns = 1: points q0 and q0 + M/2 of each hop). */
template <int LOGM>
struct QuadLin {                       /* cf32, the quad's windows in one buffer */
    const float2 *p;                   /* at slot c of hop ta, branch j */
    __device__ __forceinline__ float2 at(int v) const { return __ldg(p + (long long)v * (1 << (LOGM - 1))); }
};
template <int LOGM>
struct QuadLin16 {                     /* raw int16 I/Q, converted on the fly */
    const short2 *p;
    float cre, cim, ks;
    __device__ __forceinline__ float2 at(int v) const {
        return conv16(__ldg(p + (long long)v * (1 << (LOGM - 1))), cre, cim, ks);
    }
};
template <int LOGM>
struct QuadMixed {                     /* cf32 state / input by index */
    const float2 *st, *in;
    long long g, head;
    __device__ __forceinline__ float2 at(int v) const {
        const long long pos = g + (long long)v * (1 << (LOGM - 1));
        return __ldg(pos < head ? st + pos : in + (pos - head));
    }
};
template <int LOGM>
struct QuadMixed16 {                   /* cf32 state / raw int16 input by index */
    const float2 *st;
    const short2 *in;
    long long g, head;
    float cre, cim, ks;
    __device__ __forceinline__ float2 at(int v) const {
        const long long pos = g + (long long)v * (1 << (LOGM - 1));
        return pos < head ? __ldg(st + pos) : conv16(__ldg(in + (pos - head)), cre, cim, ks);
    }
};

/* acc[t][i]: hop ta + t, branch q_i. tq: this thread's 2K taps at stride MP
 * (tap v of class c, branch j). nq: valid hops of the quad (1..4). */
template <int LOGOS, class LD>
__device__ __forceinline__ void fold_quad(float2 (&acc)[4][2], const float *__restrict__ tq, int MP, int K,
                                          int nq, const LD &ld) {
    constexpr int D = 2 >> LOGOS;      /* v-shift per hop */
    constexpr int W = 4 * D;           /* tap window (a power of two) */
    const int V = 2 * K;               /* taps per class */
    const int vend = V + (nq - 1) * D; /* one past the last sample position */
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[t][0] = acc[t][1] = make_float2(-0.0f, -0.0f);
    float T[W];
#pragma unroll
    for (int w = 0; w < W; ++w) T[w] = 0.0f;
    for (int v0 = 0; v0 < vend; v0 += W) {
        if (v0 >= W - D && v0 + W <= V && nq == 4) {
            /* every hop in its window: no conditions */
#pragma unroll
            for (int s = 0; s < W; ++s) {
                const int v = v0 + s;
                T[s] = __ldg(tq + (long long)v * MP);
                const float2 x = ld.at(v);
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int sv = (s - t * D) & (W - 1);       /* slot of tap v - t*D */
                    const int par = LOGOS ? ((s - t) & 1) : (s & 1);
                    mac(acc[t][par], T[sv], x);
                }
            }
        } else {
#pragma unroll
            for (int s = 0; s < W; ++s) {
                const int v = v0 + s;
                if (v < V) T[s] = __ldg(tq + (long long)v * MP);
                if (v < vend) {
                    const float2 x = ld.at(v);
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const int vt = v - t * D;
                        const int sv = (s - t * D) & (W - 1);
                        const int par = LOGOS ? ((s - t) & 1) : (s & 1);
                        if (t < nq && vt >= 0 && vt < V) mac(acc[t][par], T[sv], x);
                    }
                }
            }
        }
    }
}

/* the radix-2 first pass (Ns = 1) of one hop: points q0 and q0 + M/2 in,
 * 2*q0 + {0, 1} out */
template <int LOGM>
__device__ __forceinline__ void first_pass2(float2 a, float2 b, double2 *sm, int t, int q0) {
    double2 x0 = make_double2((double)a.x, (double)a.y), x1 = make_double2((double)b.x, (double)b.y);
    dft2(x0, x1);
    if (IDX_OK((t << LOGM) + 2 * q0 + 1 < TILE_POINTS)) {
        sm[SW((t << LOGM) + 2 * q0)] = x0;
        sm[SW((t << LOGM) + 2 * q0 + 1)] = x1;
    }
}

template <int LOGM, int LOGOS>
__device__ __forceinline__ void fold_tile_quad(const atkb_job &J, const atkb_bank &B, long long h0,
                                               int nvalid, double2 *sm) {
    constexpr int M = 1 << LOGM;
    constexpr int LOGMP = LOGM - LOGP;
    constexpr int MP = 1 << LOGMP;
    constexpr int HOP = M >> LOGOS;
    static_assert(PTS == 8 && LOGM <= 10 && LOGOS <= 1, "quad fold: PTS 8, four hops a tile");
    const int tid = threadIdx.x;
    const int j = tid & (MP - 1);
    const int c = (tid >> LOGMP) & 3;
    const int ta = (tid >> (LOGMP + 2)) * 4;
    const int nq = min(4, nvalid - ta);
    float2 acc[4][2];
    if (nq > 0) {
        const float *tq = B.tapsQ + (long long)c * (2 * B.K) * MP + j;
        const long long w0 = h0 * (long long)HOP;
        const long long w1 = (h0 + nvalid - 1) * (long long)HOP + B.L;
        const long long off = (h0 + ta) * (long long)HOP + c * MP + j;
        if (w0 >= J.head) {
            if (J.in_kind) {
                const QuadLin16<LOGM> ld{(const short2 *)J.in + (off - J.head), J.cre, J.cim, J.kscale};
                fold_quad<LOGOS>(acc, tq, MP, B.K, nq, ld);
            } else {
                const QuadLin<LOGM> ld{(const float2 *)J.in + (off - J.head)};
                fold_quad<LOGOS>(acc, tq, MP, B.K, nq, ld);
            }
        } else if (w1 <= J.head) {
            const QuadLin<LOGM> ld{(const float2 *)J.state + off};
            fold_quad<LOGOS>(acc, tq, MP, B.K, nq, ld);
        } else if (J.in_kind) {
            const QuadMixed16<LOGM> ld{(const float2 *)J.state, (const short2 *)J.in, off, J.head,
                                       J.cre, J.cim, J.kscale};
            fold_quad<LOGOS>(acc, tq, MP, B.K, nq, ld);
        } else {
            const QuadMixed<LOGM> ld{(const float2 *)J.state, (const float2 *)J.in, off, J.head};
            fold_quad<LOGOS>(acc, tq, MP, B.K, nq, ld);
        }
    } else {
#pragma unroll
        for (int t = 0; t < 4; ++t) acc[t][0] = acc[t][1] = make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) first_pass2<LOGM>(acc[t][0], acc[t][1], sm, ta + t, j + c * MP);
}

template <int LOGM, int LOGOS>
__device__ void tile_quad(const atkb_job &J, const atkb_bank &B, long long h0, int nvalid, double2 *sm,
                          float2 *tile_out) {
    constexpr int M = 1 << LOGM;
    fold_tile_quad<LOGM, LOGOS>(J, B, h0, nvalid, sm);
    /* a quad's M/2 threads hold its four hops' points through the passes
     * before the last (bfly gives each hop M/8 consecutive threads) */
    constexpr int G0 = M / 2;
    constexpr int G = G0 < 32 ? 32 : G0 > NT ? NT : G0;
    group_sync<G>();
    fft_rest<LOGM, 1, 1, G>(sm, (const double2 *)B.wpass, B.plan.twoff, tile_out, B, J, h0);
    write_tile<LOGM>(J, h0, nvalid, tile_out);
    if (J.w2) w2_partial<LOGM>(J, h0, nvalid, tile_out);
}

/* fold + first Stockham pass (Ns = 1, radix PTS, no twiddles) of one hop
 * and PTS branches per thread, into the tile's shared points */
template <int LOGM>
__device__ __forceinline__ void fold_first_unpaired(const atkb_job &J, const atkb_bank &B, long long h0,
                                                    int nvalid, double2 *sm) {
    constexpr int MP = (1 << LOGM) >> LOGP;
    const int tid = threadIdx.x;
    const int tt = tid >> (LOGM - LOGP);
    const int j = tid & (MP - 1);
    double2 v[PTS];
    if (!fold_tile_staged<LOGM>(v, J, B, h0, nvalid, tt, j, sm)) {
        if (tt < nvalid) {
            const long long w0 = h0 * (long long)B.hop;                       /* first window start */
            const long long w1 = (h0 + nvalid - 1) * (long long)B.hop + B.L;  /* last window end */
            const long long off = (h0 + tt) * (long long)B.hop + j;
            if (w0 >= J.head) {
                if (J.in_kind)
                    foldP<LOGM, 1>(v, J, B, h0, tt, j, (const short2 *)J.in + (off - J.head));
                else
                    foldP<LOGM, 0>(v, J, B, h0, tt, j, (const float2 *)J.in + (off - J.head));
            } else if (w1 <= J.head) {
                foldP<LOGM, 0>(v, J, B, h0, tt, j, (const float2 *)J.state + off);
            } else {
                foldP<LOGM, 2>(v, J, B, h0, tt, j, nullptr);
            }
        } else {
#pragma unroll
            for (int r = 0; r < PTS; ++r) v[r] = make_double2(0.0, 0.0);
        }
    }
    dftR<PTS>(v);
#pragma unroll
    for (int r = 0; r < PTS; ++r) sm[SW((tt << LOGM) + j * PTS + r)] = v[r];
}

/* nchan 4096: a tile is two hops, computed in turn. Hop a's outputs wait in
 * a side buffer (4096 float2 after the FFT tile, 96 KB in all) while hop b
 * is computed, so the write covers two hops per channel: lanes 2l and 2l+1
 * write the two adjacent outputs of one channel, half the sectors of
 * single-hop writes (a single hop's 4096 outputs land in 4096 rows). */
__device__ void tile_4096x2(const atkb_job &J, const atkb_bank &B, long long h0, int nvalid, double2 *sm) {
    constexpr int LOGM = 12;
    constexpr int M = 1 << LOGM;
    constexpr int MP = M >> LOGP;
    static_assert(NT == MP, "one thread per branch group");
    float2 *tile_out = (float2 *)sm;       /* pass_last: hop at tile_out[kb * 2] */
    float2 *side = (float2 *)(sm + M);
    const double2 *wp = (const double2 *)B.wpass;
    const int tid = threadIdx.x;
#pragma unroll 1
    for (int sub = 0; sub < 2 && sub < nvalid; ++sub) {
        fold_first_unpaired<LOGM>(J, B, h0 + sub, 1, sm);
        __syncthreads();
        fft_rest<LOGM, LOGP, 1, NT>(sm, wp, B.plan.twoff, tile_out, B, J, h0 + sub);
        if (sub == 0) {
#pragma unroll
            for (int u = 0; u < PTS; ++u) side[tid + u * MP] = tile_out[(tid + u * MP) * 2];
            __syncthreads();                 /* read before hop b's first pass */
        }
    }
    const int t2 = tid & 1;
    if (t2 < nvalid) {
        const int kb0 = tid >> 1;
        float2 *o = (float2 *)J.out + (J.out_col + h0 + t2) + (long long)kb0 * J.ldo;
        const long long step = (long long)(NT / 2) * J.ldo;
#pragma unroll 4
        for (int u = 0; u < 2 * PTS; ++u) {
            const int kb = kb0 + u * (NT / 2);
            *o = t2 ? tile_out[kb * 2] : side[kb];
            o += step;
        }
    }
}

/* nchan 4096 at oversample 1/2/4: the same two-hop tile with the paired
 * fold. Thread j folds both hops over the even branches, then over the odd
 * ones (each sample and tap loaded once for the two hops); the even sums
 * wait in the side buffer, so each hop's 8 branches meet in registers for a
 * radix-8 first pass (the 4-pass plan). Hop b's sums wait in the side
 * buffer while hop a is transformed; then hop a's outputs take their place. */
template <int LOGOS>
__device__ void tile_4096x2_pair(const atkb_job &J, const atkb_bank &B, long long h0, int nvalid,
                                 double2 *sm) {
    constexpr int LOGM = 12;
    constexpr int M = 1 << LOGM;
    constexpr int MP = M >> LOGP;
    static_assert(NT == MP && PTS == 8, "one thread per branch group");
    float2 *tile_out = (float2 *)sm;       /* pass_last: hop at tile_out[kb * 2] */
    float2 *side = (float2 *)(sm + M);     /* [8][MP] float2, slot (row, j) owned by thread j */
    const double2 *wp = (const double2 *)B.wpass;
    const int j = threadIdx.x;
    const bool tb_ok = nvalid > 1;
    float2 a[4], b[4];
    fold_pair_global<LOGM, LOGOS>(a, b, J, B, h0, nvalid, 0, 0, j, tb_ok);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        side[i * MP + j] = a[i];           /* rows 0-3: hop a, even branches */
        side[(4 + i) * MP + j] = b[i];     /* rows 4-7: hop b, even branches */
    }
    fold_pair_global<LOGM, LOGOS>(a, b, J, B, h0, nvalid, 0, 1, j, tb_ok);
    {
        double2 v[PTS];                    /* branch r = c + 2i of hop a */
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 e = side[i * MP + j];
            v[2 * i] = make_double2((double)e.x, (double)e.y);
            v[2 * i + 1] = make_double2((double)a[i].x, (double)a[i].y);
            side[i * MP + j] = b[i];       /* rows 0-3 now: hop b, odd branches */
        }
        dftR<PTS>(v);
#pragma unroll
        for (int r = 0; r < PTS; ++r) sm[SW(j * PTS + r)] = v[r];
    }
    __syncthreads();
    fft_rest<LOGM, LOGP, 1, NT>(sm, wp, B.plan.twoff, tile_out, B, J, h0);
    if (tb_ok) {
        double2 v[PTS];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 e = side[(4 + i) * MP + j], o = side[i * MP + j];
            v[2 * i] = make_double2((double)e.x, (double)e.y);
            v[2 * i + 1] = make_double2((double)o.x, (double)o.y);
        }
#pragma unroll
        for (int u = 0; u < PTS; ++u) side[u * MP + j] = tile_out[(j + u * MP) * 2];   /* hop a's outputs */
        __syncthreads();                   /* tile_out read before hop b's first pass */
        dftR<PTS>(v);
#pragma unroll
        for (int r = 0; r < PTS; ++r) sm[SW(j * PTS + r)] = v[r];
        __syncthreads();
        fft_rest<LOGM, LOGP, 1, NT>(sm, wp, B.plan.twoff, tile_out, B, J, h0 + 1);
    } else {
#pragma unroll
        for (int u = 0; u < PTS; ++u) side[u * MP + j] = tile_out[(j + u * MP) * 2];
        __syncthreads();
    }
    const int tid = threadIdx.x;
    const int t2 = tid & 1;
    if (t2 < nvalid) {
        const int kb0 = tid >> 1;
        float2 *o = (float2 *)J.out + (J.out_col + h0 + t2) + (long long)kb0 * J.ldo;
        const long long step = (long long)(NT / 2) * J.ldo;
#pragma unroll 4
        for (int u = 0; u < 2 * PTS; ++u) {
            const int kb = kb0 + u * (NT / 2);
            *o = t2 ? tile_out[kb * 2] : side[kb];
            o += step;
        }
    }
}

/* LOGOS < 0: one hop and PTS branches per thread, first pass radix PTS;
 * LOGOS = log2(os) in 0..2: the paired fold, first pass radix 4 */
template <int LOGM, int LOGOS>
__device__ void tile_fast(const atkb_job &J, const atkb_bank &B, long long h0, int nvalid,
                          double2 *sm, float2 *tile_out) {
    constexpr int M = 1 << LOGM;
    constexpr int LOGNH = 12 - LOGM;
    constexpr int NH = 1 << LOGNH;
    constexpr int MP = M >> LOGP;
    static_assert(LOGM > LOGP, "the fast path needs nchan > PTS");
    const int tid = threadIdx.x;

    if constexpr (LOGOS >= 0) {
        static_assert(PTS == 8 && LOGM <= 11 && LOGOS <= 2, "paired fold: PTS 8, two hops a tile");
        fold_tile_pair<LOGM, LOGOS>(J, B, h0, nvalid, sm);
    } else {
        fold_first_unpaired<LOGM>(J, B, h0, nvalid, sm);
    }
    /* from here to the last pass each hop group (the threads of a hop pair,
     * or of one hop) touches only its own points: group barriers suffice.
     * The region was last used by the previous tile's write, fenced by the
     * CTA-wide barrier that ends every tile. */
    constexpr int G0 = (LOGOS >= 0 ? M / 4 : M / PTS);
    constexpr int G = G0 < 32 ? 32 : G0 > NT ? NT : G0;
    group_sync<G>();

    fft_rest<LOGM, (LOGOS >= 0 ? 2 : LOGP), 1, G>(sm, (const double2 *)B.wpass, B.plan.twoff, tile_out, B,
                                                   J, h0);

    write_tile<LOGM>(J, h0, nvalid, tile_out);
    if (J.w2) w2_partial<LOGM>(J, h0, nvalid, tile_out);
}

/* ---- generic path: any nchan >= 2 ----------------------------------------- */
__device__ void pass_generic(const double2 *src, double2 *dst, int M, int Ns, int R, int nh,
                             const double2 *W) {
    const int MR = M / R;
    const int NsR = Ns * R;
    const int stride = M / NsR;
    for (int bi = threadIdx.x; bi < nh * MR; bi += NT) {
        const int tt = bi / MR;
        const int j = bi - tt * MR;
        const int k = j % Ns;
        const double2 *s = src + tt * M + j;
        double2 *d = dst + tt * M + (j - k) * R + k;
        if (R == 2 || R == 3 || R == 4 || R == 8 || R == 16) {
            double2 v[16];
            for (int r = 0; r < R; ++r) {
                v[r] = s[r * MR];
                if (r) v[r] = cmul(v[r], __ldg(W + r * k * stride));
            }
            if (R == 2) dft2(v[0], v[1]);
            else if (R == 3) dft3(v[0], v[1], v[2]);
            else if (R == 4) dft4(v[0], v[1], v[2], v[3]);
            else if (R == 8) dft8(v);
            else dft16(v);
            for (int r = 0; r < R; ++r) d[r * Ns] = v[r];
        } else {
            /* direct DFT with the twiddle folded in: W_{NsR}^{r (k + o Ns)} */
            for (int o = 0; o < R; ++o) {
                double2 acc = make_double2(0.0, 0.0);
                for (int r = 0; r < R; ++r) {
                    const long long e = ((long long)r * (k + o * Ns)) % NsR;
                    const double2 w = __ldg(W + e * stride);
                    const double2 x = s[r * MR];
                    acc.x += x.x * w.x - x.y * w.y;
                    acc.y += x.x * w.y + x.y * w.x;
                }
                d[o * Ns] = acc;
            }
        }
    }
    __syncthreads();
}

__device__ void tile_generic(const atkb_job &J, const atkb_bank &B, long long h0, int nvalid,
                             double2 *sm) {
    const int M = B.nchan;
    const int nh = B.tile_hops;
    double2 *A = sm, *Bf = sm + (size_t)nh * M;
    const Src src{(const float2 *)J.state, J.in, J.head, J.in_kind, J.cre, J.cim, J.kscale};
    for (int e = threadIdx.x; e < nh * M; e += NT) {
        const int tt = e / M;
        const int q = e - tt * M;
        double2 v = make_double2(0.0, 0.0);
        if (tt < nvalid) {
            const long long base = (h0 + tt) * (long long)B.hop + q;
            float2 x = src.at(base);
            float h = __ldg(B.taps + q);
            float fr = __fmul_rn(h, x.x), fi = __fmul_rn(h, x.y);
            for (int k = 1; k < B.K; ++k) {
                h = __ldg(B.taps + (long long)k * M + q);
                x = src.at(base + (long long)k * M);
                fr = __fadd_rn(fr, __fmul_rn(h, x.x));
                fi = __fadd_rn(fi, __fmul_rn(h, x.y));
            }
            v = make_double2((double)fr, (double)fi);
        }
        A[e] = v;
    }
    __syncthreads();
    const double2 *W = (const double2 *)B.wfull;
    int Ns = 1;
    double2 *cur = A, *nxt = Bf;
    for (int p = 0; p < B.plan.npass; ++p) {
        const int R = B.plan.radix[p];
        pass_generic(cur, nxt, M, Ns, R, nh, W);
        Ns *= R;
        double2 *t = cur; cur = nxt; nxt = t;
    }
    const double2 *twd = (const double2 *)B.twd;
    const float2 *cal = (const float2 *)J.cal;
    float2 *out = (float2 *)J.out;
    const int os = B.os, hop = B.hop;
    for (int e = threadIdx.x; e < nvalid * M; e += NT) {
        const int kb = e / nvalid;
        const int tt = e - kb * nvalid;
        double2 X = cur[tt * M + kb];
        const long long b = J.b0 + h0 + tt;
        const int s = (int)((b + 1) % os);
        const int jr = (int)(((long long)kb * s) % os);
        X = cmul_rn(X, __ldg(twd + (jr ? M - jr * hop : 0)));
        if (cal) {
            const float2 c = __ldg(cal + kb);
            X = cmul_rn(X, make_double2((double)c.x, (double)c.y));
        }
        out[(long long)kb * J.ldo + J.out_col + h0 + tt] =
            make_float2(__double2float_rn(X.x), __double2float_rn(X.y));
    }
}

/* The CTA's next tile (warp 0, all lanes): claim it from the counter, find
 * its job (the last whose first tile <= tile) by a 32-ary search over the
 * tile prefix table, and copy the job and its bank into shared slot `slot`
 * with asynchronous copies that land while the CTA works on the current
 * tile (the caller waits for them before the next barrier). */
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void fetch_tile(const atkb_job *__restrict__ jobs, const int *__restrict__ tile_start,
                                           int njobs, int total, int *counters, int *s_tile, int *s_local,
                                           atkb_job *s_job, atkb_bank *s_bank, int slot) {
    static_assert(sizeof(atkb_job) % 4 == 0 && sizeof(atkb_bank) % 4 == 0, "word copies");
    const int lane = threadIdx.x & 31;
    int tile = 0;
    if (lane == 0) tile = atomicAdd(&counters[0], 1);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (lane == 0) s_tile[slot] = tile;
    if (tile >= total) return;
    int lo = 0, hi = njobs - 1;                  /* tile_start[lo] <= tile throughout */
    while (lo < hi) {
        const int step = (hi - lo + 32) >> 5;    /* ceil(span / 32) */
        const int idx = lo + lane * step;
        const bool ok = idx <= hi && tile_start[idx] <= tile;
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        lo += (31 - __clz(m)) * step;            /* lane 0 is always set */
        hi = min(hi, lo + step - 1);
    }
    const int *js = (const int *)(jobs + lo);
    int *jd = (int *)(s_job + slot);
    for (int w = lane; w < (int)(sizeof(atkb_job) / 4); w += 32) cp_async4(jd + w, js + w);
    const int *bs = (const int *)jobs[lo].bank;
    int *bd = (int *)(s_bank + slot);
    for (int w = lane; w < (int)(sizeof(atkb_bank) / 4); w += 32) cp_async4(bd + w, bs + w);
    if (lane == 0) s_local[slot] = tile - tile_start[lo];
}

/* dst[0, len) = s[from, from + len), eight loads in flight per thread before
 * their stores (a load-store loop would wait one memory round trip per
 * step: the compiler cannot tell dst from the sources) */
template <int T>
__device__ __forceinline__ void carry_copy(const Src &src, float2 *dst, long long from, long long len) {
    for (long long i0 = threadIdx.x; i0 < len; i0 += 8LL * T) {
        float2 v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const long long i = i0 + (long long)u * T;
            if (i < len) v[u] = src.at(from + i);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const long long i = i0 + (long long)u * T;
            if (i < len) dst[i] = v[u];
        }
    }
}

#ifndef ATKB_TILE_MINB
#define ATKB_TILE_MINB (PTS == 8 ? 2 : 2)
#endif
__global__ void __launch_bounds__(NT, ATKB_TILE_MINB)
pfb_tiles_kernel(const atkb_job *__restrict__ jobs, const int *__restrict__ tile_start,
                 const atkb_carry *__restrict__ carries, int njobs, const int *__restrict__ d_njobs,
                 int *counters) {
    extern __shared__ double2 sm[];
    /* launched as a programmatic dependent of the kernel that fills the job
     * table (atkb_pfb_launch_pdl): wait for it before the first read; a no-op
     * for an ordinary launch */
    asm volatile("griddepcontrol.wait;" ::: "memory");
    if (d_njobs) njobs = min(njobs, *d_njobs);      /* a server round: count set per launch */
    unsigned dyn_smem;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_smem));
    const int total_tiles = njobs > 0 ? tile_start[njobs] : 0;
    /* two slots: warp 0 fetches tile i+1 into one while the CTA works on
     * tile i from the other */
    __shared__ int s_tile[2], s_local[2];
    __shared__ atkb_bank s_bank[2];
    __shared__ atkb_job s_job[2];
    if (threadIdx.x < 32) fetch_tile(jobs, tile_start, njobs, total_tiles, counters, s_tile, s_local, s_job, s_bank, 0);
    for (int slot = 0;; slot ^= 1) {
        if (threadIdx.x < 32) cp_async_wait_all();  /* this slot's copies, issued by warp 0 */
        __syncthreads();
        const int tile = s_tile[slot];
        if (tile >= total_tiles) break;
        if (threadIdx.x < 32)
            fetch_tile(jobs, tile_start, njobs, total_tiles, counters, s_tile, s_local, s_job, s_bank, slot ^ 1);
        const atkb_job &J = s_job[slot];
        const atkb_bank &SB = s_bank[slot];
        const long long h0 = (long long)s_local[slot] * SB.tile_hops;
        const long long left = J.hops - h0;
        const int nvalid = (int)(left < SB.tile_hops ? left : SB.tile_hops);
        const int lm = SB.plan.fast ? SB.logm : 0;
        int key = SB.plan.quad ? 80 + 16 * (SB.os == 1 ? 0 : 1) + lm
                : SB.plan.pair ? 16 * (1 + (SB.os == 1 ? 0 : SB.os == 2 ? 1 : 2)) + lm : lm;
        /* a launch with less dynamic shared memory than the bank's tile needs
         * skips the tile (its outputs stay unwritten) instead of running off
         * the end of shared memory */
        if ((unsigned)SB.smem_bytes > dyn_smem) key = -1;
        /* bounds, uniform across the CTA: the tile's last window must end
         * within the job's samples and its columns within the output rows */
        {
            unsigned bad = 0;
            if ((h0 + nvalid - 1) * (long long)SB.hop + SB.L > J.nsrc || h0 + nvalid > J.hops) bad |= ATKB_FAULT_WINDOW;
            if (J.out_col + h0 + nvalid > J.ldo) bad |= ATKB_FAULT_OUTPUT;
            if (bad) {
                if (threadIdx.x == 0) atomicOr((unsigned *)&counters[ATKB_FAULT_WORD], bad);
                key = -1;
            }
        }
        float2 *to = (float2 *)sm;
        switch (key) {
#define UNPAIRED(L) case L: tile_fast<L, -1>(J, SB, h0, nvalid, sm, to); break;
#define PAIRED(L)                                                              \
        case 16 + L: tile_fast<L, 0>(J, SB, h0, nvalid, sm, to); break;    \
        case 32 + L: tile_fast<L, 1>(J, SB, h0, nvalid, sm, to); break;    \
        case 48 + L: tile_fast<L, 2>(J, SB, h0, nvalid, sm, to); break;
        UNPAIRED(4) UNPAIRED(5) UNPAIRED(6) UNPAIRED(7) UNPAIRED(8) UNPAIRED(9) UNPAIRED(10)
        UNPAIRED(11)
        case 12:
            if (!SB.plan.ptaps) tile_4096x2(J, SB, h0, nvalid, sm);
            else if (SB.os == 1) tile_4096x2_pair<0>(J, SB, h0, nvalid, sm);
            else if (SB.os == 2) tile_4096x2_pair<1>(J, SB, h0, nvalid, sm);
            else tile_4096x2_pair<2>(J, SB, h0, nvalid, sm);
            break;
        PAIRED(4) PAIRED(5) PAIRED(6) PAIRED(7) PAIRED(8) PAIRED(9) PAIRED(10) PAIRED(11)
#define QUAD(L)                                                                \
        case 80 + L: tile_quad<L, 0>(J, SB, h0, nvalid, sm, to); break;    \
        case 96 + L: tile_quad<L, 1>(J, SB, h0, nvalid, sm, to); break;
        QUAD(4) QUAD(5) QUAD(6) QUAD(7) QUAD(8) QUAD(9) QUAD(10)
#undef UNPAIRED
#undef PAIRED
#undef QUAD
        case -1: break;
        default: tile_generic(J, SB, h0, nvalid, sm); break;
        }
        /* the barrier at the top of the loop fences this tile's reads of sm
         * and of its slot from the next tile's writes */
    }
    /* this CTA's tiles are done: a programmatic dependent (the W2 finish of
     * atkdsp_gpu_pfb_process_w12) may be scheduled once every CTA is here; it
     * waits for this grid's completion before it reads anything */
    asm volatile("griddepcontrol.launch_dependents;");
    /* then the state carries, one job's per claim, the CTA's threads copying
     * s[from, from + len) into the other state buffer (no tile reads it) */
    __shared__ int s_carry;
    for (;;) {
        if (threadIdx.x == 0) s_carry = atomicAdd(&counters[2], 1);
        __syncthreads();
        const int ci = s_carry;
        __syncthreads();                  /* read before thread 0 claims again */
        if (ci >= njobs) break;
        const atkb_carry &C = carries[ci];
        const Src src{(const float2 *)C.state, C.in, C.head, C.in_kind, C.cre, C.cim, C.kscale};
        float2 *dst = (float2 *)C.dst;
        const long long from = C.from, len = C.len;
        if (from < 0 || len < 0 || from + len > C.nsrc || len > C.cap) {   /* uniform: skip it */
            if (threadIdx.x == 0) atomicOr((unsigned *)&counters[ATKB_FAULT_WORD], ATKB_FAULT_CARRY);
            continue;
        }
        carry_copy<NT>(src, dst, from, len);
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const int done = atomicAdd(&counters[1], 1);
        if (done == (int)gridDim.x - 1) {      /* the last CTA out resets */
            atomicExch(&counters[0], 0);
            atomicExch(&counters[2], 0);
            atomicExch(&counters[1], 0);
        }
    }
}

/* ---- large filterbanks: nchan beyond one CTA's shared memory --------------
 * A power of two above 4096 or any other nchan above 6400 has no in-CTA tile:
 * a hop's M points (16 M bytes in double) do not fit beside a second buffer.
 * Such a filterbank runs one hop chunk at a time through device scratch:
 *   fold      one thread per (hop, branch), the reference's operation order
 *             (a rounded multiply, then a rounded add, k ascending);
 *   FFT       the plan's Stockham passes, each one kernel over the chunk,
 *             ping-ponging between the two scratch halves (mixed radix 2, 3,
 *             4, 8, 16, and a direct DFT for any other prime factor);
 *   epilogue  rotation, cal and rounding as the tile kernel does them, written
 *             channel-major (a warp's lanes on consecutive hops of a channel).
 * Slower than the tile kernel (every pass goes through HBM), but any nchan
 * the reference accepts runs, with the same results. */
__global__ void __launch_bounds__(256)
big_fold_kernel(const atkb_job J, const float *__restrict__ taps, int M, int K, int hop, long long h0, int nh,
                double2 *__restrict__ F) {
    float cre = J.cre, cim = J.cim;
    if (J.doff) doff_consts(J.doff, J.kscale, cre, cim);
    const Src src{(const float2 *)J.state, J.in, J.head, J.in_kind, cre, cim, J.kscale};
    const long long total = (long long)nh * M;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int t = (int)(e / M);
        const int q = (int)(e - (long long)t * M);
        const long long base = (h0 + t) * (long long)hop + q;
        float h = __ldg(taps + q);
        float2 x = src.at(base);
        float fr = __fmul_rn(h, x.x), fi = __fmul_rn(h, x.y);
        for (int k = 1; k < K; ++k) {
            h = __ldg(taps + (long long)k * M + q);
            x = src.at(base + (long long)k * M);
            fr = __fadd_rn(fr, __fmul_rn(h, x.x));
            fi = __fadd_rn(fi, __fmul_rn(h, x.y));
        }
        F[e] = make_double2((double)fr, (double)fi);
    }
}

__global__ void __launch_bounds__(256)
big_pass_kernel(const double2 *__restrict__ src, double2 *__restrict__ dst, int M, int Ns, int R, int nh,
                const double2 *__restrict__ W) {
    const int MR = M / R;
    const int NsR = Ns * R;
    const int stride = M / NsR;
    const long long total = (long long)nh * MR;
    for (long long bi = (long long)blockIdx.x * blockDim.x + threadIdx.x; bi < total;
         bi += (long long)gridDim.x * blockDim.x) {
        const int tt = (int)(bi / MR);
        const int j = (int)(bi - (long long)tt * MR);
        const int k = j % Ns;
        const double2 *s = src + (long long)tt * M + j;
        double2 *d = dst + (long long)tt * M + (long long)(j - k) * R + k;
        if (R == 2 || R == 3 || R == 4 || R == 8 || R == 16) {
            double2 v[16];
            for (int r = 0; r < R; ++r) {
                v[r] = s[(long long)r * MR];
                if (r) v[r] = cmul(v[r], __ldg(W + (long long)r * k * stride));
            }
            if (R == 2) dft2(v[0], v[1]);
            else if (R == 3) dft3(v[0], v[1], v[2]);
            else if (R == 4) dft4(v[0], v[1], v[2], v[3]);
            else if (R == 8) dft8(v);
            else dft16(v);
            for (int r = 0; r < R; ++r) d[(long long)r * Ns] = v[r];
        } else {
            /* direct DFT with the twiddle folded in: W_{NsR}^{r (k + o Ns)} */
            for (int o = 0; o < R; ++o) {
                double2 acc = make_double2(0.0, 0.0);
                for (int r = 0; r < R; ++r) {
                    const long long ex = ((long long)r * (k + (long long)o * Ns)) % NsR;
                    const double2 w = __ldg(W + ex * stride);
                    const double2 x = s[(long long)r * MR];
                    acc.x += x.x * w.x - x.y * w.y;
                    acc.y += x.x * w.y + x.y * w.x;
                }
                d[(long long)o * Ns] = acc;
            }
        }
    }
}

__global__ void __launch_bounds__(256)
big_out_kernel(const double2 *__restrict__ X, const atkb_job J, const double2 *__restrict__ twd, int M, int os,
               int hop, long long h0, int nh) {
    const float2 *cal = (const float2 *)J.cal;
    float2 *out = (float2 *)J.out;
    const long long total = (long long)nh * M;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int kb = (int)(e / nh);
        const int tt = (int)(e - (long long)kb * nh);
        double2 v = X[(long long)tt * M + kb];
        const long long b = J.b0 + h0 + tt;
        const int s = (int)((b + 1) % os);
        const int jr = (int)(((long long)kb * s) % os);
        v = cmul_rn(v, __ldg(twd + (jr ? M - jr * hop : 0)));
        if (cal) {
            const float2 c = __ldg(cal + kb);
            v = cmul_rn(v, make_double2((double)c.x, (double)c.y));
        }
        out[(long long)kb * J.ldo + J.out_col + h0 + tt] = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
    }
}


/* ---- small calls: one CTA per hop ------------------------------------------
 * A host call of a few thousand samples completes a few dozen hops; the tile
 * kernel would run them as one tile in one CTA, whose fold and passes take
 * ~20 us of latency. Here every hop of every job gets its own CTA of
 * HOPS_NT threads (power-of-two nchan 16..1024 on the fast plan), and the
 * jobs' state carries one CTA each after them:
 *   fold    thread per branch q, k ascending, a rounded multiply then a
 *           rounded add: the bits of every tile shape's fold;
 *   FFT     the bank's own plan, pass by pass between two shared-memory
 *           buffers: the first pass (radix plan.radix[0], Ns = 1) without
 *           twiddles, the others with tw_powers of the bank's per-pass table
 *           and cmul, the last fused with finish_bin -- the arithmetic of the
 *           tile kernel's passes, so the outputs equal the tile path's bits.
 * The uniform bounds checks are the tile kernel's (window, output, carry). */
#define HOPS_NT 128
#define HOPS_MAXM 1024

template <int R>
__device__ __forceinline__ void hop_pass(const double2 *__restrict__ src, double2 *__restrict__ dst, int M, int Ns,
                                         const double2 *__restrict__ tw, bool first) {
    const int MR = M / R;
    for (int j = threadIdx.x; j < MR; j += HOPS_NT) {
        const int k = j & (Ns - 1);
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[j + r * MR];
        if (!first) {
            double2 w[R];
            tw_powers<R>(__ldg(tw + k), w);
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
        }
        dftR<R>(v);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[d + r * Ns] = v[r];
    }
}

template <int R>
__device__ __forceinline__ void hop_pass_last(const double2 *__restrict__ src, int M, int Ns,
                                              const double2 *__restrict__ tw, bool first, const atkb_bank &B,
                                              const atkb_job &J, long long t) {
    const int MR = M / R;                       /* == Ns */
    const double2 *twd = (const double2 *)B.twd;
    const float2 *cal = (const float2 *)J.cal;
    float2 *out = (float2 *)J.out;
    const int osm = B.os - 1;
    const int s = (int)(J.b0 + t + 1) & osm;
    for (int j = threadIdx.x; j < MR; j += HOPS_NT) {
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[j + r * MR];
        if (!first) {
            double2 w[R];
            tw_powers<R>(__ldg(tw + j), w);
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
        }
        dftR<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int kb = j + r * Ns;
            out[(long long)kb * J.ldo + J.out_col + t] = finish_bin(v[r], kb, s, M, osm + 1, B.hop, true, twd, cal);
        }
    }
}

__global__ void __launch_bounds__(HOPS_NT)
pfb_hops_kernel(const atkb_job *__restrict__ jobs, const atkb_carry *__restrict__ carries, int njobs, int m,
                int *counters) {
    __shared__ double2 buf[2][HOPS_MAXM];
    __shared__ atkb_bank SB;
    const int b = blockIdx.x;
    if (b >= njobs * m) {                       /* a state carry */
        const int ci = b - njobs * m;
        if (ci >= njobs) return;
        const atkb_carry &C = carries[ci];
        const long long from = C.from, len = C.len;
        if (from < 0 || len < 0 || from + len > C.nsrc || len > C.cap) {
            if (threadIdx.x == 0) atomicOr((unsigned *)&counters[ATKB_FAULT_WORD], ATKB_FAULT_CARRY);
            return;
        }
        const Src src{(const float2 *)C.state, C.in, C.head, C.in_kind, C.cre, C.cim, C.kscale};
        float2 *dst = (float2 *)C.dst;
        carry_copy<HOPS_NT>(src, dst, from, len);
        return;
    }
    const atkb_job &J = jobs[b / m];
    const long long t = b % m;
    {
        static_assert(sizeof(atkb_bank) % 4 == 0, "word copies");
        const int *bs = (const int *)J.bank;
        int *bd = (int *)&SB;
        for (int w = threadIdx.x; w < (int)(sizeof(atkb_bank) / 4); w += HOPS_NT) bd[w] = bs[w];
    }
    __syncthreads();
    const int M = SB.nchan;
    /* uniform across the CTA: a shape this kernel does not run, a window past
     * the job's samples or a column past the row stride skips the hop */
    {
        unsigned bad = 0;
        if (t >= J.hops || t * SB.hop + SB.L > J.nsrc) bad |= ATKB_FAULT_WINDOW;
        if (J.out_col + t + 1 > J.ldo) bad |= ATKB_FAULT_OUTPUT;
        if (!SB.plan.fast || M > HOPS_MAXM || M < 16) bad |= ATKB_FAULT_INDEX;
        for (int p = 0; p < SB.plan.npass; ++p)
            if (SB.plan.radix[p] != 2 && SB.plan.radix[p] != 4 && SB.plan.radix[p] != 8) bad |= ATKB_FAULT_INDEX;
        if (bad) {
            if (threadIdx.x == 0) atomicOr((unsigned *)&counters[ATKB_FAULT_WORD], bad);
            return;
        }
    }
    /* the fold, one branch per thread and step, eight taps' loads in flight */
    {
        const Src src{(const float2 *)J.state, J.in, J.head, J.in_kind, J.cre, J.cim, J.kscale};
        const float *taps = SB.taps;
        const int K = SB.K;
        const long long base = t * SB.hop;
        for (int q = threadIdx.x; q < M; q += HOPS_NT) {
            float fr = -0.0f, fi = -0.0f;
            for (int k0 = 0; k0 < K; k0 += 8) {
                float h[8];
                float2 x[8];
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (k0 + u < K) {
                        h[u] = __ldg(taps + (long long)(k0 + u) * M + q);
                        x[u] = src.at(base + (long long)(k0 + u) * M + q);
                    }
#pragma unroll
                for (int u = 0; u < 8; ++u)
                    if (k0 + u < K) {
                        fr = __fadd_rn(fr, __fmul_rn(h[u], x[u].x));
                        fi = __fadd_rn(fi, __fmul_rn(h[u], x[u].y));
                    }
            }
            buf[0][q] = make_double2((double)fr, (double)fi);
        }
    }
    __syncthreads();
    /* the plan's passes */
    const double2 *wp = (const double2 *)SB.wpass;
    int Ns = 1, cur = 0;
    for (int p = 0; p < SB.plan.npass; ++p) {
        const int R = SB.plan.radix[p];
        const double2 *tw = wp + SB.plan.twoff[p];
        const bool first = p == 0;
        if (p == SB.plan.npass - 1) {
            if (R == 8) hop_pass_last<8>(buf[cur], M, Ns, tw, first, SB, J, t);
            else if (R == 4) hop_pass_last<4>(buf[cur], M, Ns, tw, first, SB, J, t);
            else hop_pass_last<2>(buf[cur], M, Ns, tw, first, SB, J, t);
        } else {
            if (R == 8) hop_pass<8>(buf[cur], buf[cur ^ 1], M, Ns, tw, first);
            else if (R == 4) hop_pass<4>(buf[cur], buf[cur ^ 1], M, Ns, tw, first);
            else hop_pass<2>(buf[cur], buf[cur ^ 1], M, Ns, tw, first);
            __syncthreads();
            cur ^= 1;
        }
        Ns *= R;
    }
}

}  // namespace

extern "C" int atkb_pfb_max_smem(void) { return 200 * 1024; }

extern "C" int atkb_pfb_grid(int dev, int smem_bytes) {
    /* the attribute is idempotent: concurrent first callers may both set it */
    static std::atomic<bool> configured[64];
    if (dev < 0 || dev >= 64) return -1;
    if (!configured[dev].load(std::memory_order_acquire)) {
        if (cudaFuncSetAttribute(pfb_tiles_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 atkb_pfb_max_smem()) != cudaSuccess)
            return -1;
        configured[dev].store(true, std::memory_order_release);
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pfb_tiles_kernel, NT, smem_bytes) !=
        cudaSuccess || per_sm < 1)
        per_sm = 1;
    return per_sm * atkb_sm_count(dev);
}

extern "C" int atkb_pfb_launch(const atkb_job *d_jobs, const int *d_tile_start, const atkb_carry *d_carry,
                               int njobs, int *d_counters, int grid, int smem_bytes, void *stream) {
    return atkb_pfb_launch_n(d_jobs, d_tile_start, d_carry, njobs, NULL, d_counters, grid, smem_bytes,
                             stream);
}

extern "C" int atkb_pfb_launch_n(const atkb_job *d_jobs, const int *d_tile_start, const atkb_carry *d_carry,
                                 int njobs, const int *d_njobs, int *d_counters, int grid, int smem_bytes,
                                 void *stream) {
    if (njobs <= 0) return ATKB_OK;
    if (grid < 1) grid = 1;
    atkb_range_push("atkdsp tile kernel launch");
    pfb_tiles_kernel<<<grid, NT, smem_bytes, (cudaStream_t)stream>>>(d_jobs, d_tile_start, d_carry, njobs,
                                                                    d_njobs, d_counters);
    atkb_range_pop();
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

/* atkb_pfb_launch as a programmatic dependent launch: its CTAs may start
 * while the previous kernel on the stream (conv_from_offset_kernel) runs,
 * and wait for that kernel's completion before reading the table */
extern "C" int atkb_pfb_launch_pdl(const atkb_job *d_jobs, const int *d_tile_start, const atkb_carry *d_carry,
                                   int njobs, int *d_counters, int grid, int smem_bytes, void *stream) {
    if (njobs <= 0) return ATKB_OK;
    if (grid < 1) grid = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = (size_t)smem_bytes;
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const int *no_count = nullptr;
    atkb_range_push("atkdsp tile kernel launch");
    const cudaError_t e = cudaLaunchKernelEx(&cfg, pfb_tiles_kernel, d_jobs, d_tile_start, d_carry, njobs, no_count,
                                             d_counters);
    atkb_range_pop();
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" long long atkb_pfb_big_hops(int nchan) {
    const long long h = (1LL << 20) / nchan;
    return h < 1 ? 1 : h;
}

extern "C" int atkb_pfb_big(const atkb_job *J, const atkb_bank *B, long long h0, int nh, void *scratch,
                            int grid, void *stream) {
    if (nh <= 0) return ATKB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const int M = B->nchan;
    double2 *A = (double2 *)scratch, *Bf = A + (size_t)nh * M;
    if (grid < 1) grid = 1;
    atkb_range_push("atkdsp large-filterbank chunk");
    big_fold_kernel<<<grid, 256, 0, st>>>(*J, B->taps, M, B->K, B->hop, h0, nh, A);
    int Ns = 1;
    double2 *cur = A, *nxt = Bf;
    for (int p = 0; p < B->plan.npass; ++p) {
        const int R = B->plan.radix[p];
        big_pass_kernel<<<grid, 256, 0, st>>>(cur, nxt, M, Ns, R, nh, (const double2 *)B->wfull);
        Ns *= R;
        double2 *t = cur; cur = nxt; nxt = t;
    }
    big_out_kernel<<<grid, 256, 0, st>>>(cur, *J, (const double2 *)B->twd, M, B->os, B->hop, h0, nh);
    atkb_range_pop();
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

/* The constants of nel device jobs (and their carries) whose int16 offset
 * lives in device memory, written into the job table after its upload and
 * before the tile kernel reads it: the tile kernel itself stays unchanged. */
__global__ void conv_from_offset_kernel(atkb_job *jobs, atkb_carry *carries, int nel) {
    /* let the tile kernel launch now: it waits for this grid's completion
     * (griddepcontrol.wait) before it reads the table */
    asm volatile("griddepcontrol.launch_dependents;");
    const int e = threadIdx.x;
    if (e >= nel || !jobs[e].doff) return;
    float cre, cim;
    doff_consts(jobs[e].doff, jobs[e].kscale, cre, cim);
    jobs[e].cre = carries[e].cre = cre;
    jobs[e].cim = carries[e].cim = cim;
}

/* A one-job table from the launch's own parameters (no host->device copy):
 * the job, its carry and the tile starts, the int16 constants derived from
 * the device-held offset when the job has one. */
__global__ void job_from_params_kernel(const atkb_job J, const atkb_carry C, int tiles, atkb_job *jobs,
                                       atkb_carry *carries, int *tile_start) {
    asm volatile("griddepcontrol.launch_dependents;");
    if (threadIdx.x != 0) return;
    atkb_job j = J;
    atkb_carry c = C;
    if (j.doff) {
        float cre, cim;
        doff_consts(j.doff, j.kscale, cre, cim);
        j.cre = c.cre = cre;
        j.cim = c.cim = cim;
    }
    jobs[0] = j;
    carries[0] = c;
    tile_start[0] = 0;
    tile_start[1] = tiles;
}

extern "C" int atkb_pfb_job_from_params(const atkb_job *J, const atkb_carry *C, int tiles, atkb_job *d_jobs,
                                        atkb_carry *d_carry, int *d_tile_start, void *stream) {
    job_from_params_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(*J, *C, tiles, d_jobs, d_carry, d_tile_start);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" int atkb_pfb_conv_from_offset(atkb_job *d_jobs, atkb_carry *d_carry, int nel, void *stream) {
    if (nel < 1 || nel > 1024) return ATKB_E_ARG;
    conv_from_offset_kernel<<<1, nel, 0, (cudaStream_t)stream>>>(d_jobs, d_carry, nel);
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

/* the small-call kernel: njobs jobs of m hops each, then their carries */
extern "C" int atkb_pfb_hops(const atkb_job *d_jobs, const atkb_carry *d_carry, int njobs, int m, int *d_counters,
                             void *stream) {
    if (njobs < 1 || m < 0) return ATKB_E_ARG;
    const long long grid = (long long)njobs * m + njobs;
    if (grid > 0x7fffffffLL) return ATKB_E_ARG;
    atkb_range_push("atkdsp small call");
    pfb_hops_kernel<<<(unsigned)grid, HOPS_NT, 0, (cudaStream_t)stream>>>(d_jobs, d_carry, njobs, m, d_counters);
    atkb_range_pop();
    return cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}

extern "C" int atkb_pfb_hops_ok(const atkb_bank *B) {
    if (!B->plan.fast || B->plan.big || B->nchan < 16 || B->nchan > HOPS_MAXM) return 0;
    for (int p = 0; p < B->plan.npass; ++p)
        if (B->plan.radix[p] != 2 && B->plan.radix[p] != 4 && B->plan.radix[p] != 8) return 0;
    return 1;
}

extern "C" unsigned atkb_pfb_debug_fault(void) {
#ifdef ATKB_DEBUG_BOUNDS
    unsigned v = 0, z = 0;
    if (cudaMemcpyFromSymbol(&v, g_atkb_debug_fault, sizeof v) != cudaSuccess) return ATKB_FAULT_INDEX;
    if (v) cudaMemcpyToSymbol(g_atkb_debug_fault, &z, sizeof z);
    return v;
#else
    return 0;
#endif
}

extern "C" int atkb_pfb_debug_build(void) {
#ifdef ATKB_DEBUG_BOUNDS
    return 1;
#else
    return 0;
#endif
}

namespace {
/* the tiles' W2 partials of one single-element job, per channel: W2 power
 * (S / m), and W1 for one element (R[k] += S, counts += m), gated like
 * atkb_w12. A block of W2F_WARPS warps takes W2F_CH = 8 channels: lane l of
 * warp w reads channel l % 8 of the tiles t = s, s + 64, ... (s = 4w + l / 8,
 * 64 tile streams; sixteen loads in flight, each quarter-warp one 64-byte
 * row segment). The 64 stream sums of a channel are then added by a fixed tree
 * (eight groups of eight in stream order, then the eight group sums in
 * order), so the result is deterministic. Eight channels a block spread the
 * reads of nchan 1024 over 128 SMs. */
#define W2F_WARPS 16
#define W2F_CH 8
#define W2F_STREAMS (W2F_WARPS * 32 / W2F_CH)
__global__ void __launch_bounds__(32 * W2F_WARPS)
w2_finish_kernel(const double *__restrict__ part, int tiles, int M, long long m, const uint8_t *__restrict__ gate,
                 float2 *__restrict__ R, uint32_t *__restrict__ counts, float *__restrict__ pwr,
                 float *__restrict__ mean_pwr) {
    /* launched as a programmatic dependent of the tile kernel: wait for it */
    asm volatile("griddepcontrol.wait;" ::: "memory");
    __shared__ double red[W2F_STREAMS][W2F_CH];
    __shared__ double grp[W2F_STREAMS / 8][W2F_CH];
    const int c = threadIdx.x % W2F_CH, sidx = threadIdx.x / W2F_CH;
    const int k = blockIdx.x * W2F_CH + c;
    double S = 0.0;
    if (k < M) {
        /* sixteen loads in flight, the ones past the last tile read as +0.0
         * (S >= +0.0, so adding it is exact and the order is unchanged) */
        for (int t = sidx; t < tiles; t += 16 * W2F_STREAMS) {
            double v[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int r = t + u * W2F_STREAMS;
                v[u] = r < tiles ? __ldg(part + (long long)r * M + k) : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 16; ++u) S += v[u];
        }
    }
    red[sidx][c] = S;
    __syncthreads();
    if (threadIdx.x < (W2F_STREAMS / 8) * W2F_CH) {
        const int g = threadIdx.x / W2F_CH;
        double G = 0.0;
#pragma unroll
        for (int j = 0; j < 8; ++j) G += red[8 * g + j][c];
        grp[g][c] = G;
    }
    __syncthreads();
    if (threadIdx.x >= W2F_CH || k >= M) return;
    S = 0.0;
#pragma unroll
    for (int g = 0; g < W2F_STREAMS / 8; ++g) S += grp[g][c];
    const double inv = m ? 1.0 / (double)m : 0.0;
    if (pwr) pwr[k] = (float)(S * inv);
    if (mean_pwr) mean_pwr[k] = (float)((S * inv) / 1.0);
    if (R && counts && (!gate || gate[k])) {
        if (m > 0) {
            const float2 v = R[k];
            R[k] = make_float2((float)((double)v.x + S), (float)((double)v.y + 0.0));
        }
        counts[k] += (uint32_t)m;
    }
}
}  // namespace

extern "C" int atkb_w2_finish(const double *part, int tiles, int nchan, long long m, const uint8_t *gate, void *R,
                              uint32_t *counts, float *pwr, float *mean_pwr, void *stream) {
    /* a programmatic dependent of the tile kernel launched just before it on
     * the stream: its launch overlaps that kernel's last tiles and carries */
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)((nchan + W2F_CH - 1) / W2F_CH));
    cfg.blockDim = dim3(32 * W2F_WARPS);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = (cudaStream_t)stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, w2_finish_kernel, part, tiles, nchan, m, gate, (float2 *)R,
                                             counts, pwr, mean_pwr);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? ATKB_OK : ATKB_E_KERNEL;
}
