/* CPU oracle for the spectrum reduction -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C99 restatement of the reference's display reduction
 * (src/fft.c:137-152 windows, :154-164 dB, :176-295 atkdsp_spectrum_reduce,
 * :315-430 atkdsp_spectrum_stats) for power-of-two lengths, run frame by
 * frame in order (the reference with one thread). Linked into
 * liboracle.so; only tests/, smoke() and bench.py's CPU leg load it.
 *
 * Pinning: tests/test_oracle_pinned.py checks it against tests/golden/
 * spectrum.npz, made by tests/golden/make_golden.py from the reference library
 * built from its own sources, run single-threaded.
 *
 * Numerics: window product and transform in double (the reference's
 * pocketfft; this file's own radix-2 transform agrees to ~1e-16); the
 * reduce's power in float from the float-rounded bin, |X|^2 / n^2 with the
 * reference's rounded steps; the stats' power and sums in double; dB with
 * sqrtf / log10f as the reference.
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#define SP_PI 3.14159265358979323846
#define SP_E_ARG -1
#define SP_E_NOMEM -2

typedef struct { float re, im; } sp_cf32;

/* window of `kind` (rect, Hann, Hamming, Blackman-Harris), src/fft.c:137-152 */
int orc_window(int kind, size_t n, float *out) {
    if (!out || n == 0) return SP_E_ARG;
    if (n == 1) { out[0] = 1.0f; return 0; }
    const double d = (double)(n - 1);
    for (size_t i = 0; i < n; ++i) {
        const double x = 2.0 * SP_PI * (double)i / d;
        double w;
        switch (kind) {
        case 0: w = 1.0; break;
        case 1: w = 0.5 - 0.5 * cos(x); break;
        case 2: w = 0.54 - 0.46 * cos(x); break;
        case 3: w = 0.35875 - 0.48829 * cos(x) + 0.14128 * cos(2 * x) - 0.01168 * cos(3 * x); break;
        default: return SP_E_ARG;
        }
        out[i] = (float)w;
    }
    return 0;
}

static void sp_fft(double *a, size_t n) {
    size_t i, j = 0;
    for (i = 1; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t = a[2 * i]; a[2 * i] = a[2 * j]; a[2 * j] = t;
            t = a[2 * i + 1]; a[2 * i + 1] = a[2 * j + 1]; a[2 * j + 1] = t;
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len >> 1;
        for (size_t k = 0; k < half; ++k) {
            const double ang = -2.0 * SP_PI * (double)k / (double)len;
            const double wr = cos(ang), wi = sin(ang);
            for (i = k; i < n; i += len) {
                double *u = a + 2 * i, *v = a + 2 * (i + half);
                const double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr; v[1] = u[1] - vi;
                u[0] += vr; u[1] += vi;
            }
        }
    }
}

/* one frame, windowed in double, transformed (src/fft.c:90-112) */
static void sp_frame(const sp_cf32 *in, const float *w, size_t n, double *sc) {
    for (size_t i = 0; i < n; ++i) {
        const double g = w ? (double)w[i] : 1.0;
        sc[2 * i] = w ? (double)in[i].re * g : (double)in[i].re;
        sc[2 * i + 1] = w ? (double)in[i].im * g : (double)in[i].im;
    }
    sp_fft(sc, n);
}

static int sp_frames(size_t n, size_t n_samples, size_t *hop, long long *frames) {
    if (n < 2 || (n & (n - 1))) return SP_E_ARG;
    if (*hop == 0 || *hop > n) *hop = n;
    *frames = n_samples < n ? 0 : (long long)((n_samples - n) / *hop + 1);
    return 0;
}

/* detector 0 max, 1 min, 2 average; one line of n dB values, fftshifted */
long long orc_spectrum_reduce(size_t n, const sp_cf32 *in, size_t n_samples, size_t hop, const float *window,
                              int detector, float *out_line) {
    long long frames;
    if (!in || !out_line || detector < 0 || detector > 2) return SP_E_ARG;
    if (sp_frames(n, n_samples, &hop, &frames)) return SP_E_ARG;
    if (frames == 0) return 0;
    double *sc = (double *)malloc(2 * n * sizeof(double));
    float *acc = (float *)malloc(n * sizeof(float));
    if (!sc || !acc) { free(sc); free(acc); return SP_E_NOMEM; }
    const size_t half = n / 2;
    const float inv2 = 1.0f / ((float)n * (float)n);
    for (long long f = 0; f < frames; ++f) {
        sp_frame(in + (size_t)f * hop, window, n, sc);
        for (size_t i = 0; i < n; ++i) {
            const size_t k = (i + half) % n;
            const float re = (float)sc[2 * k], im = (float)sc[2 * k + 1];
            const float pw = (re * re + im * im) * inv2;
            if (f == 0) { acc[i] = pw; continue; }
            if (detector == 0) { if (pw > acc[i]) acc[i] = pw; }
            else if (detector == 1) { if (pw < acc[i]) acc[i] = pw; }
            else acc[i] += pw;
        }
    }
    const float scale = detector == 2 ? 1.0f / (float)frames : 1.0f;
    for (size_t i = 0; i < n; ++i) {
        const float mag = sqrtf(acc[i] * scale);
        out_line[i] = 20.0f * log10f(mag + 1e-12f);
    }
    free(sc); free(acc);
    return frames;
}

/* per bin: peak, mean and floor power in dB and the spectral kurtosis
 * M * sum P^2 / (sum P)^2 (1.0 for one frame); any output may be NULL */
long long orc_spectrum_stats(size_t n, const sp_cf32 *in, size_t n_samples, size_t hop, const float *window,
                             float *max_db, float *avg_db, float *min_db, float *sk) {
    long long frames;
    if (!in || (!max_db && !avg_db && !min_db && !sk)) return SP_E_ARG;
    if (sp_frames(n, n_samples, &hop, &frames)) return SP_E_ARG;
    if (frames == 0) return 0;
    double *sc = (double *)malloc(2 * n * sizeof(double));
    double *st = (double *)malloc(4 * n * sizeof(double));
    if (!sc || !st) { free(sc); free(st); return SP_E_NOMEM; }
    double *mx = st, *mn = st + n, *su = st + 2 * n, *s2 = st + 3 * n;
    const size_t half = n / 2;
    const double inv2 = 1.0 / ((double)n * (double)n);
    for (long long f = 0; f < frames; ++f) {
        sp_frame(in + (size_t)f * hop, window, n, sc);
        for (size_t i = 0; i < n; ++i) {
            const size_t k = (i + half) % n;
            const double re = sc[2 * k], im = sc[2 * k + 1];
            const double pw = (re * re + im * im) * inv2;
            if (f == 0) { mx[i] = mn[i] = su[i] = pw; s2[i] = pw * pw; continue; }
            if (pw > mx[i]) mx[i] = pw;
            if (pw < mn[i]) mn[i] = pw;
            su[i] += pw;
            s2[i] += pw * pw;
        }
    }
    const double M = (double)frames;
    for (size_t i = 0; i < n; ++i) {
        if (max_db) max_db[i] = 10.0f * log10f((float)mx[i] + 1e-12f);
        if (min_db) min_db[i] = 10.0f * log10f((float)mn[i] + 1e-12f);
        if (avg_db) avg_db[i] = 10.0f * log10f((float)(su[i] / M) + 1e-12f);
        if (sk) {
            const double den = su[i] * su[i];
            sk[i] = (frames < 2 || den <= 0.0) ? 1.0f : (float)(M * s2[i] / den);
        }
    }
    free(sc); free(st);
    return frames;
}
