/* CPU stand-ins for the device shim, so that the CFAR's host code
 * (atkdsp_b200/csrc/cfar_host.c: solver, tables, pass pipeline, column
 * selection, tracker) runs without a GPU -- TEST INFRASTRUCTURE ONLY, built
 * by tests/test_cfar_host.py into a temporary library. Memory is host
 * memory, copies are memcpy, streams and events are no-ops, and the four
 * CFAR kernels of cfar.cu are restated as plain loops in the same order
 * (the OS statistic by sorting, which gives the same value as counting). */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "internal.h"
int atkb_map_rc(int rc) { return rc == 0 ? 0 : rc == -1 ? -1 : rc == -2 ? -2 : rc == -3 ? -3 : -4; }
int atkb_stream_create(void **s) { *s = (void *)1; return 0; }
void atkb_stream_destroy(void *s) { (void)s; }
int atkb_stream_sync(void *s) { (void)s; return 0; }
int atkb_event_create(void **e) { *e = (void *)1; return 0; }
void atkb_event_destroy(void *e) { (void)e; }
int atkb_event_record(void *e, void *s) { (void)e; (void)s; return 0; }
int atkb_event_sync(void *e) { (void)e; return 0; }
int atkb_stream_wait(void *s, void *e) { (void)e; (void)s; return 0; }
int atkb_malloc(void **p, size_t b) { *p = malloc(b ? b : 1); return *p ? 0 : -2; }
void atkb_free(void *p) { free(p); }
int atkb_host_alloc(void **p, size_t b) { *p = malloc(b ? b : 1); return *p ? 0 : -2; }
void atkb_host_free(void *p) { free(p); }
int atkb_h2d(void *d, const void *s, size_t b, void *st) { (void)st; memcpy(d, s, b); return 0; }
int atkb_d2h(void *d, const void *s, size_t b, void *st) { (void)st; memcpy(d, s, b); return 0; }
int atkb_d2d(void *d, const void *s, size_t b, void *st) { (void)st; memcpy(d, s, b); return 0; }
int atkb_memset(void *p, int v, size_t b, void *st) { (void)st; memset(p, v, b); return 0; }
int atkb_cfar_raw(const float *frames, int units, long long f0, int nf, long long nbins, double *raw, int ring,
                  void *stream) {
    (void)stream;
    for (long long e = 0; e < (long long)nf * nbins; ++e) {
        long long j = e / nbins, i = e - j * nbins;
        double v = frames[e];
        if (units == 0) { if (v < -300.0) v = -300.0; v = exp(v * 0.23025850929940458); }
        else if (v < 1e-30) v = 1e-30;
        raw[((f0 + j) % ring) * nbins + i] = v;
    }
    return 0;
}
static int cmpd(const void *a, const void *b) { double x = *(const double *)a, y = *(const double *)b; return x < y ? -1 : x > y; }
int atkb_cfar_test(const double *raw, int ring, long long f0, long long t0, int nf, long long nbins, int k, int mode,
                   int n_ref, int N, int os_k, double alpha, double alpha_ca, double et, const uint8_t *ok,
                   const uint8_t *sided, const int32_t *idx, double *X, double *noise, double *thr, uint8_t *hits,
                   uint32_t *bits, long long words, void *stream) {
    (void)stream;
    double *sel = malloc(N * sizeof(double));
    for (long long f = t0; f < f0 + nf; ++f) {
        double *Xr = X + (f - f0) * nbins;
        for (long long i = 0; i < nbins; ++i) {
            double s = 0.0;
            for (int r = 0; r < k; ++r) s += raw[((f - k + 1 + r) % ring) * nbins + i];
            Xr[i] = s / k;
        }
        long long row = (f - f0) * nbins;
        for (long long i = 0; i < nbins; ++i) {
            if (!ok[i]) { noise[row + i] = NAN; thr[row + i] = NAN; hits[row + i] = 0; continue; }
            double Z, a = alpha, scale = et;
            if (mode == 1) {
                int nan = 0;
                for (int q = 0; q < N; ++q) { sel[q] = Xr[idx[(long long)q * nbins + i]]; nan |= isnan(sel[q]); }
                if (nan) Z = NAN; else { qsort(sel, N, sizeof(double), cmpd); Z = sel[os_k - 1]; }
            } else if ((mode == 2 || mode == 3) && sided[i]) {
                double L = 0, R = 0;
                for (int q = 0; q < n_ref; ++q) L += Xr[idx[(long long)q * nbins + i]];
                for (int q = n_ref; q < N; ++q) R += Xr[idx[(long long)q * nbins + i]];
                L /= n_ref; R /= n_ref;
                if (isnan(L) || isnan(R)) Z = NAN; else Z = mode == 2 ? (L > R ? L : R) : (L < R ? L : R);
            } else {
                double s = 0;
                for (int q = 0; q < N; ++q) s += Xr[idx[(long long)q * nbins + i]];
                Z = s / N;
                if (mode == 2 || mode == 3) { a = alpha_ca; scale = 1.0; }
            }
            thr[row + i] = a * Z; noise[row + i] = Z / scale; hits[row + i] = Xr[i] > thr[row + i];
        }
        for (long long w = 0; w < words; ++w) {
            uint32_t m = 0;
            for (int b = 0; b < 32; ++b) { long long i = w * 32 + b; if (i < nbins && hits[row + i]) m |= 1u << b; }
            bits[(f - f0) * words + w] = m;
        }
    }
    free(sel);
    return 0;
}

int atkb_cfar_gather(const double *X, const double *noise, long long nbins, int rows, const double *raw, int ring,
                     long long rf0, int nraw, const int32_t *cols, int ncol, double *Xc, double *Nc, double *Rc,
                     void *stream) {
    (void)stream;
    for (int r = 0; r < rows; ++r) for (int q = 0; q < ncol; ++q) {
        Xc[(long long)r * ncol + q] = X[r * nbins + cols[q]]; Nc[(long long)r * ncol + q] = noise[r * nbins + cols[q]]; }
    for (int r = 0; r < nraw; ++r) for (int q = 0; q < ncol; ++q)
        Rc[(long long)r * ncol + q] = raw[((rf0 + r) % ring) * nbins + cols[q]];
    return 0;
}
