/* Host side of the device spectrum reduction, in C99: the reference's
 * argument rules for atkdsp_spectrum_reduce / atkdsp_spectrum_stats
 * (src/fft.c:176-187, :315-325) and the plan's device tables. The frames
 * are split into contiguous runs, one per CTA (at most two per SM), whose
 * partial lines live in the plan (allocated by create; a call allocates
 * nothing). */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdlib.h>

#include "host_internal.h"

#define SPEC_PI 3.14159265358979323846

struct atkdsp_gpu_spectrum {
    size_t n;
    int logn;
    int maxblk;                   /* partial lines held */
    void *d_tw;                   /* n double2: (cos, -sin)(2 pi j / n) */
    void *d_part;                 /* maxblk * 4 * n doubles */
};

ATKDSP_API void atkdsp_gpu_spectrum_destroy(atkdsp_gpu_spectrum *p) {
    if (!p) return;
    atkb_free(p->d_tw);
    atkb_free(p->d_part);
    free(p);
}

ATKDSP_API atkdsp_gpu_spectrum *atkdsp_gpu_spectrum_create(size_t n) {
    if (n < 16 || n > ATKB_SPEC_NMAX || (n & (n - 1))) return NULL;
    atkdsp_gpu_spectrum *p = (atkdsp_gpu_spectrum *)calloc(1, sizeof *p);
    if (!p) return NULL;
    p->n = n;
    while (((size_t)1 << p->logn) < n) ++p->logn;
    int dev = 0, rc = atkb_get_device(&dev);
    p->maxblk = 2 * atkb_sm_count(dev);
    double *tw = (double *)malloc(2 * n * sizeof(double));
    if (!tw) rc = ATKB_E_NOMEM;
    if (rc == ATKB_OK) rc = atkb_malloc(&p->d_tw, 2 * n * sizeof(double));
    if (rc == ATKB_OK) rc = atkb_malloc(&p->d_part, (size_t)p->maxblk * 4 * n * sizeof(double));
    if (rc == ATKB_OK) {
        size_t j;
        for (j = 0; j < n; ++j) {
            const double a = 2.0 * SPEC_PI * (double)j / (double)n;
            tw[2 * j] = cos(a);
            tw[2 * j + 1] = -sin(a);
        }
        rc = atkb_h2d(p->d_tw, tw, 2 * n * sizeof(double), NULL);
        if (rc == ATKB_OK) rc = atkb_stream_sync(NULL);
    }
    free(tw);
    if (rc != ATKB_OK) {
        atkdsp_gpu_spectrum_destroy(p);
        return NULL;
    }
    return p;
}

static ptrdiff_t spec_run(atkdsp_gpu_spectrum *p, int mode, const atkdsp_cf32 *d_in, size_t n_samples, size_t hop,
                          const float *d_window, float *o0, float *o1, float *o2, float *o3, void *stream) {
    const size_t n = p->n;
    if (hop == 0 || hop > n) hop = n;
    if (n_samples < n) return 0;
    const long long frames = (long long)((n_samples - n) / hop + 1);
    long long nblk = frames < p->maxblk ? frames : p->maxblk;
    const long long per = (frames + nblk - 1) / nblk;
    nblk = (frames + per - 1) / per;
    const int rc = atkb_spec_launch(mode, d_in, frames, (long long)hop, p->logn, d_window, p->d_tw, (int)nblk,
                                    (int)per, p->d_part, o0, o1, o2, o3, stream);
    return rc == ATKB_OK ? (ptrdiff_t)frames : atkb_map_rc(rc);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_spectrum_reduce(atkdsp_gpu_spectrum *p, const atkdsp_cf32 *d_in, size_t n_samples,
                                                size_t hop, const float *d_window, int detector, float *d_out_line,
                                                void *stream) {
    if (!p || !d_in || !d_out_line) return ATKDSP_E_ARG;
    if (detector < 0 || detector > 2) return ATKDSP_E_ARG;
    return spec_run(p, detector, d_in, n_samples, hop, d_window, d_out_line, NULL, NULL, NULL, stream);
}

ATKDSP_API ptrdiff_t atkdsp_gpu_spectrum_stats(atkdsp_gpu_spectrum *p, const atkdsp_cf32 *d_in, size_t n_samples,
                                               size_t hop, const float *d_window, float *d_max_db, float *d_avg_db,
                                               float *d_min_db, float *d_sk, void *stream) {
    if (!p || !d_in) return ATKDSP_E_ARG;
    if (!d_max_db && !d_avg_db && !d_min_db && !d_sk) return ATKDSP_E_ARG;
    return spec_run(p, 3, d_in, n_samples, hop, d_window, d_max_db, d_avg_db, d_min_db, d_sk, stream);
}
