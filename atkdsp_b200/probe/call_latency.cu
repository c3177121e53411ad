/* Per-call latency of the drop-in host call (atkdsp_pfb_process) on the
 * single-stream workload: nchan 64, critically sampled, 16 taps per branch,
 * beta 8, 2^20 cf32 samples fed in blocks of 1, 999, 4096, 7 (cycling), for
 * the default tile shape and each autotuner choice. Also a floor for the
 * same box: host->device and device->host copies of the same sizes around an
 * empty kernel, completion polled as the library polls it.
 *
 *   make -C atkdsp_b200 probe && atkdsp_b200/lib/atkdsp_call_latency
 *
 * Prints one line per measurement (medians over the calls). */
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "atkdsp.h"
#include "atkdsp_gpu.h"

__global__ void empty_kernel(float *p) {
    if (threadIdx.x == 0xffff) p[0] = 1.0f;
}

static double now_us() {
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

static double median(std::vector<double> v) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    return v[v.size() / 2];
}

static int floor_probe() {
    cudaStream_t st;
    cudaEvent_t ev;
    char *h_in, *h_out, *d_in, *d_out;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaHostAlloc(&h_in, 1 << 20, 0) != cudaSuccess || cudaHostAlloc(&h_out, 1 << 20, 0) != cudaSuccess ||
        cudaMalloc(&d_in, 1 << 20) != cudaSuccess || cudaMalloc(&d_out, 1 << 20) != cudaSuccess)
        return 1;
    const char *names[3] = {"copy 40 KB up + empty kernel + copy 32 KB down", "empty kernel alone",
                            "the two copies alone"};
    for (int variant = 0; variant < 3; ++variant) {
        std::vector<double> t;
        for (int it = 0; it < 2000; ++it) {
            const double t0 = now_us();
            if (variant != 1) cudaMemcpyAsync(d_in, h_in, 40000, cudaMemcpyHostToDevice, st);
            if (variant != 2) empty_kernel<<<2, 128, 0, st>>>((float *)d_out);
            if (variant != 1) cudaMemcpyAsync(h_out, d_out, 32768, cudaMemcpyDeviceToHost, st);
            cudaEventRecord(ev, st);
            while (cudaEventQuery(ev) == cudaErrorNotReady) {
            }
            if (it >= 100) t.push_back(now_us() - t0);
        }
        printf("floor: %s: %.1f us\n", names[variant], median(t));
    }
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFreeHost(h_in);
    cudaFreeHost(h_out);
    cudaEventDestroy(ev);
    cudaStreamDestroy(st);
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

int main() {
    if (floor_probe() != 0) {
        fprintf(stderr, "no usable GPU\n");
        return 1;
    }
    const size_t N = 1 << 20;
    std::vector<atkdsp_cf32> x(N), out(64 * 128);
    srand(1);
    for (size_t i = 0; i < N; ++i) {
        x[i].re = rand() / (float)RAND_MAX - 0.5f;
        x[i].im = rand() / (float)RAND_MAX - 0.5f;
    }
    const double atten = 8.0 / 0.1102 + 8.7;            /* Kaiser beta 8 */
    const size_t blocks[4] = {1, 999, 4096, 7};
    const int before = atkdsp_gpu_tune_get(64, 1, 16);
    for (int choice = -1; choice <= 5; ++choice) {
        if (choice >= 0 && atkdsp_gpu_tune_set(64, 1, 16, choice) != 0) continue;   /* no such shape */
        atkdsp_pfb *p = atkdsp_pfb_create(2.4e6, 64, 1, 16, atten, 1);
        if (!p) {
            fprintf(stderr, "atkdsp_pfb_create failed\n");
            return 1;
        }
        std::vector<double> per[4];
        size_t pos = 0;
        int i = 0;
        const double t_start = now_us();
        while (pos + 4096 < N) {
            const size_t b = blocks[i % 4];
            const double t0 = now_us();
            const ptrdiff_t r = atkdsp_pfb_process(p, x.data() + pos, b, out.data(), out.size());
            per[i % 4].push_back(now_us() - t0);
            if (r < 0) {
                fprintf(stderr, "atkdsp_pfb_process: %td\n", r);
                return 1;
            }
            pos += b;
            ++i;
        }
        const double t_all = now_us() - t_start;
        printf("tile shape %2d: %.1f MS/s; us per call: 1: %.1f  999: %.1f  4096: %.1f  7: %.1f\n", choice,
               pos / t_all, median(per[0]), median(per[1]), median(per[2]), median(per[3]));
        atkdsp_pfb_destroy(p);
    }
    atkdsp_gpu_tune_set(64, 1, 16, before);
    return 0;
}
