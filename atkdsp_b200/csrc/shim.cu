/* The thin C-ABI shim between the C99 host layer and the CUDA runtime.
 * Every function returns an ATKB_* status; no CUDA type crosses into C. */
#include <cuda_runtime.h>
#include <stdint.h>
#include <atomic>
#include <nvtx3/nvToolsExt.h>
#include "internal.h"

static int st(cudaError_t e) {
    if (e == cudaSuccess) return ATKB_OK;
    if (e == cudaErrorMemoryAllocation) return ATKB_E_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice)
        return ATKB_E_NODEV;
    return ATKB_E_KERNEL;
}

extern "C" int atkb_get_device(int *dev) { return st(cudaGetDevice(dev)); }
extern "C" int atkb_set_device(int dev) { return st(cudaSetDevice(dev)); }

extern "C" int atkb_sm_count(int dev) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) n = 1;
    return n;
}

extern "C" int atkb_stream_create(void **stream) {
    cudaStream_t s = nullptr;
    const int rc = st(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    *stream = (void *)s;
    return rc;
}
extern "C" void atkb_stream_destroy(void *stream) {
    if (stream) cudaStreamDestroy((cudaStream_t)stream);
}
extern "C" int atkb_stream_sync(void *stream) { return st(cudaStreamSynchronize((cudaStream_t)stream)); }

/* Allocation fault injection (host side, no device fault): when armed with
 * n > 0, the n-th device, pool or pinned allocation from then on fails with
 * ATKB_E_NOMEM as a real out-of-memory would, and the hook disarms itself. */
static std::atomic<long long> g_fail_countdown{0};
static bool inject_alloc_failure() {
    long long c = g_fail_countdown.load(std::memory_order_relaxed);
    while (c > 0) {
        if (g_fail_countdown.compare_exchange_weak(c, c - 1, std::memory_order_relaxed))
            return c == 1;
    }
    return false;
}
extern "C" void atkb_fail_alloc_after(long long n) { g_fail_countdown.store(n > 0 ? n : 0); }

extern "C" int atkb_malloc(void **p, size_t bytes) {
    *p = nullptr;
    if (inject_alloc_failure()) return ATKB_E_NOMEM;
    return st(cudaMalloc(p, bytes ? bytes : 256));
}
extern "C" void atkb_free(void *p) {
    if (p) cudaFree(p);
}
/* a stream-ordered pool on `dev` that keeps freed memory for reuse (release
 * threshold at its maximum): allocations from it in steady state map nothing
 * and wait for nothing */
extern "C" int atkb_pool_create(int dev, void **pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t mp = nullptr;
    *pool = nullptr;
    int rc = st(cudaMemPoolCreate(&mp, &props));
    if (rc != ATKB_OK) return rc;
    uint64_t thr = ~(uint64_t)0;
    rc = st(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &thr));
    if (rc != ATKB_OK) { cudaMemPoolDestroy(mp); return rc; }
    *pool = (void *)mp;
    return ATKB_OK;
}
extern "C" void atkb_pool_destroy(void *pool) {
    if (pool) cudaMemPoolDestroy((cudaMemPool_t)pool);
}
/* bytes the pool holds but no allocation uses */
extern "C" size_t atkb_pool_idle_bytes(void *pool) {
    uint64_t res = 0, used = 0;
    if (!pool) return 0;
    if (cudaMemPoolGetAttribute((cudaMemPool_t)pool, cudaMemPoolAttrReservedMemCurrent, &res) != cudaSuccess ||
        cudaMemPoolGetAttribute((cudaMemPool_t)pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess)
        return 0;
    return res > used ? (size_t)(res - used) : 0;
}
extern "C" int atkb_malloc_pool(void **p, size_t bytes, void *pool, void *stream) {
    *p = nullptr;
    if (inject_alloc_failure()) return ATKB_E_NOMEM;
    return st(cudaMallocFromPoolAsync(p, bytes ? bytes : 256, (cudaMemPool_t)pool, (cudaStream_t)stream));
}
extern "C" void atkb_free_async(void *p, void *stream) {
    if (p) cudaFreeAsync(p, (cudaStream_t)stream);
}
extern "C" int atkb_host_alloc(void **p, size_t bytes) {
    *p = nullptr;
    if (inject_alloc_failure()) return ATKB_E_NOMEM;
    return st(cudaMallocHost(p, bytes ? bytes : 256));
}
extern "C" void atkb_host_free(void *p) {
    if (p) cudaFreeHost(p);
}
extern "C" int atkb_host_dev_ptr(void *h, void **d) {
    *d = nullptr;
    const cudaError_t e = cudaHostGetDevicePointer(d, h, 0);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();        /* not sticky: leave no error for the next launch check */
        *d = nullptr;
    }
    return st(e);
}
extern "C" int atkb_h2d(void *dst, const void *src, size_t bytes, void *stream) {
    if (!bytes) return ATKB_OK;
    return st(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream));
}
extern "C" int atkb_d2h(void *dst, const void *src, size_t bytes, void *stream) {
    if (!bytes) return ATKB_OK;
    return st(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream));
}
extern "C" int atkb_d2d(void *dst, const void *src, size_t bytes, void *stream) {
    if (!bytes) return ATKB_OK;
    return st(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
}
extern "C" int atkb_d2h_2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width,
                           size_t height, void *stream) {
    if (!width || !height) return ATKB_OK;
    return st(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, height, cudaMemcpyDeviceToHost,
                                (cudaStream_t)stream));
}
extern "C" int atkb_memset(void *p, int v, size_t bytes, void *stream) {
    if (!bytes) return ATKB_OK;
    return st(cudaMemsetAsync(p, v, bytes, (cudaStream_t)stream));
}
extern "C" int atkb_mem_info(size_t *free_bytes, size_t *total_bytes) {
    return st(cudaMemGetInfo(free_bytes, total_bytes));
}

extern "C" int atkb_event_create(void **ev) {
    cudaEvent_t e = nullptr;
    const int rc = st(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    *ev = (void *)e;
    return rc;
}
extern "C" void atkb_event_destroy(void *ev) {
    if (ev) cudaEventDestroy((cudaEvent_t)ev);
}
extern "C" int atkb_event_record(void *ev, void *stream) {
    return st(cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream));
}
extern "C" int atkb_event_sync(void *ev) { return st(cudaEventSynchronize((cudaEvent_t)ev)); }
extern "C" int atkb_stream_wait(void *stream, void *ev) {
    return st(cudaStreamWaitEvent((cudaStream_t)stream, (cudaEvent_t)ev, 0));
}

extern "C" int atkb_graph_begin(void *stream) {
    return st(cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal));
}
extern "C" int atkb_graph_end(void *stream, void **exec) {
    cudaGraph_t g = nullptr;
    *exec = nullptr;
    int rc = st(cudaStreamEndCapture((cudaStream_t)stream, &g));
    if (rc != ATKB_OK) return rc;
    cudaGraphExec_t x = nullptr;
    rc = st(cudaGraphInstantiate(&x, g, 0));
    cudaGraphDestroy(g);
    *exec = (void *)x;
    return rc;
}
/* NVTX ranges (header-only NVTX 3: free unless a profiler injects itself) on
 * the host timeline around every graph replay and tile-kernel launch, so a
 * trace shows when each batch or server round was enqueued */
extern "C" void atkb_range_push(const char *name) { nvtxRangePushA(name); }
extern "C" void atkb_range_pop(void) { nvtxRangePop(); }

extern "C" int atkb_graph_launch(void *exec, void *stream) {
    nvtxRangePushA("atkdsp graph launch");
    const int rc = st(cudaGraphLaunch((cudaGraphExec_t)exec, (cudaStream_t)stream));
    nvtxRangePop();
    return rc;
}
extern "C" void atkb_graph_destroy(void *exec) {
    if (exec) cudaGraphExecDestroy((cudaGraphExec_t)exec);
}

extern "C" int atkb_event_create_timed(void **ev) {
    cudaEvent_t e = nullptr;
    const int rc = st(cudaEventCreate(&e));
    *ev = (void *)e;
    return rc;
}
extern "C" int atkb_event_record_node(void *ev, void *stream) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing((cudaStream_t)stream, &cs) != cudaSuccess) return ATKB_E_KERNEL;
    if (cs == cudaStreamCaptureStatusActive)
        return st(cudaEventRecordWithFlags((cudaEvent_t)ev, (cudaStream_t)stream, cudaEventRecordExternal));
    return st(cudaEventRecord((cudaEvent_t)ev, (cudaStream_t)stream));
}
extern "C" int atkb_event_elapsed_ms(float *ms, void *start, void *stop) {
    const int rc = st(cudaEventSynchronize((cudaEvent_t)stop));
    if (rc != ATKB_OK) return rc;
    return st(cudaEventElapsedTime(ms, (cudaEvent_t)start, (cudaEvent_t)stop));
}

/* wait for an event by polling it: no sleep-and-wake in the driver's
 * synchronisation, for the short waits of small synchronous calls */
extern "C" int atkb_event_spin(void *ev) {
    for (;;) {
        const cudaError_t e = cudaEventQuery((cudaEvent_t)ev);
        if (e == cudaSuccess) return ATKB_OK;
        if (e != cudaErrorNotReady) return st(e);
    }
}
extern "C" int atkb_event_query(void *ev) {
    const cudaError_t e = cudaEventQuery((cudaEvent_t)ev);
    if (e == cudaSuccess) return ATKB_OK;
    if (e == cudaErrorNotReady) return 1;
    return st(e);
}
