// Device memory pool and shared cuBLAS handles.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>

#include "cs_internal.h"

namespace cs {

namespace {
constexpr int kMaxDevices = 64;
std::once_flag g_pool_once[kMaxDevices];

void prepare_pool(int dev) {
    std::call_once(g_pool_once[dev], [dev] {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return;
        // keep freed blocks reserved for this process (released when the context ends)
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    });
}

// CS_B200_POISON_ALLOC=1 fills every new block with 0xFF bytes (NaN as FP64), so that a read of
// memory no kernel has written shows up in the results instead of depending on what the pool
// held before.
bool poison_allocations() {
    static const bool on = [] {
        const char* v = std::getenv("CS_B200_POISON_ALLOC");
        return v && v[0] == '1';
    }();
    return on;
}
}  // namespace

void* device_alloc(size_t bytes) {
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < kMaxDevices) prepare_pool(dev);
    void* p = nullptr;
    cudaError_t e = cudaMallocAsync(&p, bytes, 0);
    if (e == cudaErrorMemoryAllocation) {
        // The pool keeps freed blocks reserved; when the device has no room left for a new
        // block, hand the reserved free blocks back (after the device has finished with them)
        // and try once more.
        cudaGetLastError();
        cudaMemPool_t pool;
        if (cudaDeviceSynchronize() == cudaSuccess &&
            cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess &&
            cudaMemPoolTrimTo(pool, 0) == cudaSuccess)
            e = cudaMallocAsync(&p, bytes, 0);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        fail(CS_ERR_CUDA, std::string("device allocation of ") + std::to_string(bytes) +
                              " bytes failed: " + cudaGetErrorString(e));
    }
    if (poison_allocations()) CS_CUDA(cudaMemsetAsync(p, 0xFF, bytes, 0));
    // usable from every stream once the allocation is ordered on the legacy stream
    CS_CUDA(cudaStreamSynchronize(0));
    return p;
}

cublasHandle_t shared_blas() {
    thread_local cublasHandle_t handles[kMaxDevices] = {};
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(CS_ERR_CUDA, "device ordinal out of range");
    if (!handles[dev] && cublasCreate(&handles[dev]) != CUBLAS_STATUS_SUCCESS)
        fail(CS_ERR_CUDA, "cublasCreate failed");
    return handles[dev];
}

cusolverDnHandle_t shared_solver() {
    thread_local cusolverDnHandle_t handles[kMaxDevices] = {};
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(CS_ERR_CUDA, "device ordinal out of range");
    if (!handles[dev] && cusolverDnCreate(&handles[dev]) != CUSOLVER_STATUS_SUCCESS)
        fail(CS_ERR_CUDA, "cusolverDnCreate failed");
    return handles[dev];
}

namespace {
thread_local cudaStream_t g_free_stream = nullptr;
}

void set_thread_free_stream(cudaStream_t s) { g_free_stream = s; }

void device_free(void* p) noexcept {
    if (!p) return;
    if (g_free_stream) {
        // ordered after the work this thread queued on its stream (the pool reuses the block
        // only once the free has executed)
        cudaFreeAsync(p, g_free_stream);
        return;
    }
    cudaDeviceSynchronize();
    cudaFreeAsync(p, 0);
}

}  // namespace cs
