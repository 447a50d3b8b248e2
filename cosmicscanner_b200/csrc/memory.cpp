// Device memory pool and the per-thread cuBLAS / cuSOLVER handles.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

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

thread_local cublasHandle_t t_blas[kMaxDevices] = {};
thread_local cusolverDnHandle_t t_solver[kMaxDevices] = {};
// Handles given back by threads that ended (release_thread_handles), reused by new threads:
// creating and destroying them per request thread costs device-wide synchronisations.
std::mutex g_handle_mu;
std::vector<cublasHandle_t> g_free_blas[kMaxDevices];
std::vector<cusolverDnHandle_t> g_free_solver[kMaxDevices];

// Gives the pool's reserved free blocks back to the device (after the device has finished
// with them), when an allocation found no room: the pool keeps freed blocks reserved, which
// neither a block of another size nor the libraries' own allocations can use.
void trim_pool(int dev) {
    cudaMemPool_t pool;
    if (cudaDeviceSynchronize() == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess)
        cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
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
        // block, hand the reserved free blocks back and try once more.
        cudaGetLastError();
        trim_pool(dev);
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
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(CS_ERR_CUDA, "device ordinal out of range");
    if (!t_blas[dev]) {
        std::lock_guard<std::mutex> lk(g_handle_mu);
        if (!g_free_blas[dev].empty()) {
            t_blas[dev] = g_free_blas[dev].back();
            g_free_blas[dev].pop_back();
        }
    }
    if (!t_blas[dev] && cublasCreate(&t_blas[dev]) != CUBLAS_STATUS_SUCCESS) {
        t_blas[dev] = nullptr;
        trim_pool(dev);
        if (cublasCreate(&t_blas[dev]) != CUBLAS_STATUS_SUCCESS) {
            t_blas[dev] = nullptr;
            fail(CS_ERR_CUDA, "cublasCreate failed");
        }
    }
    return t_blas[dev];
}

cusolverDnHandle_t shared_solver() {
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(CS_ERR_CUDA, "device ordinal out of range");
    if (!t_solver[dev]) {
        std::lock_guard<std::mutex> lk(g_handle_mu);
        if (!g_free_solver[dev].empty()) {
            t_solver[dev] = g_free_solver[dev].back();
            g_free_solver[dev].pop_back();
        }
    }
    if (!t_solver[dev] && cusolverDnCreate(&t_solver[dev]) != CUSOLVER_STATUS_SUCCESS) {
        t_solver[dev] = nullptr;
        trim_pool(dev);
        if (cusolverDnCreate(&t_solver[dev]) != CUSOLVER_STATUS_SUCCESS) {
            t_solver[dev] = nullptr;
            fail(CS_ERR_CUDA, "cusolverDnCreate failed");
        }
    }
    return t_solver[dev];
}

void release_thread_handles() noexcept {
    // back to the free lists, bound to the legacy stream (the thread's own stream is about to
    // be destroyed; every user sets its stream before use)
    std::lock_guard<std::mutex> lk(g_handle_mu);
    for (int d = 0; d < kMaxDevices; ++d) {
        if (t_blas[d]) {
            cublasSetStream(t_blas[d], 0);
            g_free_blas[d].push_back(t_blas[d]);
            t_blas[d] = nullptr;
        }
        if (t_solver[d]) {
            cusolverDnSetStream(t_solver[d], 0);
            g_free_solver[d].push_back(t_solver[d]);
            t_solver[d] = nullptr;
        }
    }
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
