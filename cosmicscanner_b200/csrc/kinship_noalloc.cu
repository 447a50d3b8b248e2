// Kinship apply for callers that must not allocate device memory.
//
// Some hosts of this library cannot let it call cudaMalloc: a process that has reserved
// nearly all of HBM up front for its own pool (for instance a serving process that keeps
// a large genotype matrix resident next to other models) would see the allocation fail
// or fragment its pool, and a latency-bound request loop cannot afford the implicit
// device-wide synchronisation a cudaMalloc/cudaFree pair can cause.  For them,
// cs_kinship_apply_noalloc computes the same FP64 Y = K X as cs_kinship_apply but takes
// its scratch from a fixed array in the library's own device memory.
//
// The scratch is a file-scope __device__ array of kNoAllocScratchDoubles doubles
// (16 MiB).  Every GPU that loads the library holds it until the process exits.  In host
// code the array's name is only a host-side stand-in, so its device address is looked up
// with cudaGetSymbolAddress once per device (with that device current) on the first call
// made on that device; that first call should therefore come before any stream capture.
// The cached address belongs to the device's current context: the library must not be used
// across a cudaDeviceReset (or any other teardown of that context).
// The operator's device must be the current device: its packed rows and lookup table live
// there, and the scratch address is that device's; a call made with another device current
// is refused with CS_ERR_INVALID_ARGUMENT rather than run on the wrong GPU.
// All calls share the one array and it keeps the previous call's contents: every scratch
// element a call reads is first written by the same call, so nothing needs clearing, but
// two calls whose work overlaps on the GPU (different streams, or different host threads
// on one device) race on the array and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "cs_internal.h"

namespace cs {

void decode_gemm_rows_fp64_unsplit(const cs_packed_view& v, const double* d_lut, const double* V,
                                   int64_t ldv, int64_t k, double* out, int64_t ldo,
                                   cudaStream_t s);
void decode_gemm_samples_fp64_unsplit(const cs_packed_view& v, const double* d_lut,
                                      const double* W, int64_t ldw, int64_t k, double* out,
                                      int64_t ldo, double scale, cudaStream_t s);

namespace {

constexpr int64_t kNoAllocScratchDoubles = int64_t(2) << 20;  // 16 MiB
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch on the current device (looked up once per device).
double* scratch_on_current_device() {
    static std::mutex mu;
    static double* addr[kMaxDevices] = {};
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(CS_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            fail(CS_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                  cudaGetErrorString(e));
        addr[dev] = static_cast<double*>(p);
    }
    return addr[dev];
}

}  // namespace

int64_t noalloc_scratch_doubles() { return kNoAllocScratchDoubles; }

// Y = K X (column-major device arrays) using only the fixed scratch array:
// X is copied row-major (n x k), U = Z^T X (n_active x k), Y_rm = Z U / M (n x k), then Y.
void kinship_apply_noalloc(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                           int64_t ldy, cudaStream_t s) {
    if (k < 0) fail(CS_ERR_INVALID_ARGUMENT, "negative column count");
    if (ldx < op->rows || ldy < op->rows)
        fail(CS_ERR_INVALID_ARGUMENT, "PlinkKinshipOperator::apply: dimension mismatch");
    int dev = 0;
    CS_CUDA(cudaGetDevice(&dev));
    if (dev != op->g->device)
        fail(CS_ERR_INVALID_ARGUMENT,
             "cs_kinship_apply_noalloc: the operator lives on device " +
                 std::to_string(op->g->device) + " but device " + std::to_string(dev) +
                 " is current");
    if (k == 0) return;
    const int64_t n = op->rows, R = op->n_active;
    const int64_t need = (2 * n + R) * k;
    if (need > kNoAllocScratchDoubles)
        fail(CS_ERR_INVALID_ARGUMENT,
             "cs_kinship_apply_noalloc: (2*rows + active variants) * k = " + std::to_string(need) +
                 " doubles exceeds the fixed scratch of " + std::to_string(kNoAllocScratchDoubles) +
                 " doubles (16 MiB); use cs_kinship_apply or fewer columns per call");
    if (R == 0) {
        CS_CUDA(cudaMemset2DAsync(Y, ldy * 8, 0, n * 8, k, s));
        return;
    }
    double* scratch = scratch_on_current_device();
    double* xrm = scratch;
    double* u = xrm + n * k;
    double* yrm = u + R * k;
    colmajor_to_rowmajor(X, ldx, n, k, xrm, k, s);
    decode_gemm_rows_fp64_unsplit(op->view, op->d_lut.get(), xrm, k, k, u, k, s);
    decode_gemm_samples_fp64_unsplit(op->view, op->d_lut.get(), u, k, k, yrm, k,
                                     1.0 / (double)op->num_variants, s);
    rowmajor_to_colmajor(yrm, k, n, k, Y, ldy, s);
}

}  // namespace cs
