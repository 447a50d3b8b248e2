// Internal definitions shared by the CUDA library's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <functional>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/cosmicscanner_b200.h"

namespace cs {

// Error carried from the implementation to the C ABI, where it becomes a status
// code plus a thread-local message (no C++ exception crosses the ABI).
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

// The calling thread's message for cs_last_error() (abi.cpp).
void set_last_error(const std::string& msg);

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) fail(CS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CS_CUDA(call) ::cs::check_cuda((call), #call)
#define CS_LAUNCH(what) ::cs::check_cuda(cudaGetLastError(), what)

// Function attributes (e.g. the dynamic shared-memory limit) belong to one device: a setup
// done once per process would leave every other device at its defaults.  PerDeviceOnce runs
// a setup once for each device it is used on (the current device at the call), from any
// thread, and reports the setup's status on every call.
struct PerDeviceOnce {
    static constexpr int kMaxDevices = 64;
    std::mutex mu;
    uint64_t done = 0;  // bit d: device d set up
    cudaError_t err[kMaxDevices] = {};
};
template <class F>
void once_per_device(PerDeviceOnce& o, F&& setup, const char* what) {
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), what);
    if (dev < 0 || dev >= PerDeviceOnce::kMaxDevices)
        fail(CS_ERR_UNSUPPORTED, std::string(what) + ": device ordinal out of range");
    cudaError_t e;
    {
        std::lock_guard<std::mutex> lk(o.mu);
        if (!((o.done >> dev) & 1u)) {
            o.err[dev] = setup();
            o.done |= uint64_t(1) << dev;
        }
        e = o.err[dev];
    }
    check_cuda(e, what);
}

// PLINK 2-bit codes (libCosmicCore/src/plink_reader.cpp:12-21):
// 00 -> 2 copies of A1, 01 -> missing, 10 -> 1, 11 -> 0.
constexpr uint8_t kMissingByte = 0x55;  // four missing codes

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Packed rows are padded to this many bytes (256 samples): every kernel may read
// whole 64-byte segments; padding samples carry the missing code and so contribute
// nothing to any product or count.
constexpr int64_t kRowAlign = 64;

// Device memory from the device's stream-ordered pool (memory.cpp).  The pool keeps freed
// blocks reserved, so handles created per request (operators, engines, their workspaces)
// reuse memory instead of paying cudaMalloc / cudaFree each time.  device_alloc returns
// memory usable from any stream; device_free waits for the device before returning the
// block (the same guarantee cudaFree gives).
void* device_alloc(size_t bytes);
void device_free(void* p) noexcept;
// For a thread whose device work all runs on one stream of its own (a request worker of the
// serving loop): the thread's frees are ordered on that stream (cudaFreeAsync there) instead of
// waiting for the whole device, so a buffer is only reused after the work queued before its
// release has finished.  nullptr restores the device-wide synchronisation.
void set_thread_free_stream(cudaStream_t s);
// Gives the calling thread's cuBLAS / cuSOLVER handles (created on first use per thread and
// device) back to a free list that later threads take them from; threads that end while the
// process goes on (the serving workers) call it last.
void release_thread_handles() noexcept;

// Device allocation that frees itself.
template <typename T>
struct DeviceBuffer {
    T* ptr = nullptr;
    size_t count = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr) device_free(ptr);
        ptr = nullptr;
        count = 0;
    }
    void resize(size_t n) {
        if (n <= count) return;
        release();
        if (n == 0) return;
        ptr = static_cast<T*>(device_alloc(n * sizeof(T)));
        count = n;
    }
    T* get() const { return ptr; }
};

}  // namespace cs

// Opaque handle bodies.
struct cs_genotypes {
    int64_t n_samples = 0;      // rows of the .fam
    int64_t n_snps = 0;         // rows of the .bim
    int64_t bytes_per_snp = 0;  // ceil(n/4), the .bed stride
    int64_t stride = 0;         // device row pitch (bytes_per_snp padded to kRowAlign)
    cs::DeviceBuffer<uint8_t> packed;
    // per-SNP statistics over all samples (plink_reader.cpp:187-239), device + host
    cs::DeviceBuffer<double> d_mean, d_inv_std;
    std::vector<double> mean, inv_std;
    std::vector<int32_t> count;
    std::vector<double> sum;
    std::vector<int32_t> code_counts;  // per SNP over all samples: codes 00, 01, 10, 11
    int device = 0;
    uint64_t uid = 0;  // distinct for every matrix created in the process (cache keys)
};

// A packed matrix of selected rows x selected samples with everything the kernels need.
struct cs_packed_view {
    const uint8_t* rows = nullptr;  // device, rows x stride bytes
    int64_t n_rows = 0;
    int64_t n_samples = 0;
    int64_t stride = 0;
};

namespace cs {
struct Workspace {
    DeviceBuffer<double> partial;
    DeviceBuffer<double> tmp_a, tmp_b, tmp_c;
};
struct MixedOperator;  // tensor-core form (kinship_mixed.cu)
void destroy_mixed(MixedOperator* m);
}  // namespace cs

// Kinship operator over a (keep, variants) selection of a cs_genotypes matrix.
struct cs_kinship {
    const cs_genotypes* g = nullptr;
    int64_t rows = 0;          // analysed samples
    int64_t num_variants = 0;  // selected variants (the 1/M scaling counts all of them)
    cs_packed_view view;       // packed rows the kernels read (own copy or g->packed)
    cs::DeviceBuffer<uint8_t> own_packed;
    int64_t n_active = 0;                  // rows of `view` (selected variants with 1/sd != 0)
    std::vector<double> mean, inv_std;     // per view row
    std::vector<int32_t> view_snp;         // per view row: its SNP (row of the .bed)
    std::vector<int32_t> view_pos;         // per view row: its position among the selected variants
    cs::DeviceBuffer<int32_t> d_view_pos;
    bool keep_identity = false;            // every sample, in .fam order
    std::vector<int32_t> counts;           // per view row: counts of codes 00,01,10,11
    cs::DeviceBuffer<double> d_lut;        // per view row: {(2-mu)s, 0, (1-mu)s, -mu s}
    cs::DeviceBuffer<double> d_lut_sq;     // squared entries (diagonal)
    cs::DeviceBuffer<double> d_mean, d_inv_std;
    cs::DeviceBuffer<int32_t> d_counts;
    double trace = 0.0;
    cs::Workspace ws;
    cs::DeviceBuffer<double> buf_x, buf_u, buf_y;
    cs::MixedOperator* mixed = nullptr;
    bool autotune = true;  // the tensor-core passes may tune their plan on new shapes
    // the samples pass may keep a sample-major copy of the packed view (one more packed matrix
    // in HBM) and read its A operand from tensor memory (six operand sets at the widths where
    // that is the default); otherwise A stays in shared memory and every samples pass runs the
    // five-set form, so a column's result does not depend on how many columns share its apply
    bool sample_major_copy = true;
    ~cs_kinship() { cs::destroy_mixed(mixed); }
};

namespace cs {

// Y_rm (rows x ldy) = K X_rm (rows x ldx), both row-major device buffers, k columns.
// Y may equal X.  precision: CS_PRECISION_*.
void kinship_apply_rowmajor(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                            int64_t ldy, int precision, cudaStream_t s);
void kinship_apply_mixed(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* Y,
                         int64_t ldy, cudaStream_t s);
// The rows-pass output of the last mixed apply: W (R x k, column-major, ld R) with
// W[t, c] = s_t^2 sum_i (G_ti - mu_t)[observed] x_ic; nullptr before any mixed apply.
const double* mixed_rows_output(const cs_kinship* op, int64_t* R, int64_t* k);
// GenotypeMatrix half-passes on tensor cores over the view rows: U (R x k, row-major) = Z^T X,
// and Y (rows x k, row-major) = Z V given W = s o V column-major (R x k).
void mixed_multiply_zt(cs_kinship* op, const double* X, int64_t ldx, int64_t k, double* U,
                       int64_t ldu, cudaStream_t s);
void mixed_multiply_z(cs_kinship* op, const double* Wcol, int64_t k, double* Y, int64_t ldy,
                      cudaStream_t s);

// The reference's Gaussian test matrix (std::normal_distribution over std::mt19937_64) on the
// device, written row-major n x ld (omega.cu).
struct OmegaWorkspace {
    DeviceBuffer<uint64_t> state, raw;
    DeviceBuffer<int32_t> counts;
    DeviceBuffer<int64_t> offsets;
    DeviceBuffer<double> pairs;
    int64_t total_pairs = 0, have = 0;  // accepted polar pairs: needed in all, drawn so far
    int64_t position = 0;               // draws taken from the engine since seeding
    DeviceBuffer<uint64_t> prefix, windows;  // parallel draws: stream prefix, chunk windows
    // the draw in flight: its attempts, count blocks and pair target; the per-block counts
    // come back to pinned host memory, signalled by `counted`
    int64_t pending_attempts = 0, pending_blocks = 0, pending_target = 0;
    int32_t* h_counts = nullptr;
    int64_t h_counts_cap = 0;
    cudaEvent_t counted = nullptr;
    OmegaWorkspace() = default;
    OmegaWorkspace(const OmegaWorkspace&) = delete;
    OmegaWorkspace& operator=(const OmegaWorkspace&) = delete;
    ~OmegaWorkspace();
};
void generate_omega_device(uint64_t seed, int64_t n, int64_t cols, double* d_out, int64_t ld,
                           OmegaWorkspace& ws, cudaStream_t s);
// The same stream in pieces: seed for total_count normals, draw until pairs_needed pairs are
// accepted, transform columns [c0, c1) (normals c0 n .. c1 n - 1).
void omega_begin(uint64_t seed, int64_t total_count, OmegaWorkspace& ws, cudaStream_t s);
void omega_ensure(OmegaWorkspace& ws, int64_t pairs_needed, cudaStream_t s);
// omega_ensure in two halves: omega_draw launches the engine and the acceptance count without
// waiting; omega_accept waits for the count, writes the accepted pairs and tops up if short.
void omega_draw(OmegaWorkspace& ws, int64_t pairs_needed, cudaStream_t s);
void omega_accept(OmegaWorkspace& ws, cudaStream_t s);
void omega_emit(OmegaWorkspace& ws, int64_t n, int64_t c0, int64_t c1, double* d_out, int64_t ld,
                cudaStream_t s);

// Tensor-core projection for the scan: T[t][c] = sum_i (g_ti - m_t)[observed] B[i][c] over
// every row of a packed view, m_t = row_mean[t] (kinship_mixed.cu).
struct MixedScan;
MixedScan* mixed_scan_create(const cs_packed_view& v, const double* row_mean, const int32_t* counts);
void mixed_scan_destroy(MixedScan* m);
void mixed_scan_project(MixedScan* m, const double* B, int64_t ldb, int64_t k, double* T,
                        int64_t ldt, cudaStream_t s);

// Per-row genotype code counts over a view's samples: c[4*t + code].
void row_code_counts(const cs_packed_view& v, int32_t* d_counts, cudaStream_t s);

// Decode-GEMM kernels (FP64).  lut[4*t + code] gives the value of code in row t.
//   pass_a:  out[t, c] = sum_i lut_t[code(t, i)] * V[i, c]      (rows t, V row-major n x ldv)
//   pass_b:  out[i, c] = sum_t lut_t[code(t, i)] * W[t, c]      (W row-major rows x ldw)
// Results are row-major with leading dimension ldo; `scale` multiplies the result.
void decode_gemm_rows_fp64(const cs_packed_view& v, const double* d_lut, const double* V,
                           int64_t ldv, int64_t k, double* out, int64_t ldo, Workspace& ws,
                           cudaStream_t s);
void decode_gemm_samples_fp64(const cs_packed_view& v, const double* d_lut, const double* W,
                              int64_t ldw, int64_t k, double* out, int64_t ldo, double scale,
                              Workspace& ws, cudaStream_t s);

// Repack selected rows/samples of a packed matrix into a new padded matrix.
void repack(const uint8_t* src, int64_t src_stride, const int32_t* d_rows, int64_t n_rows,
            const int32_t* d_keep, int64_t n_keep, uint8_t* dst, int64_t dst_stride,
            cudaStream_t s);

// Column-major (ld) <-> row-major (n x kp, zero padded) conversion on the device.
void colmajor_to_rowmajor(const double* src, int64_t ld, int64_t n, int64_t k, double* dst,
                          int64_t kp, cudaStream_t s);
void rowmajor_to_colmajor(const double* src, int64_t kp, int64_t n, int64_t k, double* dst,
                          int64_t ld, cudaStream_t s);

int num_sms();

// The low-rank engine's view of the kinship operator: its row count, trace and an apply
// Y = K X on row-major device blocks (lowrank.cu).
struct LowRankTarget {
    int64_t rows = 0;
    double trace = 0.0;
    // the final sketch apply also carries [X | y - mean(y)] (the scan then takes Z^T X and
    // Z^T y from its rows pass instead of a narrow genotype pass)
    bool fuse_scan_columns = false;
    std::function<void(const double* X, int64_t ldx, int64_t k, double* Y, int64_t ldy,
                       cudaStream_t s)>
        apply;
};
cs_lmm* lmm_create();
void lmm_destroy(cs_lmm* l);
// The y columns (n x t) of the traits that the next scans of this sketch fit in turn: the first
// scan projects all of them, the others reuse that projection (lowrank.cu).
void lmm_set_scan_traits(cs_lmm* l, const double* Y, int64_t t);
void lmm_prepare_lowrank_target(cs_lmm* l, const LowRankTarget& target, const double* y,
                                const double* X, int64_t p, int rank, int oversample,
                                int64_t seed, double trace_threshold, int min_rank,
                                cs_lowrank_diagnostics* diag, cudaStream_t s);
void lmm_fit_reml(cs_lmm* l, const double* y, const double* X, int64_t p,
                  cs_lowrank_diagnostics* diag, cudaStream_t s);
// The last sketch's basis: selected rank, U (n x rank, row-major, device), its eigenvalues
// (largest first) and the tail-mean residual eigenvalue.
int64_t lmm_rank(const cs_lmm* l);
const double* lmm_basis_device(const cs_lmm* l);
std::vector<double> lmm_eigenvalues(const cs_lmm* l);
double lmm_residual_eigenvalue(const cs_lmm* l);
// Scan of SNPs [snp_begin, snp_end) of g; per-SNP outputs have snp_end - snp_begin entries.
void lmm_scan_window(cs_lmm* l, const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                     int64_t snp_begin, int64_t snp_end, double min_maf, int precision,
                     double* beta, double* se, double* pvalue, double* log10p, double* freq,
                     int32_t* tested, cudaStream_t s);

// The tensor-core autotuner's table as JSON (kinship_mixed.cu).
std::string autotune_json();

namespace prof {
// Counts one kernel launch; with profiling enabled, times it with events on stream s.
// flops / bytes are the launch's algorithmic work, reported beside the time.
class Scope {
   public:
    Scope(const char* name, cudaStream_t s, double flops = 0.0, double bytes = 0.0);
    ~Scope();
    Scope(const Scope&) = delete;
    Scope& operator=(const Scope&) = delete;

   private:
    const char* name_;
    cudaStream_t s_;
    double flops_, bytes_;
    cudaEvent_t a_ = nullptr;
};
// Wall-clock time of a host-side stage, reported with the kernels when profiling is on.
class HostScope {
   public:
    explicit HostScope(const char* name);
    ~HostScope();
    HostScope(const HostScope&) = delete;
    HostScope& operator=(const HostScope&) = delete;

   private:
    const char* name_;
    double t0_ = -1.0;
};
bool enabled();
void set_enabled(bool on);
int64_t launches();
std::string summary_json();
}  // namespace prof

}  // namespace cs
