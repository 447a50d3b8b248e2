// Serving loop: a resident genotype matrix answering association requests with continuous
// batching of kinship applies.
//
// No reference counterpart: the reference runs one `gwas` job per process.  A request is the
// reference's matrix-free LMM job (`gwas --model lmm --fastlmm --fastlmm-matrix-free`,
// src/gwas_scanner.cpp:121-129, 314-447) on a cohort subset with 1..t traits and a scan
// window: low-rank sketch of the subset's kinship (lmm_engine.cpp:897-1003), REML per trait
// (:1010-1073) and scanLowRank over the window (:1269-1361).
//
// Batching.  The subset kinship K_S = (Z Z^T / M)[S, S] is a principal block of the full
// operator (the standardisation uses every .fam sample, kinship_operator.cpp:67), so an
// apply for request r is: embed its block X_r (|S_r| x k_r) into the full sample space
// (zeros elsewhere), apply K, read back rows S_r.  One GPU thread owns the full operator;
// request workers hand it their applies, and whenever the GPU is free it stacks every
// pending block, of any subset size, into one multi-right-hand-side apply (up to a column
// budget) and returns each block its rows.  Requests arriving while others run are admitted
// as memory and worker slots free up, so their applies join the next stacked apply.  A
// request's columns never mix with another's: each output column depends only on its own
// input column, so a result is the same alone and in the mix up to the order of FP64 slice
// sums.
//
// Small cohorts.  Embedding costs the full operator's work (all N samples) for every column;
// a request whose cohort is below `subset_fraction` of N instead gets its own operator over a
// repacked copy of its samples (the same K_S: statistics and 1/M from the full matrix) and
// runs its applies on its own stream, so its tensor work scales with its own sample count.
// Whether a request is embedded or repacked depends only on its size, so it takes the same
// path alone and in the mix.
//
// Admission.  Requests are admitted FIFO while a worker slot is free and their estimated
// working set (sketch blocks, scan window and, for repacked requests, the packed copy, its
// tensor-core operands and the sketch rows kept for the scan) fits the memory budget: by
// default the device's free memory at server creation less a 4 GB reserve and less the shared
// apply's own buffers at the full column budget (stacked blocks in and out, the rows-pass
// output, operand pieces and slice partials over all N samples and M SNPs).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cs_internal.h"

namespace cs {
cs_kinship* kinship_create(const cs_genotypes* g, const int32_t* keep, int64_t n_keep,
                           const int32_t* variants, int64_t n_var);
void kinship_diagonal(cs_kinship* op, double* diag_host);
}  // namespace cs

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct ApplyJob {
    const int32_t* d_rows = nullptr;
    int64_t n_sub = 0, k = 0;
    const double* X = nullptr;
    int64_t ldx = 0;
    double* Y = nullptr;
    int64_t ldy = 0;
    bool done = false;
    std::string error;
};

struct Request {
    int64_t id = 0;
    bool own_view = false;  // repacked subset operator instead of the shared full-space applies
    std::vector<int32_t> samples;
    std::vector<double> Y, X;  // column-major n x t, n x p
    int32_t t = 0, p = 0;
    int64_t begin = 0, end = 0;
    uint64_t seed = 42;
    int state = 0;  // 0 queued, 1 running, 2 done, -1 failed
    std::string error;
    double t_submit = 0, t_start = 0, t_done = 0;
    int64_t est_bytes = 0;
    int32_t effective_rank = 0;
    std::vector<double> sigma2;  // (sg2, se2) per trait
    std::vector<double> beta, se, pval, l10, freq;  // t x window
    std::vector<int32_t> tested;
    std::thread worker;
};

// xs[rows[i], off + c] = X[i, c]
__global__ void k_embed(const double* __restrict__ X, int64_t ldx, int64_t n, int64_t k,
                        const int32_t* __restrict__ rows, double* __restrict__ xs, int64_t ld,
                        int64_t off) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / k, c = e - i * k;
        xs[(int64_t)rows[i] * ld + off + c] = X[i * ldx + c];
    }
}

// Y[i, c] = ys[rows[i], off + c]
__global__ void k_extract(const double* __restrict__ ys, int64_t ld, int64_t off,
                          const int32_t* __restrict__ rows, int64_t n, int64_t k,
                          double* __restrict__ Y, int64_t ldy) {
    const int64_t total = n * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e / k, c = e - i * k;
        Y[i * ldy + c] = ys[(int64_t)rows[i] * ld + off + c];
    }
}

unsigned grid_for(int64_t total) {
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>((total + 255) / 256, 32LL * cs::num_sms()));
}

}  // namespace

struct cs_server {
    const cs_genotypes* g = nullptr;
    cs_kinship* op = nullptr;
    std::vector<int32_t> variants;  // the GRM selection (empty: every SNP)
    int64_t budget_bytes = 0;
    std::vector<double> diag_full;
    cs_server_options opt{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<ApplyJob*> jobs;
    std::deque<int64_t> queue;
    std::map<int64_t, std::unique_ptr<Request>> reqs;
    int64_t next_id = 1;
    int active = 0;
    int64_t mem_in_use = 0;
    bool stop = false;
    std::thread gpu_thread, dispatch_thread;
    // statistics
    int64_t applies = 0, apply_cols = 0, submitted = 0, completed = 0, failed = 0;
    int64_t max_jobs_per_apply = 0, max_active = 0, own_view_requests = 0;
    std::vector<double> latencies;
    double first_submit = -1.0, last_done = 0.0;
    cs::DeviceBuffer<double> xs, ys;

    ~cs_server() {
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (dispatch_thread.joinable()) dispatch_thread.join();
        for (auto& kv : reqs)
            if (kv.second->worker.joinable()) kv.second->worker.join();
        {
            std::lock_guard<std::mutex> lk(mu);
            stop = true;
        }
        cv.notify_all();
        if (gpu_thread.joinable()) gpu_thread.join();
        delete op;
    }

    void gpu_loop();
    void dispatch_loop();
    void run_request(Request* r);
    void apply(const int32_t* d_rows, int64_t n_sub, const double* X, int64_t ldx, int64_t k,
               double* Y, int64_t ldy, cudaStream_t s);
};

void cs_server::gpu_loop() {
    cudaSetDevice(device);
    cudaStream_t s;
    cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    const int64_t N = op->rows;
    for (;;) {
        std::vector<ApplyJob*> batch;
        int64_t K = 0;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return !jobs.empty() || (stop && active == 0); });
            if (jobs.empty()) break;
            if (opt.batch_window_ms > 0.0) {
                // hold the stack open for the other running requests' applies
                cv.wait_for(lk, std::chrono::duration<double, std::milli>(opt.batch_window_ms),
                            [&] { return (int)jobs.size() >= active || stop; });
            }
            while (!jobs.empty() &&
                   (batch.empty() || K + jobs.front()->k <= opt.max_batch_columns)) {
                batch.push_back(jobs.front());
                K += jobs.front()->k;
                jobs.pop_front();
            }
        }
        std::string err;
        try {
            xs.resize(N * K);
            ys.resize(N * K);
            CS_CUDA(cudaMemsetAsync(xs.get(), 0, 8 * N * K, s));
            int64_t off = 0;
            for (ApplyJob* j : batch) {
                cs::prof::Scope ps("serve_embed", s, 0.0, 16.0 * j->n_sub * j->k);
                k_embed<<<grid_for(j->n_sub * j->k), 256, 0, s>>>(j->X, j->ldx, j->n_sub, j->k,
                                                                  j->d_rows, xs.get(), K, off);
                CS_LAUNCH("serve_embed");
                off += j->k;
            }
            cs::kinship_apply_rowmajor(op, xs.get(), K, K, ys.get(), K, opt.precision, s);
            off = 0;
            for (ApplyJob* j : batch) {
                cs::prof::Scope ps("serve_extract", s, 0.0, 16.0 * j->n_sub * j->k);
                k_extract<<<grid_for(j->n_sub * j->k), 256, 0, s>>>(ys.get(), K, off, j->d_rows,
                                                                    j->n_sub, j->k, j->Y, j->ldy);
                CS_LAUNCH("serve_extract");
                off += j->k;
            }
            CS_CUDA(cudaStreamSynchronize(s));
        } catch (const std::exception& e) {
            err = e.what();
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            for (ApplyJob* j : batch) {
                j->error = err;
                j->done = true;
            }
            ++applies;
            apply_cols += K;
            max_jobs_per_apply = std::max<int64_t>(max_jobs_per_apply, (int64_t)batch.size());
        }
        cv.notify_all();
    }
    cudaStreamSynchronize(s);
    cs::release_thread_handles();
    cudaStreamDestroy(s);
}

void cs_server::apply(const int32_t* d_rows, int64_t n_sub, const double* X, int64_t ldx, int64_t k,
                      double* Y, int64_t ldy, cudaStream_t s) {
    CS_CUDA(cudaStreamSynchronize(s));  // X is complete before the GPU thread reads it
    ApplyJob job;
    job.d_rows = d_rows;
    job.n_sub = n_sub;
    job.k = k;
    job.X = X;
    job.ldx = ldx;
    job.Y = Y;
    job.ldy = ldy;
    {
        std::unique_lock<std::mutex> lk(mu);
        jobs.push_back(&job);
        cv.notify_all();
        cv.wait(lk, [&] { return job.done; });
    }
    if (!job.error.empty()) cs::fail(CS_ERR_CUDA, "serving apply failed: " + job.error);
}

void cs_server::dispatch_loop() {
    for (;;) {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] {
                if (stop) return true;
                if (queue.empty() || active >= opt.max_active) return false;
                const Request* f = reqs[queue.front()].get();
                return active == 0 || mem_in_use + f->est_bytes <= budget_bytes;
            });
            if (stop) break;
            r = reqs[queue.front()].get();
            queue.pop_front();
            ++active;
            max_active = std::max<int64_t>(max_active, active);
            mem_in_use += r->est_bytes;
            r->state = 1;
            r->t_start = now_s();
        }
        r->worker = std::thread([this, r] { run_request(r); });
    }
}

void cs_server::run_request(Request* r) {
    cudaSetDevice(device);
    cudaStream_t st = nullptr;
    std::string err;
    try {
        CS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        cs::set_thread_free_stream(st);
        const int64_t n = (int64_t)r->samples.size();
        cs::DeviceBuffer<int32_t> d_rows;
        d_rows.resize(n);
        CS_CUDA(cudaMemcpyAsync(d_rows.get(), r->samples.data(), 4 * n, cudaMemcpyHostToDevice, st));
        cs::LowRankTarget target;
        target.rows = n;
        double tr = 0.0;
        for (int32_t i : r->samples) tr += diag_full[i];
        target.trace = tr;
        const int32_t* rows = d_rows.get();
        std::unique_ptr<cs_kinship> sub;
        if (r->own_view) {
            sub.reset(cs::kinship_create(g, r->samples.data(), n,
                                         variants.empty() ? nullptr : variants.data(),
                                         (int64_t)variants.size()));
            sub->autotune = false;  // per-request shapes: the default plans, no tuning passes
            // the five-set form at every width (same result alone and in a stack), and no
            // sample-major copy (memory the admission budget does not count)
            sub->sample_major_copy = false;
            cs_kinship* so = sub.get();
            const int prec = opt.precision;
            target.apply = [so, prec](const double* X, int64_t ldx, int64_t k, double* Y,
                                      int64_t ldy, cudaStream_t s) {
                cs::kinship_apply_rowmajor(so, X, ldx, k, Y, ldy, prec, s);
            };
        } else {
            target.apply = [this, rows, n](const double* X, int64_t ldx, int64_t k, double* Y,
                                           int64_t ldy, cudaStream_t s) {
                apply(rows, n, X, ldx, k, Y, ldy, s);
            };
        }
        cs_lmm* lmm = cs::lmm_create();
        struct Guard {
            cs_lmm* l;
            ~Guard() { cs::lmm_destroy(l); }
        } guard{lmm};
        // destroyed first: on an error, the request's stream drains before its buffers go
        struct SyncGuard {
            cudaStream_t s;
            ~SyncGuard() { cudaStreamSynchronize(s); }
        } sync_guard{st};
        const int rank = std::max(1, std::min<int>(opt.rank, (int)n - 1));
        const int64_t W = r->end - r->begin;
        r->sigma2.assign(2 * r->t, 0.0);
        for (auto* v : {&r->beta, &r->se, &r->pval, &r->l10, &r->freq}) v->assign(r->t * W, 0.0);
        r->tested.assign(r->t * W, 0);
        cs_lowrank_diagnostics d{};
        for (int32_t j = 0; j < r->t; ++j) {
            const double* yj = r->Y.data() + (int64_t)j * n;
            if (j == 0) {
                cs::lmm_prepare_lowrank_target(lmm, target, yj, r->X.data(), r->p, rank,
                                               opt.oversample, (int64_t)r->seed, opt.trace_threshold,
                                               opt.min_rank, &d, st);
                // every trait's scan shares one projection of the window
                cs::lmm_set_scan_traits(lmm, r->Y.data(), r->t);
            } else
                cs::lmm_fit_reml(lmm, yj, r->X.data(), r->p, &d, st);
            r->effective_rank = d.effective_rank;
            r->sigma2[2 * j] = d.sigma2_g;
            r->sigma2[2 * j + 1] = d.sigma2_e;
            cs::lmm_scan_window(lmm, g, r->samples.data(), n, r->begin, r->end, opt.min_maf,
                                opt.precision, r->beta.data() + j * W, r->se.data() + j * W,
                                r->pval.data() + j * W, r->l10.data() + j * W,
                                r->freq.data() + j * W, r->tested.data() + j * W, st);
        }
        CS_CUDA(cudaStreamSynchronize(st));
    } catch (const std::exception& e) {
        err = e.what();
    }
    cs::set_thread_free_stream(nullptr);
    if (st) cudaStreamSynchronize(st);
    // this thread ends here: its library handles go back to the free list for the next worker
    cs::release_thread_handles();
    if (st) cudaStreamDestroy(st);
    {
        std::lock_guard<std::mutex> lk(mu);
        r->t_done = now_s();
        r->error = err;
        r->state = err.empty() ? 2 : -1;
        --active;
        mem_in_use -= r->est_bytes;
        if (err.empty()) {
            ++completed;
            latencies.push_back(r->t_done - r->t_submit);
            last_done = std::max(last_done, r->t_done);
        } else {
            ++failed;
        }
    }
    cv.notify_all();
}

namespace cs {

void server_default_options(cs_server_options* o) {
    o->rank = 256;
    o->oversample = 10;
    o->trace_threshold = 0.95;
    o->min_rank = 1;
    o->min_maf = 0.01;
    o->precision = CS_PRECISION_MIXED;
    o->max_batch_columns = 4096;
    o->memory_budget_gb = 0.0;
    o->max_active = 8;
    o->batch_window_ms = 0.0;
    o->subset_fraction = 0.5;
}

cs_server* server_create(const cs_genotypes* g, const int32_t* variants, int64_t n_var,
                         const cs_server_options* opt_in) {
    if (!g) fail(CS_ERR_INVALID_ARGUMENT, "null genotypes handle");
    auto* sv = new cs_server();
    try {
        if (opt_in) sv->opt = *opt_in;
        else server_default_options(&sv->opt);
        if (sv->opt.max_batch_columns < 1 || sv->opt.max_active < 1 || sv->opt.rank < 1 ||
            !(sv->opt.batch_window_ms >= 0.0) || !(sv->opt.subset_fraction >= 0.0))
            fail(CS_ERR_INVALID_ARGUMENT, "bad server options");
        CS_CUDA(cudaGetDevice(&sv->device));
        sv->g = g;
        sv->op = kinship_create(g, nullptr, 0, variants, n_var);
        sv->op->autotune = false;  // stacked widths vary from apply to apply
        // the five-set form at every width (same result alone and in a stack), and no second
        // resident copy of the matrix
        sv->op->sample_major_copy = false;
        if (variants && n_var > 0) sv->variants.assign(variants, variants + n_var);
        if (sv->opt.memory_budget_gb > 0.0) {
            sv->budget_bytes = (int64_t)(sv->opt.memory_budget_gb * 1e9);
        } else {
            size_t free_b = 0, total_b = 0;
            CS_CUDA(cudaMemGetInfo(&free_b, &total_b));
            const int64_t N = sv->op->rows, R = sv->op->n_active;
            const int64_t B = round_up(sv->opt.max_batch_columns, 16) + 16;
            const int64_t n_pad = round_up(N, 256), r_pad = round_up(R, 256);
            const int64_t shared = 8 * B * (2 * N + R + r_pad + 4 * n_pad) + 3 * B * n_pad +
                                   5 * B * r_pad;
            sv->budget_bytes = std::max<int64_t>(0, (int64_t)free_b - (int64_t)4e9 - shared);
        }
        sv->diag_full.resize(sv->op->rows);
        kinship_diagonal(sv->op, sv->diag_full.data());
        sv->gpu_thread = std::thread([sv] { sv->gpu_loop(); });
        sv->dispatch_thread = std::thread([sv] { sv->dispatch_loop(); });
    } catch (...) {
        delete sv;
        throw;
    }
    return sv;
}

int64_t server_submit(cs_server* sv, const cs_serve_request* q) {
    if (!q || !q->samples || q->n_samples <= 1 || q->n_traits < 1 || !q->Y || q->p < 0 ||
        (q->p > 0 && !q->X))
        fail(CS_ERR_INVALID_ARGUMENT, "serve request: bad arguments");
    const int64_t N = sv->g->n_samples, n = q->n_samples;
    if (q->snp_begin < 0 || q->snp_end > sv->g->n_snps || q->snp_begin >= q->snp_end)
        fail(CS_ERR_INVALID_ARGUMENT, "serve request: SNP window out of range");
    if (n <= q->p + 1) fail(CS_ERR_INVALID_ARGUMENT, "serve request: too few samples");
    std::vector<char> seen(N, 0);
    for (int64_t i = 0; i < n; ++i) {
        const int32_t s = q->samples[i];
        if (s < 0 || s >= N) fail(CS_ERR_INVALID_ARGUMENT, "serve request: sample index out of range");
        if (seen[s]) fail(CS_ERR_INVALID_ARGUMENT, "serve request: duplicate sample index");
        seen[s] = 1;
    }
    auto r = std::make_unique<Request>();
    r->samples.assign(q->samples, q->samples + n);
    r->Y.assign(q->Y, q->Y + n * q->n_traits);
    if (q->p > 0) r->X.assign(q->X, q->X + n * q->p);
    r->t = q->n_traits;
    r->p = q->p;
    r->begin = q->snp_begin;
    r->end = q->snp_end;
    r->seed = q->seed;
    const int64_t sk = std::min<int64_t>(n, sv->opt.rank + sv->opt.oversample);
    const int64_t W = r->end - r->begin;
    r->own_view = (double)n < sv->opt.subset_fraction * (double)N;
    r->est_bytes = 8 * n * sk * 4 + W * ((n + 3) / 4 + 64 + 8 * (sk + r->p + 2)) + 64 * n;
    if (r->own_view) {
        // the packed copy of the cohort's columns, the right-hand-side pieces of both passes
        // and the FP64 slice partials of the tensor-core form
        const int64_t rows = sv->op->num_variants, n_pad = round_up(n, 256);
        const int64_t kp = round_up(sk + r->p + 1, 16);
        r->est_bytes += rows * round_up((n + 3) / 4, kRowAlign) + 3 * kp * n_pad +
                        5 * kp * round_up(rows, 256) + 8 * 8 * kp * std::max(n_pad, rows) +
                        3 * 8 * kp * rows;  // rows-pass output, its copy for the scan, buf_u
    }
    std::lock_guard<std::mutex> lk(sv->mu);
    r->id = sv->next_id++;
    r->t_submit = now_s();
    if (sv->first_submit < 0) sv->first_submit = r->t_submit;
    const int64_t id = r->id;
    if (r->own_view) ++sv->own_view_requests;
    sv->reqs[id] = std::move(r);
    sv->queue.push_back(id);
    ++sv->submitted;
    sv->cv.notify_all();
    return id;
}

void server_wait(cs_server* sv, int64_t id, double timeout_s, cs_serve_status* out) {
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) fail(CS_ERR_INVALID_ARGUMENT, "unknown request id");
    Request* r = it->second.get();
    auto done = [&] { return r->state == 2 || r->state == -1; };
    if (timeout_s < 0)
        sv->cv.wait(lk, done);
    else
        sv->cv.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
    if (out) {
        out->state = r->state;
        out->latency_s = done() ? r->t_done - r->t_submit : -1.0;
        out->queue_s = r->state != 0 ? r->t_start - r->t_submit : -1.0;
        out->effective_rank = r->effective_rank;
    }
    if (r->state == -1) fail(CS_ERR_CUDA, "request failed: " + r->error);
}

void server_result(cs_server* sv, int64_t id, int32_t trait, double* sigma2, double* beta,
                   double* se, double* pval, double* log10p, double* freq, int32_t* tested) {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) fail(CS_ERR_INVALID_ARGUMENT, "unknown request id");
    Request* r = it->second.get();
    if (r->state != 2) fail(CS_ERR_INVALID_ARGUMENT, "request has not completed");
    if (trait < 0 || trait >= r->t) fail(CS_ERR_INVALID_ARGUMENT, "trait index out of range");
    const int64_t W = r->end - r->begin, o = trait * W;
    if (sigma2) {
        sigma2[0] = r->sigma2[2 * trait];
        sigma2[1] = r->sigma2[2 * trait + 1];
    }
    auto cp = [&](const std::vector<double>& v, double* d) {
        if (d) std::copy(v.begin() + o, v.begin() + o + W, d);
    };
    cp(r->beta, beta);
    cp(r->se, se);
    cp(r->pval, pval);
    cp(r->l10, log10p);
    cp(r->freq, freq);
    if (tested) std::copy(r->tested.begin() + o, r->tested.begin() + o + W, tested);
}

void server_release(cs_server* sv, int64_t id) {
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        auto it = sv->reqs.find(id);
        if (it == sv->reqs.end()) fail(CS_ERR_INVALID_ARGUMENT, "unknown request id");
        if (it->second->state == 0 || it->second->state == 1)
            fail(CS_ERR_INVALID_ARGUMENT, "request still running");
        r = std::move(it->second);
        sv->reqs.erase(it);
    }
    if (r->worker.joinable()) r->worker.join();
}

void server_stats(cs_server* sv, cs_server_statistics* out) {
    std::lock_guard<std::mutex> lk(sv->mu);
    *out = cs_server_statistics{};
    out->submitted = sv->submitted;
    out->completed = sv->completed;
    out->failed = sv->failed;
    out->applies = sv->applies;
    out->apply_columns = sv->apply_cols;
    out->max_requests_per_apply = sv->max_jobs_per_apply;
    out->max_concurrent = sv->max_active;
    out->own_view_requests = sv->own_view_requests;
    out->memory_budget_gb = (double)sv->budget_bytes / 1e9;
    std::vector<double> l = sv->latencies;
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
        if (l.empty()) return 0.0;
        const double pos = q * (double)(l.size() - 1);
        const size_t a = (size_t)pos, b = std::min(l.size() - 1, a + 1);
        return l[a] + (l[b] - l[a]) * (pos - (double)a);
    };
    out->p50_s = pct(0.50);
    out->p99_s = pct(0.99);
    double sum = 0.0;
    for (double v : l) sum += v;
    out->mean_s = l.empty() ? 0.0 : sum / (double)l.size();
    out->wall_s = sv->completed ? sv->last_done - sv->first_submit : 0.0;
    out->throughput_rps = out->wall_s > 0 ? (double)sv->completed / out->wall_s : 0.0;
}

void server_destroy(cs_server* sv) { delete sv; }

}  // namespace cs
