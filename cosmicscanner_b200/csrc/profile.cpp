// Launch counting and optional CUDA-event timing of the library's own kernels.
//
// Every kernel launch site is wrapped in a prof::Scope.  The launch counter always runs;
// when profiling is enabled the scope also records a start/stop event pair on the
// launching stream, and cs_profile_summary() reports per kernel name the launches, the
// summed device time and the algorithmic FLOPs / bytes the launch site declared.
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "cs_internal.h"

namespace cs {
namespace prof {

namespace {
struct Record {
    const char* name;
    cudaEvent_t a, b;
    double flops, bytes;
};
std::atomic<int64_t> g_launches{0};
std::atomic<bool> g_enabled{false};
std::mutex g_mu;
std::vector<Record> g_records;
std::vector<cudaEvent_t> g_pool;
std::map<std::string, std::pair<int64_t, double>> g_host;  // name -> (calls, seconds)

double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    CS_CUDA(cudaEventCreate(&e));
    return e;
}
}  // namespace

bool enabled() { return g_enabled.load(std::memory_order_relaxed); }

Scope::Scope(const char* name, cudaStream_t s, double flops, double bytes)
    : name_(name), s_(s), flops_(flops), bytes_(bytes) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (!enabled()) return;
    std::lock_guard<std::mutex> lk(g_mu);
    a_ = take_event();
    CS_CUDA(cudaEventRecord(a_, s_));
}

Scope::~Scope() {
    if (!a_) return;
    std::lock_guard<std::mutex> lk(g_mu);
    cudaEvent_t b = take_event();
    cudaEventRecord(b, s_);
    g_records.push_back(Record{name_, a_, b, flops_, bytes_});
}

HostScope::HostScope(const char* name) : name_(name) {
    if (enabled()) t0_ = now_seconds();
}

HostScope::~HostScope() {
    if (t0_ < 0.0) return;
    const double dt = now_seconds() - t0_;
    std::lock_guard<std::mutex> lk(g_mu);
    auto& e = g_host[name_];
    e.first += 1;
    e.second += dt;
}

int64_t launches() { return g_launches.load(); }

void set_enabled(bool on) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto& r : g_records) {
        g_pool.push_back(r.a);
        g_pool.push_back(r.b);
    }
    g_records.clear();
    g_host.clear();
    g_enabled = on;
}

std::string summary_json() {
    std::lock_guard<std::mutex> lk(g_mu);
    CS_CUDA(cudaDeviceSynchronize());
    struct Agg {
        int64_t n = 0;
        double ms = 0, flops = 0, bytes = 0, max_ms = 0;
    };
    std::map<std::string, Agg> agg;
    for (auto& r : g_records) {
        float ms = 0.f;
        CS_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        Agg& a = agg[r.name];
        a.n += 1;
        a.ms += ms;
        a.flops += r.flops;
        a.bytes += r.bytes;
        if (ms > a.max_ms) a.max_ms = ms;
    }
    std::string out = "{\"kernels\": [";
    bool first = true;
    char buf[512];
    for (auto& kv : agg) {
        std::snprintf(buf, sizeof buf,
                      "%s{\"name\": \"%s\", \"launches\": %lld, \"ms\": %.6f, \"max_ms\": %.6f, "
                      "\"flops\": %.6e, \"bytes\": %.6e}",
                      first ? "" : ", ", kv.first.c_str(), (long long)kv.second.n, kv.second.ms,
                      kv.second.max_ms, kv.second.flops, kv.second.bytes);
        out += buf;
        first = false;
    }
    out += "], \"host\": [";
    first = true;
    for (auto& kv : g_host) {
        std::snprintf(buf, sizeof buf, "%s{\"name\": \"%s\", \"calls\": %lld, \"ms\": %.6f}",
                      first ? "" : ", ", kv.first.c_str(), (long long)kv.second.first,
                      kv.second.second * 1e3);
        out += buf;
        first = false;
    }
    out += "], \"autotune\": " + autotune_json() + "}";
    return out;
}

}  // namespace prof
}  // namespace cs
