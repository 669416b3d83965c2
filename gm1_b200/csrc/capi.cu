// capi.cu - version, error reporting and the launch profiler of libgm1b.so.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "gm1b_common.cuh"

namespace {
thread_local char g_error[512] = "";

struct Pending {
    const char *name;
    cudaEvent_t start, stop;
};

struct Profiler {
    std::mutex mu;
    bool on = false;
    std::vector<cudaEvent_t> pool;  // free events
    std::vector<Pending> pending;
    cudaEvent_t take() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        return e;
    }
};

Profiler &profiler() {
    static Profiler p;
    return p;
}
}  // namespace

void gm1b_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

namespace gm1b {

ProfScope::ProfScope(const char *name, cudaStream_t st) : name_(name), st_(st), start_(nullptr) {
    Profiler &p = profiler();
    if (!p.on) return;
    std::lock_guard<std::mutex> g(p.mu);
    start_ = p.take();
    if (start_ != nullptr) cudaEventRecord(start_, st_);
}

void ProfScope::stop() {
    if (start_ == nullptr) return;
    Profiler &p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    cudaEvent_t e = p.take();
    if (e == nullptr) {
        p.pool.push_back(start_);
        start_ = nullptr;
        return;
    }
    cudaEventRecord(e, st_);
    p.pending.push_back(Pending{name_, start_, e});
    start_ = nullptr;
}

}  // namespace gm1b

extern "C" int32_t gm1b_abi_version(void) { return GM1B_ABI_VERSION; }

extern "C" const char *gm1b_last_error(void) { return g_error; }

extern "C" int32_t gm1b_profiler_enable(int32_t on) {
    Profiler &p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    p.on = on != 0;
    return GM1B_OK;
}

extern "C" int32_t gm1b_profiler_collect(gm1b_kernel_stat *out, int32_t capacity, int32_t *count) {
    if (count == nullptr || (out == nullptr && capacity > 0)) {
        gm1b_set_error("gm1b_profiler_collect: NULL output");
        return GM1B_ERR_ARGUMENT;
    }
    Profiler &p = profiler();
    std::lock_guard<std::mutex> g(p.mu);
    std::vector<gm1b_kernel_stat> stats;
    int32_t status = GM1B_OK;
    for (const Pending &q : p.pending) {
        float ms = 0.0f;
        cudaError_t e = cudaEventSynchronize(q.stop);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, q.start, q.stop);
        if (e != cudaSuccess) {
            gm1b_set_error("gm1b_profiler_collect: %s", cudaGetErrorString(e));
            status = GM1B_ERR_CUDA;
        }
        size_t k = 0;
        for (; k < stats.size(); ++k)
            if (std::strncmp(stats[k].name, q.name, sizeof(stats[k].name)) == 0) break;
        if (k == stats.size()) {
            gm1b_kernel_stat s{};
            std::snprintf(s.name, sizeof(s.name), "%s", q.name);
            stats.push_back(s);
        }
        stats[k].launches += 1;
        stats[k].total_ms += ms;
        p.pool.push_back(q.start);
        p.pool.push_back(q.stop);
    }
    p.pending.clear();
    for (size_t a = 0; a < stats.size(); ++a)
        for (size_t b = a + 1; b < stats.size(); ++b)
            if (stats[b].total_ms > stats[a].total_ms) std::swap(stats[a], stats[b]);
    const int32_t n = (int32_t)stats.size();
    *count = n;
    for (int32_t q = 0; q < n && q < capacity; ++q) out[q] = stats[q];
    return status;
}
