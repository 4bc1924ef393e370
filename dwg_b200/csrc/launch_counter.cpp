// launch_counter.cpp -- kernel launch census for the benchmark (built as its
// own liblaunch_counter.so; the product library does not depend on it).
//
// Uses the CUPTI activity API (concurrent-kernel records, which include the
// kernels of CUDA graph replays) to count the kernels that run between
// dwglc_start() and dwglc_stop(), with their device time, by name.
#include <cupti.h>
#include <cxxabi.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

namespace {

struct Stat {
    long long count = 0;
    unsigned long long ns = 0;
};

std::mutex g_mu;
std::map<std::string, Stat> g_stats;
bool g_registered = false;

void CUPTIAPI buffer_requested(uint8_t** buffer, size_t* size, size_t* max_records) {
    *size = 8u << 20;
    *buffer = static_cast<uint8_t*>(aligned_alloc(8, *size));
    *max_records = 0;
}

std::string short_name(const char* mangled) {
    if (!mangled) return "?";
    int st = 0;
    char* d = abi::__cxa_demangle(mangled, nullptr, nullptr, &st);
    std::string s = (st == 0 && d) ? std::string(d) : std::string(mangled);
    free(d);
    const size_t p = s.find('(');
    if (p != std::string::npos) s = s.substr(0, p);
    return s;
}

void CUPTIAPI buffer_completed(CUcontext, uint32_t, uint8_t* buffer, size_t, size_t valid) {
    CUpti_Activity* rec = nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    while (cuptiActivityGetNextRecord(buffer, valid, &rec) == CUPTI_SUCCESS) {
        if (rec->kind != CUPTI_ACTIVITY_KIND_CONCURRENT_KERNEL && rec->kind != CUPTI_ACTIVITY_KIND_KERNEL) continue;
        const auto* k = reinterpret_cast<const CUpti_ActivityKernel9*>(rec);
        Stat& s = g_stats[short_name(k->name)];
        s.count += 1;
        if (k->end > k->start) s.ns += k->end - k->start;
    }
    free(buffer);
}

}  // namespace

extern "C" {

// 0 on success, else the CUPTI result code
int dwglc_start(void) {
    if (!g_registered) {
        CUptiResult r = cuptiActivityRegisterCallbacks(buffer_requested, buffer_completed);
        if (r != CUPTI_SUCCESS) return (int)r;
        g_registered = true;
    }
    {
        std::lock_guard<std::mutex> lock(g_mu);
        g_stats.clear();
    }
    return (int)cuptiActivityEnable(CUPTI_ACTIVITY_KIND_CONCURRENT_KERNEL);
}

int dwglc_stop(void) {
    CUptiResult r = cuptiActivityFlushAll(1);
    CUptiResult r2 = cuptiActivityDisable(CUPTI_ACTIVITY_KIND_CONCURRENT_KERNEL);
    return r != CUPTI_SUCCESS ? (int)r : (int)r2;
}

// "name<TAB>count<TAB>total_ns" lines; returns the bytes needed (incl. NUL)
int dwglc_report(char* buf, int buflen) {
    std::string out;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        for (const auto& kv : g_stats) {
            char line[64];
            snprintf(line, sizeof(line), "\t%lld\t%llu\n", kv.second.count, kv.second.ns);
            out += kv.first;
            out += line;
        }
    }
    if (buf && buflen > 0) {
        const size_t n = out.size() < (size_t)buflen - 1 ? out.size() : (size_t)buflen - 1;
        memcpy(buf, out.data(), n);
        buf[n] = 0;
    }
    return (int)out.size() + 1;
}

}  // extern "C"
