// Registry of the host-side region timers (profiler.h) and their C ABI:
// enable / reset / a text report sorted by total time, in the spirit of
// TinyProfiler's end-of-run table.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "bamrex_cuda.h"
#include "profiler.h"

namespace bamrex {

namespace {

int env_on()
{
    const char* v = std::getenv("BAMREX_TINY_PROFILE");
    return (v && v[0] && std::strcmp(v, "0") != 0) ? 1 : 0;
}

struct Region {
    long long calls = 0;
    double total = 0, max = 0;
};

std::mutex& reg_mutex()
{
    static std::mutex m;
    return m;
}

std::unordered_map<std::string, Region>& regions()
{
    static std::unordered_map<std::string, Region> r;
    return r;
}

}  // namespace

std::atomic<int> g_profile_on{ env_on() };

void profile_record(const char* name, double seconds)
{
    std::lock_guard<std::mutex> lk(reg_mutex());
    Region& r = regions()[name];
    r.calls += 1;
    r.total += seconds;
    r.max = std::max(r.max, seconds);
}

}  // namespace bamrex

extern "C" int bamrex_profile_enable(int on) { return bamrex::g_profile_on.exchange(on ? 1 : 0); }

extern "C" int bamrex_profile_reset(void)
{
    std::lock_guard<std::mutex> lk(bamrex::reg_mutex());
    bamrex::regions().clear();
    return BAMREX_OK;
}

extern "C" int bamrex_profile_report(char* out, int cap, int* needed)
{
    std::vector<std::pair<std::string, bamrex::Region>> rows;
    {
        std::lock_guard<std::mutex> lk(bamrex::reg_mutex());
        rows.assign(bamrex::regions().begin(), bamrex::regions().end());
    }
    std::sort(rows.begin(), rows.end(), [](const auto& a, const auto& b) {
        return a.second.total != b.second.total ? a.second.total > b.second.total : a.first < b.first;
    });
    std::string s = "region calls total_s avg_ms max_ms\n";
    char line[512];
    for (const auto& r : rows) {
        std::snprintf(line, sizeof(line), "%s %lld %.6f %.4f %.4f\n", r.first.c_str(), r.second.calls, r.second.total,
                      1e3 * r.second.total / (double)std::max(1LL, r.second.calls), 1e3 * r.second.max);
        s += line;
    }
    if (needed) *needed = (int)s.size() + 1;
    if (out && cap > 0) {
        const size_t n = std::min((size_t)cap - 1, s.size());
        std::memcpy(out, s.data(), n);
        out[n] = '\0';
    }
    return BAMREX_OK;
}
