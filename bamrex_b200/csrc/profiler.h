// Host-side region timers, the library's counterpart of AMReX's
// BL_PROFILE / TinyProfiler scopes (e.g. Source/AmrLevelAdv_advance.cpp:24,
// Source/main.cpp:21): BX_PROFILE("name") times the enclosing scope in wall
// clock and accumulates calls, total and maximum per name.  Off unless
// bamrex_profile_enable(1) or the environment variable BAMREX_TINY_PROFILE
// is set (non-empty, not "0"); when off a scope costs one relaxed atomic
// load.  Device work is not synchronised: a region that only enqueues
// kernels measures the enqueue.
#pragma once

#include <atomic>
#include <chrono>

namespace bamrex {

extern std::atomic<int> g_profile_on;
void profile_record(const char* name, double seconds);

class ProfScope {
public:
    explicit ProfScope(const char* name) : name_(name), on_(g_profile_on.load(std::memory_order_relaxed) != 0)
    {
        if (on_) t0_ = std::chrono::steady_clock::now();
    }
    ~ProfScope()
    {
        if (on_) profile_record(name_, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count());
    }
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;

private:
    const char* name_;
    bool on_;
    std::chrono::steady_clock::time_point t0_;
};

// Consecutive phases of one function: each next() closes the running phase
// and opens the next; the destructor closes the last.
class ProfPhases {
public:
    explicit ProfPhases(const char* first) : name_(first), on_(g_profile_on.load(std::memory_order_relaxed) != 0)
    {
        if (on_) t0_ = std::chrono::steady_clock::now();
    }
    void next(const char* name)
    {
        if (!on_) return;
        const auto t = std::chrono::steady_clock::now();
        profile_record(name_, std::chrono::duration<double>(t - t0_).count());
        name_ = name;
        t0_ = t;
    }
    ~ProfPhases()
    {
        if (on_) profile_record(name_, std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count());
    }
    ProfPhases(const ProfPhases&) = delete;
    ProfPhases& operator=(const ProfPhases&) = delete;

private:
    const char* name_;
    bool on_;
    std::chrono::steady_clock::time_point t0_;
};

}  // namespace bamrex

#define BX_PROFILE_CAT2(a, b) a##b
#define BX_PROFILE_CAT(a, b) BX_PROFILE_CAT2(a, b)
#define BX_PROFILE(name) ::bamrex::ProfScope BX_PROFILE_CAT(bx_prof_scope_, __LINE__)(name)
