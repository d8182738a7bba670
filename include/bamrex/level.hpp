// C++ host-side mirror of the reference's level surface over the C ABI
// (include/bamrex_cuda.h): bamrex::Level has AmrLevelAdv's names
// (advance, estTimeStep, computeNewDt-style run) and bamrex::Parm mirrors
// Parm (Source/System/Parm.H:14-61).  Header-only; errors become
// bamrex::Error exceptions on this side of the ABI.
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

#include "../bamrex_cuda.h"

namespace bamrex {

class Error : public std::runtime_error {
public:
    Error(int status, const std::string& msg) : std::runtime_error(msg), status_(status) {}
    int status() const { return status_; }

private:
    int status_;
};

inline void check(int rc, const bamrex_level* level = nullptr)
{
    if (rc == BAMREX_OK) return;
    std::string msg = level ? bamrex_level_last_error(level) : "";
    if (msg.empty()) msg = bamrex_last_error();
    if (msg.empty()) msg = bamrex_status_string(rc);
    throw Error(rc, msg);
}

// FluidSystem::set_parm_defaults + init_parm for a spacedim-dimensional fluid.
inline bamrex_parm make_parm(int spacedim, double adiabatic, double epsilon = 1.0, int limiter = BAMREX_VAN_LEER)
{
    bamrex_parm p;
    check(bamrex_parm_set_defaults(&p, spacedim));
    p.adiabatic = adiabatic;
    p.epsilon = epsilon;
    p.limiter = limiter;
    check(bamrex_parm_init(&p));
    return p;
}

// One AMR level's state on the device, advanced like AmrLevelAdv.
class Level {
public:
    Level(const bamrex_level_desc& desc, void* stream = nullptr) { check(bamrex_level_create(&h_, &desc, stream)); }
    ~Level() { bamrex_level_destroy(h_); }
    Level(const Level&) = delete;
    Level& operator=(const Level&) = delete;

    long long numCells() const { return bamrex_level_num_cells(h_); }

    // valid cells of every box, box-major, component-slowest
    void copyIn(const double* src) { check(bamrex_level_copy_in(h_, src), h_); }
    void copyOut(double* dst) { check(bamrex_level_copy_out(h_, dst), h_); }
    void sync() { check(bamrex_level_sync(h_), h_); }
    bamrex_array4 fab(int box) const
    {
        bamrex_array4 a;
        check(bamrex_level_fab(h_, box, &a), h_);
        return a;
    }

    // AmrLevelAdv::advance(time, dt, iteration, ncycle) (Source/AmrLevelAdv.H:110-111)
    double advance(double time, double dt, int iteration = 1, int ncycle = 1)
    {
        double used = 0.0;
        check(bamrex_level_advance(h_, time, dt, iteration, ncycle, &used), h_);
        return used;
    }

    // AmrLevelAdv::estTimeStep (Source/AmrLevelAdv.cpp:395-477)
    double estTimeStep()
    {
        double dt = 0.0;
        check(bamrex_level_est_time_step(h_, &dt), h_);
        return dt;
    }

    // The coarse-step loop with computeInitialDt / computeNewDt on the device:
    // returns the number of steps taken; time is updated.
    int run(int nsteps, double stop_time, double& time, bool use_graph = true)
    {
        int steps = 0;
        check(bamrex_level_run(h_, nsteps, stop_time, use_graph ? 1 : 0, &time, &steps), h_);
        return steps;
    }

    bamrex_level* handle() { return h_; }

private:
    bamrex_level* h_ = nullptr;
};

}  // namespace bamrex
