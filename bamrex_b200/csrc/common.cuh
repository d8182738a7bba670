// Shared device/host types of the B200 explicit finite-volume path.
#pragma once

#include <cstdint>

namespace bamrex {

constexpr int kMaxComp = 8;

// Per-run physical and limiter constants.  Everything derived from gamma is
// computed on the host with the reference's own expressions
// (Source/Fluxes/HLLC.H:269-280, Source/System/FluidSystem.cpp:73-101) so the
// device sees bit-identical values.
struct Consts {
    double gamma;       // adiabatic
    double eps;         // epsilon (low-Mach scaling)
    double inv_eps;     // 1/epsilon
    double gm1;         // gamma - 1
    double half_gm1;    // (gamma - 1) / 2
    double z;           // (gamma - 1) / (2 gamma)
    double neg_z;       // -z
    double inv_z;       // 1 / z
    double gp1_2g;      // (gamma + 1) / (2 gamma)
    double gamma_inv_eps;  // gamma / epsilon
    // Fast roots: when 1/z is (to rounding) the integer root_k, the powers
    // p^-z and x^(1/z) are evaluated as a Newton-refined k-th root / integer
    // power plus a first-order correction for the tiny exponent offsets
    // root_dneg = 1/k - z and root_dpos = 1/z - k.  root_k = 0: use pow().
    int root_k;
    double root_dneg;
    double root_dpos;
    double root_dneg_l2;   // root_dneg * ln 2 (applied to log2 x)
    double root_dpos_l2;   // root_dpos * ln 2
    double half_eps;       // 0.5 * epsilon
    int limiter;        // BAMREX_MINBEE ..
    // Limiting variable per component (Parm::limiter_indices /
    // limit_on_primv, Source/Fluxes/CalcLimitingVal.H:9-22).  uniform_var >= 0
    // when every component limits on the same conserved variable.
    int uniform_var;
    int need_prim;
    int lim_var[kMaxComp];
    int lim_prim[kMaxComp];
};

// A fab (amrex::Array4 geometry) on the device.
// p points at elements of the storage type (double, or float for the
// FP32-storage variant); strides count elements.
struct FabDev {
    void* p;
    template <typename T>
    __host__ __device__ __forceinline__ T* ptr() const { return static_cast<T*>(p); }
    long long js, ks, ns;
    int b0, b1, b2;  // begin corner
};

// One box of a sweep launch.
struct SweepBox {
    int lo[3], hi[3];
    FabDev in, out, flux;      // flux.p == nullptr: no flux output
    long long item_begin;      // first work item of this box
    int nseg;                  // segments along the sweep direction
    int ngroup;                // lane groups of 32 columns (marching sweeps)
    int seglen;                // cells per segment (the last one may be shorter)
    // TMA-staged sweeps (sweep_tma.cuh): the tensor map of `in` for this
    // direction (device memory), lines of a lane group along the faster
    // transverse direction, and the elements between the map's x origin
    // (the 256-byte aligned start of the padded row) and in.b0
    const void* tmap;
    int wa;
    int xoff;
    // marching x sweep: the same-level fab holding all of this box's ghost
    // cells below lo (xnb[0]) / above hi (xnb[1]) in x, read in place of
    // the ghost cells when SweepArgs::xnb_on (p == nullptr: none)
    FabDev xnb[2];
};

// Device-resident step scalars (graph-friendly time stepping).
struct StepScalars {
    double time;
    double dt;
    double stop_time;          // < 0: none
    unsigned long long ws_bits;  // max wave speed as ordered bits (>= 0 doubles)
    int done;                  // time reached stop_time: kernels return early
    int steps;                 // steps taken
    int status;                // BAMREX_* error raised on the device
    int pad;
};

struct SweepArgs {
    const SweepBox* boxes;     // device box table, or nullptr: use `one`
    SweepBox one;              // single box passed by value (per-box calls)
    int nboxes;
    long long total_items;
    int seglen;                // the level's segment length (boxes hold their own)
    int halo;                  // 2 for reconstructing methods, 1 for first order
    double dt_host;
    const StepScalars* scal;   // non-null: dt from scal->dt, skip if done
    double dx;                 // dx[dir]
    Consts k;
    unsigned long long* ws_max;  // non-null: reduce max wave speed of Uout
    int do_update;             // 0: flux-only mode
    int* status;
    int xnb_on;                // marching x sweep: read x halos from SweepBox::xnb
};

}  // namespace bamrex
