// Coarse/fine coupling of two AMR levels: tables shared by the host builder
// (amr.cu) and the kernels (amr_kernels.cu).
//
// The arithmetic AMReX performs for the reference at these call sites
// (FillPatch with cell_cons_interp and time interpolation, FluxRegister
// Reflux, average_down) lives in AMReX, which is not part of the reference;
// the kernels here implement the published methods:
//  * time interpolation: alpha * S_old + beta * S_new with
//    alpha = (t_new - t) / (t_new - t_old), beta = (t - t_old) / (t_new - t_old),
//    and the old or new state itself when t is within 1e-3 (t_new - t_old) of
//    either end;
//  * spatial interpolation: conservative piecewise-linear reconstruction from
//    the coarse cell with monotonized-central slopes (van Leer 1977) and a
//    Barth-Jespersen (1989) scale that keeps every fine value inside the
//    range of the coarse cell and its face neighbours;
//  * average_down: the mean of the r^D fine cells over each covered coarse
//    cell;
//  * reflux: each coarse cell next to the fine region is corrected by
//    -/+ (sum of dt-and-area-scaled fine fluxes - scaled coarse flux) / V.
#pragma once

#include "common.cuh"
#include "launch.h"

namespace bamrex {

// A fine ghost region filled by interpolation: fine cells [lo, hi] of box
// dst (unshifted index space), whose periodic image is cell + shift; the
// coarse patch [plo, plo + pn) of the image starts at patch_begin.
struct CfRegion {
    int dst;
    int lo[3], hi[3];
    int shift[3];
    int plo[3], pn[3];
    int pad;
    long long patch_begin;
    long long cell_begin;
};

// Coarse cells [lo, hi] of coarse box `crse` covered by fine box `fine`.
struct AvgOp {
    int crse, fine;
    int lo[3], hi[3];
    long long cell_begin;
};

// Coarse cell corrected by one flux-register slot, and the side it sits on
// (sign -1: the face is its high face, +1: its low face).
struct RefluxRec {
    int box;
    int i, j, k;
    int sign;
};

struct CfInterpArgs {
    const CfRegion* regions;
    int nregions;
    long long ncells;
    const double* patch;  // NC * npatch, component-major
    long long npatch;
    const FabDev* fine0;  // both state buffers of the fine level
    const FabDev* fine1;
    int D, NC, ratio;
};

// Which box of a level holds each cell, at the granularity of the level's
// box corners: blocks of g[0] x g[1] x g[2] cells from the domain's low
// corner; owner[(K * nb[1] + J) * nb[0] + I] is the box covering block
// (I, J, K), -1 where no box does.
struct OwnerMap {
    const int* owner;
    int lo[3], g[3], nb[3];
};

// The coarse domain and its boundary kinds: a patch cell outside it is read
// at its periodic image, its mirror image (with the normal momentum
// negated) or the nearest domain cell, by the side's boundary kind.
struct CoarseDomain {
    int lo[3], hi[3];
    int bc_lo[3], bc_hi[3];
    int D;
};

// The coarse patches of a set of regions, gathered cell by cell: patch cell
// e lies in the region whose [patch_begin, patch_begin + volume) holds e, at
// plo + (x, y, z) with x fastest; its coarse cell is mapped into the domain
// and looked up in the owner map.
// Time stepping of a hierarchy on the device (a coarse step replayed as one
// CUDA graph): the coarse time, the stop time, every level's time step and
// the start time of every level's current substep, computed there with the
// host recursion's own arithmetic (Source/AmrLevelAdv.cpp:487-619).
constexpr int kAmrMaxLevels = 8;
struct AmrDev {
    double time;       // coarse time at the start of the step (host-written)
    double stop_time;  // < 0: none (host-written)
    double dt0;        // the coarse step's dt
    int status;        // BAMREX_* raised during the step
    int pad;
    double dt[kAmrMaxLevels];     // dt of each level
    double t_sub[kAmrMaxLevels];  // start time of each level's current substep
};

// Per-level arguments of the device time step (by value).
struct AmrLevelsArg {
    StepScalars* scal[kAmrMaxLevels];
    double dx[kAmrMaxLevels][3];
    double cfl[kAmrMaxLevels];
    int nl, D, ratio;
};

struct CfGatherArgs {
    const CfRegion* regions;  // ascending patch_begin
    int nregions;
    long long npatch;
    OwnerMap own;
    CoarseDomain dom;
    const double* patch_old;  // the coarse old values of the patch cells (saved by mode 4)
    const FabDev* crse_new;
    int NC;
    // 0 old, 1 new, 2 a_old * old + a_new * new, 3 check the owners only,
    // 4 save: the current coarse values of the patch cells as they are (no
    // boundary sign) into `patch`, which then serves as patch_old
    int mode;
    double a_old, a_new;
    double* patch;            // NC * npatch, component-major (not written in mode 3)
    unsigned long long* bad;  // mode 3: lowered to the first patch cell with no owner
    // non-null: mode and weights from the device times of the coarse level
    // lc (its substep start and dt) and the fine level lc + 1, decided as
    // bamrex_coupling_fill_patch decides them on the host
    const AmrDev* amr;
    int lc;
};

cudaError_t launch_cf_gather(bool fp32, const CfGatherArgs& a, cudaStream_t s);
// The coarse step's dt from every level's max wave speed (est_time_step +
// computeNewDt without a regrid) into a->dt and each level's scalars; the
// first level status (a rigid-body or staging failure of an earlier step)
// or a non-finite estimate into a->status.
cudaError_t launch_amr_dt(AmrDev* a, const AmrLevelsArg& lv, cudaStream_t s);
// t_sub[l] = t_sub[l - 1] + i * dt[l]: the start of substep i of level l.
cudaError_t launch_amr_substep(AmrDev* a, int l, int i, cudaStream_t s);

cudaError_t launch_cf_interp(bool fp32, const CfInterpArgs& a, cudaStream_t s);
cudaError_t launch_avg_down(int D, int NC, int ratio, bool fp32, const AvgOp* ops, int nops, long long ncells,
                            const FabDev* crse, const FabDev* fine, cudaStream_t s);
cudaError_t launch_reflux(int NC, bool fp32, const RefluxRec* recs, int nslots, const double* reg, double vol,
                          const FabDev* crse, cudaStream_t s);
// Tagging criteria of AmrLevelAdv::errorEst (Source/AmrLevelAdv.cpp:711-832):
// state_error on err_var >= err_thr, grad_error on grad_var with relative
// threshold grad_thr; *_primv selects the primitive vector.
struct TagSpec {
    int do_err, err_var, err_primv;
    int do_grad, grad_var, grad_primv;
    double err_thr, grad_thr;
    // box_error: cell centres (i + 1/2) dx + prob_lo inside [box_lo, box_hi]
    int do_box;
    double box_lo[3], box_hi[3], dx[3], prob_lo[3];
    // a rigid body's level set (component 0 of its fabs) and GFM flags (one
    // byte per cell), per box; flag_tab non-null: ghost_error clears solid
    // cells not at the interface; do_iface: interface_error with lstol
    const FabDev* ls_tab;
    const FabDev* flag_tab;
    int do_iface;
    double lstol;
};

// errorEst tagging (Source/Src_K/tagging_K.H:9-105: state_error,
// grad_error, box_error, interface_error, then ghost_error) over the valid
// cells of a level, tags (0/1) in the packed cell order.
cudaError_t launch_tag(int D, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes, long long ncells,
                       const Consts& k, const TagSpec& spec, char* tags, cudaStream_t s);

}  // namespace bamrex
