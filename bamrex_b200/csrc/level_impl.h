// Private host-side definition of bamrex_level and the level-step helpers,
// shared by the C ABI (abi.cu) and the coarse/fine coupling (amr.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "bamrex_cuda.h"
#include "devmem.h"
#include "launch.h"
#include "profiler.h"

namespace bamrex {

// Error reporting shared by every entry point (thread-local message).
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
const char* last_error_text();

#define BX_CK(call)                                                  \
    do {                                                             \
        cudaError_t e_ = (call);                                     \
        if (e_ != cudaSuccess) return ::bamrex::cuda_fail(e_, #call); \
    } while (0)

#define BX_TRY(call)                      \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ != BAMREX_OK) return rc_; \
    } while (0)

size_t align_up(size_t v, size_t a);

// Faces whose flux a level step records into a flux register (the FluxRegister
// CrseInit / FineAdd calls of AmrLevelAdv::advance,
// Source/AmrLevelAdv_advance.cpp:236-254).  One slot per coarse face; a slot
// takes `per_slot` consecutive face records.
struct FaceRec {
    int box;
    int i, j, k;  // face index: the face between cells (i,j,k) - e_dir and (i,j,k)
};

struct RegisterTask {
    const FaceRec* faces = nullptr;  // device, nslots * per_slot records
    int nslots = 0;
    int per_slot = 1;
    double* reg = nullptr;  // device, NC * nslots (component-major)
    int mode = 0;           // 0: reg = -(F * scale) (CrseInit); 1: reg += F * scale per face (FineAdd)
};

// Rigid body of a level (gfm.cu).
struct BodyState;

}  // namespace bamrex

struct bamrex_level {
    int D = 0, NC = 0, ngrow = 0, method = 0;
    bool fp32 = false;   // FP32-storage variant
    size_t esize = 8;    // bytes per stored value
    double cfl = 0.9;
    bamrex_parm parm;
    bamrex::Consts k;
    bamrex_box domain;
    double dx[3] = { 1, 1, 1 };
    double prob_lo[3] = { 0, 0, 0 };
    int bc_lo[3] = { 0, 0, 0 }, bc_hi[3] = { 0, 0, 0 };
    std::vector<bamrex_box> boxes;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;

    // device memory (one arena)
    char* arena = nullptr;
    char* state[2] = { nullptr, nullptr };
    double* d_box_sums = nullptr;  // nboxes x NC, conserved sums
    std::vector<bamrex::FabDev> fab[2];
    bamrex::FabDev* d_fab[2] = { nullptr, nullptr };
    bamrex::SweepBox* d_sweep[3][2] = {};
    long long items[3] = { 0, 0, 0 };
    int seglen[3] = { 0, 0, 0 };
    bool x_march = false;  // x sweep by the marching (thread-per-row) kernel
    // x halos read from the neighbouring boxes by the marching x sweep: the
    // step's x ghost fill then runs the ops left (d_ghost_x), not d_ghost[0]
    bool x_fused = false;
    bamrex::GhostOp* d_ghost_x = nullptr;
    int nghost_x = 0, ghost_chunks_x = 0;
    // kernel of each direction's sweep: BAMREX_STAGING_REGISTERS (sweep.cuh),
    // _TMA (per-warp march, sweep_tma.cuh) or _WAVE (block wavefront,
    // sweep_wave.cuh)
    int sweep_kind[3] = { BAMREX_STAGING_REGISTERS, BAMREX_STAGING_REGISTERS, BAMREX_STAGING_REGISTERS };
    bool tma(int d) const { return sweep_kind[d] == BAMREX_STAGING_TMA || sweep_kind[d] == BAMREX_STAGING_WAVE; }
    char* d_tmap[3][2] = {};  // tensor maps of the TMA-staged directions (per parity, one per box)
    int xoff = 0;             // elements between a fab's padded row start and its first element
    bool wave(int d) const { return sweep_kind[d] == BAMREX_STAGING_WAVE; }
    bamrex::GhostOp* d_ghost[3] = { nullptr, nullptr, nullptr };
    int nghost[3] = { 0, 0, 0 };
    int ghost_chunks[3] = { 0, 0, 0 };
    bamrex::PackBox* d_pack = nullptr;
    long long ncells = 0;
    size_t state_bytes = 0;  // bytes of one state buffer
    double* staging = nullptr;  // host copies, allocated on first use
    char* tag_buf = nullptr;    // errorEst tags, allocated on first use
    bamrex::StepScalars* d_scal = nullptr;
    bamrex::StepScalars* h_scal = nullptr;  // pinned
    int cur = 0;
    bool ws_valid = false;

    // flux-register recording by direction (set by the coarse/fine coupling)
    std::vector<bamrex::RegisterTask> reg_tasks[3];

    // halo exchange with other ranks, per direction: ops of the send and
    // receive buffers (device tables, one fab table per parity)
    struct Halo {
        bamrex::PackBox* boxes = nullptr;  // region + buffer cell offset
        bamrex::FabDev* fabs[2] = { nullptr, nullptr };
        int nops = 0;
        long long cells = 0;
    };
    Halo halo_send[3], halo_recv[3];
    char* halo_mem[3] = { nullptr, nullptr, nullptr };
    // the sweep of a direction split in two launches over complementary box
    // sets (bamrex_level_set_sweep_split): part 0 the boxes whose ghost cells
    // in that direction are all local, part 1 the others; per direction,
    // parity and part a box table (item_begin from 0) and its work items
    bamrex::SweepBox* d_split[3][2][2] = {};
    long long split_items[3][2] = {};
    int split_nboxes[3][2] = {};
    char* split_mem[3] = { nullptr, nullptr, nullptr };

    // accounting
    long long launches = 0;
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    std::vector<int> event_dir;
    size_t ev_used = 0;
    double sweep_ms = 0.0;
    long long sweep_launches = 0;
    double dir_ms[3] = { 0, 0, 0 };
    long long dir_launches[3] = { 0, 0, 0 };

    // streams, events and output staging of bamrex_level_step_host
    struct HostStream {
        cudaStream_t h2d = nullptr, d2h = nullptr;
        cudaEvent_t start = nullptr;
        std::vector<cudaEvent_t> in, out, done;  // per slab: unpacked, packed, downloaded
        double* staging_out = nullptr;
        // TMA-staged directions: one box-table entry per (direction, input
        // parity, slab) and its work items, for `slabs` slabs
        bamrex::SweepBox* slab_tab = nullptr;
        std::vector<long long> slab_items;
        int slabs = 0;
    };
    HostStream* hs = nullptr;

    // static rigid body by the ghost-fluid method (bamrex_level_set_body)
    bamrex::BodyState* body = nullptr;

    cudaGraphExec_t graph[2] = { nullptr, nullptr };
    bool run_pending = false;
    int run_start_parity = 0;
    std::string err;

    int set_err(int code);
};

namespace bamrex {

// Uniform bucket grid over the domain for box-intersection queries.
struct BoxIndex {
    int D = 0;
    int lo[3] = { 0, 0, 0 }, bs[3] = { 1, 1, 1 }, nb[3] = { 1, 1, 1 };
    std::vector<std::vector<int>> buckets;
    const std::vector<bamrex_box>* boxes = nullptr;

    void build(const bamrex_box& dom, const std::vector<bamrex_box>& bxs, int D_);
    // indices of the boxes intersecting [rlo, rhi]
    void query(const int* rlo, const int* rhi, std::vector<int>& out) const;
};

int level_launch(bamrex_level* L, cudaError_t e, const char* what);
// The level's buffer for host copies (packed layout, ncells x NC doubles),
// allocated on first use.
int level_staging_ready(bamrex_level* L);
int level_fill(bamrex_level* L, int d, int parity, const StepScalars* scal);
// One sweep of direction d from buffer `parity` into parity ^ 1; reduce_ws:
// also reduce the max wave speed of the output into d_scal->ws_bits.
int level_sweep(bamrex_level* L, int d, int parity, double dt_host, const StepScalars* scal, bool reduce_ws,
                bool allow_timing, int part = -1);
// One split step starting from buffer `parity`; the result lands in
// parity ^ (D & 1).  dt from the host (scal == nullptr) or from the device;
// next_dt (device dt only): end the step with the level's own next dt
// (time, step count, CFL estimate); off inside a hierarchy's coarse step,
// whose levels keep the dt the hierarchy gave them.
int level_step(bamrex_level* L, int parity, double dt_host, StepScalars* scal, bool allow_timing, bool next_dt = true);
// The rigid-body ghost fill of buffer `parity` (gfm.cu); gate: the step
// scalars whose `done` flag skips the work in device-stepped runs.
int body_fill(bamrex_level* L, int parity, const StepScalars* gate);
void body_destroy(bamrex_level* L);
// The rigid body's level-set and GFM-flag fab tables (device), or false
// when the level has no body.
bool body_tag_tables(const bamrex_level* L, const FabDev** ls_tab, const FabDev** flag_tab);

// Face fluxes of direction `dir` recomputed from the sweep input `in` at the
// faces of a register task (face_flux.cu); xsw (direction 0 only, or null):
// the x sweep's box table, whose neighbour fabs stand in for x ghost cells
// the step's x fill skipped.
cudaError_t launch_register_faces(int D, int dir, int method, bool fp32, const Consts& k, const FabDev* in,
                                  const RegisterTask& t, int NC, double dt, double dx_dir, double scale,
                                  const StepScalars* scal, double area1, double area2, cudaStream_t s,
                                  const SweepBox* xsw = nullptr);
// Whether the x sweep of a step reads its x halos from the neighbouring
// boxes (and the step's x ghost fill skips them).
inline bool x_halos_fused(const bamrex_level* L) { return L->x_fused && !L->body; }

// The network's 3x3 convolutions (16 -> 16, 2 -> 16, 16 -> 1) on the
// tcgen05 tensor cores (conv_tc.cu): NCHW FP32 activations, BF16-rounded
// weights [co][ci][9] and biases; widths that are multiples of 128.
// *status is set to BAMREX_ERR_TIMEOUT by a block that gave up waiting
// for its MMAs.
bool conv_tc_supported(int cin, int cout, int H, int W);
cudaError_t launch_conv_tc(int cin, int cout, const float* x, float* y, const float* w, const float* bias, int H, int W,
                           int batch, int relu, int* status, cudaStream_t s);

// The preconditioner network (precnet.cu) on device buffers: its input
// buffer (batch x 2 x ny x nx floats), output buffer (batch x ny x nx),
// size, and a forward pass on stream s.
float* precnet_input(bamrex_precnet* N);
const float* precnet_output(bamrex_precnet* N);
void precnet_size(const bamrex_precnet* N, int* nx, int* ny, int* batch);
int precnet_run(bamrex_precnet* N, cudaStream_t s);

}  // namespace bamrex
