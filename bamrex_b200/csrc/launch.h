// Host-side launch interface between the C ABI / level driver (abi.cu) and
// the kernel translation units.  `fp32` selects the FP32-storage kernels
// (state in float); the per-box reference surface is FP64 only.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace bamrex {

// Ghost-cell copy: dst box cell c takes src box cell s with
// s_d = off[d] + mul[d] * c_d (mul 1: copy / periodic shift, -1: mirror,
// 0: clamp to a boundary layer); components in negmask change sign.
struct GhostOp {
    int dst, src;
    int lo[3], hi[3];
    int off[3], mul[3];
    int negmask;
    int chunk_begin;  // first block-sized chunk of this op (number_ghost_ops)
    long long cell_begin;
};

// Cells per warp of the ghost-fill kernel; every op starts a new chunk, so a
// warp finds its op once instead of every thread searching per cell, and
// small ops (the ghost slabs of narrow boxes) still fill whole warps.
constexpr int kGhostChunk = 32;

__host__ __device__ inline long long ghost_op_cells(const GhostOp& o)
{
    return (long long)(o.hi[0] - o.lo[0] + 1) * (o.hi[1] - o.lo[1] + 1) * (o.hi[2] - o.lo[2] + 1);
}

// Sets cell_begin and chunk_begin of every op; returns the number of chunks.
// On the device the ops are followed by the op index of every chunk
// (ghost_chunk_table), which launch_ghost_fill expects.
inline int number_ghost_ops(std::vector<GhostOp>& ops)
{
    long long cells = 0, chunks = 0;
    for (auto& op : ops) {
        op.cell_begin = cells;
        op.chunk_begin = (int)chunks;
        const long long n = ghost_op_cells(op);
        cells += n;
        chunks += (n + kGhostChunk - 1) / kGhostChunk;
    }
    return (int)chunks;
}

inline std::vector<int> ghost_chunk_table(const std::vector<GhostOp>& ops, int nchunks)
{
    std::vector<int> t((size_t)nchunks);
    for (size_t i = 0; i < ops.size(); ++i) {
        const int end = i + 1 < ops.size() ? ops[i + 1].chunk_begin : nchunks;
        for (int q = ops[i].chunk_begin; q < end; ++q) t[(size_t)q] = (int)i;
    }
    return t;
}

// Bytes of the device copy of ops + chunk table.
inline size_t ghost_table_bytes(size_t nops, int nchunks) { return sizeof(GhostOp) * nops + sizeof(int) * (size_t)nchunks; }

// Valid region of a box in the packed (box-major, SoA) host layout.
struct PackBox {
    int lo[3], hi[3];
    long long cell_begin;
};

struct UpdateArgs {
    int lo[3], hi[3];
    FabDev out, in, flux[3];
    double dtdx[3];
};

int device_sm_count();

// march: run the x sweep (dir 0, D >= 2) as one thread per row instead of
// one warp per row segment; the box table's items must be laid out to match
// (sweep_items).
cudaError_t launch_sweep(int D, int dir, int method, bool fp32, const SweepArgs& a, cudaStream_t s,
                         bool march = false);

// Warps of the sweep kernel that fit on the device at once (for choosing
// segment lengths); 0 for an unsupported combination.
long long sweep_resident_warps(int D, int dir, int method, bool fp32, const Consts& k, bool march = false);

// The fast-path limiter for this configuration (MUSCL-Hancock, energy
// limiting, gamma with 1/z = 7), or -1 for the general kernels.
int fast_limiter(int D, int method, const Consts& k);

// TMA-staged sweeps: the per-warp march (sweep_tma.cuh) and the block
// wavefront (sweep_wave.cuh, wave = true), for the fast path in 2D and 3D.
// An item takes tma_item_lines lines (lane groups of wa along the faster
// transverse direction); the wavefront walks tma_pass_positions positions
// per pass.  encode_sweep_tmap writes the 128-byte tensor map (host memory
// at `out`) of one fab for the kernel of direction dir (row_start: the
// 256-byte aligned start of the fab's first padded row); the launch runs
// over a level's box table (boxes carry tmap, wa, xoff).  Resident units:
// warps (march) or blocks (wavefront).
bool tma_supported(int D, int method, const Consts& k);
int tma_item_lines(bool wave, int dir);
int tma_pass_positions(bool wave, int dir);
cudaError_t encode_sweep_tmap(void* out, bool fp32, int D, int NC, int dir, bool wave, int wa, const void* row_start,
                              long long js, long long ks, long long ns, int nyg, int nzg);
cudaError_t launch_sweep_tma(int D, int dir, bool fp32, int lim, bool wave, const SweepArgs& a, cudaStream_t s);
long long sweep_tma_resident_units(int D, int dir, bool fp32, int lim, bool wave);

cudaError_t launch_ghost_fill(int NC, bool fp32, const GhostOp* ops, int nops, int nchunks, const FabDev* fabs,
                              const StepScalars* scal, cudaStream_t s);

// Packed buffer is always double; fabs are double or float.
// One slab of one box between its fab and the packed layout of the whole box.
cudaError_t launch_pack_slab(int NC, bool fp32, const FabDev& fab, const PackBox& box, const PackBox& slab,
                             double* packed, int to_packed, cudaStream_t s);
cudaError_t launch_pack(int NC, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes,
                        long long total_cells, double* packed, int to_packed, cudaStream_t s);

cudaError_t launch_max_wave_speed(int D, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes,
                                  long long total_cells, const Consts& k, unsigned long long* ws_bits,
                                  const StepScalars* scal, cudaStream_t s);

// Per-box sums of each component over valid cells, accumulated in double in
// a fixed order (one block per box); sums[b * NC + n].
cudaError_t launch_box_sums(int NC, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes, double* sums,
                            cudaStream_t s);

// Time-step bookkeeping on the device (computeInitialDt / computeNewDt).
// mode 0: initial dt from ws_bits at the current time; mode 1: end of a
// step (time += dt, steps++, then the next dt).
cudaError_t launch_step_dt(StepScalars* scal, int D, double dx0, double dx1, double dx2, double cfl, int mode,
                           cudaStream_t s);

cudaError_t launch_flux_LR(int D, int dir, int kind, const int* lo, const int* hi, const FabDev& flux,
                           const FabDev& cL, const FabDev& cR, const Consts& k, double dx, double dt,
                           cudaStream_t s);

cudaError_t launch_sweep_update(int D, int dir, const UpdateArgs& u, cudaStream_t s);

cudaError_t launch_conservative_update(int D, const UpdateArgs& u, cudaStream_t s);

}  // namespace bamrex
