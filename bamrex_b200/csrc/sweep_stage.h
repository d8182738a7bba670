// Shared-memory staging of the marching x sweep (sweep.cuh): each warp moves
// its 32 rows through a [component][row][kStageW] buffer with row pitch
// kStagePitch (which keeps the lanes' 64-bit reads of one column free of
// bank conflicts), so global loads and stores stay coalesced (8 rows x 4
// cells per instruction) while each lane marches its own row.  One input and
// one output buffer per warp.
#pragma once

namespace bamrex {

constexpr int kStageW = 4;
constexpr int kStagePitch = 5;
constexpr int kStageBlockThreads = 128;  // threads per block of the sweep kernels

template <typename T, int NC>
constexpr int stage_elems_per_warp() { return 2 * NC * 32 * kStagePitch; }

// Dynamic shared memory of one block of the marching x sweep.
inline int march_x_smem_bytes(int D, bool fp32)
{
    return (kStageBlockThreads / 32) * 2 * (D + 2) * 32 * kStagePitch * (fp32 ? 4 : 8);
}

}  // namespace bamrex
