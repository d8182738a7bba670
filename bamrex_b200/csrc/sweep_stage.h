// Shared-memory staging of the marching x sweep (sweep.cuh): each warp moves
// its 32 rows through [component][row][kStageW] buffers, so global loads and
// stores stay coalesced (8 rows x 4 cells per instruction) while each lane
// marches its own row.  The cell of a row sits at a column rotated by
// row / 4 (stage_slot), which keeps both access patterns free of bank
// conflicts: a lane reading its own row at one column, and 8 rows x 4 cells
// written or read together.  Two input buffers per warp (the chunk being
// read and the next one, copied asynchronously with cp.async while the
// current one is processed) and one output buffer.
#pragma once

namespace bamrex {

constexpr int kStageW = 4;
constexpr int kStageBlockThreads = 128;  // threads per block of the sweep kernels

template <typename T, int NC>
constexpr int stage_elems_per_warp() { return 3 * NC * 32 * kStageW; }

// Element of row `row` (component-major rows), column c of a buffer.
__host__ __device__ constexpr int stage_slot(int row, int c) { return row * kStageW + ((c + (row >> 2)) & (kStageW - 1)); }

// Dynamic shared memory of one block of the marching x sweep: the buffers,
// then per warp the offsets of its 32 rows in the input and output fabs and
// in the fabs of the x neighbours below and above.
inline int march_x_smem_bytes(int D, bool fp32)
{
    return (kStageBlockThreads / 32) * (3 * (D + 2) * 32 * kStageW * (fp32 ? 4 : 8) + 128 * 8);
}

#ifdef __CUDACC__
// One element copied global -> shared without passing through registers
// (PTX cp.async, cached at all levels); visible after cp_async_wait_all and
// a warp barrier.
__device__ __forceinline__ void cp_async_elem(double* dst, const double* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(float* dst, const float* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }
#endif

}  // namespace bamrex
