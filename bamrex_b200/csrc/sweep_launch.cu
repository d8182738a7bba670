// Launch of the fused sweep kernels: kernel choice (storage type, fast or
// general path), persistent grid size from the occupancy of the chosen
// kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "common.cuh"
#include "euler.cuh"
#include "launch.h"
#include "sweep_stage.h"

namespace bamrex {

template <typename T>
const void* pick_sweep_kernel(int D, int dir, int method, int fast_lim, bool march);
extern template const void* pick_sweep_kernel<double>(int, int, int, int, bool);
extern template const void* pick_sweep_kernel<float>(int, int, int, int, bool);

constexpr int kLaunchThreads = 128;  // kSweepThreads of sweep.cuh

namespace {

const void* pick(int D, int dir, int method, bool fp32, int fast_lim, bool march)
{
    return fp32 ? pick_sweep_kernel<float>(D, dir, method, fast_lim, march)
                : pick_sweep_kernel<double>(D, dir, method, fast_lim, march);
}

// Resident blocks per SM of each kernel on the current device (with its
// dynamic shared memory, which is raised above the default limit once).
int blocks_per_sm(const void* fn, int smem)
{
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto& c = cache[dev & 63];
    auto it = c.find(fn);
    if (it != c.end()) return it->second;
    if (smem > 48 * 1024) cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kLaunchThreads, smem) != cudaSuccess || n < 1) n = 1;
    c[fn] = n;
    return n;
}

}  // namespace

int fast_limiter(int D, int method, const Consts& k)
{
    if (method != M_MUSCL || k.root_k != 7 || k.uniform_var != D + 1) return -1;
    return k.limiter;
}

cudaError_t launch_sweep(int D, int dir, int method, bool fp32, const SweepArgs& a, cudaStream_t s, bool march)
{
    march = march && dir == 0 && D >= 2;
    const void* fn = pick(D, dir, method, fp32, fast_limiter(D, method, a.k), march);
    if (!fn) return cudaErrorInvalidValue;
    if (a.total_items <= 0) return cudaSuccess;
    const int smem = march ? march_x_smem_bytes(D, fp32) : 0;
    // Persistent grid: every resident warp loops over the items.
    const long long warps_per_block = kLaunchThreads / 32;
    const long long need = (a.total_items + warps_per_block - 1) / warps_per_block;
    const long long cap = (long long)device_sm_count() * blocks_per_sm(fn, smem);
    const int grid = (int)std::max(1LL, std::min(need, cap));
    void* args[] = { (void*)&a };
    return cudaLaunchKernel(fn, dim3(grid), dim3(kLaunchThreads), args, (size_t)smem, s);
}

long long sweep_resident_warps(int D, int dir, int method, bool fp32, const Consts& k, bool march)
{
    march = march && dir == 0 && D >= 2;
    const void* fn = pick(D, dir, method, fp32, fast_limiter(D, method, k), march);
    if (!fn) return 0;
    return (long long)device_sm_count() * blocks_per_sm(fn, march ? march_x_smem_bytes(D, fp32) : 0) *
           (kLaunchThreads / 32);
}

}  // namespace bamrex
