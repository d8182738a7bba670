// Instantiation and launch of the fused sweep kernels (sweep.cuh) for every
// dimension / direction / method of the explicit path.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "launch.h"
#include "sweep.cuh"

namespace bamrex {

namespace {

template <int D, int DIR, int M, int LIM>
const void* kernel_ptr()
{
    if constexpr (DIR == 0) {
        if constexpr (BAMREX_X_SMEM) return (const void*)sweep_x_kernel<D, M, LIM>;
        else return (const void*)sweep_x_shfl_kernel<D, M, LIM>;
    }
    else return (const void*)sweep_s_kernel<D, DIR, M, LIM>;
}

// fast_lim >= 0: the fast MUSCL-Hancock path with that limiter; -1: general
template <int D, int DIR>
const void* pick_method(int method, int fast_lim)
{
    if (method == M_MUSCL && fast_lim >= 0) {
        switch (fast_lim) {
        case LIM_MINBEE: return kernel_ptr<D, DIR, M_MUSCL, LIM_MINBEE>();
        case LIM_VAN_LEER: return kernel_ptr<D, DIR, M_MUSCL, LIM_VAN_LEER>();
        case LIM_VAN_ALBADA: return kernel_ptr<D, DIR, M_MUSCL, LIM_VAN_ALBADA>();
        case LIM_SUPERBEE: return kernel_ptr<D, DIR, M_MUSCL, LIM_SUPERBEE>();
        default: return nullptr;
        }
    }
    switch (method) {
    case M_MUSCL: return kernel_ptr<D, DIR, M_MUSCL, -1>();
    case M_HLLC: return kernel_ptr<D, DIR, M_HLLC, -1>();
    case M_SLIC: return kernel_ptr<D, DIR, M_SLIC, -1>();
    case M_FORCE: return kernel_ptr<D, DIR, M_FORCE, -1>();
    case M_LF: return kernel_ptr<D, DIR, M_LF, -1>();
    default: return nullptr;
    }
}

const void* pick(int D, int dir, int method, int fast_lim)
{
    if (D == 1 && dir == 0) return pick_method<1, 0>(method, fast_lim);
    if (D == 2 && dir == 0) return pick_method<2, 0>(method, fast_lim);
    if (D == 2 && dir == 1) return pick_method<2, 1>(method, fast_lim);
    if (D == 3 && dir == 0) return pick_method<3, 0>(method, fast_lim);
    if (D == 3 && dir == 1) return pick_method<3, 1>(method, fast_lim);
    if (D == 3 && dir == 2) return pick_method<3, 2>(method, fast_lim);
    return nullptr;
}

// Resident blocks per SM of each kernel on the current device.
int blocks_per_sm(const void* fn)
{
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto& c = cache[dev & 63];
    auto it = c.find(fn);
    if (it != c.end()) return it->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, kSweepThreads, 0) != cudaSuccess || n < 1) n = 1;
    c[fn] = n;
    return n;
}

}  // namespace

int fast_limiter(int D, int method, const Consts& k)
{
    if (method != M_MUSCL || k.root_k != 7 || k.uniform_var != D + 1) return -1;
    return k.limiter;
}

cudaError_t launch_sweep(int D, int dir, int method, const SweepArgs& a, cudaStream_t s)
{
    const void* fn = pick(D, dir, method, fast_limiter(D, method, a.k));
    if (!fn) return cudaErrorInvalidValue;
    if (a.total_items <= 0) return cudaSuccess;
    // Persistent grid: every resident warp loops over the items.
    const long long warps_per_block = kSweepThreads / 32;
    const long long need = (a.total_items + warps_per_block - 1) / warps_per_block;
    const long long cap = (long long)device_sm_count() * blocks_per_sm(fn);
    const int grid = (int)std::max(1LL, std::min(need, cap));
    void* args[] = { (void*)&a };
    return cudaLaunchKernel(fn, dim3(grid), dim3(kSweepThreads), args, 0, s);
}

long long sweep_resident_warps(int D, int dir, int method, const Consts& k)
{
    const void* fn = pick(D, dir, method, fast_limiter(D, method, k));
    if (!fn) return 0;
    return (long long)device_sm_count() * blocks_per_sm(fn) * (kSweepThreads / 32);
}

}  // namespace bamrex
