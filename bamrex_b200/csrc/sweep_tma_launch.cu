// Host side of the TMA-staged sweeps: tensor maps of the level fabs
// (cuTensorMapEncodeTiled, reached through the runtime's driver entry point
// so the library needs no link against libcuda), occupancy and launch.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>

#include "common.cuh"
#include "launch.h"
#include "sweep_tma.cuh"
#include "sweep_wave.cuh"

namespace bamrex {

template <typename T>
const void* pick_tma_kernel(int D, int dir, int lim, bool ws, bool wave);
extern template const void* pick_tma_kernel<double>(int, int, int, bool, bool);
extern template const void* pick_tma_kernel<float>(int, int, int, bool, bool);

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

template <int D, int DIR>
int smem_bytes_t(bool fp32, bool wave)
{
    if (wave) return fp32 ? wave_smem_bytes<float, D, DIR>() : wave_smem_bytes<double, D, DIR>();
    return fp32 ? tma_smem_bytes<float, D, DIR>() : tma_smem_bytes<double, D, DIR>();
}

int smem_bytes(int D, int dir, bool fp32, bool wave)
{
    if (D == 2) return dir == 0 ? smem_bytes_t<2, 0>(fp32, wave) : smem_bytes_t<2, 1>(fp32, wave);
    return dir == 0 ? smem_bytes_t<3, 0>(fp32, wave) : dir == 1 ? smem_bytes_t<3, 1>(fp32, wave) : smem_bytes_t<3, 2>(fp32, wave);
}

const void* pick(int D, int dir, bool fp32, int lim, bool ws, bool wave)
{
    return fp32 ? pick_tma_kernel<float>(D, dir, lim, ws, wave) : pick_tma_kernel<double>(D, dir, lim, ws, wave);
}

int blocks_per_sm(const void* fn, int smem, int threads)
{
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache[64];
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto& c = cache[dev & 63];
    auto it = c.find(fn);
    if (it != c.end()) return it->second;
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem) != cudaSuccess || n < 1) n = 1;
    c[fn] = n;
    return n;
}

}  // namespace

bool tma_supported(int D, int method, const Consts& k) { return D >= 2 && fast_limiter(D, method, k) >= 0; }

int tma_item_lines(bool wave, int dir) { return wave ? (dir == 0 ? WaveShape<double, 2, 0>::NL : WaveShape<double, 2, 1>::NL) : 32; }

int tma_pass_positions(bool wave, int dir) { return wave ? (dir == 0 ? WaveShape<double, 2, 0>::PW : WaveShape<double, 2, 1>::PW) : 1; }

cudaError_t encode_sweep_tmap(void* out, bool fp32, int D, int NC, int dir, bool wave, int wa, const void* row_start,
                              long long js, long long ks, long long ns, int nyg, int nzg)
{
    auto fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    const int es = fp32 ? 4 : 8;
    // positions per tile along dir, lines across it
    const int S = wave ? tma_pass_positions(true, dir) : (fp32 ? TmaShape<float, 2, 1>::S : TmaShape<double, 2, 1>::S);
    const int NL = tma_item_lines(wave, dir);
    const int wb = NL / wa;
    cuuint64_t dims[4], strides[3];
    cuuint32_t box[4], estr[4] = { 1, 1, 1, 1 };
    const int rank = D + 1;
    dims[0] = (cuuint64_t)js;
    dims[1] = (cuuint64_t)nyg;
    strides[0] = (cuuint64_t)js * es;
    if (D == 2) {
        dims[2] = (cuuint64_t)NC;
        strides[1] = (cuuint64_t)ns * es;
        if (dir == 0) {
            box[0] = S; box[1] = NL; box[2] = NC;
        } else {
            box[0] = NL; box[1] = S; box[2] = NC;
        }
    } else {
        dims[2] = (cuuint64_t)nzg;
        dims[3] = (cuuint64_t)NC;
        strides[1] = (cuuint64_t)ks * es;
        strides[2] = (cuuint64_t)ns * es;
        if (dir == 0) {
            box[0] = S; box[1] = wa; box[2] = wb; box[3] = NC;
        } else if (dir == 1) {
            box[0] = wa; box[1] = S; box[2] = wb; box[3] = NC;
        } else {
            box[0] = wa; box[1] = wb; box[2] = S; box[3] = NC;
        }
    }
    // the march's x tiles are rows of 32 bytes, one per lane: swizzled so
    // that the 32 lanes' reads spread over the banks
    const bool swz = !wave && dir == 0;
    const CUresult r = fn(reinterpret_cast<CUtensorMap*>(out), fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                          (cuuint32_t)rank, const_cast<void*>(row_start), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, swz ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_NONE,
                          swz ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B : CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_sweep_tma(int D, int dir, bool fp32, int lim, bool wave, const SweepArgs& a, cudaStream_t s)
{
    const void* fn = pick(D, dir, fp32, lim, a.ws_max != nullptr, wave);
    if (!fn || !a.boxes) return cudaErrorInvalidValue;
    if (a.total_items <= 0) return cudaSuccess;
    const int threads = wave ? kWaveThreads : kTmaThreads;
    const int smem = smem_bytes(D, dir, fp32, wave);
    // the march takes an item per warp, the wavefront an item per block
    const long long need = wave ? a.total_items : (a.total_items + kTmaWarps - 1) / kTmaWarps;
    const long long cap = (long long)device_sm_count() * blocks_per_sm(fn, smem, threads);
    const int grid = (int)std::max(1LL, std::min(need, cap));
    void* args[] = { (void*)&a };
    return cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, (size_t)smem, s);
}

long long sweep_tma_resident_units(int D, int dir, bool fp32, int lim, bool wave)
{
    const void* fn = pick(D, dir, fp32, lim, false, wave);
    if (!fn) return 0;
    const int threads = wave ? kWaveThreads : kTmaThreads;
    const long long blocks = (long long)device_sm_count() * blocks_per_sm(fn, smem_bytes(D, dir, fp32, wave), threads);
    return wave ? blocks : blocks * kTmaWarps;
}

}  // namespace bamrex
