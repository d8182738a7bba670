// Kernel selection of the TMA-staged sweeps (per-warp march, block
// wavefront); instantiated once per storage type (sweep_tma_f64.cu,
// sweep_tma_f32.cu) so the two compile in parallel.
#pragma once

#include "sweep_tma.cuh"
#include "sweep_wave.cuh"

namespace bamrex {

// wave: the block wavefront kernel (sweep_wave.cuh) instead of the per-warp
// march (sweep_tma.cuh)
template <typename T>
const void* pick_tma_kernel(int D, int dir, int lim, bool ws, bool wave);

namespace detail {

template <typename T, int D, int DIR, int LIM, bool WS>
const void* tma_kernel_ptr(bool wave)
{
    return wave ? (const void*)sweep_wave_kernel<T, D, DIR, LIM, WS> : (const void*)sweep_tma_kernel<T, D, DIR, LIM, WS>;
}

template <typename T, int D, int DIR>
const void* pick_tma_lim(int lim, bool ws, bool wave)
{
    switch (lim) {
    case LIM_MINBEE: return ws ? tma_kernel_ptr<T, D, DIR, LIM_MINBEE, true>(wave)
                               : tma_kernel_ptr<T, D, DIR, LIM_MINBEE, false>(wave);
    case LIM_VAN_LEER: return ws ? tma_kernel_ptr<T, D, DIR, LIM_VAN_LEER, true>(wave)
                                 : tma_kernel_ptr<T, D, DIR, LIM_VAN_LEER, false>(wave);
    case LIM_VAN_ALBADA: return ws ? tma_kernel_ptr<T, D, DIR, LIM_VAN_ALBADA, true>(wave)
                                   : tma_kernel_ptr<T, D, DIR, LIM_VAN_ALBADA, false>(wave);
    case LIM_SUPERBEE: return ws ? tma_kernel_ptr<T, D, DIR, LIM_SUPERBEE, true>(wave)
                                 : tma_kernel_ptr<T, D, DIR, LIM_SUPERBEE, false>(wave);
    default: return nullptr;
    }
}

}  // namespace detail

template <typename T>
const void* pick_tma_kernel(int D, int dir, int lim, bool ws, bool wave)
{
    using namespace detail;
    if (D == 2 && dir == 0) return pick_tma_lim<T, 2, 0>(lim, ws, wave);
    if (D == 2 && dir == 1) return pick_tma_lim<T, 2, 1>(lim, ws, wave);
    if (D == 3 && dir == 0) return pick_tma_lim<T, 3, 0>(lim, ws, wave);
    if (D == 3 && dir == 1) return pick_tma_lim<T, 3, 1>(lim, ws, wave);
    if (D == 3 && dir == 2) return pick_tma_lim<T, 3, 2>(lim, ws, wave);
    return nullptr;
}

}  // namespace bamrex
