// Kernel selection for the sweep launches; instantiated once per storage
// type (sweep_f64.cu, sweep_f32.cu) so the two compile in parallel.
#pragma once

#include "sweep.cuh"

namespace bamrex {

// march: the x sweep as one thread per row (D >= 2); ignored for y / z.
template <typename T>
const void* pick_sweep_kernel(int D, int dir, int method, int fast_lim, bool march);

namespace detail {

template <typename T, int D, int DIR, bool MARCH, int M, int LIM>
const void* kernel_ptr()
{
    if constexpr (DIR == 0 && !MARCH) return (const void*)sweep_x_kernel<T, D, M, LIM>;
    else return (const void*)sweep_s_kernel<T, D, DIR, M, LIM>;
}

// fast_lim >= 0: the fast MUSCL-Hancock path with that limiter; -1: general
template <typename T, int D, int DIR, bool MARCH>
const void* pick_method(int method, int fast_lim)
{
    if (method == M_MUSCL && fast_lim >= 0) {
        switch (fast_lim) {
        case LIM_MINBEE: return kernel_ptr<T, D, DIR, MARCH, M_MUSCL, LIM_MINBEE>();
        case LIM_VAN_LEER: return kernel_ptr<T, D, DIR, MARCH, M_MUSCL, LIM_VAN_LEER>();
        case LIM_VAN_ALBADA: return kernel_ptr<T, D, DIR, MARCH, M_MUSCL, LIM_VAN_ALBADA>();
        case LIM_SUPERBEE: return kernel_ptr<T, D, DIR, MARCH, M_MUSCL, LIM_SUPERBEE>();
        default: return nullptr;
        }
    }
    switch (method) {
    case M_MUSCL: return kernel_ptr<T, D, DIR, MARCH, M_MUSCL, -1>();
    case M_HLLC: return kernel_ptr<T, D, DIR, MARCH, M_HLLC, -1>();
    case M_SLIC: return kernel_ptr<T, D, DIR, MARCH, M_SLIC, -1>();
    case M_FORCE: return kernel_ptr<T, D, DIR, MARCH, M_FORCE, -1>();
    case M_LF: return kernel_ptr<T, D, DIR, MARCH, M_LF, -1>();
    default: return nullptr;
    }
}

}  // namespace detail

template <typename T>
const void* pick_sweep_kernel(int D, int dir, int method, int fast_lim, bool march)
{
    using namespace detail;
    if (D == 1 && dir == 0) return pick_method<T, 1, 0, false>(method, fast_lim);
    if (D == 2 && dir == 0)
        return march ? pick_method<T, 2, 0, true>(method, fast_lim) : pick_method<T, 2, 0, false>(method, fast_lim);
    if (D == 2 && dir == 1) return pick_method<T, 2, 1, false>(method, fast_lim);
    if (D == 3 && dir == 0)
        return march ? pick_method<T, 3, 0, true>(method, fast_lim) : pick_method<T, 3, 0, false>(method, fast_lim);
    if (D == 3 && dir == 1) return pick_method<T, 3, 1, false>(method, fast_lim);
    if (D == 3 && dir == 2) return pick_method<T, 3, 2, false>(method, fast_lim);
    return nullptr;
}

}  // namespace bamrex
