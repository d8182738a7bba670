// Flux-register faces: the interface flux of one sweep recomputed at a list
// of faces (coarse/fine boundary faces) from the sweep's input state, scaled
// by dt and the face area, and stored (CrseInit) or accumulated (FineAdd)
// into a flux register (AMReX FluxRegister as used by AmrLevelAdv::advance,
// Source/AmrLevelAdv_advance.cpp:192-254).  The cell and face stages are the
// sweep kernels' own (Scheme<>), evaluated on the same inputs, so the
// recorded flux is the flux the sweep applied.
#pragma once

#include "common.cuh"
#include "euler.cuh"
#include "level_impl.h"

namespace bamrex {

constexpr int kRegThreads = 128;

template <typename T, int D, int DIR, int METHOD, int LIM>
__global__ void __launch_bounds__(kRegThreads) register_faces_kernel(const FabDev* __restrict__ fabs, const RegisterTask t,
                                                                     const Consts kc, double dt, double dx,
                                                                     double scale, const StepScalars* scal,
                                                                     double area1, double area2,
                                                                     const SweepBox* __restrict__ xsw)
{
    using S = Scheme<T, D, DIR, METHOD, LIM>;
    constexpr int NC = D + 2;
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= t.nslots) return;
    const K<T> k(kc);
    if (scal) {
        // dt on the device: the sweep's own, and the face scale as the host
        // forms it (dt times the other directions' spacings, in order)
        if (scal->done) return;
        dt = scal->dt;
        scale = dt * area1;
        scale = scale * area2;
    }
    // the sweep kernels' step factors (sweep.cuh, step_factors)
    const T hdtdx = (T)(0.5 * dt / dx);
    const T half_dx_dt = (T)(0.5 * dx / dt);
    const T dt_2dx = (T)(dt / (2 * dx));

    double acc[NC];
#pragma unroll
    for (int n = 0; n < NC; ++n) acc[n] = t.mode == 1 ? t.reg[(long long)n * t.nslots + slot] : 0.0;

    for (int f = 0; f < t.per_slot; ++f) {
        const FaceRec r = t.faces[(long long)slot * t.per_slot + f];
        const FabDev fb = fabs[r.box];
        const long long s = DIR == 0 ? 1 : (DIR == 1 ? fb.js : fb.ks);
        const T* p = fb.ptr<T>() + (long long)(r.i - fb.b0) + (long long)(r.j - fb.b1) * fb.js +
                     (long long)(r.k - fb.b2) * fb.ks;
        T Um2[NC], Um1[NC], U0[NC], Up1[NC];
        if (DIR == 0 && xsw) {
            // x halos read where the marching x sweep reads them: from the
            // neighbouring box that holds them (the step's x ghost fill
            // skips those ghost cells)
            const SweepBox& B = xsw[r.box];
            auto ld = [&](int x, T (&u)[NC]) {
                const FabDev* g = &fb;
                if (x < B.lo[0] && B.xnb[0].p) g = &B.xnb[0];
                else if (x > B.hi[0] && B.xnb[1].p) g = &B.xnb[1];
                const T* q = g->ptr<T>() + (long long)(x - g->b0) + (long long)(r.j - g->b1) * g->js +
                             (long long)(r.k - g->b2) * g->ks;
#pragma unroll
                for (int n = 0; n < NC; ++n) u[n] = q[n * g->ns];
            };
            ld(r.i - 2, Um2);
            ld(r.i - 1, Um1);
            ld(r.i, U0);
            ld(r.i + 1, Up1);
        } else {
#pragma unroll
            for (int n = 0; n < NC; ++n) {
                Um2[n] = p[n * fb.ns - 2 * s];
                Um1[n] = p[n * fb.ns - s];
                U0[n] = p[n * fb.ns];
                Up1[n] = p[n * fb.ns + s];
            }
        }
        T ULa[NC], URa[NC], ULb[NC], URb[NC], F[NC];
        S::cell(Um2, Um1, U0, k, hdtdx, ULa, URa);  // cell left of the face
        S::cell(Um1, U0, Up1, k, hdtdx, ULb, URb);  // cell right of the face
        S::face(URa, ULb, k, half_dx_dt, dt_2dx, F);
#pragma unroll
        for (int n = 0; n < NC; ++n) {
            const double v = (double)F[n] * scale;  // fluxes[d].mult(scaleFactor)
            if (t.mode == 0) acc[n] = -v;           // CrseInit(..., -1)
            else acc[n] = acc[n] + v;               // FineAdd(..., +1)
        }
    }
#pragma unroll
    for (int n = 0; n < NC; ++n) t.reg[(long long)n * t.nslots + slot] = acc[n];
}

template <typename T>
const void* pick_register_kernel(int D, int dir, int method, int fast_lim);

namespace detail {

template <typename T, int D, int DIR>
const void* pick_reg_method(int method, int fast_lim)
{
    if (method == M_MUSCL && fast_lim >= 0) {
        switch (fast_lim) {
        case LIM_MINBEE: return (const void*)register_faces_kernel<T, D, DIR, M_MUSCL, LIM_MINBEE>;
        case LIM_VAN_LEER: return (const void*)register_faces_kernel<T, D, DIR, M_MUSCL, LIM_VAN_LEER>;
        case LIM_VAN_ALBADA: return (const void*)register_faces_kernel<T, D, DIR, M_MUSCL, LIM_VAN_ALBADA>;
        case LIM_SUPERBEE: return (const void*)register_faces_kernel<T, D, DIR, M_MUSCL, LIM_SUPERBEE>;
        default: return nullptr;
        }
    }
    switch (method) {
    case M_MUSCL: return (const void*)register_faces_kernel<T, D, DIR, M_MUSCL, -1>;
    case M_HLLC: return (const void*)register_faces_kernel<T, D, DIR, M_HLLC, -1>;
    case M_SLIC: return (const void*)register_faces_kernel<T, D, DIR, M_SLIC, -1>;
    case M_FORCE: return (const void*)register_faces_kernel<T, D, DIR, M_FORCE, -1>;
    case M_LF: return (const void*)register_faces_kernel<T, D, DIR, M_LF, -1>;
    default: return nullptr;
    }
}

}  // namespace detail

template <typename T>
const void* pick_register_kernel(int D, int dir, int method, int fast_lim)
{
    using namespace detail;
    if (D == 1 && dir == 0) return pick_reg_method<T, 1, 0>(method, fast_lim);
    if (D == 2 && dir == 0) return pick_reg_method<T, 2, 0>(method, fast_lim);
    if (D == 2 && dir == 1) return pick_reg_method<T, 2, 1>(method, fast_lim);
    if (D == 3 && dir == 0) return pick_reg_method<T, 3, 0>(method, fast_lim);
    if (D == 3 && dir == 1) return pick_reg_method<T, 3, 1>(method, fast_lim);
    if (D == 3 && dir == 2) return pick_reg_method<T, 3, 2>(method, fast_lim);
    return nullptr;
}

}  // namespace bamrex
