// The first-order IMEX step on the device: one SP111 stage of
// advance_imex_rk (Source/IMEX/IMEX_RK.cpp:23-86; a_11 = b_1 = 1, so the
// stage input is the step input and the summed flux is the stage flux) with
// the linearised pressure equation of compute_flux_imex_o1
// (Source/IMEX/IMEX_O1.cpp:19-176):
//   1. explicit advection of the state by the Rusanov flux, or by the
//      MUSCL-Rusanov flux with its local half step (advance_rusanov_adv,
//      advance_MUSCL_rusanov_adv, Source/IMEX/IMEX_Fluxes.cpp:11-323), on the
//      valid box grown by one;
//   2. enthalpy (grown box), kinetic energy, velocity and the pressure source
//      (compute_enthalpy, compute_ke, compute_velocity,
//      pressure_source_vector, IMEX_O1.cpp:178-290, 420-453);
//   3. the pressure equation (A = 1, B = dt^2, C = -eps dt / 2 with the split
//      kinetic energy, a = eps / (gamma - 1), b = the enthalpy averaged to
//      faces; setup_pressure_op / solve_pressure, IMEX_O1.cpp:570-640)
//      solved by the library's Helmholtz operator (BiCGStab + multigrid, or
//      FGMRES with the learned preconditioner);
//   4. the momentum and energy fluxes (update_momentum_flux,
//      update_energy_flux, IMEX_O1.cpp:480-556) and the conservative update
//      (Source/Fluxes/Update.H:99-130).
// The domain is one box; ghost cells come from the boundary rules (periodic
// images, first-order extrapolation, even reflection with the normal
// momentum negated), filled one direction after the other.  Every kernel is
// HBM-bound and elementwise or a short stencil.  This file is compiled with
// -fmad=false: each operation rounds as written, so a CPU restatement
// reproduces everything but the solve bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>

#include "bamrex_cuda.h"
#include "level_impl.h"

using namespace bamrex;

namespace {

constexpr int kThreads = 256;

// A dense box of cells [lo, lo + N) in valid-cell coordinates, i fastest.
struct Grid3 {
    int lo[3], N[3];
    __host__ __device__ long long size() const { return (long long)N[0] * N[1] * N[2]; }
    __device__ __forceinline__ long long at(int i, int j, int k) const
    {
        return (long long)(i - lo[0]) + (long long)N[0] * ((long long)(j - lo[1]) + (long long)N[1] * (k - lo[2]));
    }
    __device__ __forceinline__ void cell(long long t, int& i, int& j, int& k) const
    {
        const int tt = (int)t;  // boxes are checked to hold fewer than 2^31 cells
        const int row = tt / N[0];
        i = lo[0] + (tt - row * N[0]);
        const int pl = row / N[1];
        j = lo[1] + (row - pl * N[1]);
        k = lo[2] + pl;
    }
};

Grid3 grown(int D, const int* n, int g, int face_dir = -1)
{
    Grid3 r;
    for (int d = 0; d < 3; ++d) {
        const int gd = d < D ? g : 0;
        r.lo[d] = -gd;
        r.N[d] = n[d] + 2 * gd + (d == face_dir ? 1 : 0);
    }
    return r;
}

struct IK {
    int D, NC;
    int n[3];
    double adia, eps;
    double dtdx[3];    // dt / dx       (the explicit advection)
    double hdtdx[3];   // 0.5 dt idx    (pressure source)
    double hdtdxe[3];  // hdtdx / eps   (energy flux)
    double dtidx[3];   // dt idx        (conservative update)
    double hadv[3];    // 0.5 (dt / dx) (local half step of MUSCL-Rusanov)
    double heps;       // 0.5 / eps
};

int grid_for(long long work)
{
    const long long want = (work + kThreads - 1) / kThreads;
    return (int)std::max(1LL, std::min(want, (long long)device_sm_count() * 8));
}

#define GRID_LOOP(t, total) \
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < (total); t += (long long)gridDim.x * blockDim.x)

// ------------------------------------------------------------ ghost cells
// Fill the ghost layers of direction d of an array on grid g (ncomp
// components of stride cs): over the padded range of the directions before
// d and the valid range of those after it.
__global__ void fill_kernel(double* __restrict__ a, Grid3 g, int ncomp, long long cs, int d, int nvalid, int G,
                            int bc_lo, int bc_hi, int vector_comp)
{
    int e1 = (d == 0) ? 1 : 0, e2 = (d == 2) ? 1 : 2;
    auto ext = [&](int e, int& lo, int& cnt) {
        if (e < d) {
            lo = g.lo[e];
            cnt = g.N[e];
        } else {
            lo = 0;
            cnt = g.N[e] + 2 * g.lo[e];  // the valid extent
        }
    };
    int lo1, c1, lo2, c2;
    ext(e1, lo1, c1);
    ext(e2, lo2, c2);
    const long long total = 2LL * G * c1 * c2;
    GRID_LOOP(t, total)
    {
        long long r = t;
        const int a1 = (int)(r % c1);
        r /= c1;
        const int a2 = (int)(r % c2);
        r /= c2;
        const int layer = (int)(r % G);
        const int side = (int)(r / G);
        const int bc = side ? bc_hi : bc_lo;
        const int gc = side ? nvalid + layer : -1 - layer;  // ghost coordinate
        int src;
        bool negate = false;
        if (bc == BAMREX_BC_PERIODIC) src = side ? layer : nvalid - 1 - layer;
        else if (bc == BAMREX_BC_REFLECTIVE) {
            src = side ? nvalid - 1 - layer : layer;
            negate = true;
        } else src = side ? nvalid - 1 : 0;
        int q[3], s[3];
        q[d] = gc;
        s[d] = src;
        q[e1] = s[e1] = lo1 + a1;
        q[e2] = s[e2] = lo2 + a2;
        const long long di = g.at(q[0], q[1], q[2]), si = g.at(s[0], s[1], s[2]);
        for (int c = 0; c < ncomp; ++c) {
            const double v = a[si + c * cs];
            a[di + c * cs] = (negate && c == vector_comp) ? -v : v;
        }
    }
}

// ------------------------------------------------------------ advection
template <int D>
__device__ __forceinline__ double kinetic_energy(const double (&u)[D + 2], double eps)
{
    double m2 = u[1] * u[1];
#pragma unroll
    for (int d = 1; d < D; ++d) m2 = m2 + u[1 + d] * u[1 + d];
    return eps * m2 / (2 * u[0]);
}

// adv_flux<dir> (Source/IMEX_K/euler_K.H)
template <int D>
__device__ __forceinline__ void adv_flux(const double (&u)[D + 2], int dir, double eps, double (&f)[D + 2])
{
    const double ud = u[1 + dir] / u[0];
    f[0] = u[1 + dir];
#pragma unroll
    for (int n = 1; n < D + 1; ++n) f[n] = u[n] * ud;
    f[1 + D] = ud * kinetic_energy<D>(u, eps);
}

template <int D>
__device__ __forceinline__ void load(const double* __restrict__ a, long long i, long long cs, double (&u)[D + 2])
{
#pragma unroll
    for (int n = 0; n < D + 2; ++n) u[n] = a[i + n * cs];
}

// Rusanov flux on face (L, R) with physical fluxes FL, FR
template <int D>
__device__ __forceinline__ void rusanov(const double (&L)[D + 2], const double (&R)[D + 2], int d, double eps,
                                        double (&F)[D + 2])
{
    double FL[D + 2], FR[D + 2];
    adv_flux<D>(L, d, eps, FL);
    adv_flux<D>(R, d, eps, FR);
    const double a = fabs(R[1 + d] / R[0]), b = fabs(L[1 + d] / L[0]);
    const double umax = a > b ? a : b;
#pragma unroll
    for (int n = 0; n < D + 2; ++n) F[n] = 0.5 * ((FR[n] + FL[n]) - umax * (R[n] - L[n]));
}

// Rusanov fluxes on the faces of direction d of the valid box grown by one
template <int D>
__global__ void rusanov_faces_kernel(const double* __restrict__ U, Grid3 gU, double* __restrict__ AF, Grid3 gF, int d,
                                     double eps)
{
    GRID_LOOP(t, gF.size())
    {
        int i, j, k;
        gF.cell(t, i, j, k);  // face f = (i, j, k) along d: between cells f - e_d and f
        int q[3] = { i, j, k };
        q[d] -= 1;
        double L[D + 2], R[D + 2], F[D + 2];
        load<D>(U, gU.at(i, j, k), gU.size(), R);
        load<D>(U, gU.at(q[0], q[1], q[2]), gU.size(), L);
        rusanov<D>(L, R, d, eps, F);
#pragma unroll
        for (int n = 0; n < D + 2; ++n) AF[t + n * gF.size()] = F[n];
    }
}

__device__ __forceinline__ double minmod(double a, double b)
{
    return (a > 0 && b > 0) ? fmin(a, b) : ((a < 0 && b < 0) ? fmax(a, b) : 0.0);
}

// MUSCL-Rusanov reconstruction on the valid box grown by two, with the local
// half step when local_step (SP111): SL[d] = U - h - hadv (F(U+h) - F(U-h)),
// SR[d] likewise
template <int D>
__global__ void muscl_states_kernel(const double* __restrict__ U, Grid3 gU, double* __restrict__ SL,
                                    double* __restrict__ SR, Grid3 g2, IK c, int local_step)
{
    const long long n2 = g2.size();
    GRID_LOOP(t, n2)
    {
        int i, j, k;
        g2.cell(t, i, j, k);
        double C[D + 2];
        load<D>(U, gU.at(i, j, k), gU.size(), C);
#pragma unroll
        for (int d = 0; d < D; ++d) {
            int m[3] = { i, j, k }, p[3] = { i, j, k };
            m[d] -= 1;
            p[d] += 1;
            double Um[D + 2], Up[D + 2], sl[D + 2], sr[D + 2];
            load<D>(U, gU.at(m[0], m[1], m[2]), gU.size(), Um);
            load<D>(U, gU.at(p[0], p[1], p[2]), gU.size(), Up);
#pragma unroll
            for (int n = 0; n < D + 2; ++n) {
                const double hdelta = 0.5 * minmod(C[n] - Um[n], Up[n] - C[n]);
                sl[n] = C[n] - hdelta;
                sr[n] = C[n] + hdelta;
            }
            const long long base = (long long)d * (D + 2) * n2 + t;
            if (local_step) {
                double fl[D + 2], fr[D + 2];
                adv_flux<D>(sl, d, c.eps, fl);
                adv_flux<D>(sr, d, c.eps, fr);
#pragma unroll
                for (int n = 0; n < D + 2; ++n) {
                    const double upd = c.hadv[d] * (fr[n] - fl[n]);
                    SL[base + n * n2] = sl[n] - upd;
                    SR[base + n * n2] = sr[n] - upd;
                }
            } else {
#pragma unroll
                for (int n = 0; n < D + 2; ++n) {
                    SL[base + n * n2] = sl[n];
                    SR[base + n * n2] = sr[n];
                }
            }
        }
    }
}

// MUSCL-Rusanov fluxes on the faces of direction d of the grown box: left
// state of cell f against the right state of cell f - e_d
template <int D>
__global__ void muscl_faces_kernel(const double* __restrict__ SL, const double* __restrict__ SR, Grid3 g2,
                                   double* __restrict__ AF, Grid3 gF, int d, double eps)
{
    const long long n2 = g2.size();
    GRID_LOOP(t, gF.size())
    {
        int i, j, k;
        gF.cell(t, i, j, k);
        int q[3] = { i, j, k };
        q[d] -= 1;
        const long long base = (long long)d * (D + 2) * n2;
        double Li[D + 2], Rm[D + 2];
        load<D>(SL + base, g2.at(i, j, k), n2, Li);
        load<D>(SR + base, g2.at(q[0], q[1], q[2]), n2, Rm);
        double FL[D + 2], FR[D + 2];
        adv_flux<D>(Li, d, eps, FL);
        adv_flux<D>(Rm, d, eps, FR);
        const double a = fabs(Li[1 + d] / Li[0]), b = fabs(Rm[1 + d] / Rm[0]);
        const double umax = a > b ? a : b;
#pragma unroll
        for (int n = 0; n < D + 2; ++n) AF[t + n * gF.size()] = 0.5 * ((FL[n] + FR[n]) - umax * (Li[n] - Rm[n]));
    }
}

// explicit update on the grown box: Uex = U - (sum_d dt/dx_d (F(f+1) - F(f)))
// with U the state to update (the implicit-stage state)
template <int D>
__global__ void explicit_update_kernel(const double* __restrict__ U, Grid3 gU, const double* __restrict__ AF0,
                                       const double* __restrict__ AF1, const double* __restrict__ AF2, Grid3 gF0,
                                       Grid3 gF1, Grid3 gF2, double* __restrict__ Uex, Grid3 g1, IK c)
{
    const double* AF[3] = { AF0, AF1, AF2 };
    const Grid3 gF[3] = { gF0, gF1, gF2 };
    GRID_LOOP(t, g1.size())
    {
        int i, j, k;
        g1.cell(t, i, j, k);
        const long long iu = gU.at(i, j, k);
#pragma unroll
        for (int n = 0; n < D + 2; ++n) {
            double acc = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                int p[3] = { i, j, k };
                p[d] += 1;
                const long long fs = gF[d].size();
                const double term = c.dtdx[d] * (AF[d][gF[d].at(p[0], p[1], p[2]) + n * fs] - AF[d][gF[d].at(i, j, k) + n * fs]);
                acc = d == 0 ? term : acc + term;
            }
            Uex[t + n * g1.size()] = U[iu + n * gU.size()] - acc;
        }
    }
}

// compute_enthalpy on the grown box; the conservative methods also set the
// pressure (the solve's initial guess) from the explicitly updated state
template <int D>
__global__ void enthalpy_kernel(const double* __restrict__ U, Grid3 gU, const double* __restrict__ Uex, Grid3 g1,
                                const double* __restrict__ pg, double* __restrict__ enth, double* __restrict__ p,
                                Grid3 gV, int method, IK c)
{
    GRID_LOOP(t, g1.size())
    {
        int i, j, k;
        g1.cell(t, i, j, k);
        double ex[D + 2];
        load<D>(Uex, t, g1.size(), ex);
        if (method == BAMREX_IMEX_ENTH_REUSE_PRESSURE) {
            enth[t] = pg[t] * c.adia / ((c.adia - 1) * ex[0]);
        } else {
            double s[D + 2];
            if (method == BAMREX_IMEX_ENTH_CONSERVATIVE) load<D>(U, gU.at(i, j, k), gU.size(), s);
            else {
#pragma unroll
                for (int n = 0; n < D + 2; ++n) s[n] = ex[n];
            }
            enth[t] = c.adia * (s[1 + D] - kinetic_energy<D>(s, c.eps)) / ex[0];
            const bool valid = i >= 0 && i < c.n[0] && j >= 0 && j < c.n[1] && k >= 0 && k < c.n[2];
            if (valid) p[gV.at(i, j, k)] = (c.adia - 1) * (ex[1 + D] - kinetic_energy<D>(ex, c.eps));
        }
    }
}

// compute_ke, compute_velocity and pressure_source_vector on the valid box
template <int D>
__global__ void source_kernel(const double* __restrict__ U, Grid3 gU, const double* __restrict__ Uex, Grid3 g1,
                              const double* __restrict__ enth, double* __restrict__ ke, double* __restrict__ vel,
                              double* __restrict__ rhs, Grid3 gV, int ke_method, IK c)
{
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        double u[D + 2], ex[D + 2];
        load<D>(U, gU.at(i, j, k), gU.size(), u);
        const long long e1 = g1.at(i, j, k);
        load<D>(Uex, e1, g1.size(), ex);
        double kv;
        if (ke_method == BAMREX_IMEX_KE_CONSERVATIVE) kv = kinetic_energy<D>(u, c.eps);
        else if (ke_method == BAMREX_IMEX_KE_EX) kv = kinetic_energy<D>(ex, c.eps);
        else {
            double dot = u[1] * ex[1];
#pragma unroll
            for (int d = 1; d < D; ++d) dot = dot + u[1 + d] * ex[1 + d];
            kv = 0.5 * c.eps * dot / u[0];
        }
        ke[t] = kv;
        if (vel) {
#pragma unroll
            for (int d = 0; d < D; ++d) vel[t + d * gV.size()] = u[1 + d] / u[0];
        }
        double acc = 0.0;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            int p[3] = { i, j, k }, m[3] = { i, j, k };
            p[d] += 1;
            m[d] -= 1;
            const long long ip = g1.at(p[0], p[1], p[2]), im = g1.at(m[0], m[1], m[2]);
            const double term = c.hdtdx[d] * (enth[ip] * Uex[ip + (1 + d) * g1.size()] - enth[im] * Uex[im + (1 + d) * g1.size()]);
            acc = d == 0 ? term : acc + term;
        }
        rhs[t] = c.eps * (ex[1 + D] - kv - acc);
    }
}

// average_cellcenter_to_face of the enthalpy on the valid faces of direction d
__global__ void bface_kernel(const double* __restrict__ enth, Grid3 g1, double* __restrict__ b, Grid3 gF, int d)
{
    GRID_LOOP(t, gF.size())
    {
        int i, j, k;
        gF.cell(t, i, j, k);
        int m[3] = { i, j, k };
        m[d] -= 1;
        b[t] = 0.5 * (enth[g1.at(m[0], m[1], m[2])] + enth[g1.at(i, j, k)]);
    }
}

// valid dense array -> valid part of a grown array
__global__ void to_grown_kernel(const double* __restrict__ v, Grid3 gV, double* __restrict__ a, Grid3 g, int ncomp)
{
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        const long long q = g.at(i, j, k);
        for (int c = 0; c < ncomp; ++c) a[q + c * g.size()] = v[t + c * gV.size()];
    }
}

__global__ void from_grown_kernel(const double* __restrict__ a, Grid3 g, double* __restrict__ v, Grid3 gV, int ncomp)
{
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        const long long q = g.at(i, j, k);
        for (int c = 0; c < ncomp; ++c) v[t + c * gV.size()] = a[q + c * g.size()];
    }
}

// update_momentum_flux + update_energy_flux on the valid faces of direction d
template <int D>
__global__ void flux_kernel(const double* __restrict__ AF, Grid3 gA, const double* __restrict__ Uex,
                            const double* __restrict__ enth, const double* __restrict__ pg, Grid3 g1,
                            double* __restrict__ FL, Grid3 gF, int d, IK c)
{
    GRID_LOOP(t, gF.size())
    {
        int i, j, k;
        gF.cell(t, i, j, k);
        int m[3] = { i, j, k };
        m[d] -= 1;
        const long long ia = gA.at(i, j, k);
        double F[D + 2];
#pragma unroll
        for (int n = 0; n < D + 2; ++n) F[n] = AF[ia + n * gA.size()];
        const long long ic = g1.at(i, j, k), im = g1.at(m[0], m[1], m[2]);
        const double pi = pg[ic], pm = pg[im], hi = enth[ic], hm = enth[im];
        const double mi = Uex[ic + (1 + d) * g1.size()], mm = Uex[im + (1 + d) * g1.size()];
        F[1 + d] += c.heps * (pi + pm);
        F[1 + D] += 0.5 * (hi * mi + hm * mm) - c.hdtdxe[d] * ((hi + hm) * (pi - pm));
#pragma unroll
        for (int n = 0; n < D + 2; ++n) FL[t + n * gF.size()] = F[n];
    }
}

// conservative update of the valid cells in place
template <int D>
__global__ void update_kernel(double* __restrict__ U, Grid3 gU, const double* __restrict__ F0,
                              const double* __restrict__ F1, const double* __restrict__ F2, Grid3 gF0, Grid3 gF1,
                              Grid3 gF2, Grid3 gV, IK c)
{
    const double* F[3] = { F0, F1, F2 };
    const Grid3 gF[3] = { gF0, gF1, gF2 };
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        const long long iu = gU.at(i, j, k);
#pragma unroll
        for (int n = 0; n < D + 2; ++n) {
            double v = U[iu + n * gU.size()];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                int p[3] = { i, j, k };
                p[d] += 1;
                const long long fs = gF[d].size();
                v = v - c.dtidx[d] * (F[d][gF[d].at(p[0], p[1], p[2]) + n * fs] - F[d][gF[d].at(i, j, k) + n * fs]);
            }
            U[iu + n * gU.size()] = v;
        }
    }
}

// The two stage states (conservative_update with two outputs,
// Source/Fluxes/Update.H:216-300): out = in - sum over the earlier stages i
// of (c_i,x dFx_i + c_i,y dFy_i [+ c_i,z dFz_i]), with c = a_i dt idx for the
// implicit (1) and explicit (2) rows of the tableau.
struct StageArgs {
    const double* F[3][3];  // [stage][direction]
    Grid3 gF[3];
    double c1[3][3], c2[3][3];  // [stage][direction]
    int nprev;
};

template <int D>
__global__ void stage_state_kernel(const double* __restrict__ U, Grid3 gU, double* __restrict__ O1,
                                   double* __restrict__ O2, Grid3 gV, StageArgs a)
{
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        const long long iu = gU.at(i, j, k);
        for (int n = 0; n < D + 2; ++n) {
            const double u = U[iu + n * gU.size()];
            double o1 = u, o2 = u;
            for (int s = 0; s < a.nprev; ++s) {
                double acc1 = 0.0, acc2 = 0.0;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    int p[3] = { i, j, k };
                    p[d] += 1;
                    const long long fs = a.gF[d].size();
                    const double df = a.F[s][d][a.gF[d].at(p[0], p[1], p[2]) + n * fs] - a.F[s][d][a.gF[d].at(i, j, k) + n * fs];
                    const double t1 = a.c1[s][d] * df, t2 = a.c2[s][d] * df;
                    acc1 = d == 0 ? t1 : acc1 + t1;
                    acc2 = d == 0 ? t2 : acc2 + t2;
                }
                o1 = o1 - acc1;
                o2 = o2 - acc2;
            }
            O1[iu + n * gU.size()] = o1;
            O2[iu + n * gU.size()] = o2;
        }
    }
}

// compute_pressure (Source/IMEX/IMEX_O1.cpp:292-378) for a later stage of the
// linearised scheme, valid cells: split kinetic energy
// (gamma-1)(E_new - eps/2 m_old . m_new / rho_old); explicit kinetic energy
// (gamma-1)(E_new - eps/2 |m_ex|^2 / rho_new) with m_ex the old stage state
// advanced by adt with its own advection fluxes AF; otherwise pressure(new).
template <int D>
__global__ void stage_pressure_kernel(const double* __restrict__ Unew, const double* __restrict__ Uold, Grid3 gU,
                                      const double* __restrict__ AF0, const double* __restrict__ AF1,
                                      const double* __restrict__ AF2, Grid3 gA0, Grid3 gA1, Grid3 gA2,
                                      double* __restrict__ p, Grid3 gV, int ke_method, IK c)
{
    const double* AF[3] = { AF0, AF1, AF2 };
    const Grid3 gA[3] = { gA0, gA1, gA2 };
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        const long long iu = gU.at(i, j, k);
        double un[D + 2], uo[D + 2];
        load<D>(Unew, iu, gU.size(), un);
        load<D>(Uold, iu, gU.size(), uo);
        double v;
        if (ke_method == BAMREX_IMEX_KE_SPLIT) {
            double dot = uo[1] * un[1];
#pragma unroll
            for (int d = 1; d < D; ++d) dot = dot + uo[1 + d] * un[1 + d];
            v = (c.adia - 1) * (un[1 + D] - 0.5 * c.eps * dot / uo[0]);
        } else if (ke_method == BAMREX_IMEX_KE_EX) {
            double ex[D + 2];
#pragma unroll
            for (int n = 0; n < D + 2; ++n) {
                double acc = 0.0;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    int q[3] = { i, j, k };
                    q[d] += 1;
                    const long long fs = gA[d].size();
                    const double term = c.dtdx[d] * (AF[d][gA[d].at(q[0], q[1], q[2]) + n * fs] - AF[d][gA[d].at(i, j, k) + n * fs]);
                    acc = d == 0 ? term : acc + term;
                }
                ex[n] = uo[n] - acc;
            }
            double m2 = ex[1] * ex[1];
#pragma unroll
            for (int d = 1; d < D; ++d) m2 = m2 + ex[1 + d] * ex[1 + d];
            v = (c.adia - 1) * (un[1 + D] - 0.5 * c.eps * m2 / un[0]);
        } else {
            v = (c.adia - 1) * (un[1 + D] - kinetic_energy<D>(un, c.eps));
        }
        p[t] = v;
    }
}

// sum_fluxes (Source/IMEX/IMEX_RK.cpp:196-235): dst = F_0 b_0 + F_1 b_1 + ...
__global__ void flux_sum_kernel(double* __restrict__ dst, const double* __restrict__ F0, const double* __restrict__ F1,
                                const double* __restrict__ F2, const double* __restrict__ F3, double b0, double b1,
                                double b2, double b3, int nstage, long long n)
{
    GRID_LOOP(t, n)
    {
        double v = F0[t] * b0;
        if (nstage > 1) v += F1[t] * b1;
        if (nstage > 2) v += F2[t] * b2;
        if (nstage > 3) v += F3[t] * b3;
        dst[t] = v;
    }
}

// pressure(U) = (gamma - 1)(E - KE) on the valid cells (copy_pressure)
template <int D>
__global__ void pressure_kernel(const double* __restrict__ U, Grid3 gU, double* __restrict__ p, Grid3 gV, IK c)
{
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        double u[D + 2];
        load<D>(U, gU.at(i, j, k), gU.size(), u);
        p[t] = (c.adia - 1) * (u[1 + D] - kinetic_energy<D>(u, c.eps));
    }
}

// max over valid cells of (|m_x| / dx + |m_y| / dy [+ |m_z| / dz]) / rho
// (max_dx_scaled_speed, Source/System/Euler/Euler.cpp:107-129), as ordered
// bits of a non-negative double; NaN reported as the NaN pattern
template <int D>
__global__ void scaled_speed_kernel(const double* __restrict__ U, Grid3 gU, Grid3 gV, double dx0, double dx1,
                                    double dx2, unsigned long long* out)
{
    const double dxs[3] = { dx0, dx1, dx2 };
    double best = 0.0;
    bool nan_seen = false;
    GRID_LOOP(t, gV.size())
    {
        int i, j, k;
        gV.cell(t, i, j, k);
        const long long q = gU.at(i, j, k);
        double s = fabs(U[q + gU.size()]) / dxs[0];
#pragma unroll
        for (int d = 1; d < D; ++d) s = s + fabs(U[q + (1 + d) * gU.size()]) / dxs[d];
        s = s / U[q];
        best = fmax(best, s);
        nan_seen = nan_seen || (s != s);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, off));
    const bool any_nan = __any_sync(0xffffffffu, nan_seen);
    if ((threadIdx.x & 31) == 0) {
        if (any_nan) atomicMax(out, 0x7ff8000000000000ull);
        else atomicMax(out, (unsigned long long)__double_as_longlong(best));
    }
}

}  // namespace

struct bamrex_imex {
    int D = 2, NC = 4, G = 2;
    int n[3] = { 1, 1, 1 };
    double dx[3] = { 1, 1, 1 }, idx[3] = { 1, 1, 1 };
    int bc_lo[3] = { 0, 0, 0 }, bc_hi[3] = { 0, 0, 0 };
    double adia = 1.4, eps = 1.0, cfl = 0.5, tol_rel = 1e-12, tol_abs = 1e-15;
    int max_iter = 1000, method = 0, enth_method = 0, ke_method = 1;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bamrex_helmholtz* H = nullptr;
    bamrex_precnet* net = nullptr;
    int net_mode = 0;
    // learned-solve policy: iterations of the last plain solve (warm-started
    // from the previous pressure it needs few), consecutive learned cycles
    // that fell back, and pressure solves so far
    int plain_last = 0;
    int learned_misses = 0;
    long long solves = 0;
    char* arena = nullptr;
    Grid3 gU, g1, g2, gV, gA[3], gF[3];
    double *U = nullptr, *Uex = nullptr, *enth = nullptr, *ke = nullptr, *vel = nullptr, *rhs = nullptr;
    double *p = nullptr, *pg = nullptr, *bf[3] = { nullptr, nullptr, nullptr };
    double *af[3] = { nullptr, nullptr, nullptr }, *fl[3] = { nullptr, nullptr, nullptr };
    double *SL = nullptr, *SR = nullptr;
    double* stage = nullptr;  // the valid state, dense, on its way to or from the caller
    // the tableau and the stage buffers
    int tab = BAMREX_IMEX_SP111, S = 1;
    double Ai[4][4] = {}, Ae[4][4] = {}, b[4] = {};
    double *Uimp = nullptr, *Uexb[2] = { nullptr, nullptr };
    double* sf[4][3] = {};  // stage fluxes [stage][direction]; stage 0 of SP111 is fl
    unsigned long long* speed = nullptr;
    long long launches = 0;
    std::string err;
    int set_err(int code)
    {
        err = last_error_text();
        return code;
    }
};

namespace {

int ifail(bamrex_imex* h, int code, const std::string& msg) { return h->set_err(fail(code, msg)); }

int ilaunch(bamrex_imex* h, const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, what));
    h->launches++;
    return BAMREX_OK;
}

#define I_TRY(h, call)                        \
    do {                                      \
        const int rc_ = (call);               \
        if (rc_ != BAMREX_OK) return rc_;     \
    } while (0)

IK make_consts(const bamrex_imex* h, double dt)
{
    IK c;
    std::memset(&c, 0, sizeof(c));
    c.D = h->D;
    c.NC = h->NC;
    for (int d = 0; d < 3; ++d) c.n[d] = h->n[d];
    c.adia = h->adia;
    c.eps = h->eps;
    for (int d = 0; d < h->D; ++d) {
        c.dtdx[d] = dt / h->dx[d];
        c.hdtdx[d] = 0.5 * dt * h->idx[d];
        c.hdtdxe[d] = c.hdtdx[d] / h->eps;
        c.dtidx[d] = dt * h->idx[d];
        c.hadv[d] = 0.5 * c.dtdx[d];
    }
    c.heps = 0.5 / h->eps;
    return c;
}

// ghost cells of the state (vector) or of the pressure (scalar)
int fill_ghosts(bamrex_imex* h, double* a, const Grid3& g, int ncomp, int G, bool vector)
{
    for (int d = 0; d < h->D; ++d) {
        int c1 = 1, c2 = 1;
        const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
        c1 = e1 < d ? g.N[e1] : g.N[e1] + 2 * g.lo[e1];
        c2 = e2 < d ? g.N[e2] : g.N[e2] + 2 * g.lo[e2];
        const long long total = 2LL * G * c1 * c2;
        fill_kernel<<<grid_for(total), kThreads, 0, h->stream>>>(a, g, ncomp, g.size(), d, h->n[d], G, h->bc_lo[d],
                                                                 h->bc_hi[d], vector ? 1 + d : -1);
        I_TRY(h, ilaunch(h, "IMEX ghost fill"));
    }
    return BAMREX_OK;
}

// compute_flux_imex_o1 (IMEX_O1.cpp:19-176): the fluxes of one implicit
// stage of size adt into out[d], from the explicit-stage state Ue (whose
// ghost cells are filled) applied to the implicit-stage state Ui; the
// pressure (valid cells, h->p) is the solve's initial guess and result
template <int D>
int stage_flux(bamrex_imex* h, const double* Ui, const double* Ue, double adt, bool local_step, double* const* out,
               int* iters, double* rel_res)
{
    const IK c = make_consts(h, adt);
    cudaStream_t s = h->stream;
    const int gV = grid_for(h->gV.size());
    // pressure ghosts (fill_pressure_boundary)
    to_grown_kernel<<<gV, kThreads, 0, s>>>(h->p, h->gV, h->pg, h->g1, 1);
    I_TRY(h, ilaunch(h, "IMEX pressure copy"));
    I_TRY(h, fill_ghosts(h, h->pg, h->g1, 1, 1, false));
    // 1. explicit advection on the grown box
    if (h->method == BAMREX_IMEX_MUSCL_RUSANOV) {
        muscl_states_kernel<D><<<grid_for(h->g2.size()), kThreads, 0, s>>>(Ue, h->gU, h->SL, h->SR, h->g2, c,
                                                                           local_step ? 1 : 0);
        I_TRY(h, ilaunch(h, "IMEX MUSCL states"));
        for (int d = 0; d < D; ++d) {
            muscl_faces_kernel<D><<<grid_for(h->gA[d].size()), kThreads, 0, s>>>(h->SL, h->SR, h->g2, h->af[d], h->gA[d], d,
                                                                                  h->eps);
            I_TRY(h, ilaunch(h, "IMEX MUSCL-Rusanov faces"));
        }
    } else {
        for (int d = 0; d < D; ++d) {
            rusanov_faces_kernel<D><<<grid_for(h->gA[d].size()), kThreads, 0, s>>>(Ue, h->gU, h->af[d], h->gA[d], d, h->eps);
            I_TRY(h, ilaunch(h, "IMEX Rusanov faces"));
        }
    }
    explicit_update_kernel<D><<<grid_for(h->g1.size()), kThreads, 0, s>>>(Ui, h->gU, h->af[0], h->af[1], h->af[2],
                                                                          h->gA[0], h->gA[1], h->gA[2], h->Uex, h->g1, c);
    I_TRY(h, ilaunch(h, "IMEX explicit update"));
    // 2. enthalpy, kinetic energy, velocity, pressure source
    enthalpy_kernel<D><<<grid_for(h->g1.size()), kThreads, 0, s>>>(Ue, h->gU, h->Uex, h->g1, h->pg, h->enth, h->p, h->gV,
                                                                   h->enth_method, c);
    I_TRY(h, ilaunch(h, "IMEX enthalpy"));
    const bool split = h->ke_method == BAMREX_IMEX_KE_SPLIT;
    source_kernel<D><<<gV, kThreads, 0, s>>>(Ue, h->gU, h->Uex, h->g1, h->enth, h->ke, split ? h->vel : nullptr, h->rhs,
                                             h->gV, h->ke_method, c);
    I_TRY(h, ilaunch(h, "IMEX pressure source"));
    for (int d = 0; d < D; ++d) {
        bface_kernel<<<grid_for(h->gF[d].size()), kThreads, 0, s>>>(h->enth, h->g1, h->bf[d], h->gF[d], d);
        I_TRY(h, ilaunch(h, "IMEX face enthalpy"));
    }
    // 3. the pressure equation
    auto hck = [&](int rc) -> int {
        if (rc != BAMREX_OK) {
            const char* m = bamrex_helmholtz_last_error(h->H);
            return ifail(h, rc, std::string("pressure operator: ") + (m ? m : ""));
        }
        return (int)BAMREX_OK;
    };
    I_TRY(h, hck(bamrex_helmholtz_set_scalars(h->H, 1.0, adt * adt, split ? -0.5 * h->eps * adt : 0.0)));
    I_TRY(h, hck(bamrex_helmholtz_set_acoeffs(h->H, nullptr, h->eps / (h->adia - 1))));
    I_TRY(h, hck(bamrex_helmholtz_set_bcoeffs(h->H, h->bf[0], h->bf[1], D > 2 ? h->bf[2] : nullptr)));
    I_TRY(h, hck(bamrex_helmholtz_set_ccoeffs(h->H, split ? h->vel : nullptr)));
    int it = 0;
    double rr = 0.0;
    // The learned cycle gets a budget of FGMRES iterations worth about the
    // plain solve it replaces (one preconditioner application per FGMRES
    // iteration, two per BiCGStab iteration): 2 x the last plain count, at
    // least 2, at most 30; when it misses the plain solve continues from its
    // iterate.  After two misses in a row the steps solve plainly, trying the
    // learned cycle again on every 16th solve.
    const bool learned = h->net && (h->learned_misses < 2 || h->solves % 16 == 0);
    ++h->solves;
    if (learned) {
        int plain = 0, fb = 0;
        const int budget = h->plain_last > 0 ? std::min(30, std::max(2, 2 * h->plain_last)) : 30;
        I_TRY(h, hck(bamrex_helmholtz_solve_learned(h->H, h->net, h->net_mode, h->p, h->rhs, h->tol_rel, h->tol_abs,
                                                    budget, budget, &it, &plain, &rr, &fb)));
        if (fb) {
            h->learned_misses++;
            h->plain_last = plain;
        } else {
            h->learned_misses = 0;
        }
        it += plain;
    } else if (h->net) {
        I_TRY(h, hck(bamrex_helmholtz_solve(h->H, h->p, h->rhs, h->tol_rel, h->tol_abs, h->max_iter, 0, &it, &rr)));
        h->plain_last = it;
    } else {
        // no CUDA graph: the scalars change every step (dt), so each step
        // would capture a new one, and the solve needs few iterations from
        // the previous pressure
        I_TRY(h, hck(bamrex_helmholtz_solve(h->H, h->p, h->rhs, h->tol_rel, h->tol_abs, h->max_iter, 0, &it, &rr)));
    }
    *iters = it;
    *rel_res = rr;
    if (!std::isfinite(rr)) return ifail(h, BAMREX_ERR_NAN, "the pressure solve produced a non-finite residual");
    // MLMG aborts when it cannot reach the tolerance; here the step stops
    // before the update (the state is unchanged, the pressure holds the
    // solver's last iterate)
    if (!(rr <= h->tol_rel) && it >= h->max_iter)
        return ifail(h, BAMREX_ERR_NOT_CONVERGED, "the pressure solve did not reach its tolerance");
    // 4. the stage fluxes
    to_grown_kernel<<<gV, kThreads, 0, s>>>(h->p, h->gV, h->pg, h->g1, 1);
    I_TRY(h, ilaunch(h, "IMEX pressure copy"));
    I_TRY(h, fill_ghosts(h, h->pg, h->g1, 1, 1, false));
    for (int d = 0; d < D; ++d) {
        flux_kernel<D><<<grid_for(h->gF[d].size()), kThreads, 0, s>>>(h->af[d], h->gA[d], h->Uex, h->enth, h->pg, h->g1,
                                                                       out[d], h->gF[d], d, c);
        I_TRY(h, ilaunch(h, "IMEX fluxes"));
    }
    return BAMREX_OK;
}

// advance_imex_rk (Source/IMEX/IMEX_RK.cpp:23-86): per stage the two stage
// states from the earlier stage fluxes, the stage pressure (later stages),
// the stage fluxes; then the b-weighted flux sum and the conservative update
template <int D>
int step_impl(bamrex_imex* h, double dt, int* iters, double* rel_res)
{
    cudaStream_t s = h->stream;
    const int gV = grid_for(h->gV.size());
    // the step input with its ghost cells (fill_consv_boundary); it stays
    // unchanged until the final update and is both stage states of stage 0
    I_TRY(h, fill_ghosts(h, h->U, h->gU, h->NC, h->G, true));
    int it_total = 0;
    double rr_max = 0.0;
    const double* Ue_prev = nullptr;
    for (int st = 0; st < h->S; ++st) {
        const double* Ui = h->U;
        const double* Ue = h->U;
        if (st > 0) {
            StageArgs a;
            std::memset(&a, 0, sizeof(a));
            a.nprev = st;
            for (int q = 0; q < st; ++q)
                for (int d = 0; d < D; ++d) {
                    a.F[q][d] = h->sf[q][d];
                    a.c1[q][d] = (h->Ai[st][q] * dt) * h->idx[d];
                    a.c2[q][d] = (h->Ae[st][q] * dt) * h->idx[d];
                }
            for (int d = 0; d < D; ++d) a.gF[d] = h->gF[d];
            double* Ue_new = h->Uexb[st % 2];
            stage_state_kernel<D><<<gV, kThreads, 0, s>>>(h->U, h->gU, h->Uimp, Ue_new, h->gV, a);
            I_TRY(h, ilaunch(h, "IMEX stage states"));
            I_TRY(h, fill_ghosts(h, h->Uimp, h->gU, h->NC, h->G, true));
            I_TRY(h, fill_ghosts(h, Ue_new, h->gU, h->NC, h->G, true));
            Ui = h->Uimp;
            Ue = Ue_new;
        }
        const double adt = h->Ai[st][st] * dt;
        if (st > 0) {
            // compute_pressure from this stage's and the previous stage's
            // explicit states
            const IK c = make_consts(h, adt);
            if (h->ke_method == BAMREX_IMEX_KE_EX) {
                if (h->method == BAMREX_IMEX_MUSCL_RUSANOV) {
                    muscl_states_kernel<D><<<grid_for(h->g2.size()), kThreads, 0, s>>>(Ue_prev, h->gU, h->SL, h->SR,
                                                                                       h->g2, c, 0);
                    I_TRY(h, ilaunch(h, "IMEX MUSCL states"));
                    for (int d = 0; d < D; ++d) {
                        muscl_faces_kernel<D><<<grid_for(h->gA[d].size()), kThreads, 0, s>>>(h->SL, h->SR, h->g2, h->af[d],
                                                                                              h->gA[d], d, h->eps);
                        I_TRY(h, ilaunch(h, "IMEX MUSCL-Rusanov faces"));
                    }
                } else {
                    for (int d = 0; d < D; ++d) {
                        rusanov_faces_kernel<D><<<grid_for(h->gA[d].size()), kThreads, 0, s>>>(Ue_prev, h->gU, h->af[d],
                                                                                                h->gA[d], d, h->eps);
                        I_TRY(h, ilaunch(h, "IMEX Rusanov faces"));
                    }
                }
            }
            stage_pressure_kernel<D><<<gV, kThreads, 0, s>>>(Ue, Ue_prev, h->gU, h->af[0], h->af[1], h->af[2], h->gA[0],
                                                             h->gA[1], h->gA[2], h->p, h->gV, h->ke_method, c);
            I_TRY(h, ilaunch(h, "IMEX stage pressure"));
        }
        int it = 0;
        double rr = 0.0;
        I_TRY(h, stage_flux<D>(h, Ui, Ue, adt, h->tab == BAMREX_IMEX_SP111, h->sf[st], &it, &rr));
        it_total += it;
        rr_max = std::max(rr_max, rr);
        Ue_prev = Ue;
    }
    if (iters) *iters = it_total;
    if (rel_res) *rel_res = rr_max;
    if (h->S > 1) {
        for (int d = 0; d < D; ++d) {
            const long long nf = (long long)h->NC * h->gF[d].size();
            flux_sum_kernel<<<grid_for(nf), kThreads, 0, s>>>(h->fl[d], h->sf[0][d], h->sf[1][d], h->S > 2 ? h->sf[2][d] : nullptr,
                                                              h->S > 3 ? h->sf[3][d] : nullptr, h->b[0], h->b[1], h->b[2],
                                                              h->b[3], h->S, nf);
            I_TRY(h, ilaunch(h, "IMEX flux sum"));
        }
    }
    const IK c = make_consts(h, dt);
    update_kernel<D><<<gV, kThreads, 0, s>>>(h->U, h->gU, h->fl[0], h->fl[1], h->fl[2], h->gF[0], h->gF[1], h->gF[2],
                                             h->gV, c);
    I_TRY(h, ilaunch(h, "IMEX update"));
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX step"));
    return BAMREX_OK;
}

}  // namespace

extern "C" int bamrex_imex_create(bamrex_imex** out, const bamrex_imex_desc* d, void* stream)
{
    if (!out || !d) return fail(BAMREX_ERR_ARG, "NULL argument");
    *out = nullptr;
    const int D = d->spacedim;
    if (D != 2 && D != 3) return fail(BAMREX_ERR_ARG, "spacedim must be 2 or 3");
    if (d->advection_flux < BAMREX_IMEX_RUSANOV || d->advection_flux > BAMREX_IMEX_MUSCL_RUSANOV)
        return fail(BAMREX_ERR_ARG, "unknown advection flux");
    if (d->enthalpy_method < BAMREX_IMEX_ENTH_REUSE_PRESSURE || d->enthalpy_method > BAMREX_IMEX_ENTH_CONSERVATIVE_EX)
        return fail(BAMREX_ERR_ARG, "unknown enthalpy method");
    if (d->ke_method < BAMREX_IMEX_KE_CONSERVATIVE || d->ke_method > BAMREX_IMEX_KE_SPLIT)
        return fail(BAMREX_ERR_ARG, "unknown kinetic-energy method");
    if (!(d->parm.adiabatic > 1.0) || !(d->parm.epsilon > 0.0)) return fail(BAMREX_ERR_ARG, "need gamma > 1 and epsilon > 0");
    const int G = d->advection_flux == BAMREX_IMEX_MUSCL_RUSANOV ? 3 : 2;
    long long cells = 1;
    for (int q = 0; q < D; ++q) {
        if (d->n[q] < G) return fail(BAMREX_ERR_ARG, "every direction needs at least as many cells as ghost layers");
        if (!(d->prob_hi[q] > d->prob_lo[q])) return fail(BAMREX_ERR_ARG, "prob_hi must exceed prob_lo");
        for (int s = 0; s < 2; ++s) {
            const int bc = s ? d->bc_hi[q] : d->bc_lo[q];
            if (bc < BAMREX_BC_TRANSMISSIVE || bc > BAMREX_BC_REFLECTIVE) return fail(BAMREX_ERR_ARG, "unknown boundary kind");
        }
        if ((d->bc_lo[q] == BAMREX_BC_PERIODIC) != (d->bc_hi[q] == BAMREX_BC_PERIODIC))
            return fail(BAMREX_ERR_ARG, "periodic boundaries must be set on both sides");
        cells *= d->n[q] + 2 * G + 2;
    }
    if (cells >= (1LL << 31)) return fail(BAMREX_ERR_ARG, "domain too large for one box (2^31 cells with ghosts)");
    std::unique_ptr<bamrex_imex> h(new (std::nothrow) bamrex_imex());
    if (!h) return fail(BAMREX_ERR_OOM, "host allocation failed");
    h->D = D;
    h->NC = D + 2;
    h->G = G;
    for (int q = 0; q < 3; ++q) {
        h->n[q] = q < D ? d->n[q] : 1;
        h->dx[q] = q < D ? (d->prob_hi[q] - d->prob_lo[q]) / (double)d->n[q] : 1.0;
        h->idx[q] = 1.0 / h->dx[q];
        h->bc_lo[q] = q < D ? d->bc_lo[q] : BAMREX_BC_PERIODIC;
        h->bc_hi[q] = q < D ? d->bc_hi[q] : BAMREX_BC_PERIODIC;
    }
    h->adia = d->parm.adiabatic;
    h->eps = d->parm.epsilon;
    h->cfl = d->cfl > 0 ? d->cfl : 0.5;
    h->tol_rel = d->tol_rel > 0 ? d->tol_rel : 1e-12;   // solve_pressure, IMEX_O1.cpp:627-628
    h->tol_abs = d->tol_abs > 0 ? d->tol_abs : 1e-15;
    h->max_iter = d->max_iter > 0 ? d->max_iter : 1000;  // setMaxIter(1000), IMEX_O1.cpp:622
    h->method = d->advection_flux;
    h->enth_method = d->enthalpy_method;
    h->ke_method = d->ke_method;
    // IMEXButcherTableau (Source/IMEX/ButcherTableau.cpp:5-98)
    h->tab = d->tableau;
    switch (h->tab) {
    case BAMREX_IMEX_SP111:
        h->S = 1;
        h->Ai[0][0] = 1;
        h->b[0] = 1;
        break;
    case BAMREX_IMEX_SSP222: {
        h->S = 2;
        const double al = 1 - 1 / std::sqrt(2.0);
        h->Ai[0][0] = al;
        h->Ai[1][0] = 1 - 2 * al;
        h->Ai[1][1] = al;
        h->Ae[1][0] = 1;
        h->b[0] = h->b[1] = 0.5;
        break;
    }
    case BAMREX_IMEX_SASSP322:
        h->S = 3;
        h->Ai[0][0] = 0.5;
        h->Ai[1][0] = -0.5;
        h->Ai[1][1] = 0.5;
        h->Ai[2][1] = 0.5;
        h->Ai[2][2] = 0.5;
        h->Ae[2][1] = 1;
        h->b[1] = h->b[2] = 0.5;
        break;
    case BAMREX_IMEX_SASSP332:
        h->S = 3;
        h->Ai[0][0] = 0.25;
        h->Ai[1][1] = 0.25;
        h->Ai[2][0] = h->Ai[2][1] = h->Ai[2][2] = (double)1 / 3;
        h->Ae[1][0] = 0.5;
        h->Ae[2][0] = h->Ae[2][1] = 0.5;
        h->b[0] = h->b[1] = h->b[2] = (double)1 / 3;
        break;
    case BAMREX_IMEX_SSP433: {
        h->S = 4;
        const double al = 0.24169426078821, be = 0.06042356519705, et = 0.12915286960590;
        h->Ai[0][0] = al;
        h->Ai[1][0] = -al;
        h->Ai[1][1] = al;
        h->Ai[2][1] = 1 - al;
        h->Ai[2][2] = al;
        h->Ai[3][0] = be;
        h->Ai[3][1] = et;
        h->Ai[3][2] = 0.5 - be - et - al;
        h->Ai[3][3] = al;
        h->Ae[2][1] = 1;
        h->Ae[3][1] = 0.25;
        h->Ae[3][2] = 0.25;
        h->b[1] = (double)1 / 6;
        h->b[2] = (double)1 / 6;
        h->b[3] = (double)2 / 3;
        break;
    }
    default:
        if (h->own_stream) cudaStreamDestroy(h->stream);
        return fail(BAMREX_ERR_ARG, "unknown Butcher tableau");
    }
    if (stream) {
        h->stream = (cudaStream_t)stream;
    } else {
        const cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreateWithFlags");
        h->own_stream = true;
    }
    h->gU = grown(D, h->n, G);
    h->g1 = grown(D, h->n, 1);
    h->g2 = grown(D, h->n, 2);
    h->gV = grown(D, h->n, 0);
    for (int q = 0; q < D; ++q) {
        h->gA[q] = grown(D, h->n, 1, q);
        h->gF[q] = grown(D, h->n, 0, q);
    }
    // one arena
    const int NC = h->NC;
    size_t off = 0;
    auto take = [&](long long elems) {
        const size_t o = off;
        off = align_up(off + (size_t)std::max(elems, 1LL) * sizeof(double), 256);
        return o;
    };
    const size_t oU = take(NC * h->gU.size()), oUex = take(NC * h->g1.size()), oEnth = take(h->g1.size());
    const size_t oKe = take(h->gV.size()), oVel = take(D * h->gV.size()), oRhs = take(h->gV.size());
    const size_t oP = take(h->gV.size()), oPg = take(h->g1.size());
    size_t oBf[3] = {}, oAf[3] = {}, oFl[3] = {};
    for (int q = 0; q < D; ++q) {
        oBf[q] = take(h->gF[q].size());
        oAf[q] = take(NC * h->gA[q].size());
        oFl[q] = take(NC * h->gF[q].size());
    }
    size_t oImp = 0, oExb[2] = { 0, 0 }, oSf[4][3] = {};
    if (h->S > 1) {
        oImp = take(NC * h->gU.size());
        oExb[0] = take(NC * h->gU.size());
        oExb[1] = take(NC * h->gU.size());
        for (int st = 0; st < h->S; ++st)
            for (int q = 0; q < D; ++q) oSf[st][q] = take(NC * h->gF[q].size());
    }
    size_t oSL = 0, oSR = 0;
    if (G == 3) {
        oSL = take((long long)D * NC * h->g2.size());
        oSR = take((long long)D * NC * h->g2.size());
    }
    const size_t oSt = take((long long)NC * h->gV.size());
    const size_t oSp = take(1);
    cudaError_t e = cudaMalloc((void**)&h->arena, off);
    if (e != cudaSuccess) {
        if (h->own_stream) cudaStreamDestroy(h->stream);
        return fail(BAMREX_ERR_OOM, std::string("cudaMalloc of the IMEX arena failed: ") + cudaGetErrorString(e));
    }
    char* A = h->arena;
    h->U = (double*)(A + oU);
    h->Uex = (double*)(A + oUex);
    h->enth = (double*)(A + oEnth);
    h->ke = (double*)(A + oKe);
    h->vel = (double*)(A + oVel);
    h->rhs = (double*)(A + oRhs);
    h->p = (double*)(A + oP);
    h->pg = (double*)(A + oPg);
    for (int q = 0; q < D; ++q) {
        h->bf[q] = (double*)(A + oBf[q]);
        h->af[q] = (double*)(A + oAf[q]);
        h->fl[q] = (double*)(A + oFl[q]);
    }
    if (G == 3) {
        h->SL = (double*)(A + oSL);
        h->SR = (double*)(A + oSR);
    }
    if (h->S > 1) {
        h->Uimp = (double*)(A + oImp);
        h->Uexb[0] = (double*)(A + oExb[0]);
        h->Uexb[1] = (double*)(A + oExb[1]);
        for (int st = 0; st < h->S; ++st)
            for (int q = 0; q < D; ++q) h->sf[st][q] = (double*)(A + oSf[st][q]);
    } else {
        for (int q = 0; q < D; ++q) h->sf[0][q] = h->fl[q];
    }
    h->stage = (double*)(A + oSt);
    h->speed = (unsigned long long*)(A + oSp);
    e = cudaMemsetAsync(h->arena, 0, off, h->stream);
    if (e != cudaSuccess) {
        cudaFree(h->arena);
        if (h->own_stream) cudaStreamDestroy(h->stream);
        return cuda_fail(e, "IMEX arena clear");
    }
    // the pressure operator on the same grid and stream
    bamrex_helmholtz_desc hd;
    std::memset(&hd, 0, sizeof(hd));
    hd.spacedim = D;
    for (int q = 0; q < 3; ++q) {
        hd.n[q] = h->n[q];
        hd.prob_lo[q] = q < D ? d->prob_lo[q] : 0.0;
        hd.prob_hi[q] = q < D ? d->prob_hi[q] : 1.0;
        // set_pressure_domain_BC (IMEX_O1.cpp:663-690) with the pressure
        // linop types of bamrexBCData (BCs.cpp:228-265): periodic stays
        // periodic, transmissive and reflective become homogeneous Neumann
        hd.bc_lo[q] = h->bc_lo[q] == BAMREX_BC_PERIODIC ? BAMREX_LINOP_PERIODIC : BAMREX_LINOP_NEUMANN;
        hd.bc_hi[q] = h->bc_hi[q] == BAMREX_BC_PERIODIC ? BAMREX_LINOP_PERIODIC : BAMREX_LINOP_NEUMANN;
    }
    const int rc = bamrex_helmholtz_create(&h->H, &hd, h->stream);
    if (rc != BAMREX_OK) {
        cudaFree(h->arena);
        if (h->own_stream) cudaStreamDestroy(h->stream);
        return rc;
    }
    *out = h.release();
    return BAMREX_OK;
}

extern "C" int bamrex_imex_destroy(bamrex_imex* h)
{
    if (!h) return BAMREX_OK;
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->H) bamrex_helmholtz_destroy(h->H);
    if (h->arena) cudaFree(h->arena);
    if (h->own_stream) cudaStreamDestroy(h->stream);
    delete h;
    return BAMREX_OK;
}

extern "C" const char* bamrex_imex_last_error(const bamrex_imex* h) { return h ? h->err.c_str() : ""; }

extern "C" bamrex_helmholtz* bamrex_imex_operator(bamrex_imex* h) { return h ? h->H : nullptr; }

extern "C" int bamrex_imex_set_state(bamrex_imex* h, const double* U, const double* p)
{
    if (!h || !U) return fail(BAMREX_ERR_ARG, "NULL argument");
    const long long nv = h->gV.size();
    double* stage = h->stage;
    const size_t bytes = sizeof(double) * h->NC * nv;
    cudaError_t e = cudaMemcpyAsync(stage, U, bytes, cudaMemcpyDefault, h->stream);
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX state copy"));
    to_grown_kernel<<<grid_for(nv), kThreads, 0, h->stream>>>(stage, h->gV, h->U, h->gU, h->NC);
    I_TRY(h, ilaunch(h, "IMEX state copy"));
    if (p) {
        e = cudaMemcpyAsync(h->p, p, sizeof(double) * nv, cudaMemcpyDefault, h->stream);
        if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX pressure copy"));
    } else {
        const IK c = make_consts(h, 0.0);
        if (h->D == 2) pressure_kernel<2><<<grid_for(nv), kThreads, 0, h->stream>>>(h->U, h->gU, h->p, h->gV, c);
        else pressure_kernel<3><<<grid_for(nv), kThreads, 0, h->stream>>>(h->U, h->gU, h->p, h->gV, c);
        I_TRY(h, ilaunch(h, "IMEX initial pressure"));
    }
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX set_state"));
    return BAMREX_OK;
}

extern "C" int bamrex_imex_get_state(bamrex_imex* h, double* U, double* p)
{
    if (!h) return fail(BAMREX_ERR_ARG, "NULL argument");
    const long long nv = h->gV.size();
    cudaError_t e = cudaSuccess;
    if (U) {
        double* stage = h->stage;
        from_grown_kernel<<<grid_for(nv), kThreads, 0, h->stream>>>(h->U, h->gU, stage, h->gV, h->NC);
        I_TRY(h, ilaunch(h, "IMEX state copy"));
        e = cudaMemcpyAsync(U, stage, sizeof(double) * h->NC * nv, cudaMemcpyDefault, h->stream);
        if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX state copy"));
    }
    if (p) {
        e = cudaMemcpyAsync(p, h->p, sizeof(double) * nv, cudaMemcpyDefault, h->stream);
        if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX pressure copy"));
    }
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX get_state"));
    return BAMREX_OK;
}

extern "C" int bamrex_imex_est_time_step(bamrex_imex* h, double* dt)
{
    if (!h || !dt) return fail(BAMREX_ERR_ARG, "NULL argument");
    cudaError_t e = cudaMemsetAsync(h->speed, 0, sizeof(unsigned long long), h->stream);
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX time step"));
    const long long nv = h->gV.size();
    if (h->D == 2)
        scaled_speed_kernel<2><<<grid_for(nv), kThreads, 0, h->stream>>>(h->U, h->gU, h->gV, h->dx[0], h->dx[1], h->dx[2], h->speed);
    else
        scaled_speed_kernel<3><<<grid_for(nv), kThreads, 0, h->stream>>>(h->U, h->gU, h->gV, h->dx[0], h->dx[1], h->dx[2], h->speed);
    I_TRY(h, ilaunch(h, "IMEX time step"));
    unsigned long long bits = 0;
    e = cudaMemcpyAsync(&bits, h->speed, sizeof(bits), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX time step"));
    double smax;
    std::memcpy(&smax, &bits, sizeof(smax));
    if (!std::isfinite(smax)) return ifail(h, BAMREX_ERR_NAN, "non-finite advective speed");
    // estTimeStep for IMEX after the acoustic start-up: 1 / max_dx_scaled_speed,
    // times cfl (Source/AmrLevelAdv.cpp:432-468)
    *dt = (1.0 / smax) * h->cfl;
    return BAMREX_OK;
}

extern "C" int bamrex_imex_set_precnet(bamrex_imex* h, bamrex_precnet* net, int mode)
{
    if (!h) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (net && (mode < BAMREX_PRECOND_NETWORK || mode > BAMREX_PRECOND_VCYCLE_NETWORK))
        return ifail(h, BAMREX_ERR_ARG, "unknown preconditioner mode");
    h->net = net;
    h->net_mode = mode;
    h->plain_last = 0;
    h->learned_misses = 0;
    h->solves = 0;
    return BAMREX_OK;
}

extern "C" int bamrex_imex_step(bamrex_imex* h, double dt, int* iters, double* rel_res)
{
    if (!h) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (!(dt > 0) || !std::isfinite(dt)) return ifail(h, BAMREX_ERR_ARG, "dt must be positive and finite");
    return h->D == 2 ? step_impl<2>(h, dt, iters, rel_res) : step_impl<3>(h, dt, iters, rel_res);
}

extern "C" int bamrex_imex_field(bamrex_imex* h, int which, double* out, long long* count)
{
    if (!h || !count) return fail(BAMREX_ERR_ARG, "NULL argument");
    const double* src = nullptr;
    long long n = 0;
    switch (which) {
    case BAMREX_IMEX_FIELD_UEX: src = h->Uex; n = h->NC * h->g1.size(); break;
    case BAMREX_IMEX_FIELD_ENTHALPY: src = h->enth; n = h->g1.size(); break;
    case BAMREX_IMEX_FIELD_KE: src = h->ke; n = h->gV.size(); break;
    case BAMREX_IMEX_FIELD_RHS: src = h->rhs; n = h->gV.size(); break;
    case BAMREX_IMEX_FIELD_PRESSURE: src = h->p; n = h->gV.size(); break;
    case BAMREX_IMEX_FIELD_FLUX_X:
    case BAMREX_IMEX_FIELD_FLUX_Y:
    case BAMREX_IMEX_FIELD_FLUX_Z: {
        const int d = which - BAMREX_IMEX_FIELD_FLUX_X;
        if (d >= h->D) return ifail(h, BAMREX_ERR_ARG, "no flux in that direction");
        src = h->fl[d];
        n = h->NC * h->gF[d].size();
        break;
    }
    default: return ifail(h, BAMREX_ERR_ARG, "unknown field");
    }
    *count = n;
    if (!out) return BAMREX_OK;
    cudaError_t e = cudaMemcpyAsync(out, src, sizeof(double) * n, cudaMemcpyDefault, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return h->set_err(cuda_fail(e, "IMEX field copy"));
    return BAMREX_OK;
}

extern "C" long long bamrex_imex_launches(const bamrex_imex* h) { return h ? h->launches : 0; }
