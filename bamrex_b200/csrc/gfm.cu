// Rigid bodies by the ghost-fluid method on one level: level set, normals,
// GFM flags, the interface ghost fill (reflective / no-slip / foextrap) and
// the fast-sweeping extrapolation into the body, all on the device.
//
// Reference behaviour followed here:
//   level set      fill_from_IF (Source/AmrLevelAdv_LSinit.cpp:13-35) with the
//                  SDFs of Source/Geometry/{Plane,Sphere,Cylinder,Union,
//                  Intersection}SDF.H, on every cell of every fab
//   normals        fill_ls_normals (Source/Geometry/Normals.cpp:12-54)
//   flags          build_gfm_flags (Source/GFM/GFMFlag.cpp:6-83)
//   interface fill fill_ghost_rb (Source/GFM/RigidBody.cpp:24-170) with
//                  bilinear_interp (Source/GFM/Interp_K.H:17-75), the exact
//                  Riemann solver (Source/System/Euler/RiemannSolver.H:112-275,
//                  Euler.H:248-333) and newton_raphson (RootFinding.H)
//   extrapolation  extrapolate_from_boundary (Source/GFM/Extrapolate.cc:9-37,
//                  Extrapolate.H:47-117) over the orderings of fast_sweep
//                  (Source/GFM/FastSweep.H:17-214)
//
// The file is compiled with -fmad=false: every product and sum is rounded
// on its own, in the reference's order, so a CPU restatement reproduces the
// results (up to pow() and the reference's long-double quotient in the
// extrapolation, a unit in the last place).
//
// The extrapolation is a Gauss-Seidel iteration whose result depends on the
// visiting order.  One sweep visits the cells in a fixed lexicographic
// order; a cell reads its axis neighbours, which lie one step earlier or
// later in that order.  Cells on the same hyperplane s0*i + s1*j + s2*k = t
// (s = the sweep's signs) never read each other, and every neighbour a cell
// reads as "already updated" lies on plane t - 1.  So one CTA per box walks
// the planes of the swept region in order, a __syncthreads between planes,
// and reproduces the serial sweep exactly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "bamrex_cuda.h"
#include "level_impl.h"

namespace bamrex {

struct BodyState {
    bamrex_body_desc desc;
    char* mem = nullptr;
    FabDev* d_ls_fab = nullptr;    // per box: D+1 doubles per cell, state fab geometry
    FabDev* d_flag_fab = nullptr;  // per box: one byte per cell, state fab geometry
    int* d_bbox = nullptr;         // per box: lo[3], hi[3] of the swept cells
    int* d_counts = nullptr;       // [0] interface cells, [1] swept cells, [2] list fill
    int* d_iface = nullptr;        // interface cells: box, i, j, k
    double* d_ival = nullptr;      // their new states, NC each
    int* d_active = nullptr;       // boxes swept by the global-memory kernel
    int* d_list_s = nullptr;       // boxes swept in shared memory
    long long* d_meta_off = nullptr;  // their first metadata cell
    double* d_wts = nullptr;       // per swept-region cell: its sweep record (rec_words)
    int ring = 1;                  // records each sweep thread keeps in flight
    int n_smem = 0;                // boxes of d_list_s
    int threads_p = 32;            // threads (pencils) and shared memory of their sweep CTAs
    size_t bytes_p = 0;
    long long n_iface = 0, n_swept = 0;
    int nactive = 0;
    char* list_mem = nullptr;      // second block: interface list and values, box lists, sweep metadata
    GhostOp* d_full = nullptr;     // every ghost cell (FillPatch / fill_consv_boundary)
    int nfull = 0, full_chunks = 0;
    GhostOp* d_inner = nullptr;    // inter-box and periodic ghost cells (FillBoundary)
    bamrex_box* d_boxes = nullptr;
    int ninner = 0, inner_chunks = 0;
};

namespace {

constexpr int kBodyThreads = 256;
constexpr int kSweepCta = 512;
constexpr int kNewtonMax = 200;

struct Sdf {
    int kind;
    double c[3], a[3];
    double r;
    int sign;  // +1: fluid inside
};

struct Shape {
    int n, combine;
    Sdf s[2];
};

// ---- signed distances, > 0 in the body ----------------------------------

__host__ __device__ double sdf_eval(const Sdf& f, int D, double x, double y, double z)
{
    // points of a 1D/2D level have zero in the unused coordinates (XDim3)
    const double p[3] = { x, D > 1 ? y : 0.0, D > 2 ? z : 0.0 };
    const double rx = p[0] - f.c[0], ry = p[1] - f.c[1], rz = p[2] - f.c[2];
    if (f.kind == BAMREX_SDF_PLANE) {
        const double dot = rx * f.a[0] + ry * f.a[1] + rz * f.a[2];
        return -1 * dot;
    }
    if (f.kind == BAMREX_SDF_SPHERE) {
        // AMREX_D_TERM sum over the level's dimensions only
        double s = rx * rx;
        if (D > 1) s = s + ry * ry;
        if (D > 2) s = s + rz * rz;
        return (sqrt(s) - f.r) * f.sign;
    }
    const double dot = rx * f.a[0] + ry * f.a[1] + rz * f.a[2];
    const double tx = rx - dot * f.a[0], ty = ry - dot * f.a[1], tz = rz - dot * f.a[2];
    return (sqrt(tx * tx + ty * ty + tz * tz) - f.r) * f.sign;
}

__host__ __device__ double shape_eval(const Shape& S, int D, double x, double y, double z)
{
    const double f1 = sdf_eval(S.s[0], D, x, y, z);
    if (S.n == 1) return f1;
    const double f2 = sdf_eval(S.s[1], D, x, y, z);
    if (S.combine == BAMREX_SDF_UNION) {
        const double outside = fmin(fmax(f1, f2), 0.);
        const double inside = sqrt(fmax(f1, 0.) * fmax(f1, 0.) + fmax(f2, 0.) * fmax(f2, 0.));
        return inside + outside;
    }
    const double inside = fmax(fmin(f1, f2), 0.);
    const double outside = -sqrt(fmin(f1, 0.) * fmin(f1, 0.) + fmin(f2, 0.) * fmin(f2, 0.));
    return inside + outside;
}

// ---- per-box cell loops ----------------------------------------------------

struct Region {
    int lo[3], n[3];
    __device__ long long size() const { return (long long)n[0] * n[1] * n[2]; }
    __device__ void cell(long long q, int& i, int& j, int& k) const
    {
        i = lo[0] + (int)(q % n[0]);
        const long long r = q / n[0];
        j = lo[1] + (int)(r % n[1]);
        k = lo[2] + (int)(r / n[1]);
    }
};

// The cells of box b's fab (valid box grown by the fab's ghost width),
// shrunk by `shrink` in the level's directions.
__device__ Region fab_region(const FabDev& f, const bamrex_box& B, int D, int shrink)
{
    Region R;
    const int b0[3] = { f.b0, f.b1, f.b2 };
    for (int d = 0; d < 3; ++d) {
        const int g = d < D ? (B.lo[d] - b0[d]) : 0;
        R.lo[d] = B.lo[d] - (g - (d < D ? shrink : 0));
        R.n[d] = (B.hi[d] - B.lo[d] + 1) + 2 * (g - (d < D ? shrink : 0));
    }
    return R;
}

// element offset of cell (i,j,k) in a fab (component 0)
__device__ __forceinline__ long long at(const FabDev& f, int i, int j, int k)
{
    return (long long)(i - f.b0) + (long long)(j - f.b1) * f.js + (long long)(k - f.b2) * f.ks;
}

__global__ void ls_fill_kernel(Shape S, int D, const bamrex_box* __restrict__ boxes, const FabDev* __restrict__ lsf,
                               double dx0, double dx1, double dx2, double plo0, double plo1, double plo2)
{
    const int b = blockIdx.y;
    const FabDev f = lsf[b];
    const Region R = fab_region(f, boxes[b], D, 0);
    double* ls = f.ptr<double>();
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < R.size();
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        R.cell(q, i, j, k);
        ls[at(f, i, j, k)] = shape_eval(S, D, (i + 0.5) * dx0 + plo0, (j + 0.5) * dx1 + plo1, (k + 0.5) * dx2 + plo2);
    }
}

__global__ void normals_kernel(int D, const bamrex_box* __restrict__ boxes, const FabDev* __restrict__ lsf, double dx0,
                               double dx1, double dx2)
{
    const int b = blockIdx.y;
    const FabDev f = lsf[b];
    const Region R = fab_region(f, boxes[b], D, 1);
    double* ls = f.ptr<double>();
    const double dx[3] = { dx0, dx1, dx2 };
    const long long off[3] = { 1, f.js, f.ks };
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < R.size();
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        R.cell(q, i, j, k);
        const long long c = at(f, i, j, k);
        double nv[3] = { 0, 0, 0 };
        for (int d = 0; d < D; ++d) {
            const double lp = ls[c + off[d]], lm = ls[c - off[d]], l0 = ls[c];
            nv[d] = ((fabs(lp) < fabs(lm)) ? lp - l0 : l0 - lm) / dx[d];
            ls[c + (1 + d) * f.ns] = nv[d];
        }
        double m2 = nv[0] * nv[0];
        for (int d = 1; d < D; ++d) m2 = m2 + nv[d] * nv[d];
        const double mag = sqrt(m2);
        if (mag != 0)
            for (int d = 0; d < D; ++d) ls[c + (1 + d) * f.ns] = nv[d] / -mag;
    }
}

// GFM flags of the valid cells (build_gfm_flags), the swept region of each
// box (ghost cells not at the interface: the cells extrapolate_from_boundary
// rewrites) and the counts.
__global__ void flags_kernel(int D, int stencil, int diag, const bamrex_box* __restrict__ boxes,
                             const FabDev* __restrict__ lsf, const FabDev* __restrict__ flf, int* __restrict__ bbox,
                             int* __restrict__ counts)
{
    const int b = blockIdx.y;
    const FabDev f = lsf[b], g = flf[b];
    const bamrex_box B = boxes[b];
    Region R;
    for (int d = 0; d < 3; ++d) {
        R.lo[d] = B.lo[d];
        R.n[d] = B.hi[d] - B.lo[d] + 1;
    }
    const double* ls = f.ptr<double>();
    unsigned char* fl = g.ptr<unsigned char>();
    const long long off[3] = { 1, f.js, f.ks };
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < R.size();
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        R.cell(q, i, j, k);
        const long long c = at(f, i, j, k);
        const double l0 = ls[c];
        int flag = 0;
        if (l0 >= 0) flag |= BAMREX_GFM_GHOST;
        bool iface = false;
        for (int d = 0; d < D; ++d) iface = iface || (l0 * ls[c + off[d]] <= 0) || (l0 * ls[c - off[d]] <= 0);
        if (iface) flag |= BAMREX_GFM_INTERFACE;
        if (l0 >= 0) {
            bool close = false;
            if (!diag) {
                for (int s = -stencil; s <= stencil; ++s)
                    for (int d = 0; d < D; ++d) close = close || (l0 * ls[c + s * off[d]] <= 0);
            } else {
                for (int ii = -stencil; ii <= stencil; ++ii) {
                    const int jr = D >= 2 ? stencil - abs(ii) : 0;
                    for (int jj = -jr; jj <= jr; ++jj) {
                        const int kr = D == 3 ? jr - abs(jj) : 0;
                        for (int kk = -kr; kk <= kr; ++kk)
                            close = close || (l0 * ls[c + ii * off[0] + jj * off[1] + kk * off[2]] <= 0);
                    }
                }
            }
            if (close) flag |= BAMREX_GFM_FILL;
        }
        fl[at(g, i, j, k)] = (unsigned char)flag;
        if ((flag & BAMREX_GFM_GHOST) && (flag & BAMREX_GFM_INTERFACE)) atomicAdd(&counts[0], 1);
        if ((flag & BAMREX_GFM_GHOST) && !(flag & BAMREX_GFM_INTERFACE)) {
            atomicAdd(&counts[1], 1);
            int* bb = bbox + 6 * b;
            atomicMin(&bb[0], i);
            atomicMin(&bb[1], j);
            atomicMin(&bb[2], k);
            atomicMax(&bb[3], i);
            atomicMax(&bb[4], j);
            atomicMax(&bb[5], k);
        }
    }
}

__global__ void iface_collect_kernel(const bamrex_box* __restrict__ boxes, const FabDev* __restrict__ flf,
                                     int* __restrict__ list, int cap, int* __restrict__ counter)
{
    const int b = blockIdx.y;
    const FabDev g = flf[b];
    const bamrex_box B = boxes[b];
    Region R;
    for (int d = 0; d < 3; ++d) {
        R.lo[d] = B.lo[d];
        R.n[d] = B.hi[d] - B.lo[d] + 1;
    }
    const unsigned char* fl = g.ptr<unsigned char>();
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < R.size();
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        R.cell(q, i, j, k);
        const int flag = fl[at(g, i, j, k)];
        if ((flag & BAMREX_GFM_GHOST) && (flag & BAMREX_GFM_INTERFACE)) {
            const int s = atomicAdd(counter, 1);
            if (s < cap) {
                list[4 * s] = b;
                list[4 * s + 1] = i;
                list[4 * s + 2] = j;
                list[4 * s + 3] = k;
            }
        }
    }
}

// ---- exact Riemann solver (EulerExactRiemannSolver<0>, interface at x = 0)

struct Prim {
    double v[5];  // rho, u (dir 0), transverse velocities, p: NC = D + 2 entries
};

__device__ double sound_speed(const Prim& q, int NC, double gamma, double eps)
{
    return sqrt(gamma * q.v[NC - 1] / (q.v[0] * eps));
}

__device__ double riemann_one_side(double p, const Prim& q, int NC, double gamma)
{
    const double pK = q.v[NC - 1];
    if (p > pK) {
        const double A = 2 / ((gamma + 1) * q.v[0]);
        const double B = ((gamma - 1) / (gamma + 1)) * pK;
        return (p - pK) * sqrt(A / (p + B));
    }
    const double cK = sound_speed(q, NC, gamma, 1);
    return 2 * cK / (gamma - 1) * (pow(p / pK, (gamma - 1) / (2 * gamma)) - 1);
}

__device__ double riemann_one_side_deriv(double p, const Prim& q, int NC, double gamma)
{
    const double pK = q.v[NC - 1];
    if (p > pK) {
        const double A = 2 / ((gamma + 1) * q.v[0]);
        const double B = ((gamma - 1) / (gamma + 1)) * pK;
        return sqrt(A / (p + B)) * (1 - (p - pK) / (2 * (B + p)));
    }
    const double cK = sound_speed(q, NC, gamma, 1);
    return pow(p / pK, -(gamma + 1) / (2 * gamma)) / (q.v[0] * cK);
}

// consv_from_primv (Source/System/Euler/Euler.H:139-165)
__device__ void consv_from_primv(const Prim& q, int D, double gamma, double eps, double* U)
{
    U[0] = q.v[0];
    for (int d = 0; d < D; ++d) U[1 + d] = q.v[0] * q.v[1 + d];
    const double vie = q.v[1 + D] / (gamma - 1);
    double usq = q.v[1] * q.v[1];
    for (int d = 1; d < D; ++d) usq = usq + q.v[1 + d] * q.v[1 + d];
    U[1 + D] = vie + 0.5 * eps * q.v[0] * usq;
}

// The left intermediate state (conserved) of the Riemann problem L | R in
// direction 0; false if the Newton iteration did not converge.
__device__ bool exact_interm_left(const Prim& L, const Prim& R, int D, double gamma, double eps, double* U)
{
    const int NC = D + 2;
    const double cL1 = sound_speed(L, NC, gamma, 1), cR1 = sound_speed(R, NC, gamma, 1);
    double p = 0.5 * (L.v[NC - 1] + R.v[NC - 1]) - 0.125 * sqrt(eps) * (R.v[1] - L.v[1]) * (L.v[0] + R.v[0]) * (cL1 + cR1);
    p = fmax(1e-6, p);
    bool conv = false;
    for (int it = 0; it < kNewtonMax; ++it) {
        const double prev = p;
        const double f = riemann_one_side(prev, L, NC, gamma) + riemann_one_side(prev, R, NC, gamma) +
                         sqrt(eps) * (R.v[1] - L.v[1]);
        const double fd = riemann_one_side_deriv(prev, L, NC, gamma) + riemann_one_side_deriv(prev, R, NC, gamma);
        p = prev - f / fd;
        if (!(fabs(p - prev) >= 1e-8 * fabs(prev))) {
            conv = true;
            break;
        }
    }
    const double uI = 0.5 * (L.v[1] + R.v[1]) +
                      0.5 * (riemann_one_side(p, R, NC, gamma) - riemann_one_side(p, L, NC, gamma)) / sqrt(eps);
    Prim I = L;
    I.v[1] = uI;
    I.v[NC - 1] = p;
    const double pL = L.v[NC - 1];
    if (p > pL) {
        const double pr = p / pL;
        const double ar = (gamma - 1) / (gamma + 1);
        I.v[0] = L.v[0] * (pr + ar) / (ar * pr + 1);
    } else {
        I.v[0] = L.v[0] * pow(p / pL, 1 / gamma);
    }
    consv_from_primv(I, D, gamma, eps, U);
    return conv;
}

// ---- interface ghost cells ----------------------------------------------

template <typename T, int D>
__device__ double src_at(const FabDev& f, int i, int j, int k, int n)
{
    return (double)f.ptr<T>()[at(f, i, j, D > 2 ? k : f.b2) + n * f.ns];
}

template <typename T, int D>
__global__ void iface_kernel(int rb_bc, int n, const int* __restrict__ list, const bamrex_box* __restrict__ boxes,
                             int ngrow, const FabDev* __restrict__ fab_tab, const FabDev* __restrict__ lsf, Consts k,
                             double dx0, double dx1, double dx2, double* __restrict__ out, StepScalars* status,
                             const StepScalars* gate)
{
    constexpr int NC = D + 2;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n || (gate && gate->done)) return;
    const int b = list[4 * e], ci = list[4 * e + 1], cj = list[4 * e + 2], ck = list[4 * e + 3];
    const FabDev f = fab_tab[b], L = lsf[b];
    const double* ls = L.ptr<double>();
    const long long c = at(L, ci, cj, ck);
    const double dx[3] = { dx0, dx1, dx2 };
    const int idx[3] = { ci, cj, ck };
    double nrm[3] = { 0, 0, 0 };
    for (int d = 0; d < D; ++d) nrm[d] = ls[c + (1 + d) * L.ns];
    const double l0 = ls[c];
    // reflection of the cell centre 1.5 dx into the fluid (x measured from
    // index 0, as bilinear_interp expects)
    const double reach = l0 + 1.5 * dx[0];
    double ijk[3] = { 0, 0, 0 };
    int i0[3] = { 0, 0, 0 }, i1[3] = { 0, 0, 0 };
    double Dx[3] = { 0, 0, 0 };
    for (int d = 0; d < D; ++d) {
        const double xg = (idx[d] + 0.5) * dx[d];
        const double xr = xg + reach * nrm[d];
        ijk[d] = xr / dx[d] - 0.5;
        i0[d] = (int)ijk[d];
        i1[d] = (int)ceil(ijk[d]);
        Dx[d] = ijk[d] - i0[d];
    }
    if (D < 3) {
        i0[2] = i1[2] = f.b2;
    }
    if (D < 2) {
        i0[1] = i1[1] = f.b1;
    }
    // the stencil must lie in the fab (ghost cells included)
    const bamrex_box& B = boxes[b];
    for (int d = 0; d < D; ++d) {
        const int a = min(i0[d], i1[d]), z = max(i0[d], i1[d]);
        if (a < B.lo[d] - ngrow || z > B.hi[d] + ngrow) {
            status->status = BAMREX_ERR_ARG;
            for (int m = 0; m < NC; ++m) out[(long long)e * NC + m] = (double)f.ptr<T>()[at(f, ci, cj, D > 2 ? ck : f.b2) + m * f.ns];
            return;
        }
    }
    double U[NC];
    for (int m = 0; m < NC; ++m) {
        const double s000 = src_at<T, D>(f, i0[0], i0[1], i0[2], m);
        const double s100 = src_at<T, D>(f, i1[0], i0[1], i0[2], m);
        const double s010 = src_at<T, D>(f, i0[0], i1[1], i0[2], m);
        const double s110 = src_at<T, D>(f, i1[0], i1[1], i0[2], m);
        const double s001 = src_at<T, D>(f, i0[0], i0[1], i1[2], m);
        const double s101 = src_at<T, D>(f, i1[0], i0[1], i1[2], m);
        const double s011 = src_at<T, D>(f, i0[0], i1[1], i1[2], m);
        const double s111 = src_at<T, D>(f, i1[0], i1[1], i1[2], m);
        const double c0 = s000;
        const double c1 = s100 - s000;
        const double c2 = s010 - s000;
        const double c3 = s001 - s000;
        const double c4 = s110 - s010 - s100 + s000;
        const double c5 = s011 - s001 - s010 + s000;
        const double c6 = s101 - s001 - s100 + s000;
        // the last two terms of c7 read component 0 whatever m is (Interp_K.H:65)
        const double c7 = s111 - s011 - s101 - s110 + s100 + s001 + src_at<T, D>(f, i0[0], i1[1], i0[2], 0) -
                          src_at<T, D>(f, i0[0], i0[1], i0[2], 0);
        U[m] = c0 + c1 * Dx[0] + c2 * Dx[1] + c3 * Dx[2] + c4 * Dx[0] * Dx[1] + c5 * Dx[1] * Dx[2] + c6 * Dx[2] * Dx[0] +
               c7 * Dx[0] * Dx[1] * Dx[2];
    }
    if (rb_bc != BAMREX_RB_FOEXTRAP) {
        // primv_from_consv (Euler.H:167-198)
        Prim q;
        q.v[0] = U[0];
        for (int d = 0; d < D; ++d) q.v[1 + d] = U[1 + d] / U[0];
        double usq = q.v[1] * q.v[1];
        for (int d = 1; d < D; ++d) usq = usq + q.v[1 + d] * q.v[1 + d];
        q.v[1 + D] = (k.gamma - 1) * (U[1 + D] - 0.5 * k.eps * U[0] * usq);
        if (rb_bc == BAMREX_RB_NO_SLIP) {
            for (int d = 0; d < D; ++d) q.v[1 + d] *= -1;
            consv_from_primv(q, D, k.gamma, k.eps, U);
        } else {
            double un = q.v[1] * nrm[0];
            for (int d = 1; d < D; ++d) un = un + q.v[1 + d] * nrm[d];
            double ut[3] = { 0, 0, 0 };
            for (int d = 0; d < D; ++d) ut[d] = q.v[1 + d] - un * nrm[d];
            // curvature = -div(normal) by central differences of the normals
            const long long off[3] = { 1, L.js, L.ks };
            double curv = -(0.5 * (1.0 / dx[0]) * (ls[c + off[0] + L.ns] - ls[c - off[0] + L.ns]));
            for (int d = 1; d < D; ++d)
                curv = curv - (0.5 * (1.0 / dx[d]) * (ls[c + off[d] + (1 + d) * L.ns] - ls[c - off[d] + (1 + d) * L.ns]));
            double ut2 = ut[0] * ut[0];
            for (int d = 1; d < D; ++d) ut2 = ut2 + ut[d] * ut[d];
            const double utl = sqrt(ut2);
            Prim PL, PR;
            for (int m = 0; m < 5; ++m) PL.v[m] = PR.v[m] = 0;
            PL.v[0] = PR.v[0] = q.v[0];
            PL.v[1] = -un;
            PR.v[1] = un;
            if (D > 1) PL.v[2] = PR.v[2] = utl;
            PL.v[1 + D] = q.v[1 + D];
            PR.v[1 + D] = fmax(q.v[1 + D] - q.v[0] * ut2 * curv * 2 * 1.5 * dx[0], 1e-14);
            double I[NC];
            if (!exact_interm_left(PL, PR, D, k.gamma, k.eps, I)) status->status = BAMREX_ERR_NOT_CONVERGED;
            U[0] = I[0];
            for (int d = 0; d < D; ++d) U[1 + d] = -I[1] * nrm[d] + ut[d] * I[0];
            U[1 + D] = I[1 + D];
        }
    }
    for (int m = 0; m < NC; ++m) out[(long long)e * NC + m] = U[m];
}

template <typename T>
__global__ void iface_store_kernel(int NC, int n, const int* __restrict__ list, const FabDev* __restrict__ fab_tab,
                                   const double* __restrict__ val, const StepScalars* gate)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n || (gate && gate->done)) return;
    const FabDev f = fab_tab[list[4 * e]];
    T* p = f.ptr<T>() + at(f, list[4 * e + 1], list[4 * e + 2], list[4 * e + 3]);
    for (int m = 0; m < NC; ++m) p[m * f.ns] = (T)val[(long long)e * NC + m];
}

// ---- fast-sweeping extrapolation ------------------------------------------

// Sweep signs of fast_sweep in its order (FastSweep.H): 2D j-major, 3D
// k-major loops.  s[d] = +1 ascending, -1 descending.
__constant__ int kOrder2[4][2] = { { 1, 1 }, { -1, 1 }, { -1, -1 }, { 1, -1 } };
__constant__ int kOrder3[8][3] = { { 1, 1, 1 },   { 1, 1, -1 }, { -1, 1, 1 },  { -1, 1, -1 },
                                   { -1, -1, 1 }, { -1, -1, -1 }, { 1, -1, 1 }, { 1, -1, -1 } };

// extrapolate_from_boundary on one box: two fast sweeps over the swept
// region in place (one CTA per box; planes of the sweep order in turn).
template <typename T, int D>
__global__ void __launch_bounds__(kSweepCta) extrap_kernel(const int* __restrict__ active, const int* __restrict__ bbox,
                                                           const FabDev* __restrict__ fab_tab,
                                                           const FabDev* __restrict__ lsf,
                                                           const FabDev* __restrict__ flf, double dx0, double dx1,
                                                           double dx2, const StepScalars* gate)
{
    constexpr int NC = D + 2;
    constexpr int NORD = D == 1 ? 2 : (D == 2 ? 4 : 8);
    if (gate && gate->done) return;
    const int b = active[blockIdx.x];
    const FabDev f = fab_tab[b], L = lsf[b], G = flf[b];
    const int lo[3] = { bbox[6 * b], bbox[6 * b + 1], bbox[6 * b + 2] };
    const int n[3] = { bbox[6 * b + 3] - lo[0] + 1, bbox[6 * b + 4] - lo[1] + 1, bbox[6 * b + 5] - lo[2] + 1 };
    const double dx[3] = { dx0, dx1, dx2 };
    const long long off[3] = { 1, f.js, f.ks };
    T* u = f.ptr<T>();
    const double* ls = L.ptr<double>();
    const unsigned char* fl = G.ptr<unsigned char>();
    const int planes = n[0] + n[1] + n[2] - 2;
    const int across = n[1] * n[2];
    for (int rep = 0; rep < 2; ++rep)
        for (int o = 0; o < NORD; ++o) {
            int s[3] = { 1, 1, 1 };
            if (D == 1) s[0] = o == 0 ? 1 : -1;
            if (D == 2) {
                s[0] = kOrder2[o][0];
                s[1] = kOrder2[o][1];
            }
            if (D == 3) {
                s[0] = kOrder3[o][0];
                s[1] = kOrder3[o][1];
                s[2] = kOrder3[o][2];
            }
            for (int t = 0; t < planes; ++t) {
                for (int q = threadIdx.x; q < across; q += blockDim.x) {
                    const int pj = q % n[1], pk = q / n[1];
                    const int pi = t - pj - pk;
                    if (pi < 0 || pi >= n[0]) continue;
                    const int i = s[0] > 0 ? lo[0] + pi : lo[0] + n[0] - 1 - pi;
                    const int j = s[1] > 0 ? lo[1] + pj : lo[1] + n[1] - 1 - pj;
                    const int k = s[2] > 0 ? lo[2] + pk : lo[2] + n[2] - 1 - pk;
                    const int flag = fl[at(G, i, j, k)];
                    if ((flag & BAMREX_GFM_INTERFACE) || !(flag & BAMREX_GFM_GHOST)) continue;
                    const long long cl = at(L, i, j, k);
                    const double sflip = (ls[cl] >= 0) ? -1 : 1;
                    double w[3];
                    long long nb[3];
                    const long long cu = at(f, i, j, k);
                    for (int d = 0; d < D; ++d) {
                        const double nd = ls[cl + (1 + d) * L.ns] / dx[d] * sflip;
                        w[d] = fabs(nd);
                        nb[d] = cu + (nd < 0 ? off[d] : -off[d]);
                    }
                    double den = w[0];
                    for (int d = 1; d < D; ++d) den = den + w[d];
                    for (int m = 0; m < NC; ++m) {
                        double num = 0.0 + w[0] * (double)u[nb[0] + m * f.ns];
                        for (int d = 1; d < D; ++d) num = num + w[d] * (double)u[nb[d] + m * f.ns];
                        u[cu + m * f.ns] = (T)(num / den);
                    }
                }
                __syncthreads();
            }
        }
}

// ---- extrapolation in shared memory ----------------------------------------
//
// The components never read each other (same neighbours and weights for
// all of them), so one CTA takes one (box, component): the swept region of
// the box plus a one-cell halo of that component lives in shared memory in
// the storage type T (every update is rounded to T as the state is), the
// neighbour choice and weights of each swept cell come precomputed, and
// each thread walks one pencil along x, taking the cell of its pencil on
// the current plane.  The weights of the next plane's cell are loaded
// before the barrier so that the plane's critical path is the shared-memory
// reads, the quotient and the barrier.

constexpr int kSmemMax = 224 * 1024;  // shared memory of one (box, component) sweep CTA
constexpr int kPencilMax = 1024;      // pencils (= threads) of one CTA

// Sweep metadata of a swept-region cell, one 16-byte aligned record of
// rec_words<D>() doubles: w_d = |n_d / dx_d| with the sign giving the
// neighbour (+: the cell at +1, -: at -1, so a zero weight is -0.0 as the
// reference's i - 1 choice), their sum (negative for a cell the sweeps skip:
// not a ghost, or at the interface) and the sum's correctly rounded
// reciprocal.
template <int D>
__host__ __device__ constexpr int rec_words() { return (D + 3) & ~1; }

template <int D>
__global__ void meta_kernel(const int* __restrict__ list, int nlist, const int* __restrict__ bbox,
                            const long long* __restrict__ meta_off, const FabDev* __restrict__ lsf,
                            const FabDev* __restrict__ flf, double dx0, double dx1, double dx2,
                            double* __restrict__ wts)
{
    constexpr int RW = rec_words<D>();
    const int li = blockIdx.y;
    if (li >= nlist) return;
    const int b = list[li];
    const int* bb = bbox + 6 * b;
    Region R;
    for (int d = 0; d < 3; ++d) {
        R.lo[d] = bb[d];
        R.n[d] = bb[3 + d] - bb[d] + 1;
    }
    const FabDev L = lsf[b], G = flf[b];
    const double* ls = L.ptr<double>();
    const unsigned char* fl = G.ptr<unsigned char>();
    const double dx[3] = { dx0, dx1, dx2 };
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < R.size();
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        R.cell(q, i, j, k);
        const int flag = fl[at(G, i, j, k)];
        double* rec = wts + (meta_off[li] + q) * RW;
        const bool swept = (flag & BAMREX_GFM_GHOST) && !(flag & BAMREX_GFM_INTERFACE);
        const long long cl = at(L, i, j, k);
        const double sflip = (ls[cl] >= 0) ? -1 : 1;
        double den = 0.0;
        for (int d = 0; d < D; ++d) {
            const double nd = ls[cl + (1 + d) * L.ns] / dx[d] * sflip;
            const double w = fabs(nd);
            rec[d] = nd < 0 ? w : -w;
            den = d == 0 ? w : den + w;
        }
        rec[D] = swept ? den : -1.0;
        rec[D + 1] = 1.0 / den;
        for (int d = D + 2; d < RW; ++d) rec[d] = 0.0;
    }
}

// The correctly rounded quotient a / b from y = RN(1/b): q = RN(a y), then
// one correction q + (a - b q) y with the remainder exact by FMA
// (P. Markstein, IBM J. Res. Dev. 34(1), 1990; the correction is exact
// rounding when y is the rounded reciprocal and q is within an ulp).  Three
// dependent operations instead of a full division on the sweep's critical
// path; checked bit for bit against IEEE division on 2e9 random operands.
__device__ __forceinline__ double div_by_rcp(double a, double b, double y)
{
    const double q = a * y;
    const double r = fma(-q, b, a);
    return fma(r, y, q);
}

// Geometry of a swept region in shared memory: extents, halo extents and
// strides, region base corner.
template <int D>
struct SweepRegion {
    int lo[3], n[3], hn0, hn1, hn2, so1, so2, hvol, vol;
    __device__ void init(const int* bb)
    {
        for (int d = 0; d < 3; ++d) {
            lo[d] = bb[d];
            n[d] = bb[3 + d] - bb[d] + 1;
        }
        hn0 = n[0] + 2;
        hn1 = n[1] + (D > 1 ? 2 : 0);
        hn2 = n[2] + (D > 2 ? 2 : 0);
        so1 = hn0;
        so2 = hn0 * hn1;
        hvol = hn0 * hn1 * hn2;
        vol = n[0] * n[1] * n[2];
    }
    __device__ int sidx(int ci, int cj, int ck) const { return (ci + 1) + (cj + (D > 1)) * so1 + (ck + (D > 2)) * so2; }
};

template <typename T, int D>
__device__ void region_load(const SweepRegion<D>& R, const FabDev& f, const T* u, T* sv)
{
#pragma unroll 4
    for (int q = threadIdx.x; q < R.hvol; q += blockDim.x) {
        const int hi = q % R.hn0, r = q / R.hn0;
        const int hj = r % R.hn1, hk = r / R.hn1;
        sv[q] = u[at(f, R.lo[0] - 1 + hi, R.lo[1] - (D > 1) + hj, R.lo[2] - (D > 2) + hk)];
    }
}

__device__ __forceinline__ void sweep_signs(int D, int o, int& s0, int& s1, int& s2)
{
    s0 = s1 = s2 = 1;
    if (D == 1) s0 = o == 0 ? 1 : -1;
    if (D == 2) {
        s0 = kOrder2[o][0];
        s1 = kOrder2[o][1];
    }
    if (D == 3) {
        s0 = kOrder3[o][0];
        s1 = kOrder3[o][1];
        s2 = kOrder3[o][2];
    }
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    const unsigned dst = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// Shared memory of a sweep CTA: the region's values with their halo, then
// each thread's ring of K metadata records.
__host__ __device__ inline size_t sweep_smem_bytes(long long hvol, size_t esize, int threads, int K, int rec_bytes)
{
    return (((size_t)hvol * esize + 15) / 16 * 16) + (size_t)threads * K * rec_bytes;
}

// One thread per pencil (up to 1024 pencils), a barrier per plane.  Each
// thread streams the metadata record of its cell K - 1 planes ahead into a
// ring of its own in shared memory (cp.async), so the plane's critical path
// is the shared-memory reads, the quotient and the barrier; K = 1 (no room
// for a ring) loads the next plane's record into registers instead.
template <typename T, int D, int K>
__global__ void __launch_bounds__(kPencilMax) extrap_smem_kernel(const int* __restrict__ list, const int* __restrict__ bbox,
                                   const long long* __restrict__ meta_off, const double* __restrict__ wts,
                                   const FabDev* __restrict__ fab_tab, const StepScalars* gate)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sv = reinterpret_cast<T*>(smem_raw);
    constexpr int NORD = D == 1 ? 2 : (D == 2 ? 4 : 8);
    constexpr int RW = rec_words<D>();
    if (gate && gate->done) return;
    const int li = blockIdx.x, m = blockIdx.y;
    const int b = list[li];
    SweepRegion<D> R;
    R.init(bbox + 6 * b);
    const double* wt = wts + meta_off[li] * RW;
    double* ring = reinterpret_cast<double*>(smem_raw + ((size_t)R.hvol * sizeof(T) + 15) / 16 * 16) +
                   (size_t)threadIdx.x * K * RW;
    const FabDev f = fab_tab[b];
    T* u = f.ptr<T>() + m * f.ns;
    region_load<T, D>(R, f, u, sv);
    __syncthreads();
    const int pencils = R.n[1] * R.n[2];
    const int q = threadIdx.x;
    const bool has = q < pencils;
    const int pj = has ? q % R.n[1] : 0, pk = has ? q / R.n[1] : 0;
    const int t0 = pj + pk;  // the plane of this thread's first cell
    const int planes = R.n[0] + R.n[1] + R.n[2] - 2;
    for (int rep = 0; rep < 2; ++rep)
        for (int o = 0; o < NORD; ++o) {
            int s0, s1, s2;
            sweep_signs(D, o, s0, s1, s2);
            const int cj = s1 > 0 ? pj : R.n[1] - 1 - pj;
            const int ck = s2 > 0 ? pk : R.n[2] - 1 - pk;
            const int ci0 = s0 > 0 ? 0 : R.n[0] - 1;
            // cell of plane t = t0 + e: x = ci0 + s0 e; record r0 + s0 e, smem cs0 + s0 e
            const int r0 = ci0 + R.n[0] * (cj + R.n[1] * ck);
            const int cs0 = R.sidx(ci0, cj, ck);
            auto on_pencil = [&](int t) { return has && (unsigned)(t - t0) < (unsigned)R.n[0]; };
            auto update = [&](int t, const double* rec) {
                const double den = rec[D];
                if (!(den >= 0)) return;
                const int cs = cs0 + s0 * (t - t0);
                double num = 0.0 + fabs(rec[0]) * (double)sv[cs + (signbit(rec[0]) ? -1 : 1)];
                if (D > 1) num = num + fabs(rec[1]) * (double)sv[cs + (signbit(rec[1]) ? -R.so1 : R.so1)];
                if (D > 2) num = num + fabs(rec[2]) * (double)sv[cs + (signbit(rec[2]) ? -R.so2 : R.so2)];
                sv[cs] = (T)div_by_rcp(num, den, rec[D + 1]);
            };
            if constexpr (K == 1) {
                // no room for a ring: the next plane's record in registers
                double nxt[RW];
                auto fetch = [&](int t) {
                    if (!on_pencil(t)) return;
                    const double* src = wt + (long long)(r0 + s0 * (t - t0)) * RW;
#pragma unroll
                    for (int w = 0; w < RW; ++w) nxt[w] = src[w];
                };
                fetch(0);
                for (int t = 0; t < planes; ++t) {
                    double cur[RW];
#pragma unroll
                    for (int w = 0; w < RW; ++w) cur[w] = nxt[w];
                    fetch(t + 1);
                    if (on_pencil(t)) update(t, cur);
                    __syncthreads();
                }
            } else {
                // the record of plane t goes to ring slot t % K (an empty
                // group off the pencil keeps one group per plane)
                auto issue = [&](int t) {
                    if (on_pencil(t)) {
                        const double* src = wt + (long long)(r0 + s0 * (t - t0)) * RW;
                        double* dst = ring + (t % K) * RW;
#pragma unroll
                        for (int w = 0; w < RW; w += 2) cp_async16(dst + w, src + w);
                    }
                    cp_async_group();
                };
#pragma unroll
                for (int t = 0; t < K - 1; ++t) issue(t);
                for (int t = 0; t < planes; ++t) {
                    issue(t + K - 1);
                    cp_async_wait<K - 1>();
                    if (on_pencil(t)) update(t, ring + (t % K) * RW);
                    __syncthreads();
                }
                cp_async_wait<0>();
            }
        }
    // swept cells back to the state
#pragma unroll 4
    for (int r = threadIdx.x; r < R.vol; r += blockDim.x) {
        if (!(wt[(long long)r * RW + D] >= 0)) continue;
        const int ci = r % R.n[0], rr = r / R.n[0];
        const int cj = rr % R.n[1], ck = rr / R.n[1];
        u[at(f, R.lo[0] + ci, R.lo[1] + cj, R.lo[2] + ck)] = sv[R.sidx(ci, cj, ck)];
    }
}

template <typename T>
__global__ void body_field_kernel(int which, const bamrex_box* __restrict__ boxes, const FabDev* __restrict__ lsf,
                                  const FabDev* __restrict__ flf, const long long* __restrict__ begin,
                                  double* __restrict__ out)
{
    const int b = blockIdx.y;
    const bamrex_box B = boxes[b];
    Region R;
    for (int d = 0; d < 3; ++d) {
        R.lo[d] = B.lo[d];
        R.n[d] = B.hi[d] - B.lo[d] + 1;
    }
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < R.size();
         q += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        R.cell(q, i, j, k);
        double v;
        if (which < 0) v = (double)flf[b].ptr<unsigned char>()[at(flf[b], i, j, k)];
        else v = lsf[b].ptr<double>()[at(lsf[b], i, j, k) + which * lsf[b].ns];
        out[begin[b] + q] = v;
    }
}

// ---- host side -----------------------------------------------------------------

// Ghost-fill ops for every ghost cell of every fab (corners included): the
// product of the per-direction maps of the domain boundary (identity inside,
// periodic shift, mirror with the normal momentum negated, or clamp).  Ops
// whose every outside direction is periodic also go to `inner` (the
// inter-box and periodic fill of FillBoundary).
void build_full_ghost_ops(const bamrex_level* L, const BoxIndex& idx, std::vector<GhostOp>& full,
                          std::vector<GhostOp>& inner)
{
    const int D = L->D, g = L->ngrow;
    std::vector<int> hits;
    for (int b = 0; b < (int)L->boxes.size(); ++b) {
        const bamrex_box& B = L->boxes[b];
        int nsel[3];
        for (int d = 0; d < 3; ++d) nsel[d] = d < D ? 3 : 1;
        for (int c2 = 0; c2 < nsel[2]; ++c2)
            for (int c1 = 0; c1 < nsel[1]; ++c1)
                for (int c0 = 0; c0 < nsel[0]; ++c0) {
                    const int cs[3] = { D > 0 ? c0 - 1 : 0, D > 1 ? c1 - 1 : 0, D > 2 ? c2 - 1 : 0 };
                    if (cs[0] == 0 && cs[1] == 0 && cs[2] == 0) continue;
                    int rlo[3], rhi[3];
                    for (int d = 0; d < 3; ++d) {
                        if (cs[d] < 0) {
                            rlo[d] = B.lo[d] - g;
                            rhi[d] = B.lo[d] - 1;
                        } else if (cs[d] > 0) {
                            rlo[d] = B.hi[d] + 1;
                            rhi[d] = B.hi[d] + g;
                        } else {
                            rlo[d] = B.lo[d];
                            rhi[d] = B.hi[d];
                        }
                    }
                    // split by the domain in every direction: part 0 below, 1 inside, 2 above
                    int plo[3][3], phi[3][3];
                    for (int d = 0; d < 3; ++d) {
                        const int dlo = L->domain.lo[d], dhi = L->domain.hi[d];
                        plo[d][0] = rlo[d];
                        phi[d][0] = std::min(rhi[d], dlo - 1);
                        plo[d][1] = std::max(rlo[d], dlo);
                        phi[d][1] = std::min(rhi[d], dhi);
                        plo[d][2] = std::max(rlo[d], dhi + 1);
                        phi[d][2] = rhi[d];
                        if (d >= D) {
                            plo[d][0] = 1;
                            phi[d][0] = 0;
                            plo[d][2] = 1;
                            phi[d][2] = 0;
                        }
                    }
                    for (int p2 = 0; p2 < 3; ++p2)
                        for (int p1 = 0; p1 < 3; ++p1)
                            for (int p0 = 0; p0 < 3; ++p0) {
                                const int ps[3] = { p0, p1, p2 };
                                int glo[3], ghi[3], mul[3], off[3], slo[3], shi[3];
                                int neg = 0;
                                bool empty = false, periodic_only = true;
                                for (int d = 0; d < 3; ++d) {
                                    glo[d] = plo[d][ps[d]];
                                    ghi[d] = phi[d][ps[d]];
                                    if (glo[d] > ghi[d]) empty = true;
                                }
                                if (empty) continue;
                                for (int d = 0; d < 3; ++d) {
                                    const int dlo = L->domain.lo[d], dhi = L->domain.hi[d], len = dhi - dlo + 1;
                                    mul[d] = 1;
                                    off[d] = 0;
                                    if (ps[d] != 1) {
                                        const int bc = ps[d] == 0 ? L->bc_lo[d] : L->bc_hi[d];
                                        if (bc == BAMREX_BC_PERIODIC) {
                                            off[d] = ps[d] == 0 ? len : -len;
                                        } else if (bc == BAMREX_BC_REFLECTIVE) {
                                            periodic_only = false;
                                            mul[d] = -1;
                                            off[d] = ps[d] == 0 ? 2 * dlo - 1 : 2 * dhi + 1;
                                            neg |= 1 << (1 + d);
                                        } else {
                                            periodic_only = false;
                                            mul[d] = 0;
                                            off[d] = ps[d] == 0 ? dlo : dhi;
                                        }
                                    }
                                    if (mul[d] == 1) {
                                        slo[d] = glo[d] + off[d];
                                        shi[d] = ghi[d] + off[d];
                                    } else if (mul[d] == -1) {
                                        slo[d] = off[d] - ghi[d];
                                        shi[d] = off[d] - glo[d];
                                    } else {
                                        slo[d] = shi[d] = off[d];
                                    }
                                }
                                idx.query(slo, shi, hits);
                                std::sort(hits.begin(), hits.end());
                                for (int sb : hits) {
                                    const bamrex_box& S = L->boxes[sb];
                                    GhostOp op;
                                    std::memset(&op, 0, sizeof(op));
                                    op.dst = b;
                                    op.src = sb;
                                    op.negmask = neg;
                                    bool none = false;
                                    for (int d = 0; d < 3; ++d) {
                                        op.mul[d] = mul[d];
                                        op.off[d] = off[d];
                                        const int a = std::max(slo[d], S.lo[d]), z = std::min(shi[d], S.hi[d]);
                                        if (a > z) {
                                            none = true;
                                            break;
                                        }
                                        if (mul[d] == 1) {
                                            op.lo[d] = a - off[d];
                                            op.hi[d] = z - off[d];
                                        } else if (mul[d] == -1) {
                                            op.lo[d] = off[d] - z;
                                            op.hi[d] = off[d] - a;
                                        } else {
                                            op.lo[d] = glo[d];
                                            op.hi[d] = ghi[d];
                                        }
                                    }
                                    if (none) continue;
                                    full.push_back(op);
                                    if (periodic_only) inner.push_back(op);
                                }
                            }
                }
    }
}

Sdf make_sdf(const bamrex_sdf& s)
{
    Sdf f;
    std::memset(&f, 0, sizeof(f));
    f.kind = s.kind;
    for (int d = 0; d < 3; ++d) {
        f.c[d] = s.center[d];
        f.a[d] = s.axis[d];
    }
    f.r = s.radius;
    f.sign = s.fluid_inside ? 1 : -1;
    if (s.kind == BAMREX_SDF_PLANE || s.kind == BAMREX_SDF_CYLINDER) {
        const double mag = std::sqrt(f.a[0] * f.a[0] + f.a[1] * f.a[1] + f.a[2] * f.a[2]);
        for (int d = 0; d < 3; ++d) f.a[d] /= mag;
    }
    return f;
}

int body_launch(bamrex_level* L, cudaError_t e, const char* what) { return level_launch(L, e, what); }

// The dynamic shared-memory limit of the sweep kernel: a property of the
// kernel, shared by every level that uses it, so it is raised to the most
// any level may ask (kSmemMax) rather than to this level's need (a level
// set up later with a smaller region must not lower it under another's).
template <int K>
cudaError_t smem_attribute(bool fp32, int D, int bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    bytes = kSmemMax;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (fp32) {
        if (D == 1) return cudaFuncSetAttribute(extrap_smem_kernel<float, 1, K>, a, bytes);
        if (D == 2) return cudaFuncSetAttribute(extrap_smem_kernel<float, 2, K>, a, bytes);
        return cudaFuncSetAttribute(extrap_smem_kernel<float, 3, K>, a, bytes);
    }
    if (D == 1) return cudaFuncSetAttribute(extrap_smem_kernel<double, 1, K>, a, bytes);
    if (D == 2) return cudaFuncSetAttribute(extrap_smem_kernel<double, 2, K>, a, bytes);
    return cudaFuncSetAttribute(extrap_smem_kernel<double, 3, K>, a, bytes);
}

int ghost_ops(bamrex_level* L, const GhostOp* ops, int nops, int nchunks, int parity, const StepScalars* gate)
{
    if (!nops) return BAMREX_OK;
    return body_launch(L, launch_ghost_fill(L->NC, L->fp32, ops, nops, nchunks, L->d_fab[parity], gate, L->stream),
                       "body ghost fill");
}

dim3 box_grid(const bamrex_level* L, long long max_cells)
{
    const long long blocks = std::min<long long>(1024, (max_cells + kBodyThreads - 1) / kBodyThreads);
    return dim3((unsigned)std::max<long long>(1, blocks), (unsigned)L->boxes.size());
}

}  // namespace

bool body_tag_tables(const bamrex_level* L, const FabDev** ls_tab, const FabDev** flag_tab)
{
    if (!L->body) return false;
    *ls_tab = L->body->d_ls_fab;
    *flag_tab = L->body->d_flag_fab;
    return true;
}

void body_destroy(bamrex_level* L)
{
    if (!L || !L->body) return;
    cudaStreamSynchronize(L->stream);
    dev_free(L->body->list_mem, L->stream);
    dev_free(L->body->mem, L->stream);
    delete L->body;
    L->body = nullptr;
}

// The rigid-body ghost fill of buffer `parity` (FillPatch, fill_ghost_rb,
// fill_consv_boundary), all in stream order.
int body_fill(bamrex_level* L, int parity, const StepScalars* gate)
{
    BodyState* S = L->body;
    if (!S) return BAMREX_OK;
    BX_TRY(ghost_ops(L, S->d_full, S->nfull, S->full_chunks, parity, gate));
    const int D = L->D;
    if (S->n_iface) {
        const int n = (int)S->n_iface;
        const int g = (n + kBodyThreads - 1) / kBodyThreads;
        const double* dx = L->dx;
        cudaError_t e;
#define BX_IFACE(T, DD)                                                                                              \
    iface_kernel<T, DD><<<g, kBodyThreads, 0, L->stream>>>(S->desc.rb_bc, n, S->d_iface, S->d_boxes, L->ngrow,          \
                                                           L->d_fab[parity], S->d_ls_fab, L->k, dx[0], dx[1], dx[2], \
                                                           S->d_ival, L->d_scal, gate)
        if (L->fp32) {
            if (D == 1) BX_IFACE(float, 1);
            else if (D == 2) BX_IFACE(float, 2);
            else BX_IFACE(float, 3);
        } else {
            if (D == 1) BX_IFACE(double, 1);
            else if (D == 2) BX_IFACE(double, 2);
            else BX_IFACE(double, 3);
        }
#undef BX_IFACE
        e = cudaGetLastError();
        BX_TRY(body_launch(L, e, "interface ghost cells"));
        if (L->fp32) iface_store_kernel<float><<<g, kBodyThreads, 0, L->stream>>>(L->NC, n, S->d_iface, L->d_fab[parity], S->d_ival, gate);
        else iface_store_kernel<double><<<g, kBodyThreads, 0, L->stream>>>(L->NC, n, S->d_iface, L->d_fab[parity], S->d_ival, gate);
        BX_TRY(body_launch(L, cudaGetLastError(), "interface ghost store"));
    }
    BX_TRY(ghost_ops(L, S->d_inner, S->ninner, S->inner_chunks, parity, gate));
    for (int r = 0; r < D + 1; ++r) {
        if (S->n_smem) {
            const dim3 g((unsigned)S->n_smem, (unsigned)L->NC);
#define BX_EXTRAP_S(T, DD, KK)                                                                               \
    extrap_smem_kernel<T, DD, KK><<<g, S->threads_p, S->bytes_p, L->stream>>>(S->d_list_s, S->d_bbox, S->d_meta_off, \
                                                                              S->d_wts, L->d_fab[parity], gate)
#define BX_EXTRAP_SK(T, DD) \
    if (S->ring == 4) BX_EXTRAP_S(T, DD, 4); else if (S->ring == 2) BX_EXTRAP_S(T, DD, 2); else BX_EXTRAP_S(T, DD, 1)
            if (L->fp32) {
                if (D == 1) { BX_EXTRAP_SK(float, 1); }
                else if (D == 2) { BX_EXTRAP_SK(float, 2); }
                else { BX_EXTRAP_SK(float, 3); }
            } else {
                if (D == 1) { BX_EXTRAP_SK(double, 1); }
                else if (D == 2) { BX_EXTRAP_SK(double, 2); }
                else { BX_EXTRAP_SK(double, 3); }
            }
#undef BX_EXTRAP_SK
#undef BX_EXTRAP_S
            BX_TRY(body_launch(L, cudaGetLastError(), "extrapolation (shared memory)"));
        }
        if (S->nactive) {
#define BX_EXTRAP(T, DD)                                                                                       \
    extrap_kernel<T, DD><<<S->nactive, kSweepCta, 0, L->stream>>>(S->d_active, S->d_bbox, L->d_fab[parity], \
                                                                  S->d_ls_fab, S->d_flag_fab, L->dx[0], L->dx[1], L->dx[2], gate)
            if (L->fp32) {
                if (D == 1) BX_EXTRAP(float, 1);
                else if (D == 2) BX_EXTRAP(float, 2);
                else BX_EXTRAP(float, 3);
            } else {
                if (D == 1) BX_EXTRAP(double, 1);
                else if (D == 2) BX_EXTRAP(double, 2);
                else BX_EXTRAP(double, 3);
            }
#undef BX_EXTRAP
            BX_TRY(body_launch(L, cudaGetLastError(), "extrapolation"));
        }
        BX_TRY(ghost_ops(L, S->d_inner, S->ninner, S->inner_chunks, parity, gate));
    }
    return ghost_ops(L, S->d_full, S->nfull, S->full_chunks, parity, gate);
}

}  // namespace bamrex

using namespace bamrex;

extern "C" int bamrex_level_set_body(bamrex_level* L, const bamrex_body_desc* desc)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    body_destroy(L);
    if (!desc) return BAMREX_OK;
    const int D = L->D;
    if (desc->nshapes < 1 || desc->nshapes > 2) return L->set_err(fail(BAMREX_ERR_ARG, "nshapes must be 1 or 2"));
    if (desc->nshapes == 2 && desc->combine != BAMREX_SDF_UNION && desc->combine != BAMREX_SDF_INTERSECTION)
        return L->set_err(fail(BAMREX_ERR_ARG, "unknown shape combination"));
    for (int s = 0; s < desc->nshapes; ++s) {
        const bamrex_sdf& f = desc->shapes[s];
        if (f.kind < BAMREX_SDF_PLANE || f.kind > BAMREX_SDF_CYLINDER) return L->set_err(fail(BAMREX_ERR_ARG, "unknown shape"));
        if (f.kind != BAMREX_SDF_SPHERE && !(f.axis[0] * f.axis[0] + f.axis[1] * f.axis[1] + f.axis[2] * f.axis[2] > 0))
            return L->set_err(fail(BAMREX_ERR_ARG, "plane normal / cylinder axis must be non-zero"));
    }
    if (desc->rb_bc < BAMREX_RB_REFLECTIVE || desc->rb_bc > BAMREX_RB_FOEXTRAP)
        return L->set_err(fail(BAMREX_ERR_ARG, "unknown rigid-body boundary condition"));
    if (desc->stencil < 1 || desc->stencil > L->ngrow)
        return L->set_err(fail(BAMREX_ERR_ARG, "stencil must be in [1, ngrow]"));
    // the interpolation stencil of an interface cell reaches its reflection
    // 1.5 dx beyond the interface plus one cell: up to ~3.2 cells (the
    // reference runs with 6 ghost cells)
    if (L->ngrow < 4) return L->set_err(fail(BAMREX_ERR_ARG, "rigid bodies need ngrow >= 4"));

    std::unique_ptr<BodyState> S(new (std::nothrow) BodyState());
    if (!S) return L->set_err(fail(BAMREX_ERR_OOM, "host allocation failed"));
    S->desc = *desc;
    const int nb = (int)L->boxes.size();

    // ghost-op tables
    BoxIndex idx;
    idx.build(L->domain, L->boxes, D);
    std::vector<GhostOp> full, inner;
    build_full_ghost_ops(L, idx, full, inner);
    S->nfull = (int)full.size();
    S->ninner = (int)inner.size();
    S->full_chunks = number_ghost_ops(full);
    S->inner_chunks = number_ghost_ops(inner);

    // one block: LS and flag fabs (state fab geometry), tables
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + std::max<size_t>(bytes, 1), 256);
        return o;
    };
    std::vector<size_t> o_ls(nb), o_fl(nb);
    long long max_cells = 1;
    for (int b = 0; b < nb; ++b) {
        o_ls[b] = take(sizeof(double) * (size_t)L->fab[0][b].ns * (D + 1));
        o_fl[b] = take((size_t)L->fab[0][b].ns);
        max_cells = std::max(max_cells, L->fab[0][b].ns);
    }
    const size_t o_lsf = take(sizeof(FabDev) * nb), o_flf = take(sizeof(FabDev) * nb);
    const size_t o_bbox = take(sizeof(int) * 6 * nb), o_counts = take(sizeof(int) * 4), o_active = take(sizeof(int) * nb);
    const size_t o_full = take(ghost_table_bytes(full.size(), S->full_chunks));
    const size_t o_inner = take(ghost_table_bytes(inner.size(), S->inner_chunks));
    const size_t o_boxes = take(sizeof(bamrex_box) * nb);
    cudaError_t e = dev_alloc((void**)&S->mem, off, L->stream);
    if (e != cudaSuccess) return L->set_err(fail(BAMREX_ERR_OOM, "allocation of the body tables failed"));
    char* M = S->mem;
    std::vector<FabDev> lsf(nb), flf(nb);
    for (int b = 0; b < nb; ++b) {
        lsf[b] = L->fab[0][b];
        lsf[b].p = M + o_ls[b];
        flf[b] = L->fab[0][b];
        flf[b].p = M + o_fl[b];
    }
    S->d_ls_fab = (FabDev*)(M + o_lsf);
    S->d_flag_fab = (FabDev*)(M + o_flf);
    S->d_bbox = (int*)(M + o_bbox);
    S->d_counts = (int*)(M + o_counts);
    S->d_active = (int*)(M + o_active);
    S->d_full = (GhostOp*)(M + o_full);
    S->d_inner = (GhostOp*)(M + o_inner);
    S->d_boxes = (bamrex_box*)(M + o_boxes);
    bamrex_box* d_boxes = S->d_boxes;
    std::vector<int> bbox0(6 * nb);
    for (int b = 0; b < nb; ++b) {
        for (int d = 0; d < 3; ++d) {
            bbox0[6 * b + d] = 0x7fffffff;
            bbox0[6 * b + 3 + d] = -0x7fffffff;
        }
    }
    const std::vector<int> ct_full = ghost_chunk_table(full, S->full_chunks), ct_inner = ghost_chunk_table(inner, S->inner_chunks);
    auto up = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, L->stream) : cudaSuccess;
    };
    e = up(S->d_ls_fab, lsf.data(), sizeof(FabDev) * nb);
    if (e == cudaSuccess) e = up(S->d_flag_fab, flf.data(), sizeof(FabDev) * nb);
    if (e == cudaSuccess) e = up(S->d_bbox, bbox0.data(), sizeof(int) * 6 * nb);
    if (e == cudaSuccess) e = cudaMemsetAsync(S->d_counts, 0, sizeof(int) * 4, L->stream);
    if (e == cudaSuccess) e = up(S->d_full, full.data(), sizeof(GhostOp) * full.size());
    if (e == cudaSuccess) e = up(S->d_full + full.size(), ct_full.data(), sizeof(int) * ct_full.size());
    if (e == cudaSuccess) e = up(S->d_inner, inner.data(), sizeof(GhostOp) * inner.size());
    if (e == cudaSuccess) e = up(S->d_inner + inner.size(), ct_inner.data(), sizeof(int) * ct_inner.size());
    if (e == cudaSuccess) e = up(d_boxes, L->boxes.data(), sizeof(bamrex_box) * nb);
    Shape sh;
    std::memset(&sh, 0, sizeof(sh));
    sh.n = desc->nshapes;
    sh.combine = desc->combine;
    for (int s = 0; s < desc->nshapes; ++s) sh.s[s] = make_sdf(desc->shapes[s]);
    const dim3 grid = box_grid(L, max_cells);
    if (e == cudaSuccess) {
        ls_fill_kernel<<<grid, kBodyThreads, 0, L->stream>>>(sh, D, d_boxes, S->d_ls_fab, L->dx[0], L->dx[1], L->dx[2],
                                                             L->prob_lo[0], L->prob_lo[1], L->prob_lo[2]);
        normals_kernel<<<grid, kBodyThreads, 0, L->stream>>>(D, d_boxes, S->d_ls_fab, L->dx[0], L->dx[1], L->dx[2]);
        flags_kernel<<<grid, kBodyThreads, 0, L->stream>>>(D, desc->stencil, desc->fill_diagonals ? 1 : 0, d_boxes,
                                                           S->d_ls_fab, S->d_flag_fab, S->d_bbox, S->d_counts);
        e = cudaGetLastError();
    }
    int counts[4] = { 0, 0, 0, 0 };
    if (e == cudaSuccess) e = cudaMemcpyAsync(counts, S->d_counts, sizeof(counts), cudaMemcpyDeviceToHost, L->stream);
    std::vector<int> bbox(6 * nb);
    if (e == cudaSuccess) e = cudaMemcpyAsync(bbox.data(), S->d_bbox, sizeof(int) * 6 * nb, cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) {
        dev_free(S->mem, L->stream);
        return L->set_err(cuda_fail(e, "rigid body set-up"));
    }
    L->launches += 3;
    S->n_iface = counts[0];
    S->n_swept = counts[1];
    // boxes with swept cells: in shared memory when the region and its halo
    // fit (one CTA per box and component), else the global-memory kernel
    std::vector<int> list_p, list_g;
    std::vector<long long> vol_p;
    size_t bytes_p = 0;
    int threads_p = 32;
    const int rec_bytes = 8 * (D == 1 ? rec_words<1>() : (D == 2 ? rec_words<2>() : rec_words<3>()));
    for (int b = 0; b < nb; ++b) {
        if (bbox[6 * b] > bbox[6 * b + 3]) continue;
        long long n[3], hv = 1, vol = 1;
        for (int d = 0; d < 3; ++d) {
            n[d] = bbox[6 * b + 3 + d] - bbox[6 * b + d] + 1;
            hv *= n[d] + (d < D ? 2 : 0);
            vol *= n[d];
        }
        const long long pencils = n[1] * n[2];
        // the region's values (a ring comes on top only where it fits)
        const size_t values = sweep_smem_bytes(hv, L->esize, 0, 1, rec_bytes);
        if (pencils > kPencilMax || values > (size_t)kSmemMax) {
            list_g.push_back(b);
        } else {
            list_p.push_back(b);
            vol_p.push_back(vol);
            bytes_p = std::max(bytes_p, values);
            threads_p = std::max(threads_p, (int)((pencils + 31) / 32 * 32));
        }
    }
    // the deepest ring (records in flight per thread) that fits
    int ring = 1;
    for (int K : { 4, 2 })
        if (bytes_p + (size_t)threads_p * K * rec_bytes <= (size_t)kSmemMax) {
            ring = K;
            break;
        }
    S->ring = ring;
    bytes_p += ring > 1 ? (size_t)threads_p * ring * rec_bytes : 0;
    const std::vector<int>& list_s = list_p;
    std::vector<long long> meta_off;
    long long meta_cells = 0;
    for (long long v : vol_p) {
        meta_off.push_back(meta_cells);
        meta_cells += v;
    }
    S->nactive = (int)list_g.size();
    S->n_smem = (int)list_s.size();
    S->bytes_p = bytes_p;
    S->threads_p = threads_p;
    // second block: interface list and values, box lists, sweep metadata
    char* M2 = nullptr;
    const size_t n_if = (size_t)std::max<long long>(1, S->n_iface);
    size_t off2 = 0;
    auto take2 = [&](size_t bytes) {
        const size_t o = off2;
        off2 = align_up(off2 + std::max<size_t>(bytes, 1), 256);
        return o;
    };
    const size_t o_if = take2(sizeof(int) * 4 * n_if), o_iv = take2(sizeof(double) * L->NC * n_if);
    const size_t o_lg = take2(sizeof(int) * list_g.size()), o_lst = take2(sizeof(int) * list_s.size());
    const size_t o_mo = take2(sizeof(long long) * meta_off.size());
    const size_t o_w = take2((size_t)rec_bytes * (size_t)meta_cells);
    e = dev_alloc((void**)&M2, off2, L->stream);
    if (e != cudaSuccess) {
        dev_free(S->mem, L->stream);
        return L->set_err(fail(BAMREX_ERR_OOM, "allocation of the interface list failed"));
    }
    S->d_iface = (int*)(M2 + o_if);
    S->d_ival = (double*)(M2 + o_iv);
    S->d_active = (int*)(M2 + o_lg);
    S->d_list_s = (int*)(M2 + o_lst);
    S->d_meta_off = (long long*)(M2 + o_mo);
    S->d_wts = (double*)(M2 + o_w);
    e = up(S->d_active, list_g.data(), sizeof(int) * list_g.size());
    if (e == cudaSuccess) e = up(S->d_list_s, list_s.data(), sizeof(int) * list_s.size());
    if (e == cudaSuccess) e = up(S->d_meta_off, meta_off.data(), sizeof(long long) * meta_off.size());
    if (e == cudaSuccess && S->n_iface) {
        iface_collect_kernel<<<grid, kBodyThreads, 0, L->stream>>>(d_boxes, S->d_flag_fab, S->d_iface, (int)S->n_iface,
                                                                   S->d_counts + 2);
        e = cudaGetLastError();
        L->launches++;
    }
    if (e == cudaSuccess && S->n_smem) {
        long long maxv = 1;
        for (size_t i = 0; i < list_s.size(); ++i)
            maxv = std::max(maxv, (i + 1 < list_s.size() ? meta_off[i + 1] : meta_cells) - meta_off[i]);
        const dim3 mg((unsigned)std::min<long long>(1024, (maxv + kBodyThreads - 1) / kBodyThreads), (unsigned)list_s.size());
        if (D == 1) meta_kernel<1><<<mg, kBodyThreads, 0, L->stream>>>(S->d_list_s, S->n_smem, S->d_bbox, S->d_meta_off, S->d_ls_fab, S->d_flag_fab, L->dx[0], L->dx[1], L->dx[2], S->d_wts);
        else if (D == 2) meta_kernel<2><<<mg, kBodyThreads, 0, L->stream>>>(S->d_list_s, S->n_smem, S->d_bbox, S->d_meta_off, S->d_ls_fab, S->d_flag_fab, L->dx[0], L->dx[1], L->dx[2], S->d_wts);
        else meta_kernel<3><<<mg, kBodyThreads, 0, L->stream>>>(S->d_list_s, S->n_smem, S->d_bbox, S->d_meta_off, S->d_ls_fab, S->d_flag_fab, L->dx[0], L->dx[1], L->dx[2], S->d_wts);
        e = cudaGetLastError();
        L->launches++;
        if (e == cudaSuccess)
            e = ring == 4 ? smem_attribute<4>(L->fp32, D, (int)bytes_p)
                          : (ring == 2 ? smem_attribute<2>(L->fp32, D, (int)bytes_p) : smem_attribute<1>(L->fp32, D, (int)bytes_p));
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) {
        dev_free(M2, L->stream);
        dev_free(S->mem, L->stream);
        return L->set_err(cuda_fail(e, "interface list"));
    }
    S->list_mem = M2;
    L->body = S.release();
    return BAMREX_OK;
}

extern "C" int bamrex_level_fill_body_ghosts(bamrex_level* L)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (!L->body) return L->set_err(fail(BAMREX_ERR_ARG, "the level has no rigid body"));
    BX_TRY(body_fill(L, L->cur, nullptr));
    StepScalars h;
    cudaError_t e = cudaMemcpyAsync(&h, L->d_scal, sizeof(h), cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "rigid-body ghost fill"));
    if (h.status == BAMREX_ERR_NOT_CONVERGED)
        return L->set_err(fail(BAMREX_ERR_NOT_CONVERGED, "exact Riemann solve at an interface cell did not converge"));
    if (h.status == BAMREX_ERR_ARG)
        return L->set_err(fail(BAMREX_ERR_ARG, "interface interpolation stencil outside the fab: raise ngrow"));
    return BAMREX_OK;
}

extern "C" int bamrex_level_body_field(bamrex_level* L, int which, double* out)
{
    if (!L || !out) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (!L->body) return L->set_err(fail(BAMREX_ERR_ARG, "the level has no rigid body"));
    if (which < -1 || which > L->D) return L->set_err(fail(BAMREX_ERR_ARG, "which must be -1 .. spacedim"));
    const int nb = (int)L->boxes.size();
    std::vector<long long> begin(nb);
    long long acc = 0, max_cells = 1;
    for (int b = 0; b < nb; ++b) {
        begin[b] = acc;
        long long n = 1;
        for (int d = 0; d < 3; ++d) n *= (long long)(L->boxes[b].hi[d] - L->boxes[b].lo[d] + 1);
        acc += n;
        max_cells = std::max(max_cells, n);
    }
    void* mem = nullptr;
    const size_t o_out = align_up(sizeof(long long) * nb, 256), o_box = o_out + align_up(sizeof(double) * acc, 256);
    cudaError_t e = dev_alloc(&mem, o_box + sizeof(bamrex_box) * nb, L->stream);
    if (e != cudaSuccess) return L->set_err(fail(BAMREX_ERR_OOM, "allocation failed"));
    char* M = (char*)mem;
    e = cudaMemcpyAsync(M, begin.data(), sizeof(long long) * nb, cudaMemcpyHostToDevice, L->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M + o_box, L->boxes.data(), sizeof(bamrex_box) * nb, cudaMemcpyHostToDevice, L->stream);
    if (e == cudaSuccess) {
        body_field_kernel<double><<<box_grid(L, max_cells), kBodyThreads, 0, L->stream>>>(
            which, (const bamrex_box*)(M + o_box), L->body->d_ls_fab, L->body->d_flag_fab, (const long long*)M,
            (double*)(M + o_out));
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, M + o_out, sizeof(double) * acc, cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    dev_free(mem, L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "body field"));
    L->launches++;
    return BAMREX_OK;
}

extern "C" int bamrex_level_body_counts(const bamrex_level* L, long long* interface_cells, long long* swept_cells)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (interface_cells) *interface_cells = L->body ? L->body->n_iface : 0;
    if (swept_cells) *swept_cells = L->body ? L->body->n_swept : 0;
    return BAMREX_OK;
}
