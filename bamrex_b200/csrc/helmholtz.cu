// The pressure Helmholtz operator of the IMEX path on the device:
//   y = A a x - B div(b grad x) + C c . grad x
// (MLABecLaplacianGrad: mlalapgrad_adotx, Source/LinearSolver/
// MLALapGrad_2D_K.H:9-33 and MLALapGrad_3D_K.H:9-38), its red-black
// Gauss-Seidel smoother (alapgrad_gsrb, MLALapGrad_2D_K.H:180-230: plain
// Gauss-Seidel in 2D; MLALapGrad_3D_K.H:258-324: over-relaxed, omega 1.15,
// in 3D), a geometric multigrid V-cycle over a hierarchy of coarsened copies
// of the operator (coefficients averaged down as averageDownCoeffs,
// MLALaplacianGrad.H:950-986), and a BiCGStab solve preconditioned by one
// V-cycle (the solve of setup_pressure_op / solve_pressure,
// Source/IMEX/IMEX_O1.cpp:570-640, to a relative residual).
//
// One box per level: the whole domain, i fastest, no ghost cells.  Domain
// boundaries are applied where a stencil leaves the box: periodic wrap, or
// the boundary value cf * x(cell) with cf = +1 (homogeneous Neumann) or -1
// (homogeneous Dirichlet on the face); the smoother moves the cf part to the
// left-hand side as the reference's cf/delta terms do.  Every kernel is
// HBM-bound; this file is compiled with -fmad=false so each operation rounds
// exactly as written and a CPU restatement reproduces apply and smooth bit
// for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "bamrex_cuda.h"
#include "level_impl.h"

using namespace bamrex;

namespace {

constexpr int kThreads = 256;
constexpr int kDotBlocks = 1184;  // 148 SMs x 8

struct HLev {
    int n[3];
    long long ncell;
    double dx[3];
    double* a;     // ncell
    double* b[3];  // faces: (n0+1)*n1*n2, n0*(n1+1)*n2, n0*n1*(n2+1)
    double* c;     // D * ncell (component-major) or nullptr
    double* phi;   // ncell
    double* rhs;   // ncell
    double* res;   // ncell
    double* tmp;   // ncell: the second buffer of the fused smoother
};

struct HOp {
    double ascal, bscal, cscal;
    int bc_lo[3], bc_hi[3];
};

__device__ __forceinline__ long long cidx(const HLev& L, int i, int j, int k)
{
    return (long long)i + (long long)L.n[0] * ((long long)j + (long long)L.n[1] * k);
}

__device__ __forceinline__ long long fidx(const HLev& L, int d, int i, int j, int k)
{
    const int nx = L.n[0] + (d == 0), ny = L.n[1] + (d == 1);
    return (long long)i + (long long)nx * ((long long)j + (long long)ny * k);
}

// Neighbour value of x at cell (i,j,k) + s e_d (s = -1 or +1).  cf
// receives the boundary factor (0 inside the domain or across a periodic
// face).
__device__ __forceinline__ double nbr(const double* __restrict__ x, const HLev& L, const HOp& op, int i, int j, int k,
                                      int d, int s, double xc, double& cf)
{
    int q[3] = { i, j, k };
    q[d] += s;
    cf = 0.0;
    if (q[d] < 0 || q[d] >= L.n[d]) {
        const int bc = s < 0 ? op.bc_lo[d] : op.bc_hi[d];
        if (bc == BAMREX_LINOP_PERIODIC) {
            q[d] = q[d] < 0 ? q[d] + L.n[d] : q[d] - L.n[d];
        } else {
            cf = bc == BAMREX_LINOP_NEUMANN ? 1.0 : -1.0;
            return cf * xc;
        }
    }
    return x[cidx(L, q[0], q[1], q[2])];
}

// y = A x (mode 0) or y = rhs - A x (mode 1), the operator of
// mlalapgrad_adotx with dhx = B dxinv^2, chdx = C c 0.5 dxinv.
struct ApplyCoef {
    double dxinv[3], dh[3];
};

__device__ __forceinline__ ApplyCoef apply_coef(const HLev& L, const HOp& op)
{
    ApplyCoef a;
    for (int d = 0; d < 3; ++d) {
        a.dxinv[d] = 1.0 / L.dx[d];
        a.dh[d] = op.bscal * a.dxinv[d] * a.dxinv[d];
    }
    return a;
}

// (A x)_c, or rhs_c - (A x)_c with mode 1.
template <int D>
__device__ __forceinline__ double apply_value(const HLev& L, const HOp& op, const ApplyCoef& ac,
                                              const double* __restrict__ x, const double* __restrict__ rhs, int mode,
                                              long long c)
{
    const double* dxinv = ac.dxinv;
    const double* dh = ac.dh;
    {
        const int i = (int)(c % L.n[0]);
        const int j = (int)((c / L.n[0]) % L.n[1]);
        const int k = (int)(c / ((long long)L.n[0] * L.n[1]));
        const double xc = x[c];
        double xm[3], xp[3], cf;
        for (int d = 0; d < D; ++d) {
            xm[d] = nbr(x, L, op, i, j, k, d, -1, xc, cf);
            xp[d] = nbr(x, L, op, i, j, k, d, +1, xc, cf);
        }
        double v = op.ascal * L.a[c] * xc;
        for (int d = 0; d < D; ++d) {
            const int ih = i + (d == 0), jh = j + (d == 1), kh = k + (d == 2);
            const double bl = L.b[d][fidx(L, d, i, j, k)], bh = L.b[d][fidx(L, d, ih, jh, kh)];
            v = v - dh[d] * (bh * (xp[d] - xc) - bl * (xc - xm[d]));
        }
        if (L.c) {
            for (int d = 0; d < D; ++d) {
                const double chd = op.cscal * L.c[(long long)d * L.ncell + c] * 0.5 * dxinv[d];
                v = v + chd * (xp[d] - xm[d]);
            }
        }
        return mode ? rhs[c] - v : v;
    }
}

template <int D>
__global__ void apply_kernel(const HLev L, const HOp op, const double* __restrict__ x, double* __restrict__ y,
                             const double* __restrict__ rhs, int mode)
{
    const ApplyCoef ac = apply_coef(L, op);
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < L.ncell;
         c += (long long)gridDim.x * blockDim.x)
        y[c] = apply_value<D>(L, op, ac, x, rhs, mode, c);
}

// The Gauss-Seidel update of one cell from its neighbours pm/pp (boundary
// factors cfm/cfp), in the operation order of alapgrad_gsrb.
struct GsCoef {
    double dh[3], cdh[3];  // B / h^2 and C / (2 h) as Fsmooth computes them
};

__device__ __forceinline__ GsCoef gs_coef(const HLev& L, const HOp& op)
{
    GsCoef g;
    for (int d = 0; d < 3; ++d) {
        g.dh[d] = op.bscal / (L.dx[d] * L.dx[d]);
        g.cdh[d] = op.cscal / (2 * L.dx[d]);
    }
    return g;
}

// The update itself from the cell's coefficients (a, the low / high face
// coefficients bl / bh, the gradient coefficients cc) and neighbours.
template <int D>
__device__ __forceinline__ double gsrb_core(const HOp& op, const GsCoef& gc, double a, const double (&bl)[3],
                                            const double (&bh)[3], const double (&cc)[3], double pc,
                                            const double (&pm)[3], const double (&pp)[3], const double (&cfm)[3],
                                            const double (&cfp)[3], double rhs)
{
    const double* dh = gc.dh;
    const double* cdh = gc.cdh;
    double gamma = op.ascal * a;
    for (int d = 0; d < D; ++d) gamma = gamma + dh[d] * (bl[d] + bh[d]);
    double delta = dh[0] * (bl[0] * cfm[0] + bh[0] * cfp[0]);
    for (int d = 1; d < D; ++d) delta = delta + dh[d] * (bl[d] * cfm[d] + bh[d] * cfp[d]);
    for (int d = 0; d < D; ++d) delta = delta + cdh[d] * cc[d] * (cfm[d] - cfp[d]);
    double rho = dh[0] * (bl[0] * pm[0] + bh[0] * pp[0]);
    for (int d = 1; d < D; ++d) rho = rho + dh[d] * (bl[d] * pm[d] + bh[d] * pp[d]);
    for (int d = 0; d < D; ++d) rho = rho - cdh[d] * cc[d] * (pp[d] - pm[d]);
    if (D == 3) {
        // MLALapGrad_3D_K.H:293-323
        const double omega = 1.15;
        const double g_m_d = gamma - delta;
        const double res = rhs - (gamma * pc - rho);
        return pc + omega / g_m_d * res;
    }
    // MLALapGrad_2D_K.H:205-228
    return (rhs + rho - pc * delta) / (gamma - delta);
}

template <int D>
__device__ __forceinline__ double gsrb_value(const HLev& L, const HOp& op, const GsCoef& gc, long long c, int i, int j,
                                             int k, double pc, const double (&pm)[3], const double (&pp)[3],
                                             const double (&cfm)[3], const double (&cfp)[3], double rhs)
{
    double bl[3], bh[3], cc[3];
    for (int d = 0; d < D; ++d) {
        const int ih = i + (d == 0), jh = j + (d == 1), kh = k + (d == 2);
        bl[d] = L.b[d][fidx(L, d, i, j, k)];
        bh[d] = L.b[d][fidx(L, d, ih, jh, kh)];
        cc[d] = L.c ? L.c[(long long)d * L.ncell + c] : 0.0;
    }
    return gsrb_core<D>(op, gc, L.a[c], bl, bh, cc, pc, pm, pp, cfm, cfp, rhs);
}

// One colour of the red-black smoother: cells with (i+j+k+color) even.
template <int D>
__global__ void gsrb_kernel(const HLev L, const HOp op, double* __restrict__ phi, const double* __restrict__ rhs,
                            int color)
{
    const GsCoef gc = gs_coef(L, op);
    const long long half = (L.ncell + 1) / 2;
    const int nxh = (L.n[0] + 1) / 2;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < half;
         t += (long long)gridDim.x * blockDim.x) {
        const long long row = t / nxh;
        const int j = (int)(row % L.n[1]);
        const int k = (int)(row / L.n[1]);
        const int i = 2 * (int)(t % nxh) + ((j + k + color) & 1);
        if (i >= L.n[0] || j >= L.n[1] || k >= L.n[2]) continue;
        const long long c = cidx(L, i, j, k);
        const double pc = phi[c];
        double pm[3], pp[3], cfm[3], cfp[3];
        for (int d = 0; d < D; ++d) {
            pm[d] = nbr(phi, L, op, i, j, k, d, -1, pc, cfm[d]);
            pp[d] = nbr(phi, L, op, i, j, k, d, +1, pc, cfp[d]);
        }
        phi[c] = gsrb_value<D>(L, op, gc, c, i, j, k, pc, pm, pp, cfm, cfp, rhs[c]);
    }
}

// A full 2D sweep (red, then black) in one launch over tiles of 32 x 16
// cells: the tile and a 2-cell halo of phi are staged in shared memory,
// red is updated on the tile grown by one cell (the halo's red cells are
// recomputed from the same inputs their own tile uses, so every value is
// the one the two half-sweeps give), then black on the tile, which is
// written to the other buffer (tiles read their halos from the old one).
// One read and one write of phi per sweep instead of two each.  Requires
// n0 % 32 == 0 and n1 % 16 == 0.
constexpr int kGsTX = 32, kGsTY = 16;
constexpr int kGsSX = kGsTX + 4, kGsSY = kGsTY + 4;   // the tile with a 2-cell halo

// One tile of the fused sweep: sp holds the tile's phi window (2-cell halo)
// on entry; the coefficients of the red pass (tile + 1-cell ring) and the
// black pass (tile) come from global memory, or, when sa is non-null, from
// the staged windows sa / sr / sbx / sby of a, rhs and the x / y face
// coefficients (same window origin; only for tiles away from the domain
// boundary, where no boundary condition applies and every neighbour is
// inside the window).
__device__ __forceinline__ void gsrb2_tile(const HLev& L, const HOp& op, const GsCoef& gc, double (*sp)[kGsSX],
                                           const double* __restrict__ rhs, int i0, int j0, const double* sa,
                                           const double* sr, const double* sbx, const double* sby)
{
    for (int pass = 0; pass < 2; ++pass) {
        // pass 0: red on [-1, TX] x [-1, TY]; pass 1: black on the tile.
        // Threads take the cells of the pass's colour only: row lj holds
        // w / 2 of them, at columns of parity (lj + pass + i0 + j0) & 1.
        const int lo = pass == 0 ? -1 : 0;
        const int w = kGsTX + (pass == 0 ? 2 : 0), h = kGsTY + (pass == 0 ? 2 : 0);
        const int wh = w / 2;
        for (int q = threadIdx.x; q < wh * h; q += blockDim.x) {
            const int lj = lo + q / wh;
            const int par = ((i0 + j0 + lj + lo + pass) & 1);  // first column of the colour in this row
            const int li = lo + 2 * (q % wh) + par;
            const double pc = sp[lj + 2][li + 2];
            double pm[3], pp[3], cfm[3] = { 0, 0, 0 }, cfp[3] = { 0, 0, 0 };
            if (sa) {
                const int o = (lj + 2) * kGsSX + li + 2;
                pm[0] = sp[lj + 2][li + 1];
                pp[0] = sp[lj + 2][li + 3];
                pm[1] = sp[lj + 1][li + 2];
                pp[1] = sp[lj + 3][li + 2];
                const double bl[3] = { sbx[o], sby[o], 0.0 }, bh[3] = { sbx[o + 1], sby[o + kGsSX], 0.0 };
                const double cc[3] = { 0.0, 0.0, 0.0 };
                sp[lj + 2][li + 2] = gsrb_core<2>(op, gc, sa[o], bl, bh, cc, pc, pm, pp, cfm, cfp, sr[o]);
                continue;
            }
            const int gi0 = i0 + li, gj0 = j0 + lj;
            // the cell itself in global indices (a periodic image for halo cells)
            int gi = gi0, gj = gj0;
            if (gi < 0 || gi >= L.n[0]) {
                if (op.bc_lo[0] != BAMREX_LINOP_PERIODIC) continue;
                gi = gi < 0 ? gi + L.n[0] : gi - L.n[0];
            }
            if (gj < 0 || gj >= L.n[1]) {
                if (op.bc_lo[1] != BAMREX_LINOP_PERIODIC) continue;
                gj = gj < 0 ? gj + L.n[1] : gj - L.n[1];
            }
            const int nn[2] = { L.n[0], L.n[1] };
            const int g[2] = { gi, gj };
            for (int d = 0; d < 2; ++d) {
                const int si = d == 0 ? 1 : 0, sj = d == 1 ? 1 : 0;
                pm[d] = sp[lj + 2 - sj][li + 2 - si];
                pp[d] = sp[lj + 2 + sj][li + 2 + si];
                if (g[d] == 0 && op.bc_lo[d] != BAMREX_LINOP_PERIODIC) {
                    cfm[d] = op.bc_lo[d] == BAMREX_LINOP_NEUMANN ? 1.0 : -1.0;
                    pm[d] = cfm[d] * pc;
                }
                if (g[d] == nn[d] - 1 && op.bc_hi[d] != BAMREX_LINOP_PERIODIC) {
                    cfp[d] = op.bc_hi[d] == BAMREX_LINOP_NEUMANN ? 1.0 : -1.0;
                    pp[d] = cfp[d] * pc;
                }
            }
            const long long c = (long long)gj * L.n[0] + gi;
            sp[lj + 2][li + 2] = gsrb_value<2>(L, op, gc, c, gi, gj, 0, pc, pm, pp, cfm, cfp, rhs[c]);
        }
        __syncthreads();
    }
}

// phi of a tile's window (periodic images; outside a non-periodic face the
// value is never read) by plain loads.
__device__ __forceinline__ void gsrb2_load_phi(const HLev& L, const HOp& op, const double* __restrict__ phi,
                                               double (*sp)[kGsSX], int i0, int j0)
{
    for (int q = threadIdx.x; q < kGsSX * kGsSY; q += blockDim.x) {
        const int li = q % kGsSX - 2, lj = q / kGsSX - 2;
        int gi = i0 + li, gj = j0 + lj;
        if (gi < 0) gi = op.bc_lo[0] == BAMREX_LINOP_PERIODIC ? gi + L.n[0] : 0;
        if (gi >= L.n[0]) gi = op.bc_hi[0] == BAMREX_LINOP_PERIODIC ? gi - L.n[0] : L.n[0] - 1;
        if (gj < 0) gj = op.bc_lo[1] == BAMREX_LINOP_PERIODIC ? gj + L.n[1] : 0;
        if (gj >= L.n[1]) gj = op.bc_hi[1] == BAMREX_LINOP_PERIODIC ? gj - L.n[1] : L.n[1] - 1;
        sp[lj + 2][li + 2] = phi[(long long)gj * L.n[0] + gi];
    }
}

__device__ __forceinline__ void gsrb2_store(const HLev& L, double* __restrict__ phi_out, double (*sp)[kGsSX], int i0,
                                            int j0)
{
    for (int q = threadIdx.x; q < kGsTX * kGsTY; q += blockDim.x) {
        const int li = q % kGsTX, lj = q / kGsTX;
        phi_out[(long long)(j0 + lj) * L.n[0] + i0 + li] = sp[lj + 2][li + 2];
    }
}

// A full 2D sweep (red, then black) in one launch over tiles of 32 x 16
// cells: the tile and a 2-cell halo of phi are staged in shared memory,
// red is updated on the tile grown by one cell (the halo's red cells are
// recomputed from the same inputs their own tile uses, so every value is
// the one the two half-sweeps give), then black on the tile, which is
// written to the other buffer (tiles read their halos from the old one).
// One read and one write of phi per sweep instead of two each.  Requires
// n0 % 32 == 0 and n1 % 16 == 0.
__global__ void __launch_bounds__(256) gsrb2_fused_kernel(const HLev L, const HOp op, const double* __restrict__ phi,
                                                          double* __restrict__ phi_out, const double* __restrict__ rhs)
{
    __shared__ double sp[kGsSY][kGsSX];
    const GsCoef gc = gs_coef(L, op);
    const int tx = L.n[0] / kGsTX, ty = L.n[1] / kGsTY;
    for (int tile = blockIdx.x; tile < tx * ty; tile += gridDim.x) {
        const int i0 = (tile % tx) * kGsTX, j0 = (tile / tx) * kGsTY;
        __syncthreads();
        gsrb2_load_phi(L, op, phi, sp, i0, j0);
        __syncthreads();
        gsrb2_tile(L, op, gc, sp, rhs, i0, j0, nullptr, nullptr, nullptr, nullptr);
        gsrb2_store(L, phi_out, sp, i0, j0);
    }
}

// The same sweep with every input of a tile staged: tiles away from the
// domain boundary copy the windows of phi, a, rhs and both face
// coefficients (20 x 36 values each, coalesced rows) into shared memory
// with cp.async, the next tile's while the current one is swept, so the
// sweep reads no global memory and waits on no load; boundary tiles take
// the plain path of gsrb2_fused_kernel.  Operators without a gradient term
// (c == nullptr).  The arithmetic is gsrb_core's, so the result is the
// plain sweep's bit for bit.
constexpr int kGsWin = kGsSX * kGsSY;                       // values of one window
constexpr int kGsStageBytes = 5 * kGsWin * (int)sizeof(double);
constexpr int kGsStagedSmem = 2 * kGsStageBytes;

__device__ __forceinline__ bool gsrb2_interior(const HLev& L, int i0, int j0)
{
    return i0 >= kGsTX && i0 + kGsTX + 2 < L.n[0] && j0 >= kGsTY && j0 + kGsTY + 2 < L.n[1];
}

__device__ __forceinline__ void cp_async8(double* dst, const double* src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}

// The five windows of an interior tile into stage st: phi, a, rhs (cells),
// x faces (row stride n0 + 1), y faces (row stride n0); origin (i0-2, j0-2).
__device__ __forceinline__ void gsrb2_prefetch(const HLev& L, const double* __restrict__ phi,
                                               const double* __restrict__ rhs, double* st, int i0, int j0)
{
    const int nx = L.n[0];
    for (int q = threadIdx.x; q < kGsWin; q += blockDim.x) {
        const int li = q % kGsSX, lj = q / kGsSX;
        const long long gc = (long long)(j0 - 2 + lj) * nx + (i0 - 2 + li);
        cp_async8(st + q, phi + gc);
        cp_async8(st + kGsWin + q, L.a + gc);
        cp_async8(st + 2 * kGsWin + q, rhs + gc);
        cp_async8(st + 3 * kGsWin + q, L.b[0] + (long long)(j0 - 2 + lj) * (nx + 1) + (i0 - 2 + li));
        cp_async8(st + 4 * kGsWin + q, L.b[1] + gc);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__global__ void __launch_bounds__(256) gsrb2_staged_kernel(const HLev L, const HOp op, const double* __restrict__ phi,
                                                           double* __restrict__ phi_out, const double* __restrict__ rhs)
{
    extern __shared__ __align__(16) double gs_stage[];
    __shared__ double sp_plain[kGsSY][kGsSX];
    const GsCoef gc = gs_coef(L, op);
    const int tx = L.n[0] / kGsTX, ty = L.n[1] / kGsTY;
    const int ntiles = tx * ty;
    auto origin = [&](int tile, int& i0, int& j0) {
        i0 = (tile % tx) * kGsTX;
        j0 = (tile / tx) * kGsTY;
    };
    int buf = 0;
    {
        int i0, j0;
        if (blockIdx.x < ntiles) {
            origin(blockIdx.x, i0, j0);
            if (gsrb2_interior(L, i0, j0)) gsrb2_prefetch(L, phi, rhs, gs_stage, i0, j0);
        }
    }
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int i0, j0;
        origin(tile, i0, j0);
        const bool staged = gsrb2_interior(L, i0, j0);
        double* st = gs_stage + buf * (5 * kGsWin);
        if (staged) asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();  // this tile's window is in; the other stage is free
        const int next = tile + gridDim.x;
        if (next < ntiles) {
            int ni, nj;
            origin(next, ni, nj);
            if (gsrb2_interior(L, ni, nj)) gsrb2_prefetch(L, phi, rhs, gs_stage + (buf ^ 1) * (5 * kGsWin), ni, nj);
        }
        if (staged) {
            double (*sp)[kGsSX] = reinterpret_cast<double (*)[kGsSX]>(st);
            gsrb2_tile(L, op, gc, sp, rhs, i0, j0, st + kGsWin, st + 2 * kGsWin, st + 3 * kGsWin, st + 4 * kGsWin);
            gsrb2_store(L, phi_out, sp, i0, j0);
        } else {
            gsrb2_load_phi(L, op, phi, sp_plain, i0, j0);
            __syncthreads();
            gsrb2_tile(L, op, gc, sp_plain, rhs, i0, j0, nullptr, nullptr, nullptr, nullptr);
            gsrb2_store(L, phi_out, sp_plain, i0, j0);
        }
        buf ^= 1;
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// rhs_c = mean of the 2^D children of the fine residual
template <int D>
__device__ __forceinline__ void restrict_cell(const HLev& F, const HLev& C, long long c)
{
    const double w = D == 3 ? 0.125 : (D == 2 ? 0.25 : 0.5);
    {
        const int i = (int)(c % C.n[0]);
        const int j = (int)((c / C.n[0]) % C.n[1]);
        const int k = (int)(c / ((long long)C.n[0] * C.n[1]));
        double s = 0.0;
        for (int kk = 0; kk < (D > 2 ? 2 : 1); ++kk)
            for (int jj = 0; jj < (D > 1 ? 2 : 1); ++jj)
                for (int ii = 0; ii < 2; ++ii)
                    s = s + F.res[cidx(F, 2 * i + ii, D > 1 ? 2 * j + jj : j, D > 2 ? 2 * k + kk : k)];
        C.rhs[c] = s * w;
        C.phi[c] = 0.0;
    }
}

template <int D>
__global__ void restrict_kernel(const HLev F, const HLev C)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < C.ncell;
         c += (long long)gridDim.x * blockDim.x)
        restrict_cell<D>(F, C, c);
}

// phi_f += phi_c(parent)
template <int D>
__device__ __forceinline__ void prolong_cell(const HLev& F, const HLev& C, long long c)
{
    const int i = (int)(c % F.n[0]);
    const int j = (int)((c / F.n[0]) % F.n[1]);
    const int k = (int)(c / ((long long)F.n[0] * F.n[1]));
    F.phi[c] = F.phi[c] + C.phi[cidx(C, i / 2, D > 1 ? j / 2 : j, D > 2 ? k / 2 : k)];
}

template <int D>
__global__ void prolong_kernel(const HLev F, const HLev C)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < F.ncell;
         c += (long long)gridDim.x * blockDim.x)
        prolong_cell<D>(F, C, c);
}

// The coarse end of a V-cycle in one block: from level 0 of `lv` (the
// first level of at most kSmallCells cells) down to the bottom and back,
// every phase a block-strided loop over the level's cells followed by a
// block barrier (the launches of the multi-block cycle, each a grid-wide
// step, become barriers): nu1 red-black sweeps, the residual, restriction,
// the bottom's sweeps, prolongation, nu2 sweeps.  The levels' coefficients
// and work arrays live in shared memory for the whole cycle (copied in at
// the start; the first level's phi copied back at the end).  Each cell's
// arithmetic is the multi-block kernels' (gsrb_value, apply_value,
// restrict_cell, prolong_cell), and a colour's cells never read each
// other, so the result is the same bit for bit; the launches and their
// global-memory round trips are gone.
constexpr int kSmallLevels = 12;
constexpr int kSmallThreads = 512;
constexpr long long kSmallCells = 1024;
constexpr int kSmallSmemMax = 200 * 1024;
struct HLevs {
    HLev lev[kSmallLevels];
    int n;
};

// doubles of one level in the shared layout: phi, rhs, res, a, the face
// coefficients of each direction, the gradient coefficients if present
__host__ __device__ __forceinline__ long long face_count(const HLev& L, int d)
{
    return (long long)(L.n[0] + (d == 0)) * (L.n[1] + (d == 1)) * (L.n[2] + (d == 2));
}
__host__ __device__ __forceinline__ long long small_level_doubles(const HLev& L, int D)
{
    long long t = 4 * L.ncell;
    for (int d = 0; d < D; ++d) t += face_count(L, d);
    if (L.c) t += (long long)D * L.ncell;
    return t;
}

template <int D>
__device__ void small_sweeps(const HLev L, const HOp& op, int sweeps)
{
    const GsCoef gc = gs_coef(L, op);
    for (int s = 0; s < sweeps; ++s)
        for (int color = 0; color < 2; ++color) {
            for (int c = threadIdx.x; c < (int)L.ncell; c += blockDim.x) {
                const int i = c % L.n[0];
                const int j = (c / L.n[0]) % L.n[1];
                const int k = c / (L.n[0] * L.n[1]);
                if ((i + j + k + color) & 1) continue;
                const double pc = L.phi[c];
                double pm[3], pp[3], cfm[3], cfp[3];
                for (int d = 0; d < D; ++d) {
                    pm[d] = nbr(L.phi, L, op, i, j, k, d, -1, pc, cfm[d]);
                    pp[d] = nbr(L.phi, L, op, i, j, k, d, +1, pc, cfp[d]);
                }
                L.phi[c] = gsrb_value<D>(L, op, gc, c, i, j, k, pc, pm, pp, cfm, cfp, L.rhs[c]);
            }
            __syncthreads();
        }
}

__device__ __forceinline__ void small_copy(double* dst, const double* src, long long n)
{
    for (long long q = threadIdx.x; q < n; q += blockDim.x) dst[q] = src[q];
}

template <int D>
__global__ void __launch_bounds__(kSmallThreads) vcycle_small_kernel(const HLevs lv, const HOp op, int nu1, int nu2,
                                                                     int bottom)
{
    extern __shared__ double small_sm[];
    __shared__ HLev S[kSmallLevels];
    const int nl = lv.n;
    if (threadIdx.x == 0) {
        long long off = 0;
        for (int l = 0; l < nl; ++l) {
            const HLev& G = lv.lev[l];
            HLev& L = S[l];
            L = G;
            L.phi = small_sm + off;
            off += G.ncell;
            L.rhs = small_sm + off;
            off += G.ncell;
            L.res = small_sm + off;
            off += G.ncell;
            L.a = small_sm + off;
            off += G.ncell;
            for (int d = 0; d < D; ++d) {
                L.b[d] = small_sm + off;
                off += face_count(G, d);
            }
            if (G.c) {
                L.c = small_sm + off;
                off += (long long)D * G.ncell;
            }
        }
    }
    __syncthreads();
    for (int l = 0; l < nl; ++l) {
        const HLev& G = lv.lev[l];
        small_copy(S[l].a, G.a, G.ncell);
        for (int d = 0; d < D; ++d) small_copy(S[l].b[d], G.b[d], face_count(G, d));
        if (G.c) small_copy(S[l].c, G.c, (long long)D * G.ncell);
    }
    small_copy(S[0].phi, lv.lev[0].phi, lv.lev[0].ncell);
    small_copy(S[0].rhs, lv.lev[0].rhs, lv.lev[0].ncell);
    __syncthreads();
    // the level descriptions in registers (the shared copies would be
    // re-read after every barrier)
    for (int l = 0; l + 1 < nl; ++l) {
        const HLev F = S[l];
        const HLev C = S[l + 1];
        small_sweeps<D>(F, op, nu1);
        const ApplyCoef ac = apply_coef(F, op);
        for (int c = threadIdx.x; c < (int)F.ncell; c += blockDim.x) F.res[c] = apply_value<D>(F, op, ac, F.phi, F.rhs, 1, c);
        __syncthreads();
        for (int c = threadIdx.x; c < (int)C.ncell; c += blockDim.x) restrict_cell<D>(F, C, c);
        __syncthreads();
    }
    small_sweeps<D>(S[nl - 1], op, bottom);
    for (int l = nl - 2; l >= 0; --l) {
        const HLev F = S[l];
        const HLev C = S[l + 1];
        for (int c = threadIdx.x; c < (int)F.ncell; c += blockDim.x) prolong_cell<D>(F, C, c);
        __syncthreads();
        small_sweeps<D>(F, op, nu2);
    }
    small_copy(lv.lev[0].phi, S[0].phi, lv.lev[0].ncell);
}

// averageDownCoeffs: cell coefficients by the mean of the children, face
// coefficients by the mean of the fine faces on each coarse face.
template <int D>
__global__ void coarsen_coeffs_kernel(const HLev F, const HLev C, int has_c)
{
    const double w = D == 3 ? 0.125 : (D == 2 ? 0.25 : 0.5);
    const double wf = D == 3 ? 0.25 : (D == 2 ? 0.5 : 1.0);
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < C.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % C.n[0]);
        const int j = (int)((c / C.n[0]) % C.n[1]);
        const int k = (int)(c / ((long long)C.n[0] * C.n[1]));
        for (int m = -1; m < (has_c ? D : 0); ++m) {
            const double* src = m < 0 ? F.a : F.c + (long long)m * F.ncell;
            double s = 0.0;
            for (int kk = 0; kk < (D > 2 ? 2 : 1); ++kk)
                for (int jj = 0; jj < (D > 1 ? 2 : 1); ++jj)
                    for (int ii = 0; ii < 2; ++ii)
                        s = s + src[cidx(F, 2 * i + ii, D > 1 ? 2 * j + jj : j, D > 2 ? 2 * k + kk : k)];
            if (m < 0) C.a[c] = s * w;
            else C.c[(long long)m * C.ncell + c] = s * w;
        }
        // faces: the low face of this coarse cell in each direction, plus the
        // high face for the last cell of a row
        for (int d = 0; d < D; ++d) {
            for (int hiface = 0; hiface < 2; ++hiface) {
                const int q[3] = { i, j, k };
                if (hiface && q[d] != C.n[d] - 1) continue;
                int cf[3] = { i, j, k };
                cf[d] += hiface;
                double s = 0.0;
                const int e1 = d == 0 ? 1 : 0, e2 = d == 2 ? 1 : 2;
                for (int t2 = 0; t2 < (D > 2 ? 2 : 1); ++t2)
                    for (int t1 = 0; t1 < (D > 1 ? 2 : 1); ++t1) {
                        int f[3];
                        f[d] = 2 * cf[d];
                        f[e1] = (e1 < D) ? 2 * cf[e1] + t1 : cf[e1];
                        f[e2] = (e2 < D && e2 != d) ? 2 * cf[e2] + t2 : cf[e2];
                        s = s + F.b[d][fidx(F, d, f[0], f[1], f[2])];
                    }
                C.b[d][fidx(C, d, cf[0], cf[1], cf[2])] = s * wf;
            }
        }
    }
}

// ---------------------------------------------------------------- vectors
// Deterministic dot product: fixed-grid partials, then one block in a
// fixed tree order.
__global__ void dot_partial_kernel(const double* __restrict__ x, const double* __restrict__ y, long long n,
                                   double* __restrict__ part)
{
    __shared__ double red[kThreads];
    double acc = 0.0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        acc = acc + x[c] * y[c];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void dot_final_kernel(const double* __restrict__ part, int nparts, double* __restrict__ out)
{
    __shared__ double red[kThreads];
    double acc = 0.0;
    for (int q = threadIdx.x; q < nparts; q += blockDim.x) acc = acc + part[q];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// BiCGStab scalars (device resident)
struct KScal {
    double rho, rho_old, alpha, omega, beta;
    double rv, ts, tt, rr, ss, bb;
    int breakdown;
    int pad;
};

__global__ void bicg_p_kernel(double* __restrict__ p, const double* __restrict__ r, const double* __restrict__ v,
                              const KScal* __restrict__ S, long long n)
{
    // p = r + beta (p - omega v), beta = (rho / rho_old) (alpha / omega)
    const double beta = (S->rho / S->rho_old) * (S->alpha / S->omega);
    const double om = S->omega;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        p[c] = r[c] + beta * (p[c] - om * v[c]);
}

__global__ void bicg_s_kernel(double* __restrict__ s, const double* __restrict__ r, const double* __restrict__ v,
                              const KScal* __restrict__ S, long long n)
{
    const double alpha = S->rho / S->rv;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        s[c] = r[c] - alpha * v[c];
}

// x += alpha phat + omega shat; r = s - omega t
__global__ void bicg_xr_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ ph,
                               const double* __restrict__ sh, const double* __restrict__ s,
                               const double* __restrict__ t, const KScal* __restrict__ S, long long n)
{
    const double alpha = S->rho / S->rv;
    const double omega = S->ts / S->tt;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        x[c] = x[c] + alpha * ph[c] + omega * sh[c];
        r[c] = s[c] - omega * t[c];
    }
}

__global__ void bicg_scalars_kernel(KScal* S, int stage)
{
    if (stage == 0) {  // start of an iteration after the first
        S->rho_old = S->rho;
    } else if (stage == 1) {  // after (t,s) and (t,t): omega for the next iteration
        S->alpha = S->rho / S->rv;
        S->omega = S->ts / S->tt;
    }
}

__global__ void copy_kernel(double* __restrict__ d, const double* __restrict__ s, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        d[c] = s[c];
}

__global__ void fill_value_kernel(double* __restrict__ d, double v, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        d[c] = v;
}

__global__ void face_avg_kernel(const double* __restrict__ cc, double* __restrict__ f, int d, int n0, int n1, int n2,
                                int periodic)
{
    const int m[3] = { n0 + (d == 0), n1 + (d == 1), n2 + (d == 2) };
    const long long nf = (long long)m[0] * m[1] * m[2];
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nf;
         q += (long long)gridDim.x * blockDim.x) {
        int p[3] = { (int)(q % m[0]), (int)((q / m[0]) % m[1]), (int)(q / ((long long)m[0] * m[1])) };
        int lo[3] = { p[0], p[1], p[2] }, hi[3] = { p[0], p[1], p[2] };
        const int nd = d == 0 ? n0 : (d == 1 ? n1 : n2);
        lo[d] = p[d] - 1;
        hi[d] = p[d];
        if (lo[d] < 0) lo[d] = periodic ? nd - 1 : 0;
        if (hi[d] >= nd) hi[d] = periodic ? 0 : nd - 1;
        const double vl = cc[(long long)lo[0] + (long long)n0 * ((long long)lo[1] + (long long)n1 * lo[2])];
        const double vh = cc[(long long)hi[0] + (long long)n0 * ((long long)hi[1] + (long long)n1 * hi[2])];
        f[q] = 0.5 * (vl + vh);
    }
}

// ---------------------------------------------------------------- FGMRES
constexpr int kMaxVec = 64;

__global__ void logbeta_cell_kernel(const double* __restrict__ beta, float* __restrict__ lb, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        lb[c] = (float)log(beta[c]);
}

// cell beta as the mean of the cell's 2D faces (for face coefficients given
// directly)
template <int D>
__global__ void logbeta_faces_kernel(const HLev L, float* __restrict__ lb)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < L.ncell;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % L.n[0]);
        const int j = (int)((c / L.n[0]) % L.n[1]);
        const int k = (int)(c / ((long long)L.n[0] * L.n[1]));
        double s = 0.0;
        for (int d = 0; d < D; ++d) {
            const int ih = i + (d == 0), jh = j + (d == 1), kh = k + (d == 2);
            s = s + L.b[d][fidx(L, d, i, j, k)] + L.b[d][fidx(L, d, ih, jh, kh)];
        }
        lb[c] = (float)log(s / (2 * D));
    }
}

__global__ void net_input_kernel(const double* __restrict__ v, double scale, const float* __restrict__ lb,
                                 float* __restrict__ in, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        in[c] = (float)(v[c] * scale);
        in[n + c] = lb[c];
    }
}

__global__ void net_output_kernel(const float* __restrict__ out, double scale, double* __restrict__ z, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        z[c] = (double)out[c] * scale;
}

__global__ void mdot_partial_kernel(const double* __restrict__ V, long long ldv, int nvec, const double* __restrict__ w,
                                    long long n, double* __restrict__ part)
{
    __shared__ double red[kThreads];
    for (int i = 0; i < nvec; ++i) {
        const double* vi = V + (long long)i * ldv;
        double acc = 0.0;
        for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
            acc = acc + vi[c] * w[c];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int s = blockDim.x / 2; s > 0; s >>= 1) {
            if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * kMaxVec + i] = red[0];
        __syncthreads();
    }
}

__global__ void mdot_final_kernel(const double* __restrict__ part, int nblocks, double* __restrict__ out, int accumulate)
{
    __shared__ double red[kThreads];
    const int i = blockIdx.x;
    double acc = 0.0;
    for (int q = threadIdx.x; q < nblocks; q += blockDim.x) acc = acc + part[(long long)q * kMaxVec + i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = red[threadIdx.x] + red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[i] = accumulate ? out[i] + red[0] : red[0];
}

// w += sign * sum_i h[i] V_i
__global__ void mupdate_kernel(double* __restrict__ w, const double* __restrict__ V, long long ldv, int nvec,
                               const double* __restrict__ h, double sign, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int i = 0; i < nvec; ++i) s = s + h[i] * V[(long long)i * ldv + c];
        w[c] = w[c] + sign * s;
    }
}

__global__ void scale_add_kernel(double* __restrict__ d, const double* __restrict__ src, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        d[c] = d[c] + src[c];
}

__global__ void scale_kernel(double* __restrict__ d, const double* __restrict__ src, double a, long long n)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        d[c] = a * src[c];
}

int grid_for(long long n)
{
    const long long want = (n + kThreads - 1) / kThreads;
    return (int)std::max(1LL, std::min(want, (long long)device_sm_count() * 8));
}

}  // namespace

struct bamrex_helmholtz {
    int D = 2;
    HOp op;
    bool staged_smoother = true;  // 2D fused sweeps with cp.async-staged tiles
    bool small_cycle = true;      // levels of <= 1024 cells cycled by one block in shared memory
    int nu1 = 2, nu2 = 2, bottom = 16;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<HLev> lev;
    char* arena = nullptr;
    bool has_c = false;
    bool coeffs_dirty = true;
    // Krylov vectors on the finest level
    double *x = nullptr, *r = nullptr, *rh = nullptr, *p = nullptr, *v = nullptr, *ph = nullptr, *s = nullptr,
           *sh = nullptr, *t = nullptr, *bvec = nullptr;
    double* part = nullptr;
    KScal* d_scal = nullptr;
    KScal* h_scal = nullptr;  // pinned
    std::vector<double*> cbufs;  // per level, D * ncell: the C coefficients
    // learned-preconditioner solve
    float* logbeta = nullptr;    // log of the cell beta (network input)
    double* krylov = nullptr;    // FGMRES: V (m + 1 vectors) then Z (m vectors)
    int krylov_m = 0;
    double* mpart = nullptr;     // multi-dot partials (kDotBlocks x kMaxVec)
    double* hdev = nullptr;      // multi-dot results (kMaxVec + 1)
    cudaGraphExec_t iter_graph = nullptr;
    long long launches = 0;
    std::string err;
};

namespace {

int hfail(bamrex_helmholtz* H, int code, const std::string& msg)
{
    const int rc = fail(code, msg);
    if (H) H->err = last_error_text();
    return rc;
}

int hck(bamrex_helmholtz* H, cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        const int rc = cuda_fail(e, what);
        H->err = last_error_text();
        return rc;
    }
    H->launches++;
    return BAMREX_OK;
}

#define H_TRY(call)                       \
    do {                                  \
        int rc_ = (call);                 \
        if (rc_ != BAMREX_OK) return rc_; \
    } while (0)

int launch_apply(bamrex_helmholtz* H, int l, const double* x, double* y, const double* rhs, int mode)
{
    const HLev& L = H->lev[l];
    const int g = grid_for(L.ncell);
    if (H->D == 3) apply_kernel<3><<<g, kThreads, 0, H->stream>>>(L, H->op, x, y, rhs, mode);
    else apply_kernel<2><<<g, kThreads, 0, H->stream>>>(L, H->op, x, y, rhs, mode);
    return hck(H, cudaGetLastError(), "helmholtz apply");
}

int launch_gsrb(bamrex_helmholtz* H, int l, int color)
{
    const HLev& L = H->lev[l];
    const int g = grid_for((L.ncell + 1) / 2);
    if (H->D == 3) gsrb_kernel<3><<<g, kThreads, 0, H->stream>>>(L, H->op, L.phi, L.rhs, color);
    else gsrb_kernel<2><<<g, kThreads, 0, H->stream>>>(L, H->op, L.phi, L.rhs, color);
    return hck(H, cudaGetLastError(), "helmholtz gsrb");
}

int smooth(bamrex_helmholtz* H, int l, int sweeps)
{
    const HLev& L = H->lev[l];
    const bool fused = H->D == 2 && L.n[0] % kGsTX == 0 && L.n[1] % kGsTY == 0;
    if (fused) {
        // ping-pong between phi and tmp; an odd count ends with a copy back
        const int tiles = (L.n[0] / kGsTX) * (L.n[1] / kGsTY);
        const int g = std::max(1, std::min(tiles, device_sm_count() * 8));
        // tiles staged by cp.async where the operator has no gradient term
        const bool staged = L.c == nullptr && H->staged_smoother;
        if (staged) {
            static bool attr_set[64] = { false };
            int dev = 0;
            cudaGetDevice(&dev);
            if (!attr_set[dev & 63]) {
                H_TRY(hck(H, cudaFuncSetAttribute(gsrb2_staged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  kGsStagedSmem),
                          "smoother shared memory"));
                attr_set[dev & 63] = true;
            }
        }
        const int gs = std::max(1, std::min(tiles, device_sm_count() * 3));
        for (int s = 0; s < sweeps; ++s) {
            const double* in = (s & 1) ? L.tmp : L.phi;
            double* out = (s & 1) ? L.phi : L.tmp;
            if (staged)
                gsrb2_staged_kernel<<<gs, 256, kGsStagedSmem, H->stream>>>(L, H->op, in, out, L.rhs);
            else
                gsrb2_fused_kernel<<<g, 256, 0, H->stream>>>(L, H->op, in, out, L.rhs);
            H_TRY(hck(H, cudaGetLastError(), "helmholtz gsrb (fused)"));
        }
        if (sweeps & 1)
            H_TRY(hck(H, cudaMemcpyAsync(L.phi, L.tmp, sizeof(double) * L.ncell, cudaMemcpyDeviceToDevice, H->stream),
                      "smoother copy"));
        return BAMREX_OK;
    }
    for (int s = 0; s < sweeps; ++s) {
        H_TRY(launch_gsrb(H, l, 0));
        H_TRY(launch_gsrb(H, l, 1));
    }
    return BAMREX_OK;
}

int vcycle(bamrex_helmholtz* H, int l)
{
    const int nl = (int)H->lev.size();
    if (H->small_cycle && H->lev[l].ncell <= kSmallCells && nl - l <= kSmallLevels) {
        // the rest of the cycle in one block, its levels in shared memory
        HLevs lv;
        lv.n = nl - l;
        long long doubles = 0;
        for (int q = l; q < nl; ++q) {
            lv.lev[q - l] = H->lev[q];
            doubles += small_level_doubles(H->lev[q], H->D);
        }
        const long long bytes = doubles * (long long)sizeof(double);
        if (bytes <= kSmallSmemMax) {
            static bool attr_set[2][64] = { { false } };
            int dev = 0;
            cudaGetDevice(&dev);
            const void* fn = H->D == 3 ? (const void*)vcycle_small_kernel<3> : (const void*)vcycle_small_kernel<2>;
            if (!attr_set[H->D == 3][dev & 63]) {
                H_TRY(hck(H, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmallSmemMax),
                          "coarse V-cycle shared memory"));
                attr_set[H->D == 3][dev & 63] = true;
            }
            if (H->D == 3)
                vcycle_small_kernel<3><<<1, kSmallThreads, (size_t)bytes, H->stream>>>(lv, H->op, H->nu1, H->nu2, H->bottom);
            else
                vcycle_small_kernel<2><<<1, kSmallThreads, (size_t)bytes, H->stream>>>(lv, H->op, H->nu1, H->nu2, H->bottom);
            return hck(H, cudaGetLastError(), "coarse V-cycle");
        }
    }
    if (l == nl - 1) return smooth(H, l, H->bottom);
    H_TRY(smooth(H, l, H->nu1));
    const HLev& F = H->lev[l];
    const HLev& C = H->lev[l + 1];
    H_TRY(launch_apply(H, l, F.phi, F.res, F.rhs, 1));
    const int g = grid_for(C.ncell);
    if (H->D == 3) restrict_kernel<3><<<g, kThreads, 0, H->stream>>>(F, C);
    else restrict_kernel<2><<<g, kThreads, 0, H->stream>>>(F, C);
    H_TRY(hck(H, cudaGetLastError(), "restrict"));
    H_TRY(vcycle(H, l + 1));
    const int gf = grid_for(F.ncell);
    if (H->D == 3) prolong_kernel<3><<<gf, kThreads, 0, H->stream>>>(F, C);
    else prolong_kernel<2><<<gf, kThreads, 0, H->stream>>>(F, C);
    H_TRY(hck(H, cudaGetLastError(), "prolong"));
    return smooth(H, l, H->nu2);
}

int coarsen_coeffs(bamrex_helmholtz* H)
{
    for (size_t l = 1; l < H->lev.size(); ++l) {
        const int g = grid_for(H->lev[l].ncell);
        if (H->D == 3) coarsen_coeffs_kernel<3><<<g, kThreads, 0, H->stream>>>(H->lev[l - 1], H->lev[l], H->has_c);
        else coarsen_coeffs_kernel<2><<<g, kThreads, 0, H->stream>>>(H->lev[l - 1], H->lev[l], H->has_c);
        H_TRY(hck(H, cudaGetLastError(), "coarsen coefficients"));
    }
    H->coeffs_dirty = false;
    return BAMREX_OK;
}

int dot(bamrex_helmholtz* H, const double* x, const double* y, double* out)
{
    const long long n = H->lev[0].ncell;
    dot_partial_kernel<<<kDotBlocks, kThreads, 0, H->stream>>>(x, y, n, H->part);
    H_TRY(hck(H, cudaGetLastError(), "dot partial"));
    dot_final_kernel<<<1, kThreads, 0, H->stream>>>(H->part, kDotBlocks, out);
    return hck(H, cudaGetLastError(), "dot final");
}

int copy_vec(bamrex_helmholtz* H, double* d, const double* s)
{
    const long long n = H->lev[0].ncell;
    copy_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(d, s, n);
    return hck(H, cudaGetLastError(), "copy");
}

// z = M y: one V-cycle from a zero guess
int precondition(bamrex_helmholtz* H, double* z, const double* y)
{
    const HLev& F = H->lev[0];
    H_TRY(copy_vec(H, F.rhs, y));
    H_TRY(hck(H, cudaMemsetAsync(F.phi, 0, sizeof(double) * F.ncell, H->stream), "memset"));
    H_TRY(vcycle(H, 0));
    return copy_vec(H, z, F.phi);
}

// One BiCGStab iteration (right preconditioning), all scalars on the device.
int bicg_iteration(bamrex_helmholtz* H)
{
    const long long n = H->lev[0].ncell;
    const int g = grid_for(n);
    KScal* S = H->d_scal;
    bicg_scalars_kernel<<<1, 1, 0, H->stream>>>(S, 0);
    H_TRY(hck(H, cudaGetLastError(), "scalars"));
    H_TRY(dot(H, H->rh, H->r, &S->rho));
    bicg_p_kernel<<<g, kThreads, 0, H->stream>>>(H->p, H->r, H->v, S, n);
    H_TRY(hck(H, cudaGetLastError(), "bicg p"));
    H_TRY(precondition(H, H->ph, H->p));
    H_TRY(launch_apply(H, 0, H->ph, H->v, nullptr, 0));
    H_TRY(dot(H, H->rh, H->v, &S->rv));
    bicg_s_kernel<<<g, kThreads, 0, H->stream>>>(H->s, H->r, H->v, S, n);
    H_TRY(hck(H, cudaGetLastError(), "bicg s"));
    H_TRY(precondition(H, H->sh, H->s));
    H_TRY(launch_apply(H, 0, H->sh, H->t, nullptr, 0));
    H_TRY(dot(H, H->t, H->s, &S->ts));
    H_TRY(dot(H, H->t, H->t, &S->tt));
    bicg_xr_kernel<<<g, kThreads, 0, H->stream>>>(H->x, H->r, H->ph, H->sh, H->s, H->t, S, n);
    H_TRY(hck(H, cudaGetLastError(), "bicg xr"));
    bicg_scalars_kernel<<<1, 1, 0, H->stream>>>(S, 1);
    H_TRY(hck(H, cudaGetLastError(), "scalars"));
    return dot(H, H->r, H->r, &S->rr);
}

bool is_device_ptr(const void* p)
{
    cudaPointerAttributes at;
    const bool dev = cudaPointerGetAttributes(&at, p) == cudaSuccess &&
                     (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    return dev;
}

int upload(bamrex_helmholtz* H, double* dst, const double* src, size_t n)
{
    return hck(H, cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDefault, H->stream), "coefficient copy");
}

}  // namespace

extern "C" int bamrex_helmholtz_create(bamrex_helmholtz** out, const bamrex_helmholtz_desc* d, void* stream)
{
    if (!out || !d) return fail(BAMREX_ERR_ARG, "NULL argument");
    *out = nullptr;
    const int D = d->spacedim;
    if (D != 2 && D != 3) return fail(BAMREX_ERR_ARG, "spacedim must be 2 or 3");
    for (int q = 0; q < D; ++q) {
        if (d->n[q] < 2) return fail(BAMREX_ERR_ARG, "at least two cells per direction");
        if (!(d->prob_hi[q] > d->prob_lo[q])) return fail(BAMREX_ERR_ARG, "prob_hi must exceed prob_lo");
        for (int s = 0; s < 2; ++s) {
            const int bc = s ? d->bc_hi[q] : d->bc_lo[q];
            if (bc < BAMREX_LINOP_PERIODIC || bc > BAMREX_LINOP_DIRICHLET) return fail(BAMREX_ERR_ARG, "unknown boundary type");
        }
        if ((d->bc_lo[q] == BAMREX_LINOP_PERIODIC) != (d->bc_hi[q] == BAMREX_LINOP_PERIODIC))
            return fail(BAMREX_ERR_ARG, "periodic boundaries must be set on both sides");
    }
    std::unique_ptr<bamrex_helmholtz> H(new (std::nothrow) bamrex_helmholtz());
    if (!H) return fail(BAMREX_ERR_OOM, "host allocation failed");
    H->D = D;
    H->op.ascal = 1.0;
    H->op.bscal = 1.0;
    H->op.cscal = 0.0;
    for (int q = 0; q < 3; ++q) {
        H->op.bc_lo[q] = q < D ? d->bc_lo[q] : BAMREX_LINOP_PERIODIC;
        H->op.bc_hi[q] = q < D ? d->bc_hi[q] : BAMREX_LINOP_PERIODIC;
    }
    H->nu1 = d->nu1 > 0 ? d->nu1 : 2;
    H->nu2 = d->nu2 > 0 ? d->nu2 : 2;
    H->bottom = d->bottom_sweeps > 0 ? d->bottom_sweeps : 16;
    // levels: halve every direction while all are even and >= 4
    int n[3] = { d->n[0], d->n[1], D > 2 ? d->n[2] : 1 };
    double dx[3];
    for (int q = 0; q < 3; ++q) dx[q] = q < D ? (d->prob_hi[q] - d->prob_lo[q]) / n[q] : 1.0;
    const int maxl = d->max_levels > 0 ? d->max_levels : 64;
    for (int l = 0; l < maxl; ++l) {
        HLev L;
        std::memset(&L, 0, sizeof(L));
        for (int q = 0; q < 3; ++q) {
            L.n[q] = n[q];
            L.dx[q] = dx[q];
        }
        L.ncell = (long long)n[0] * n[1] * n[2];
        H->lev.push_back(L);
        bool can = true;
        for (int q = 0; q < D; ++q) can = can && n[q] % 2 == 0 && n[q] >= 4;
        if (!can) break;
        for (int q = 0; q < D; ++q) {
            n[q] /= 2;
            dx[q] *= 2;
        }
    }
    // one arena: per level a, b[D], c[D], phi, rhs, res; Krylov vectors; partials
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + std::max<size_t>(bytes, 8), 256);
        return o;
    };
    struct Offs {
        size_t a, b[3], c, phi, rhs, res, tmp;
    };
    std::vector<Offs> lo(H->lev.size());
    for (size_t l = 0; l < H->lev.size(); ++l) {
        const HLev& L = H->lev[l];
        lo[l].a = take(sizeof(double) * L.ncell);
        for (int q = 0; q < 3; ++q) {
            const long long nf = (long long)(L.n[0] + (q == 0)) * (L.n[1] + (q == 1)) * (L.n[2] + (q == 2));
            lo[l].b[q] = q < D ? take(sizeof(double) * nf) : 0;
        }
        lo[l].c = take(sizeof(double) * D * L.ncell);
        lo[l].phi = take(sizeof(double) * L.ncell);
        lo[l].rhs = take(sizeof(double) * L.ncell);
        lo[l].res = take(sizeof(double) * L.ncell);
        lo[l].tmp = take(sizeof(double) * L.ncell);
    }
    const long long n0 = H->lev[0].ncell;
    size_t ov[10];
    for (int q = 0; q < 10; ++q) ov[q] = take(sizeof(double) * n0);
    const size_t opart = take(sizeof(double) * kDotBlocks);
    const size_t oscal = take(sizeof(KScal));
    cudaError_t e = cudaMalloc((void**)&H->arena, off);
    if (e != cudaSuccess) return fail(BAMREX_ERR_OOM, std::string("cudaMalloc of the Helmholtz arena failed: ") + cudaGetErrorString(e));
    e = cudaMallocHost((void**)&H->h_scal, sizeof(KScal));
    if (e != cudaSuccess) {
        cudaFree(H->arena);
        return fail(BAMREX_ERR_OOM, "cudaMallocHost failed");
    }
    char* A = H->arena;
    for (size_t l = 0; l < H->lev.size(); ++l) {
        HLev& L = H->lev[l];
        L.a = (double*)(A + lo[l].a);
        for (int q = 0; q < 3; ++q) L.b[q] = q < D ? (double*)(A + lo[l].b[q]) : nullptr;
        L.c = nullptr;  // set when C coefficients are given
        L.phi = (double*)(A + lo[l].phi);
        L.rhs = (double*)(A + lo[l].rhs);
        L.res = (double*)(A + lo[l].res);
        L.tmp = (double*)(A + lo[l].tmp);
    }
    std::vector<double*> cbuf(H->lev.size());
    for (size_t l = 0; l < H->lev.size(); ++l) cbuf[l] = (double*)(A + lo[l].c);
    double** vv[10] = { &H->x, &H->r, &H->rh, &H->p, &H->v, &H->ph, &H->s, &H->sh, &H->t, &H->bvec };
    for (int q = 0; q < 10; ++q) *vv[q] = (double*)(A + ov[q]);
    H->part = (double*)(A + opart);
    H->d_scal = (KScal*)(A + oscal);
    e = cudaMemset(H->arena, 0, off);
    if (e != cudaSuccess) {
        cudaFree(H->arena);
        cudaFreeHost(H->h_scal);
        return cuda_fail(e, "memset");
    }
    H->cbufs = cbuf;
    if (stream) {
        H->stream = (cudaStream_t)stream;
    } else {
        e = cudaStreamCreateWithFlags(&H->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            cudaFree(H->arena);
            cudaFreeHost(H->h_scal);
            return cuda_fail(e, "cudaStreamCreateWithFlags");
        }
        H->own_stream = true;
    }
    e = cudaMalloc((void**)&H->logbeta, sizeof(float) * n0);
    if (e == cudaSuccess) e = cudaMalloc((void**)&H->mpart, sizeof(double) * ((size_t)kDotBlocks * kMaxVec + kMaxVec + 1));
    if (e != cudaSuccess) {
        cudaFree(H->arena);
        cudaFreeHost(H->h_scal);
        if (H->logbeta) cudaFree(H->logbeta);
        if (H->own_stream) cudaStreamDestroy(H->stream);
        return fail(BAMREX_ERR_OOM, "cudaMalloc of the Krylov workspace failed");
    }
    H->hdev = H->mpart + (size_t)kDotBlocks * kMaxVec;
    cudaMemset(H->logbeta, 0, sizeof(float) * n0);  // log(1): the default b = 1
    // default coefficients: a = 1, b = 1
    for (size_t l = 0; l < H->lev.size(); ++l) {
        HLev& L = H->lev[l];
        std::vector<double> ones((size_t)L.ncell, 1.0);
        cudaMemcpy(L.a, ones.data(), sizeof(double) * L.ncell, cudaMemcpyHostToDevice);
        for (int q = 0; q < D; ++q) {
            const long long nf = (long long)(L.n[0] + (q == 0)) * (L.n[1] + (q == 1)) * (L.n[2] + (q == 2));
            std::vector<double> fo((size_t)nf, 1.0);
            cudaMemcpy(L.b[q], fo.data(), sizeof(double) * nf, cudaMemcpyHostToDevice);
        }
    }
    // the default-stream memsets and copies above are complete before any
    // kernel on the operator's (non-blocking) stream reads them
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cuda_fail(e, "set-up");
    *out = H.release();
    return BAMREX_OK;
}

extern "C" int bamrex_helmholtz_destroy(bamrex_helmholtz* H)
{
    if (!H) return BAMREX_OK;
    if (H->stream) cudaStreamSynchronize(H->stream);
    if (H->iter_graph) cudaGraphExecDestroy(H->iter_graph);
    if (H->krylov) cudaFree(H->krylov);
    if (H->logbeta) cudaFree(H->logbeta);
    if (H->mpart) cudaFree(H->mpart);
    if (H->arena) cudaFree(H->arena);
    if (H->h_scal) cudaFreeHost(H->h_scal);
    if (H->own_stream) cudaStreamDestroy(H->stream);
    delete H;
    return BAMREX_OK;
}

extern "C" const char* bamrex_helmholtz_last_error(const bamrex_helmholtz* H) { return H ? H->err.c_str() : ""; }

extern "C" int bamrex_helmholtz_num_levels(const bamrex_helmholtz* H) { return H ? (int)H->lev.size() : 0; }

extern "C" int bamrex_helmholtz_set_scalars(bamrex_helmholtz* H, double a, double b, double c)
{
    if (!H) return fail(BAMREX_ERR_ARG, "NULL operator");
    H->op.ascal = a;
    H->op.bscal = b;
    H->op.cscal = c;
    if (H->iter_graph) {
        cudaGraphExecDestroy(H->iter_graph);
        H->iter_graph = nullptr;
    }
    return BAMREX_OK;
}

extern "C" int bamrex_helmholtz_set_acoeffs(bamrex_helmholtz* H, const double* alpha, double alpha_const)
{
    if (!H) return fail(BAMREX_ERR_ARG, "NULL operator");
    HLev& L = H->lev[0];
    if (alpha) {
        H_TRY(upload(H, L.a, alpha, (size_t)L.ncell));
    } else {
        fill_value_kernel<<<grid_for(L.ncell), kThreads, 0, H->stream>>>(L.a, alpha_const, L.ncell);
        H_TRY(hck(H, cudaGetLastError(), "a coefficients"));
    }
    H->coeffs_dirty = true;
    return BAMREX_OK;
}

extern "C" int bamrex_helmholtz_set_bcoeffs(bamrex_helmholtz* H, const double* bx, const double* by, const double* bz)
{
    if (!H) return fail(BAMREX_ERR_ARG, "NULL operator");
    const double* src[3] = { bx, by, bz };
    HLev& L = H->lev[0];
    for (int q = 0; q < H->D; ++q) {
        if (!src[q]) return hfail(H, BAMREX_ERR_ARG, "missing face coefficients");
        const long long nf = (long long)(L.n[0] + (q == 0)) * (L.n[1] + (q == 1)) * (L.n[2] + (q == 2));
        H_TRY(upload(H, L.b[q], src[q], (size_t)nf));
    }
    if (H->logbeta) {
        if (H->D == 3) logbeta_faces_kernel<3><<<grid_for(L.ncell), kThreads, 0, H->stream>>>(L, H->logbeta);
        else logbeta_faces_kernel<2><<<grid_for(L.ncell), kThreads, 0, H->stream>>>(L, H->logbeta);
        H_TRY(hck(H, cudaGetLastError(), "log beta"));
    }
    H->coeffs_dirty = true;
    return BAMREX_OK;
}

extern "C" int bamrex_helmholtz_set_bcoeffs_from_cell(bamrex_helmholtz* H, const double* beta_cc)
{
    if (!H || !beta_cc) return fail(BAMREX_ERR_ARG, "NULL argument");
    HLev& L = H->lev[0];
    const double* src = beta_cc;
    if (!is_device_ptr(beta_cc)) {
        H_TRY(upload(H, H->bvec, beta_cc, (size_t)L.ncell));
        src = H->bvec;
    }
    for (int q = 0; q < H->D; ++q) {
        const long long nf = (long long)(L.n[0] + (q == 0)) * (L.n[1] + (q == 1)) * (L.n[2] + (q == 2));
        face_avg_kernel<<<grid_for(nf), kThreads, 0, H->stream>>>(src, L.b[q], q, L.n[0], L.n[1], L.n[2],
                                                                 H->op.bc_lo[q] == BAMREX_LINOP_PERIODIC);
        H_TRY(hck(H, cudaGetLastError(), "face average"));
    }
    if (H->logbeta) {
        logbeta_cell_kernel<<<grid_for(L.ncell), kThreads, 0, H->stream>>>(src, H->logbeta, L.ncell);
        H_TRY(hck(H, cudaGetLastError(), "log beta"));
    }
    H->coeffs_dirty = true;
    return BAMREX_OK;
}

extern "C" int bamrex_helmholtz_set_ccoeffs(bamrex_helmholtz* H, const double* c)
{
    if (!H) return fail(BAMREX_ERR_ARG, "NULL operator");
    if (!c) {
        for (auto& L : H->lev) L.c = nullptr;
        H->has_c = false;
    } else {
        for (size_t l = 0; l < H->lev.size(); ++l) H->lev[l].c = H->cbufs[l];
        H_TRY(upload(H, H->lev[0].c, c, (size_t)H->D * H->lev[0].ncell));
        H->has_c = true;
    }
    if (H->iter_graph) {
        cudaGraphExecDestroy(H->iter_graph);
        H->iter_graph = nullptr;
    }
    H->coeffs_dirty = true;
    return BAMREX_OK;
}

static int prepare(bamrex_helmholtz* H)
{
    if (H->coeffs_dirty) {
        H_TRY(coarsen_coeffs(H));
        if (H->iter_graph) {
            cudaGraphExecDestroy(H->iter_graph);
            H->iter_graph = nullptr;
        }
    }
    return BAMREX_OK;
}

// In/out vectors may be host or device memory: host data go through the
// finest level's work vectors.
extern "C" int bamrex_helmholtz_apply(bamrex_helmholtz* H, const double* x, double* y)
{
    if (!H || !x || !y) return fail(BAMREX_ERR_ARG, "NULL argument");
    const long long n = H->lev[0].ncell;
    const bool dx = is_device_ptr(x), dy = is_device_ptr(y);
    const double* xi = x;
    if (!dx) {
        H_TRY(upload(H, H->p, x, (size_t)n));
        xi = H->p;
    }
    double* yo = dy ? y : H->v;
    H_TRY(launch_apply(H, 0, xi, yo, nullptr, 0));
    if (!dy) H_TRY(hck(H, cudaMemcpyAsync(y, yo, sizeof(double) * n, cudaMemcpyDeviceToHost, H->stream), "copy out"));
    return hck(H, cudaStreamSynchronize(H->stream), "sync");
}

extern "C" int bamrex_helmholtz_smooth(bamrex_helmholtz* H, double* phi, const double* rhs, int redblack)
{
    if (!H || !phi || !rhs) return fail(BAMREX_ERR_ARG, "NULL argument");
    HLev& L = H->lev[0];
    const long long n = L.ncell;
    H_TRY(upload(H, L.phi, phi, (size_t)n));
    H_TRY(upload(H, L.rhs, rhs, (size_t)n));
    H_TRY(launch_gsrb(H, 0, redblack & 1));
    H_TRY(hck(H, cudaMemcpyAsync(phi, L.phi, sizeof(double) * n, cudaMemcpyDefault, H->stream), "copy out"));
    return hck(H, cudaStreamSynchronize(H->stream), "sync");
}

extern "C" int bamrex_helmholtz_vcycle(bamrex_helmholtz* H, double* z, const double* r)
{
    if (!H || !z || !r) return fail(BAMREX_ERR_ARG, "NULL argument");
    H_TRY(prepare(H));
    const long long n = H->lev[0].ncell;
    H_TRY(upload(H, H->s, r, (size_t)n));
    H_TRY(precondition(H, H->sh, H->s));
    H_TRY(hck(H, cudaMemcpyAsync(z, H->sh, sizeof(double) * n, cudaMemcpyDefault, H->stream), "copy out"));
    return hck(H, cudaStreamSynchronize(H->stream), "sync");
}

extern "C" int bamrex_helmholtz_solve(bamrex_helmholtz* H, double* x, const double* rhs, double tol_rel, double tol_abs,
                                      int max_iter, int use_graph, int* iters, double* rel_res)
{
    if (!H || !x || !rhs) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (max_iter < 1) return hfail(H, BAMREX_ERR_ARG, "max_iter must be >= 1");
    H_TRY(prepare(H));
    const long long n = H->lev[0].ncell;
    KScal* S = H->d_scal;
    H_TRY(upload(H, H->x, x, (size_t)n));
    H_TRY(upload(H, H->bvec, rhs, (size_t)n));
    // r = b - A x, rhat = r; rho = alpha = omega = 1, p = v = 0
    H_TRY(launch_apply(H, 0, H->x, H->r, H->bvec, 1));
    H_TRY(copy_vec(H, H->rh, H->r));
    H_TRY(hck(H, cudaMemsetAsync(H->p, 0, sizeof(double) * n, H->stream), "memset"));
    H_TRY(hck(H, cudaMemsetAsync(H->v, 0, sizeof(double) * n, H->stream), "memset"));
    KScal init;
    std::memset(&init, 0, sizeof(init));
    init.rho = init.alpha = init.omega = init.rv = init.ts = init.tt = 1.0;
    *H->h_scal = init;
    H_TRY(hck(H, cudaMemcpyAsync(S, H->h_scal, sizeof(KScal), cudaMemcpyHostToDevice, H->stream), "scalars"));
    H_TRY(dot(H, H->bvec, H->bvec, &S->bb));
    H_TRY(dot(H, H->r, H->r, &S->rr));
    H_TRY(hck(H, cudaMemcpyAsync(H->h_scal, S, sizeof(KScal), cudaMemcpyDeviceToHost, H->stream), "scalars"));
    H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
    const double bnorm = std::sqrt(H->h_scal->bb);
    double rnorm = std::sqrt(H->h_scal->rr);
    const double target = std::max(tol_rel * bnorm, tol_abs);
    int it = 0;
    while (rnorm > target && it < max_iter) {
        if (use_graph) {
            if (!H->iter_graph) {
                cudaGraph_t g = nullptr;
                H_TRY(hck(H, cudaStreamBeginCapture(H->stream, cudaStreamCaptureModeThreadLocal), "begin capture"));
                const long long before = H->launches;
                const int rc = bicg_iteration(H);
                cudaError_t e = cudaStreamEndCapture(H->stream, &g);
                if (rc != BAMREX_OK) {
                    if (g) cudaGraphDestroy(g);
                    return rc;
                }
                H_TRY(hck(H, e, "end capture"));
                H->launches = before;
                e = cudaGraphInstantiate(&H->iter_graph, g, 0);
                cudaGraphDestroy(g);
                H_TRY(hck(H, e, "graph instantiate"));
            }
            H_TRY(hck(H, cudaGraphLaunch(H->iter_graph, H->stream), "graph launch"));
        } else {
            H_TRY(bicg_iteration(H));
        }
        H_TRY(hck(H, cudaMemcpyAsync(H->h_scal, S, sizeof(KScal), cudaMemcpyDeviceToHost, H->stream), "scalars"));
        H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
        ++it;
        rnorm = std::sqrt(H->h_scal->rr);
        if (!std::isfinite(rnorm)) return hfail(H, BAMREX_ERR_NAN, "BiCGStab breakdown (non-finite residual)");
    }
    H_TRY(hck(H, cudaMemcpyAsync(x, H->x, sizeof(double) * n, cudaMemcpyDefault, H->stream), "copy out"));
    H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
    if (iters) *iters = it;
    if (rel_res) *rel_res = bnorm > 0 ? rnorm / bnorm : rnorm;
    return BAMREX_OK;
}

extern "C" long long bamrex_helmholtz_launches(const bamrex_helmholtz* H) { return H ? H->launches : 0; }

// ---------------------------------------------------------------- learned
namespace {

int mdot(bamrex_helmholtz* H, const double* V, long long ldv, int nvec, const double* w, double* out, int accumulate)
{
    const long long n = H->lev[0].ncell;
    mdot_partial_kernel<<<kDotBlocks, kThreads, 0, H->stream>>>(V, ldv, nvec, w, n, H->mpart);
    H_TRY(hck(H, cudaGetLastError(), "multi-dot partial"));
    mdot_final_kernel<<<nvec, kThreads, 0, H->stream>>>(H->mpart, kDotBlocks, out, accumulate);
    return hck(H, cudaGetLastError(), "multi-dot final");
}

// z = M v with the network: input (v / rms(v), log beta), output scaled by
// rms(v) dx0 dx1 / B.  rms_v is known on the host.
int net_precondition(bamrex_helmholtz* H, bamrex_precnet* N, const double* v, double rms_v, double* z)
{
    const HLev& L = H->lev[0];
    const long long n = L.ncell;
    float* in = precnet_input(N);
    net_input_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(v, 1.0 / rms_v, H->logbeta, in, n);
    H_TRY(hck(H, cudaGetLastError(), "network input"));
    const int rc = precnet_run(N, H->stream);
    if (rc != BAMREX_OK) {
        H->err = last_error_text();
        return rc;
    }
    H->launches += 20;
    const double scale = rms_v * L.dx[0] * L.dx[1] / H->op.bscal;
    net_output_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(precnet_output(N), scale, z, n);
    return hck(H, cudaGetLastError(), "network output");
}

}  // namespace

extern "C" int bamrex_helmholtz_solve_learned(bamrex_helmholtz* H, bamrex_precnet* N, int mode, double* x,
                                              const double* rhs, double tol_rel, double tol_abs, int max_iter, int restart,
                                              int* iters, int* plain_iters, double* rel_res, int* fell_back)
{
    if (!H || !x || !rhs) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (mode < BAMREX_PRECOND_NETWORK || mode > BAMREX_PRECOND_VCYCLE_NETWORK) return hfail(H, BAMREX_ERR_ARG, "unknown mode");
    if (!N && mode != BAMREX_PRECOND_VCYCLE) return hfail(H, BAMREX_ERR_ARG, "the mode needs a network");
    if (H->D != 2) return hfail(H, BAMREX_ERR_UNSUPPORTED, "the learned preconditioner is two-dimensional");
    if (restart < 1 || restart + 1 > kMaxVec) return hfail(H, BAMREX_ERR_ARG, "restart must be in [1, 63]");
    if (max_iter < 0) return hfail(H, BAMREX_ERR_ARG, "max_iter must be >= 0");
    const HLev& L = H->lev[0];
    if (N) {
        int nnx, nny, nb;
        precnet_size(N, &nnx, &nny, &nb);
        if (nnx != L.n[0] || nny != L.n[1] || nb != 1)
            return hfail(H, BAMREX_ERR_ARG, "the network workspace must match the operator grid with batch 1");
    }
    for (int q = 0; q < 2 && N; ++q)
        if (H->op.bc_lo[q] != BAMREX_LINOP_PERIODIC)
            return hfail(H, BAMREX_ERR_UNSUPPORTED, "the network pads periodically: periodic domains only");
    H_TRY(prepare(H));
    const long long n = L.ncell;
    const int m = restart;
    if (H->krylov_m < m) {
        if (H->krylov) cudaFree(H->krylov);
        H->krylov = nullptr;
        H->krylov_m = 0;
        const cudaError_t e = cudaMalloc((void**)&H->krylov, sizeof(double) * (size_t)n * (2 * m + 1));
        if (e != cudaSuccess) return hfail(H, BAMREX_ERR_OOM, "cudaMalloc of the FGMRES basis failed");
        H->krylov_m = m;
    }
    double* V = H->krylov;
    double* Z = H->krylov + (size_t)n * (m + 1);
    double* hd = H->hdev;
    H_TRY(upload(H, H->x, x, (size_t)n));
    H_TRY(upload(H, H->bvec, rhs, (size_t)n));
    H_TRY(dot(H, H->bvec, H->bvec, &hd[0]));
    double hb = 0;
    H_TRY(hck(H, cudaMemcpyAsync(&hb, hd, sizeof(double), cudaMemcpyDeviceToHost, H->stream), "copy"));
    H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
    const double bnorm = std::sqrt(hb);
    const double target = std::max(tol_rel * bnorm, tol_abs);
    const double rms_unit = 1.0 / std::sqrt((double)n);  // rms of a unit vector
    std::vector<double> Hm((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), hv(kMaxVec + 1);
    int total = 0;
    double rnorm = 0.0;
    for (;;) {
        // r = b - A x into V_0, beta = ||r||
        H_TRY(launch_apply(H, 0, H->x, V, H->bvec, 1));
        H_TRY(dot(H, V, V, &hd[0]));
        H_TRY(hck(H, cudaMemcpyAsync(&hb, hd, sizeof(double), cudaMemcpyDeviceToHost, H->stream), "copy"));
        H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
        rnorm = std::sqrt(hb);
        if (rnorm <= target || total >= max_iter || !std::isfinite(rnorm)) break;
        scale_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(V, V, 1.0 / rnorm, n);
        H_TRY(hck(H, cudaGetLastError(), "scale"));
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = rnorm;
        int k = 0;
        for (int j = 0; j < m && total < max_iter; ++j) {
            double* vj = V + (size_t)j * n;
            double* zj = Z + (size_t)j * n;
            double* w = V + (size_t)(j + 1) * n;
            if (mode == BAMREX_PRECOND_VCYCLE) {
                H_TRY(precondition(H, zj, vj));
            } else if (mode == BAMREX_PRECOND_VCYCLE_NETWORK) {
                // z = V(v); z += N(v - A z): the network on what the V-cycle left
                H_TRY(precondition(H, zj, vj));
                H_TRY(launch_apply(H, 0, zj, H->t, vj, 1));
                H_TRY(dot(H, H->t, H->t, &hd[kMaxVec]));
                double tt = 0;
                H_TRY(hck(H, cudaMemcpyAsync(&tt, &hd[kMaxVec], sizeof(double), cudaMemcpyDeviceToHost, H->stream), "copy"));
                H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
                if (tt > 0) {
                    H_TRY(net_precondition(H, N, H->t, std::sqrt(tt / (double)n), H->sh));
                    scale_add_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(zj, H->sh, n);
                    H_TRY(hck(H, cudaGetLastError(), "combine"));
                }
            } else {
                H_TRY(net_precondition(H, N, vj, rms_unit, zj));
                if (mode == BAMREX_PRECOND_NETWORK_VCYCLE) {
                    // z += V(v - A z): one V-cycle on what the network left
                    H_TRY(launch_apply(H, 0, zj, H->t, vj, 1));
                    H_TRY(precondition(H, H->sh, H->t));
                    scale_add_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(zj, H->sh, n);
                    H_TRY(hck(H, cudaGetLastError(), "combine"));
                }
            }
            H_TRY(launch_apply(H, 0, zj, w, nullptr, 0));
            // classical Gram-Schmidt, twice
            H_TRY(mdot(H, V, n, j + 1, w, hd, 0));
            mupdate_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(w, V, n, j + 1, hd, -1.0, n);
            H_TRY(hck(H, cudaGetLastError(), "orthogonalise"));
            H_TRY(mdot(H, V, n, j + 1, w, hd + kMaxVec / 2, 0));
            mupdate_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(w, V, n, j + 1, hd + kMaxVec / 2, -1.0, n);
            H_TRY(hck(H, cudaGetLastError(), "orthogonalise"));
            H_TRY(dot(H, w, w, hd + kMaxVec));
            H_TRY(hck(H, cudaMemcpyAsync(hv.data(), hd, sizeof(double) * (kMaxVec + 1), cudaMemcpyDeviceToHost, H->stream),
                      "copy"));
            H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
            for (int i = 0; i <= j; ++i) Hm[(size_t)i * m + j] = hv[i] + hv[kMaxVec / 2 + i];
            const double hn = std::sqrt(hv[kMaxVec]);
            Hm[(size_t)(j + 1) * m + j] = hn;
            if (hn > 0) {
                scale_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(w, w, 1.0 / hn, n);
                H_TRY(hck(H, cudaGetLastError(), "scale"));
            }
            // Givens rotations on the new column
            for (int i = 0; i < j; ++i) {
                const double a = Hm[(size_t)i * m + j], b = Hm[(size_t)(i + 1) * m + j];
                Hm[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
                Hm[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
            }
            const double a = Hm[(size_t)j * m + j], b = Hm[(size_t)(j + 1) * m + j];
            const double den = std::hypot(a, b);
            cs[j] = den > 0 ? a / den : 1.0;
            sn[j] = den > 0 ? b / den : 0.0;
            Hm[(size_t)j * m + j] = den;
            Hm[(size_t)(j + 1) * m + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            ++total;
            k = j + 1;
            if (std::fabs(g[j + 1]) <= target || hn == 0.0) break;
        }
        // y = R^{-1} g; x += Z y
        for (int i = k - 1; i >= 0; --i) {
            double sres = g[i];
            for (int q = i + 1; q < k; ++q) sres -= Hm[(size_t)i * m + q] * y[q];
            y[i] = sres / Hm[(size_t)i * m + i];
        }
        H_TRY(hck(H, cudaMemcpyAsync(hd, y.data(), sizeof(double) * k, cudaMemcpyHostToDevice, H->stream), "copy"));
        mupdate_kernel<<<grid_for(n), kThreads, 0, H->stream>>>(H->x, Z, n, k, hd, 1.0, n);
        H_TRY(hck(H, cudaGetLastError(), "update x"));
    }
    int fb = 0, pit = 0;
    double rr = bnorm > 0 ? rnorm / bnorm : rnorm;
    if (!(rnorm <= target)) {
        // fallback: the plain solve from the current iterate
        fb = 1;
        H_TRY(hck(H, cudaMemcpyAsync(x, H->x, sizeof(double) * n, cudaMemcpyDefault, H->stream), "copy out"));
        H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
        H_TRY(bamrex_helmholtz_solve(H, x, rhs, tol_rel, tol_abs, 1000, 1, &pit, &rr));
    } else {
        H_TRY(hck(H, cudaMemcpyAsync(x, H->x, sizeof(double) * n, cudaMemcpyDefault, H->stream), "copy out"));
        H_TRY(hck(H, cudaStreamSynchronize(H->stream), "sync"));
    }
    if (iters) *iters = total;
    if (plain_iters) *plain_iters = pit;
    if (rel_res) *rel_res = rr;
    if (fell_back) *fell_back = fb;
    return BAMREX_OK;
}
