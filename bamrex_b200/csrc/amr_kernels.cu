// Kernels of the coarse/fine coupling (time and space interpolation of fine
// ghost cells, average_down, reflux) and of grad_error / state_error
// tagging.  This file is compiled with -fmad=false: every product and sum
// is rounded separately, so the results are reproducible operation by
// operation by a CPU restatement.
#include <cuda_runtime.h>

#include <algorithm>

#include "amr.h"
#include "bamrex_cuda.h"
#include "common.cuh"
#include "euler.cuh"

namespace bamrex {

namespace {

constexpr int kThreads = 256;

int grid_for(long long work)
{
    const long long want = (work + kThreads - 1) / kThreads;
    const long long cap = (long long)device_sm_count() * 8;
    return (int)std::max(1LL, std::min(want, cap));
}

__device__ __forceinline__ long long fidx(const FabDev& f, int i, int j, int k)
{
    return (long long)(i - f.b0) + (long long)(j - f.b1) * f.js + (long long)(k - f.b2) * f.ks;
}

template <typename V>
__device__ __forceinline__ int find_begin(const V* v, int n, long long idx)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (v[mid].cell_begin <= idx) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// ------------------------------------------------------------ coarse patch
__device__ __forceinline__ int find_patch_begin(const CfRegion* v, int n, long long idx)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (v[mid].patch_begin <= idx) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Coarse cell c mapped into the domain by the boundary kinds; a mirror
// image flips the sign of the normal momentum (bit 1 + d of negmask).
__device__ __forceinline__ void map_into_domain(const CoarseDomain& dm, int* c, int& negmask)
{
    for (int d = 0; d < dm.D; ++d) {
        const int lo = dm.lo[d], hi = dm.hi[d], len = hi - lo + 1;
        if (c[d] >= lo && c[d] <= hi) continue;
        const int bc = c[d] < lo ? dm.bc_lo[d] : dm.bc_hi[d];
        if (bc == BAMREX_BC_PERIODIC) {
            c[d] = lo + (((c[d] - lo) % len) + len) % len;
        } else if (bc == BAMREX_BC_REFLECTIVE) {
            c[d] = c[d] < lo ? 2 * lo - 1 - c[d] : 2 * hi + 1 - c[d];
            negmask ^= 1 << (1 + d);
        } else {
            c[d] = c[d] < lo ? lo : hi;
        }
    }
}

__device__ __forceinline__ int owner_of(const OwnerMap& m, const int* c)
{
    int blk[3];
    for (int d = 0; d < 3; ++d) {
        const int off = c[d] - m.lo[d];
        if (off < 0) return -1;
        blk[d] = off / m.g[d];
        if (blk[d] >= m.nb[d]) return -1;
    }
    return m.owner[((long long)blk[2] * m.nb[1] + blk[1]) * m.nb[0] + blk[0]];
}

// mode 0: old state, 1: new state, 2: a_old * old + a_new * new, 3: only
// check that every patch cell has an owner
template <typename T>
__global__ void cf_gather_kernel(const CfGatherArgs a)
{
    const long long n = a.npatch;
    int mode = a.mode;
    double a_old = a.a_old, a_new = a.a_new;
    if (a.amr) {
        // bamrex_coupling_fill_patch's choice, from the device times
        const double t_old = a.amr->t_sub[a.lc];
        const double t_new = t_old + a.amr->dt[a.lc];
        const double time = a.amr->t_sub[a.lc + 1];
        const double span = t_new - t_old;
        const double teps = 1e-3 * span;
        mode = 2;
        if (fabs(time - t_old) < teps) {
            mode = 0;
        } else if (fabs(time - t_new) < teps) {
            mode = 1;
        } else {
            a_old = (t_new - time) / span;
            a_new = (time - t_old) / span;
        }
    }
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        const CfRegion& R = a.regions[find_patch_begin(a.regions, a.nregions, e)];
        const long long local = e - R.patch_begin;
        const long long row = local / R.pn[0];
        int c[3] = { R.plo[0] + (int)(local - row * R.pn[0]), R.plo[1] + (int)(row % R.pn[1]),
                     R.plo[2] + (int)(row / R.pn[1]) };
        int neg = 0;
        map_into_domain(a.dom, c, neg);
        const int b = owner_of(a.own, c);
        if (mode == 3) {
            if (b < 0) atomicMin(a.bad, (unsigned long long)e);
            continue;
        }
        if (b < 0) {
            // not reached: the coupling checks every patch cell when it is made
            for (int m = 0; m < a.NC; ++m) a.patch[(long long)m * n + e] = 0.0;
            continue;
        }
        const FabDev& fn = a.crse_new[b];
        const long long in = fidx(fn, c[0], c[1], c[2]);
        if (mode == 4) {
            for (int m = 0; m < a.NC; ++m) a.patch[(long long)m * n + e] = (double)fn.ptr<T>()[in + m * fn.ns];
            continue;
        }
        for (int m = 0; m < a.NC; ++m) {
            double v;
            if (mode == 0) v = a.patch_old[(long long)m * n + e];
            else if (mode == 1) v = (double)fn.ptr<T>()[in + m * fn.ns];
            else v = a_old * a.patch_old[(long long)m * n + e] + a_new * (double)fn.ptr<T>()[in + m * fn.ns];
            if ((neg >> m) & 1) v = -v;
            a.patch[(long long)m * n + e] = v;
        }
    }
}

// ------------------------------------------------------------ interpolation
template <typename T>
__global__ void cf_interp_kernel(const CfInterpArgs a)
{
    const int r = a.ratio;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < a.ncells;
         idx += (long long)gridDim.x * blockDim.x) {
        const CfRegion& R = a.regions[find_begin(a.regions, a.nregions, idx)];
        // 32-bit index arithmetic: a region is a ghost slab or one fine box
        const int local = (int)(idx - R.cell_begin);
        const int nx = R.hi[0] - R.lo[0] + 1, ny = R.hi[1] - R.lo[1] + 1;
        const int row = local / nx, kk = row / ny;
        const int f[3] = { R.lo[0] + (local - row * nx), R.lo[1] + (row - kk * ny), R.lo[2] + kk };
        int c[3];
        double xi[3];
        for (int d = 0; d < 3; ++d) {
            const int w = f[d] + R.shift[d];
            c[d] = d < a.D ? floor_div(w, r) : w;
            // fine-cell centre relative to the coarse centre, in coarse cells
            xi[d] = d < a.D ? (double)(2 * (w - c[d] * r) + 1 - r) / (double)(2 * r) : 0.0;
        }
        const long long pc = R.patch_begin + ((long long)(c[2] - R.plo[2]) * R.pn[1] + (c[1] - R.plo[1])) * R.pn[0] +
                             (c[0] - R.plo[0]);
        const long long pstride[3] = { 1, R.pn[0], (long long)R.pn[0] * R.pn[1] };
        // the largest |xi| of any fine cell in a coarse cell
        const double xmax = (double)(r - 1) / (double)(2 * r);
        const FabDev& d0 = a.fine0[R.dst];
        const FabDev& d1 = a.fine1[R.dst];
        const long long i0 = fidx(d0, f[0], f[1], f[2]), i1 = fidx(d1, f[0], f[1], f[2]);
        for (int m = 0; m < a.NC; ++m) {
            const double* P = a.patch + (long long)m * a.npatch;
            const double uc = P[pc];
            double umin = uc, umax = uc, ext = 0.0, s = 0.0;
            double slope[3] = { 0.0, 0.0, 0.0 };
            for (int d = 0; d < a.D; ++d) {
                const double ul = P[pc - pstride[d]], ur = P[pc + pstride[d]];
                const double dc = 0.5 * (ur - ul);
                const double dl = 2.0 * (uc - ul);
                const double dr = 2.0 * (ur - uc);
                double sl = 0.0;
                if (dl * dr > 0.0) sl = copysign(fmin(fabs(dc), fmin(fabs(dl), fabs(dr))), dc);
                slope[d] = sl;
                umin = fmin(umin, fmin(ul, ur));
                umax = fmax(umax, fmax(ul, ur));
                ext = ext + fabs(sl) * xmax;
            }
            double alpha = 1.0;
            if (ext > 0.0) {
                alpha = fmin(alpha, (umax - uc) / ext);
                alpha = fmin(alpha, (uc - umin) / ext);
            }
            for (int d = 0; d < a.D; ++d) s = s + slope[d] * xi[d];
            const T v = (T)(uc + alpha * s);
            d0.ptr<T>()[i0 + m * d0.ns] = v;
            d1.ptr<T>()[i1 + m * d1.ns] = v;
        }
    }
}

// ------------------------------------------------------------ average_down
template <typename T>
__global__ void avg_down_kernel(int D, int NC, int r, const AvgOp* __restrict__ ops, int nops, long long n,
                                const FabDev* __restrict__ crse, const FabDev* __restrict__ fine)
{
    const int rz = D > 2 ? r : 1, ry = D > 1 ? r : 1;
    const double w = 1.0 / (double)(r * ry * rz);  // exact: r^D is a power of two
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
         idx += (long long)gridDim.x * blockDim.x) {
        const AvgOp& op = ops[find_begin(ops, nops, idx)];
        const int local = (int)(idx - op.cell_begin);  // one coarse/fine box intersection
        const int nx = op.hi[0] - op.lo[0] + 1, ny = op.hi[1] - op.lo[1] + 1;
        const int row = local / nx, kk0 = row / ny;
        const int i = op.lo[0] + (local - row * nx);
        const int j = op.lo[1] + (row - kk0 * ny);
        const int k = op.lo[2] + kk0;
        const FabDev& fc = crse[op.crse];
        const FabDev& ff = fine[op.fine];
        const long long ic = fidx(fc, i, j, k);
        const long long if0 = fidx(ff, i * r, D > 1 ? j * r : j, D > 2 ? k * r : k);
        for (int m = 0; m < NC; ++m) {
            const T* p = ff.ptr<T>() + if0 + m * ff.ns;
            double sum = 0.0;
            for (int kk = 0; kk < rz; ++kk)
                for (int jj = 0; jj < ry; ++jj)
                    for (int ii = 0; ii < r; ++ii) sum = sum + (double)p[ii + jj * ff.js + kk * ff.ks];
            fc.ptr<T>()[ic + m * fc.ns] = (T)(sum * w);
        }
    }
}

// ------------------------------------------------------------ reflux
template <typename T>
__global__ void reflux_kernel(int NC, const RefluxRec* __restrict__ recs, int nslots, const double* __restrict__ reg,
                              double vol, const FabDev* __restrict__ crse)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nslots) return;
    const RefluxRec rc = recs[s];
    const FabDev& f = crse[rc.box];
    T* p = f.ptr<T>() + fidx(f, rc.i, rc.j, rc.k);
    for (int m = 0; m < NC; ++m) {
        const double corr = ((double)rc.sign * reg[(long long)m * nslots + s]) / vol;
        p[m * f.ns] = (T)((double)p[m * f.ns] + corr);
    }
}

// ------------------------------------------------------------ tagging
template <typename T, int D>
__device__ __forceinline__ double tag_value(const FabDev& f, int i, int j, int k, const K<T>& kk, int var, int primv)
{
    constexpr int NC = D + 2;
    const T* p = f.ptr<T>() + fidx(f, i, j, k);
    if (!primv) return (double)p[var * f.ns];
    T U[NC], q[NC], ir;
#pragma unroll
    for (int n = 0; n < NC; ++n) U[n] = p[n * f.ns];
    to_prim<T, D>(U, kk, q, ir);
    return (double)sel(q, var);
}

template <typename T, int D>
__global__ void tag_kernel(const FabDev* __restrict__ fab_tab, const PackBox* __restrict__ boxes, int nboxes,
                           long long total, const Consts kc, const TagSpec spec, char* __restrict__ tags)
{
    const K<T> kk(kc);
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        const int b = find_begin(boxes, nboxes, c);
        const PackBox& B = boxes[b];
        const int nx = B.hi[0] - B.lo[0] + 1, ny = B.hi[1] - B.lo[1] + 1;
        const long long local = c - B.cell_begin;
        const int i = B.lo[0] + (int)(local % nx);
        const int j = B.lo[1] + (int)((local / nx) % ny);
        const int k = B.lo[2] + (int)(local / ((long long)nx * ny));
        const FabDev& f = fab_tab[b];
        char t = 0;
        // state_error (tagging_K.H:9-19)
        if (spec.do_err && tag_value<T, D>(f, i, j, k, kk, spec.err_var, spec.err_primv) >= spec.err_thr) t = 1;
        // grad_error (tagging_K.H:21-60)
        if (spec.do_grad) {
            const int var = spec.grad_var, pv = spec.grad_primv;
            const double v = tag_value<T, D>(f, i, j, k, kk, var, pv);
            double ax = fabs(tag_value<T, D>(f, i - 1, j, k, kk, var, pv) - v);
            ax = fmax(ax, fabs(v - tag_value<T, D>(f, i + 1, j, k, kk, var, pv)));
            double ay = 0.0, az = 0.0;
            if (D > 1) {
                ay = fabs(tag_value<T, D>(f, i, j - 1, k, kk, var, pv) - v);
                ay = fmax(ay, fabs(v - tag_value<T, D>(f, i, j + 1, k, kk, var, pv)));
            }
            if (D > 2) {
                az = fabs(tag_value<T, D>(f, i, j, k - 1, kk, var, pv) - v);
                az = fmax(az, fabs(v - tag_value<T, D>(f, i, j, k + 1, kk, var, pv)));
            }
            if (fmax(ax, fmax(ay, az)) >= spec.grad_thr * fmax(fabs(v), 1e-14)) t = 1;
        }
        // box_error (tagging_K.H:87-103)
        if (spec.do_box) {
            const int ijk[3] = { i, j, k };
            bool in = true;
            for (int d = 0; d < D; ++d) {
                const double p = (ijk[d] + 0.5) * spec.dx[d] + spec.prob_lo[d];
                in = in && spec.box_lo[d] <= p && p <= spec.box_hi[d];
            }
            if (in) t = 1;
        }
        if (spec.flag_tab) {
            const FabDev& ff = spec.flag_tab[b];
            const int fl = ((const unsigned char*)ff.p)[fidx(ff, i, j, k)];
            // interface_error (tagging_K.H:62-72)
            if (spec.do_iface) {
                const FabDev& lf = spec.ls_tab[b];
                if ((fl & BAMREX_GFM_INTERFACE) || fabs(lf.ptr<double>()[fidx(lf, i, j, k)]) <= spec.lstol) t = 1;
            }
            // ghost_error (tagging_K.H:74-84)
            if ((fl & BAMREX_GFM_GHOST) && !(fl & BAMREX_GFM_INTERFACE)) t = 0;
        }
        tags[c] = t;
    }
}

// computeNewDt of a hierarchy without a regrid (Source/AmrLevelAdv.cpp:
// 487-619 with AMReX's Amr::computeNewDt): each level's estTimeStep from its
// max wave speed, the coarse dt the smallest of n_l * dt_l, clamped to the
// stop time, and dt / n_l on level l; the same operations in the same order
// as the host path (bamrex_level_est_time_step, compute_dt), so the values
// are equal bit for bit.  A non-finite or non-positive estimate, or a level
// status, goes to a->status; the host reads it before it steps.
__global__ void amr_dt_kernel(AmrDev* a, const AmrLevelsArg lv)
{
    int status = 0;
    for (int l = 0; l < lv.nl; ++l)
        if (!status && lv.scal[l]->status) status = lv.scal[l]->status;
    double dt0 = 1.0e100;
    long long nf = 1;
    for (int l = 0; l < lv.nl; ++l) {
        const double ms = __longlong_as_double((long long)lv.scal[l]->ws_bits);
        double e = 1.0e20;
        for (int d = 0; d < lv.D; ++d) {
            const double x = lv.dx[l][d] / ms;
            e = (x < e) ? x : e;
        }
        e = e * lv.cfl[l];
        if (!isfinite(e) || !(e > 0.0)) status = status ? status : 3; /* BAMREX_ERR_NAN */
        if (l > 0) nf *= lv.ratio;
        const double c = (double)nf * e;
        dt0 = (c < dt0) ? c : dt0;
    }
    const double eps = 0.001 * dt0;
    if (a->stop_time >= 0.0 && (a->time + dt0) > (a->stop_time - eps)) dt0 = a->stop_time - a->time;
    if (!(dt0 > 0.0) || !isfinite(dt0)) status = status ? status : 3;
    nf = 1;
    for (int l = 0; l < lv.nl; ++l) {
        if (l > 0) nf *= lv.ratio;
        a->dt[l] = dt0 / (double)nf;
        lv.scal[l]->dt = a->dt[l];
        lv.scal[l]->done = 0;
    }
    a->t_sub[0] = a->time;
    a->dt0 = dt0;
    a->status = status;
}

__global__ void amr_substep_kernel(AmrDev* a, int l, int i)
{
    a->t_sub[l] = a->t_sub[l - 1] + (double)i * a->dt[l];
}

}  // namespace

cudaError_t launch_amr_dt(AmrDev* a, const AmrLevelsArg& lv, cudaStream_t s)
{
    amr_dt_kernel<<<1, 1, 0, s>>>(a, lv);
    return cudaGetLastError();
}

cudaError_t launch_amr_substep(AmrDev* a, int l, int i, cudaStream_t s)
{
    amr_substep_kernel<<<1, 1, 0, s>>>(a, l, i);
    return cudaGetLastError();
}

cudaError_t launch_cf_gather(bool fp32, const CfGatherArgs& a, cudaStream_t s)
{
    if (a.npatch <= 0) return cudaSuccess;
    const int g = grid_for(a.npatch);
    if (fp32) cf_gather_kernel<float><<<g, kThreads, 0, s>>>(a);
    else cf_gather_kernel<double><<<g, kThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_cf_interp(bool fp32, const CfInterpArgs& a, cudaStream_t s)
{
    if (a.ncells <= 0) return cudaSuccess;
    const int g = grid_for(a.ncells);
    if (fp32) cf_interp_kernel<float><<<g, kThreads, 0, s>>>(a);
    else cf_interp_kernel<double><<<g, kThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_avg_down(int D, int NC, int ratio, bool fp32, const AvgOp* ops, int nops, long long ncells,
                            const FabDev* crse, const FabDev* fine, cudaStream_t s)
{
    if (ncells <= 0) return cudaSuccess;
    const int g = grid_for(ncells);
    if (fp32) avg_down_kernel<float><<<g, kThreads, 0, s>>>(D, NC, ratio, ops, nops, ncells, crse, fine);
    else avg_down_kernel<double><<<g, kThreads, 0, s>>>(D, NC, ratio, ops, nops, ncells, crse, fine);
    return cudaGetLastError();
}

cudaError_t launch_reflux(int NC, bool fp32, const RefluxRec* recs, int nslots, const double* reg, double vol,
                          const FabDev* crse, cudaStream_t s)
{
    if (nslots <= 0) return cudaSuccess;
    const int g = (nslots + kThreads - 1) / kThreads;
    if (fp32) reflux_kernel<float><<<g, kThreads, 0, s>>>(NC, recs, nslots, reg, vol, crse);
    else reflux_kernel<double><<<g, kThreads, 0, s>>>(NC, recs, nslots, reg, vol, crse);
    return cudaGetLastError();
}

cudaError_t launch_tag(int D, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes, long long ncells,
                       const Consts& k, const TagSpec& spec, char* tags, cudaStream_t s)
{
    if (ncells <= 0) return cudaSuccess;
    const int g = grid_for(ncells);
#define BX_TAG(TT, DD) tag_kernel<TT, DD><<<g, kThreads, 0, s>>>(fabs, boxes, nboxes, ncells, k, spec, tags)
    if (fp32) {
        if (D == 1) BX_TAG(float, 1);
        else if (D == 2) BX_TAG(float, 2);
        else BX_TAG(float, 3);
    } else {
        if (D == 1) BX_TAG(double, 1);
        else if (D == 2) BX_TAG(double, 2);
        else BX_TAG(double, 3);
    }
#undef BX_TAG
    return cudaGetLastError();
}

}  // namespace bamrex
