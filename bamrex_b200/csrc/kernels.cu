// Light kernels of the explicit path: ghost fill (FillBoundary + physical
// boundary conditions), pack/unpack of valid cells, the stand-alone max
// wave speed reduction, per-box conserved sums, device time-step
// bookkeeping, and the per-box left/right flux and update kernels of the
// Fluxes.H / Update.H surface.  Level kernels are templated on the storage
// type (double, or float for the FP32-storage variant).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "euler.cuh"
#include "launch.h"

namespace bamrex {

namespace {

constexpr int kThreads = 256;

int grid_for(long long work, int per_thread = 1)
{
    const long long want = (work + (long long)kThreads * per_thread - 1) / ((long long)kThreads * per_thread);
    const long long cap = (long long)device_sm_count() * 8;
    return (int)std::max(1LL, std::min(want, cap));
}

__device__ __forceinline__ long long fab_index(const FabDev& f, int i, int j, int k)
{
    return (long long)(i - f.b0) + (long long)(j - f.b1) * f.js + (long long)(k - f.b2) * f.ks;
}

template <typename V>
__device__ __forceinline__ int find_by_begin(const V* v, int n, long long idx)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (v[mid].cell_begin <= idx) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------- ghosts
// bamrexBCData::fill_consv_boundary (Source/BoundaryConditions/BCs.cpp:429-442)
// expressed as a table of region copies built on the host.
template <typename T>
__global__ void ghost_fill_kernel(int NC, const GhostOp* __restrict__ ops, int nops, int nchunks,
                                  const FabDev* __restrict__ fabs, const StepScalars* scal)
{
    static_assert(kGhostChunk == 32, "one ghost chunk per warp");
    if (scal && scal->done) return;
    const int* __restrict__ chunk_op = reinterpret_cast<const int*>(ops + nops);
    const int lane = threadIdx.x & 31;
    const int w = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int nw = (int)((gridDim.x * blockDim.x) >> 5);
    for (int q = w; q < nchunks; q += nw) {
        const GhostOp& op = ops[chunk_op[q]];
        // 32-bit index arithmetic: a copy op is a ghost slab, far below 2^31 cells
        const int local = (q - op.chunk_begin) * kGhostChunk + lane;
        const int nx = op.hi[0] - op.lo[0] + 1, ny = op.hi[1] - op.lo[1] + 1;
        if (local < (int)ghost_op_cells(op)) {
            const int row = local / nx;
            const int ci = op.lo[0] + (local - row * nx);
            const int kk = row / ny;
            const int cj = op.lo[1] + (row - kk * ny);
            const int ck = op.lo[2] + kk;
            const int si = op.off[0] + op.mul[0] * ci;
            const int sj = op.off[1] + op.mul[1] * cj;
            const int sk = op.off[2] + op.mul[2] * ck;
            const FabDev& d = fabs[op.dst];
            const FabDev& s = fabs[op.src];
            const T* ps = s.ptr<T>() + fab_index(s, si, sj, sk);
            T* pd = d.ptr<T>() + fab_index(d, ci, cj, ck);
            // every load issued before the first store (the compiler cannot
            // tell that source and destination do not alias)
            T v[kMaxComp];
#pragma unroll
            for (int n = 0; n < kMaxComp; ++n)
                if (n < NC) v[n] = ps[n * s.ns];
#pragma unroll
            for (int n = 0; n < kMaxComp; ++n)
                if (n < NC) pd[n * d.ns] = ((op.negmask >> n) & 1) ? -v[n] : v[n];
        }
    }
}

// ---------------------------------------------------------------- pack
// packed element e = cell_begin*NC + n*ncells_box + cell (always double)
template <typename T>
__global__ void pack_kernel(int NC, const FabDev* __restrict__ fabs, const PackBox* __restrict__ boxes, int nboxes,
                            long long total, double* __restrict__ packed, int to_packed)
{
    const long long nel = total * NC;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nel;
         e += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nboxes - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (boxes[mid].cell_begin * NC <= e) lo = mid; else hi = mid - 1;
        }
        const PackBox& B = boxes[lo];
        const int nx = B.hi[0] - B.lo[0] + 1, ny = B.hi[1] - B.lo[1] + 1, nz = B.hi[2] - B.lo[2] + 1;
        const long long ncell = (long long)nx * ny * nz;
        const long long local = e - B.cell_begin * NC;
        const int n = (int)(local / ncell);
        const long long c = local % ncell;
        const int i = B.lo[0] + (int)(c % nx);
        const int j = B.lo[1] + (int)((c / nx) % ny);
        const int k = B.lo[2] + (int)(c / ((long long)nx * ny));
        const FabDev& f = fabs[lo];
        T* pf = f.ptr<T>() + fab_index(f, i, j, k) + n * f.ns;
        if (to_packed) packed[e] = (double)*pf;
        else *pf = (T)packed[e];
    }
}

// One slab of one box (full extent in the other directions) between the fab
// and the packed layout of the whole box ([n][cells of the box], x fastest).
template <typename T>
__global__ void pack_slab_kernel(int NC, const FabDev f, const PackBox box, const PackBox slab, double* __restrict__ packed,
                                 int to_packed)
{
    const int bx = box.hi[0] - box.lo[0] + 1, by = box.hi[1] - box.lo[1] + 1, bz = box.hi[2] - box.lo[2] + 1;
    const long long ncells = (long long)bx * by * bz;
    const int sx = slab.hi[0] - slab.lo[0] + 1, sy = slab.hi[1] - slab.lo[1] + 1, sz = slab.hi[2] - slab.lo[2] + 1;
    const long long scells = (long long)sx * sy * sz;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < scells * NC;
         e += (long long)gridDim.x * blockDim.x) {
        const int n = (int)(e / scells);
        const long long c = e - n * scells;
        const int i = slab.lo[0] + (int)(c % sx);
        const int j = slab.lo[1] + (int)((c / sx) % sy);
        const int k = slab.lo[2] + (int)(c / ((long long)sx * sy));
        const long long q = n * ncells + (i - box.lo[0]) + (long long)bx * ((j - box.lo[1]) + (long long)by * (k - box.lo[2]));
        T* pf = f.ptr<T>() + fab_index(f, i, j, k) + n * f.ns;
        if (to_packed) packed[q] = (double)*pf;
        else *pf = (T)packed[q];
    }
}

// ---------------------------------------------------------------- max speed
// max_wave_speed (Source/System/Euler/Euler.cpp:46-74) over valid cells.
template <typename T, int D>
__global__ void max_ws_kernel(const FabDev* __restrict__ fabs, const PackBox* __restrict__ boxes, int nboxes,
                              long long total, const Consts kc, unsigned long long* ws_bits, const StepScalars* scal)
{
    if (scal && scal->done) return;
    constexpr int NC = D + 2;
    const K<T> k(kc);
    double wmax = 0.0;
    bool nan_seen = false;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        const int b = find_by_begin(boxes, nboxes, c);
        const PackBox& B = boxes[b];
        const int nx = B.hi[0] - B.lo[0] + 1, ny = B.hi[1] - B.lo[1] + 1;
        const long long local = c - B.cell_begin;
        const int i = B.lo[0] + (int)(local % nx);
        const int j = B.lo[1] + (int)((local / nx) % ny);
        const int kk = B.lo[2] + (int)(local / ((long long)nx * ny));
        const FabDev& f = fabs[b];
        const T* p = f.ptr<T>() + fab_index(f, i, j, kk);
        T U[NC];
        for (int n = 0; n < NC; ++n) U[n] = p[n * f.ns];
        const double w = (double)wave_speed<T, D>(U, k);
        wmax = fmax(wmax, w);
        nan_seen = nan_seen || (w != w);
    }
    for (int off = 16; off > 0; off >>= 1) wmax = fmax(wmax, __shfl_xor_sync(0xffffffffu, wmax, off));
    const bool any_nan = __any_sync(0xffffffffu, nan_seen);
    if ((threadIdx.x & 31) == 0) {
        if (any_nan) atomicMax(ws_bits, 0x7ff8000000000000ull);
        else if (wmax > 0.0) atomicMax(ws_bits, (unsigned long long)__double_as_longlong(wmax));
    }
}

// ---------------------------------------------------------------- box sums
// One block per box; each thread sums a fixed strided subset of cells in
// double, then a fixed-shape tree reduction: the result does not depend on
// scheduling, so repeated runs give identical totals.
template <typename T>
__global__ void box_sums_kernel(int NC, const FabDev* __restrict__ fabs, const PackBox* __restrict__ boxes,
                                double* __restrict__ sums)
{
    __shared__ double red[256];
    const int b = blockIdx.x;
    const PackBox& B = boxes[b];
    const FabDev& f = fabs[b];
    const int nx = B.hi[0] - B.lo[0] + 1, ny = B.hi[1] - B.lo[1] + 1, nz = B.hi[2] - B.lo[2] + 1;
    const long long ncell = (long long)nx * ny * nz;
    for (int n = 0; n < NC; ++n) {
        double acc = 0.0;
        for (long long c = threadIdx.x; c < ncell; c += blockDim.x) {
            const int i = B.lo[0] + (int)(c % nx);
            const int j = B.lo[1] + (int)((c / nx) % ny);
            const int k = B.lo[2] + (int)(c / ((long long)nx * ny));
            acc += (double)f.ptr<T>()[fab_index(f, i, j, k) + n * f.ns];
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) sums[(long long)b * NC + n] = red[0];
        __syncthreads();
    }
}

// ---------------------------------------------------------------- dt
// estTimeStep (Source/AmrLevelAdv.cpp:395-477 -> FluidSystem.cpp:194-206):
// cfl * min_d dx_d / max_speed, then the stop-time clamp of
// computeInitialDt / computeNewDt (Source/AmrLevelAdv.cpp:513-523, 600-611).
__global__ void step_dt_kernel(StepScalars* s, int D, double dx0, double dx1, double dx2, double cfl, int mode)
{
    if (s->done) return;
    if (mode == 1) {
        s->time = s->time + s->dt;
        s->steps += 1;
    }
    const double ms = __longlong_as_double((long long)s->ws_bits);
    double dt_est = 1.0e20;
    const double dxs[3] = { dx0, dx1, dx2 };
    for (int d = 0; d < D; ++d) dt_est = fmin(dt_est, dxs[d] / ms);
    dt_est *= cfl;
    double dt_0 = dt_est;
    if (s->stop_time >= 0.0) {
        const double eps = 0.001 * dt_0;
        if ((s->time + dt_0) > (s->stop_time - eps)) dt_0 = s->stop_time - s->time;
        if (!(s->time < s->stop_time)) s->done = 1;
    }
    if (!(dt_est > 0.0) || dt_est != dt_est || isinf(dt_est)) {
        s->status = 3; /* BAMREX_ERR_NAN */
        s->done = 1;
    }
    s->dt = dt_0;
    s->ws_bits = 0ull;
}

// ---------------------------------------------------------------- LR flux
// compute_HLLC_flux_LR / compute_force_flux_LR on a box: one thread per face.
template <int D, int DIR, int KIND>
__global__ void flux_lr_kernel(int lo0, int lo1, int lo2, int hi0, int hi1, int hi2, const FabDev flux,
                               const FabDev cL, const FabDev cR, const Consts kc, double half_dx_dt, double dt_2dx)
{
    constexpr int NC = D + 2;
    const K<double> k(kc);
    const int fhi[3] = { hi0 + (DIR == 0), hi1 + (DIR == 1), hi2 + (DIR == 2) };
    const int nx = fhi[0] - lo0 + 1, ny = fhi[1] - lo1 + 1, nz = fhi[2] - lo2 + 1;
    const long long total = (long long)nx * ny * nz;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = lo0 + (int)(idx % nx);
        const int j = lo1 + (int)((idx / nx) % ny);
        const int kk = lo2 + (int)(idx / ((long long)nx * ny));
        double L[NC], R[NC], F[NC];
        const double* pl = cL.ptr<double>() + fab_index(cL, i - (DIR == 0), j - (DIR == 1), kk - (DIR == 2));
        const double* pr = cR.ptr<double>() + fab_index(cR, i, j, kk);
        for (int n = 0; n < NC; ++n) {
            L[n] = pl[n * cL.ns];
            R[n] = pr[n * cR.ns];
        }
        if (KIND == M_HLLC) hllc_face<double, D, DIR>(L, R, k, F);
        else force_face<double, D, DIR>(L, R, k, half_dx_dt, dt_2dx, F);
        double* pf = flux.ptr<double>() + fab_index(flux, i, j, kk);
        for (int n = 0; n < NC; ++n) pf[n * flux.ns] = F[n];
    }
}

// ---------------------------------------------------------------- updates
// AmrLevelAdv_advance.cpp:330-341 (sweep, dt/dx division form)
template <int D, int DIR>
__global__ void sweep_update_kernel(const UpdateArgs u)
{
    constexpr int NC = D + 2;
    const int nx = u.hi[0] - u.lo[0] + 1, ny = u.hi[1] - u.lo[1] + 1, nz = u.hi[2] - u.lo[2] + 1;
    const long long total = (long long)nx * ny * nz;
    const FabDev& fl = u.flux[0];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = u.lo[0] + (int)(idx % nx);
        const int j = u.lo[1] + (int)((idx / nx) % ny);
        const int k = u.lo[2] + (int)(idx / ((long long)nx * ny));
        const double* pin = u.in.ptr<double>() + fab_index(u.in, i, j, k);
        const double* pf0 = fl.ptr<double>() + fab_index(fl, i, j, k);
        const double* pf1 = fl.ptr<double>() + fab_index(fl, i + (DIR == 0), j + (DIR == 1), k + (DIR == 2));
        double* po = u.out.ptr<double>() + fab_index(u.out, i, j, k);
        // explicit rounding of the product: no FMA contraction, so the
        // stand-alone update rounds exactly as the scalar reference does
        for (int n = 0; n < NC; ++n)
            po[n * u.out.ns] = pin[n * u.in.ns] - __dmul_rn(u.dtdx[0], pf1[n * fl.ns] - pf0[n * fl.ns]);
    }
}

// conservative_update(bx, ...) (Source/Fluxes/Update.H:99-130, dt*idx form)
template <int D>
__global__ void cons_update_kernel(const UpdateArgs u)
{
    constexpr int NC = D + 2;
    const int nx = u.hi[0] - u.lo[0] + 1, ny = u.hi[1] - u.lo[1] + 1, nz = u.hi[2] - u.lo[2] + 1;
    const long long total = (long long)nx * ny * nz;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int i = u.lo[0] + (int)(idx % nx);
        const int j = u.lo[1] + (int)((idx / nx) % ny);
        const int k = u.lo[2] + (int)(idx / ((long long)nx * ny));
        const double* pin = u.in.ptr<double>() + fab_index(u.in, i, j, k);
        double* po = u.out.ptr<double>() + fab_index(u.out, i, j, k);
        for (int n = 0; n < NC; ++n) {
            double v = pin[n * u.in.ns];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                const FabDev& f = u.flux[d];
                const double a = f.ptr<double>()[fab_index(f, i + (d == 0), j + (d == 1), k + (d == 2)) + n * f.ns];
                const double b = f.ptr<double>()[fab_index(f, i, j, k) + n * f.ns];
                v = v - __dmul_rn(u.dtdx[d], a - b);
            }
            po[n * u.out.ns] = v;
        }
    }
}

}  // namespace

int device_sm_count()
{
    static int cache[64] = { 0 };
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!cache[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 148;
    }
    return cache[dev];
}

cudaError_t launch_ghost_fill(int NC, bool fp32, const GhostOp* ops, int nops, int nchunks, const FabDev* fabs,
                              const StepScalars* scal, cudaStream_t s)
{
    if (nops == 0 || nchunks == 0) return cudaSuccess;
    const long long warps = kThreads / 32;
    const int g = (int)std::min<long long>((nchunks + warps - 1) / warps, (long long)device_sm_count() * 8);
    if (fp32) ghost_fill_kernel<float><<<g, kThreads, 0, s>>>(NC, ops, nops, nchunks, fabs, scal);
    else ghost_fill_kernel<double><<<g, kThreads, 0, s>>>(NC, ops, nops, nchunks, fabs, scal);
    return cudaGetLastError();
}

cudaError_t launch_pack_slab(int NC, bool fp32, const FabDev& fab, const PackBox& box, const PackBox& slab,
                             double* packed, int to_packed, cudaStream_t s)
{
    const long long cells = (long long)(slab.hi[0] - slab.lo[0] + 1) * (slab.hi[1] - slab.lo[1] + 1) * (slab.hi[2] - slab.lo[2] + 1);
    if (cells <= 0) return cudaSuccess;
    const int g = grid_for(cells * NC, 4);
    if (fp32) pack_slab_kernel<float><<<g, kThreads, 0, s>>>(NC, fab, box, slab, packed, to_packed);
    else pack_slab_kernel<double><<<g, kThreads, 0, s>>>(NC, fab, box, slab, packed, to_packed);
    return cudaGetLastError();
}

cudaError_t launch_pack(int NC, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes,
                        long long total_cells, double* packed, int to_packed, cudaStream_t s)
{
    if (total_cells == 0) return cudaSuccess;
    const int g = grid_for(total_cells * NC, 4);
    if (fp32) pack_kernel<float><<<g, kThreads, 0, s>>>(NC, fabs, boxes, nboxes, total_cells, packed, to_packed);
    else pack_kernel<double><<<g, kThreads, 0, s>>>(NC, fabs, boxes, nboxes, total_cells, packed, to_packed);
    return cudaGetLastError();
}

template <typename T>
static cudaError_t max_ws_dispatch(int D, const FabDev* fabs, const PackBox* boxes, int nboxes, long long total_cells,
                                   const Consts& k, unsigned long long* ws_bits, const StepScalars* scal,
                                   cudaStream_t s)
{
    const int g = grid_for(total_cells, 4);
    switch (D) {
    case 1: max_ws_kernel<T, 1><<<g, kThreads, 0, s>>>(fabs, boxes, nboxes, total_cells, k, ws_bits, scal); break;
    case 2: max_ws_kernel<T, 2><<<g, kThreads, 0, s>>>(fabs, boxes, nboxes, total_cells, k, ws_bits, scal); break;
    case 3: max_ws_kernel<T, 3><<<g, kThreads, 0, s>>>(fabs, boxes, nboxes, total_cells, k, ws_bits, scal); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_max_wave_speed(int D, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes,
                                  long long total_cells, const Consts& k, unsigned long long* ws_bits,
                                  const StepScalars* scal, cudaStream_t s)
{
    if (fp32) return max_ws_dispatch<float>(D, fabs, boxes, nboxes, total_cells, k, ws_bits, scal, s);
    return max_ws_dispatch<double>(D, fabs, boxes, nboxes, total_cells, k, ws_bits, scal, s);
}

cudaError_t launch_box_sums(int NC, bool fp32, const FabDev* fabs, const PackBox* boxes, int nboxes, double* sums,
                            cudaStream_t s)
{
    if (nboxes == 0) return cudaSuccess;
    if (fp32) box_sums_kernel<float><<<nboxes, 256, 0, s>>>(NC, fabs, boxes, sums);
    else box_sums_kernel<double><<<nboxes, 256, 0, s>>>(NC, fabs, boxes, sums);
    return cudaGetLastError();
}

cudaError_t launch_step_dt(StepScalars* scal, int D, double dx0, double dx1, double dx2, double cfl, int mode,
                           cudaStream_t s)
{
    step_dt_kernel<<<1, 1, 0, s>>>(scal, D, dx0, dx1, dx2, cfl, mode);
    return cudaGetLastError();
}

template <int D, int DIR>
static cudaError_t flux_lr_dispatch(int kind, const int* lo, const int* hi, const FabDev& flux, const FabDev& cL,
                                    const FabDev& cR, const Consts& k, double half_dx_dt, double dt_2dx,
                                    cudaStream_t s)
{
    long long faces = 1;
    for (int d = 0; d < 3; ++d) faces *= (long long)(hi[d] - lo[d] + 1 + (d == DIR));
    const int g = grid_for(faces);
    if (kind == M_HLLC)
        flux_lr_kernel<D, DIR, M_HLLC><<<g, 128, 0, s>>>(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], flux, cL, cR, k,
                                                         half_dx_dt, dt_2dx);
    else
        flux_lr_kernel<D, DIR, M_FORCE><<<g, 128, 0, s>>>(lo[0], lo[1], lo[2], hi[0], hi[1], hi[2], flux, cL, cR, k,
                                                          half_dx_dt, dt_2dx);
    return cudaGetLastError();
}

cudaError_t launch_flux_LR(int D, int dir, int kind, const int* lo, const int* hi, const FabDev& flux,
                           const FabDev& cL, const FabDev& cR, const Consts& k, double dx, double dt,
                           cudaStream_t s)
{
    const double half_dx_dt = 0.5 * dx / dt, dt_2dx = dt / (2 * dx);
#define BAMREX_LR(DD, DR) \
    if (D == DD && dir == DR) return flux_lr_dispatch<DD, DR>(kind, lo, hi, flux, cL, cR, k, half_dx_dt, dt_2dx, s);
    BAMREX_LR(1, 0)
    BAMREX_LR(2, 0)
    BAMREX_LR(2, 1)
    BAMREX_LR(3, 0)
    BAMREX_LR(3, 1)
    BAMREX_LR(3, 2)
#undef BAMREX_LR
    return cudaErrorInvalidValue;
}

cudaError_t launch_sweep_update(int D, int dir, const UpdateArgs& u, cudaStream_t s)
{
    long long cells = 1;
    for (int d = 0; d < 3; ++d) cells *= (long long)(u.hi[d] - u.lo[d] + 1);
    const int g = grid_for(cells);
#define BAMREX_UP(DD, DR) \
    if (D == DD && dir == DR) { sweep_update_kernel<DD, DR><<<g, kThreads, 0, s>>>(u); return cudaGetLastError(); }
    BAMREX_UP(1, 0)
    BAMREX_UP(2, 0)
    BAMREX_UP(2, 1)
    BAMREX_UP(3, 0)
    BAMREX_UP(3, 1)
    BAMREX_UP(3, 2)
#undef BAMREX_UP
    return cudaErrorInvalidValue;
}

cudaError_t launch_conservative_update(int D, const UpdateArgs& u, cudaStream_t s)
{
    long long cells = 1;
    for (int d = 0; d < 3; ++d) cells *= (long long)(u.hi[d] - u.lo[d] + 1);
    const int g = grid_for(cells);
    switch (D) {
    case 1: cons_update_kernel<1><<<g, kThreads, 0, s>>>(u); break;
    case 2: cons_update_kernel<2><<<g, kThreads, 0, s>>>(u); break;
    case 3: cons_update_kernel<3><<<g, kThreads, 0, s>>>(u); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace bamrex
