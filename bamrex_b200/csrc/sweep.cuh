// Fused split-sweep kernels: per box, the interface flux of one direction
// and the conservative update (compute_*_flux + the update lambda of
// AmrLevelAdv::advance_explicit, Source/AmrLevelAdv_advance.cpp:290-341),
// in one pass that reads U once and writes U once.  T is the storage and
// arithmetic type (double: the drop-in path; float: the FP32-storage
// variant); the wave-speed reduction is carried out in double either way.
//
// Work decomposition: a launch covers every box of a sweep (the device box
// table); each warp takes work items from a grid-stride loop.
//  * x sweep (contiguous direction): an item is a segment of one row.  The
//    warp marches along the row in 32-cell chunks, lane t holding cell
//    x0+t; neighbour states come from warp shuffles, and the values of
//    earlier chunks carry the stencil across chunk boundaries.
//  * y / z sweeps (strided directions): an item is a group of 32 adjacent
//    columns x and a segment along the sweep; each thread marches its column
//    keeping the stencil in registers.  Loads and stores are coalesced
//    across the warp (32 consecutive values per component).
// Both are software-pipelined: the face stage of an iteration uses cell
// stages finished in earlier iterations, so the cell stage (reconstruction
// + half step) and the face stage (Riemann flux) of one iteration are
// independent instruction streams the scheduler can interleave.
#pragma once

#include "common.cuh"
#include "euler.cuh"
#include "sweep_stage.h"

namespace bamrex {

constexpr int kSweepThreads = 128;
// Resident 128-thread blocks per SM the sweep kernels are compiled for
// (register budget 65536 / (128 * blocks)).  3 measured best for FP64
// (2 and 4 were slower on the 4096^2 MUSCL-Hancock step).
#ifndef BAMREX_SWEEP_MIN_BLOCKS
#define BAMREX_SWEEP_MIN_BLOCKS 3
#endif
constexpr int kSweepMinBlocks = BAMREX_SWEEP_MIN_BLOCKS;
// The FP32-storage kernels hold half the registers per state value.
#ifndef BAMREX_SWEEP_MIN_BLOCKS_F32
#define BAMREX_SWEEP_MIN_BLOCKS_F32 4
#endif
template <typename T>
constexpr int min_blocks() { return sizeof(T) == 4 ? BAMREX_SWEEP_MIN_BLOCKS_F32 : kSweepMinBlocks; }
// Unroll factor of the strided march loop.
#ifndef BAMREX_MARCH_UNROLL
#define BAMREX_MARCH_UNROLL 1
#endif
constexpr int kMarchUnroll = BAMREX_MARCH_UNROLL;
static_assert(kSweepThreads == kStageBlockThreads, "staging sized for the sweep block");
// Unroll factor of the x-sweep chunk loop.
#ifndef BAMREX_XCHUNK_UNROLL
#define BAMREX_XCHUNK_UNROLL 1
#endif
constexpr int kXChunkUnroll = BAMREX_XCHUNK_UNROLL;

__device__ __forceinline__ int find_box(const SweepBox* boxes, int nboxes, long long item)
{
    int lo = 0, hi = nboxes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (boxes[mid].item_begin <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <typename T>
struct StepFactors {
    T dtdx, hdtdx, half_dx_dt, dt_2dx;
};

template <typename T>
__device__ __forceinline__ bool step_factors(const SweepArgs& a, StepFactors<T>& s)
{
    double dt = a.dt_host;
    if (a.scal) {
        if (a.scal->done) return false;
        dt = a.scal->dt;
    }
    s.dtdx = (T)(dt / a.dx);               // (dt / dx[d]), AmrLevelAdv_advance.cpp:337
    s.hdtdx = (T)(0.5 * dt / a.dx);        // Flux_Helpers.cpp:138
    s.half_dx_dt = (T)(0.5 * a.dx / dt);   // Force.cpp:77, 144
    s.dt_2dx = (T)(dt / (2 * a.dx));       // Force.cpp:91
    return true;
}

// A benign state used for lanes that have nothing to load: keeps the
// arithmetic of idle lanes finite.
template <typename T, int NC>
__device__ __forceinline__ void benign(T (&u)[NC])
{
    u[0] = T(1);
#pragma unroll
    for (int n = 1; n < NC - 1; ++n) u[n] = T(0);
    u[NC - 1] = T(1);
}

template <typename T, int NC>
__device__ __forceinline__ void ld_state(const T* __restrict__ p, long long ns, T (&u)[NC])
{
#pragma unroll
    for (int n = 0; n < NC; ++n) u[n] = __ldg(p + n * ns);
}

template <typename T, int NC>
__device__ __forceinline__ void copy_state(const T (&s)[NC], T (&d)[NC])
{
#pragma unroll
    for (int n = 0; n < NC; ++n) d[n] = s[n];
}

template <typename T, int NC>
__device__ __forceinline__ void shfl_carry(const T (&cur)[NC], const T (&prev)[NC], int lane, int shift,
                                           T (&out)[NC])
{
    // lane t receives cur[t-shift], or prev[32+t-shift] for t < shift
    const bool from_prev = lane >= 32 - shift;
#pragma unroll
    for (int n = 0; n < NC; ++n)
        out[n] = __shfl_sync(0xffffffffu, from_prev ? prev[n] : cur[n], (lane + 32 - shift) & 31);
}

// Warp max of the wave speed, then one atomicMax per warp on the ordered bit
// pattern (non-negative doubles order like their bits).  A NaN anywhere is
// reported as the NaN bit pattern, which is larger than every finite value,
// so the time step becomes NaN and the host sees BAMREX_ERR_NAN.
__device__ __forceinline__ void reduce_ws(double ws, bool nan_seen, unsigned long long* dst)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) ws = fmax(ws, __shfl_xor_sync(0xffffffffu, ws, off));
    const bool any_nan = __any_sync(0xffffffffu, nan_seen);
    if ((threadIdx.x & 31) == 0) {
        if (any_nan) atomicMax(dst, 0x7ff8000000000000ull);
        else if (ws > 0.0) atomicMax(dst, (unsigned long long)__double_as_longlong(ws));
    }
}

__device__ __forceinline__ void track_ws(double w, double& wsmax, bool& nan_seen)
{
    wsmax = fmax(wsmax, w);
    nan_seen = nan_seen || (w != w);
}

// ------------------------------------------------------------------ x sweep
// Chunk x0, lane t: load A = U(x0+t+2); cell stage of cell x0+t+1; face
// x0-31+t from the previous chunk's cell stages; update of cell x0-32+t.
template <typename T, int D, int METHOD, int LIM>
__global__ void __launch_bounds__(kSweepThreads, min_blocks<T>()) sweep_x_kernel(const SweepArgs a)
{
    using S = Scheme<T, D, 0, METHOD, LIM>;
    constexpr int NC = D + 2;
    constexpr int H = S::kHalo;
    StepFactors<T> f;
    if (!step_factors(a, f)) return;
    const K<T> k(a.k);
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    double wsmax = 0.0;
    bool nan_seen = false;

    for (long long it = gw; it < a.total_items; it += nw) {
        const int b = a.boxes ? find_box(a.boxes, a.nboxes, it) : 0;
        const SweepBox& B = a.boxes ? a.boxes[b] : a.one;
        const long long local = it - B.item_begin;
        const int seg = (int)(local % B.nseg);
        const long long row = local / B.nseg;
        const int ny = B.hi[1] - B.lo[1] + 1;
        const int j = B.lo[1] + (int)(row % ny);
        const int kk = B.lo[2] + (int)(row / ny);
        const int s0 = B.lo[0] + seg * B.seglen;
        const int s1 = min(s0 + B.seglen, B.hi[0] + 1);
        const bool last_seg = (s1 == B.hi[0] + 1);

        // row pointers indexed by the absolute x, and the component strides,
        // held in registers for the whole item
        const T* __restrict__ in = B.in.ptr<T>() + (long long)(j - B.in.b1) * B.in.js + (long long)(kk - B.in.b2) * B.in.ks - B.in.b0;
        T* __restrict__ out = B.out.ptr<T>() + (long long)(j - B.out.b1) * B.out.js + (long long)(kk - B.out.b2) * B.out.ks - B.out.b0;
        T* __restrict__ fl = B.flux.p ? B.flux.ptr<T>() + (long long)(j - B.flux.b1) * B.flux.js + (long long)(kk - B.flux.b2) * B.flux.ks - B.flux.b0 : nullptr;
        const long long ins = B.in.ns, ons = B.out.ns, fns = B.flux.ns;
        const bool do_update = a.do_update != 0;
        const bool ws_on = a.ws_max != nullptr;

        auto load = [&](int x0, T (&u)[NC]) {
            const int xl = x0 + lane + 2;
            if (xl >= s0 - H && xl <= s1 - 1 + H) ld_state(in + xl, ins, u);
            else benign(u);
        };

        // carried across chunks
        T Ap[NC];               // previous chunk's loads
        T ULp[NC], URp[NC];     // previous chunk's cell stages
        T URpp[NC];             // the chunk before that (its lane 31 is used)
        T Fp[NC];               // previous chunk's faces (lane 31 used)
        T Um2p[NC];             // previous chunk's U(x0-32+t)
        benign(Ap);
        benign(ULp);
        benign(URp);
        benign(URpp);
        benign(Um2p);
#pragma unroll
        for (int n = 0; n < NC; ++n) Fp[n] = T(0);

        T An[NC];
        load(s0 - 32, An);
#pragma unroll kXChunkUnroll
        for (int x0 = s0 - 32; x0 < s1 + 32; x0 += 32) {
            T A[NC];
            copy_state(An, A);
            load(x0 + 32, An);
            // cell stage of cell x0+t+1 (this chunk)
            T Um1[NC], Um2[NC];
            shfl_carry(A, Ap, lane, 1, Um1);  // U(x0+t+1)
            shfl_carry(A, Ap, lane, 2, Um2);  // U(x0+t)
            T UL[NC], UR[NC];
            S::cell(Um2, Um1, A, k, f.hdtdx, UL, UR);
            // face x0-31+t from the previous chunk: UR(x0-32+t), UL(x0-31+t)
            T URf[NC];
            shfl_carry(URp, URpp, lane, 1, URf);
            T F[NC];
            S::face(URf, ULp, k, f.half_dx_dt, f.dt_2dx, F);
            // update of cell o = x0-32+t from faces o and o+1
            T Fm[NC];
            shfl_carry(F, Fp, lane, 1, Fm);
            const int o = x0 - 32 + lane;
            // the update is computed by every lane (idle lanes hold benign
            // states) and stored by the lanes that own a cell, so the chunk
            // stays one basic block
            const bool upd = do_update && o >= s0 && o < s1;
            T Un[NC];
#pragma unroll
            for (int n = 0; n < NC; ++n) Un[n] = Um2p[n] - f.dtdx * (F[n] - Fm[n]);
            if (upd) {
#pragma unroll
                for (int n = 0; n < NC; ++n) out[o + n * ons] = Un[n];
            }
            if (ws_on) {
                const double w = (double)S::speed(Un, k);
                track_ws(upd ? w : 0.0, wsmax, nan_seen);
            }
            if (fl) {
                const int fo = o + 1;
                if (fo >= s0 && (fo < s1 || (fo == s1 && last_seg))) {
#pragma unroll
                    for (int n = 0; n < NC; ++n) fl[fo + n * fns] = F[n];
                }
            }
            copy_state(A, Ap);
            copy_state(URp, URpp);
            copy_state(UR, URp);
            copy_state(UL, ULp);
            copy_state(F, Fp);
            copy_state(Um2, Um2p);
        }
    }
    if (a.ws_max) reduce_ws(wsmax, nan_seen, a.ws_max);
}

// ----------------------------------------------------- marching sweeps
// y / z sweeps, and the x sweep of levels made of narrow boxes: each thread
// marches one column (one row for DIR = 0) keeping the stencil in
// registers; the 32 lanes of a warp take 32 adjacent columns across x (for
// DIR = 0: 32 adjacent rows across y, staged through shared memory so that
// global loads and stores stay coalesced; see sweep_stage.h).
// Iteration o: load U(o+4); cell stage of cell o+2; face o+1 from the cell
// stages of cells o and o+1 (earlier iterations); update of cell o.
template <typename T, int D, int DIR, int METHOD, int LIM>
__global__ void __launch_bounds__(kSweepThreads, min_blocks<T>()) sweep_s_kernel(const SweepArgs a)
{
    using S = Scheme<T, D, DIR, METHOD, LIM>;
    constexpr int NC = D + 2;
    constexpr int H = S::kHalo;
    StepFactors<T> f;
    if (!step_factors(a, f)) return;
    const K<T> k(a.k);
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    double wsmax = 0.0;
    bool nan_seen = false;

    for (long long it = gw; it < a.total_items; it += nw) {
        const int b = a.boxes ? find_box(a.boxes, a.nboxes, it) : 0;
        const SweepBox& B = a.boxes ? a.boxes[b] : a.one;
        const long long local = it - B.item_begin;
        const int seg = (int)(local % B.nseg);
        const long long rest = local / B.nseg;
        const int grp = (int)rest;
        // The lanes take 32 consecutive columns of the plane across DIR,
        // numbered with LD fastest then OT, so boxes narrower than 32 cells
        // still fill the warp (a group may span several OT planes).
        constexpr int LD = (DIR == 0) ? 1 : 0;  // the faster direction across the lanes
        constexpr int OT = (DIR == 2) ? 1 : 2;  // the slower one
        const int nld = B.hi[LD] - B.lo[LD] + 1;
        const int ncol = nld * (B.hi[OT] - B.lo[OT] + 1);
        const int fi = grp * 32 + lane;
        const bool active = fi < ncol;
        const int fa = active ? fi : 0;
        const int lp = B.lo[LD] + fa % nld;
        const int tr = B.lo[OT] + fa / nld;
        const int s0 = B.lo[DIR] + seg * B.seglen;
        const int s1 = min(s0 + B.seglen, B.hi[DIR] + 1);
        const bool last_seg = (s1 == B.hi[DIR] + 1);

        // column base offsets (position along DIR added per access): cell
        // (i, j, k) sits at (i - b0) + (j - b1) js + (k - b2) ks
        auto column = [&](const FabDev& G, long long& off, long long& step) {
            if (DIR == 0) {
                off = (long long)(lp - G.b1) * G.js + (long long)(tr - G.b2) * G.ks - (long long)G.b0;
                step = 1;
            } else if (DIR == 1) {
                off = (long long)(lp - G.b0) + (long long)(tr - G.b2) * G.ks - (long long)G.b1 * G.js;
                step = G.js;
            } else {
                off = (long long)(lp - G.b0) + (long long)(tr - G.b1) * G.js - (long long)G.b2 * G.ks;
                step = G.ks;
            }
        };
        long long inoff, outoff, floff = 0;
        long long ins, outs, fls = 0;
        column(B.in, inoff, ins);
        column(B.out, outoff, outs);
        if (B.flux.p) column(B.flux, floff, fls);
        const T* __restrict__ in = B.in.ptr<T>() + inoff;
        T* __restrict__ out = B.out.ptr<T>() + outoff;
        T* __restrict__ fl = B.flux.p ? B.flux.ptr<T>() + floff : nullptr;
        const long long inns = B.in.ns, ons = B.out.ns, fns = B.flux.ns;
        const bool do_update = a.do_update != 0;
        const bool ws_on = a.ws_max != nullptr;

        const int plo = s0 - H, phi = s1 - 1 + H;  // loadable positions
        // x sweep: the staged rows; positions are read in order, so a
        // warp-uniform test switches input buffers every kStageW reads, and
        // the updates leave through the output buffer every kStageW cells
        T* sin = nullptr;   // two input buffers: the chunk being read, the next one in flight
        T* sout = nullptr;
        int pbase = 0, pnext = 0, obase = s0, cur = 0;
        const int rows_left = ncol - grp * 32;
        const T* gin = nullptr;   // row 0 of the input / output fab, cell (lane % 4) of a chunk
        T* gout = nullptr;
        long long* srow = nullptr;  // per warp: the 32 rows' offsets in the input and output fabs
                                    // and in the x neighbours' fabs (below, above)
        // x halos read from the neighbouring boxes' fabs (null: from this
        // box's ghost cells)
        const T* xlo = nullptr;
        const T* xhi = nullptr;
        long long xlo_ns = 0, xhi_ns = 0;
        // start the asynchronous copy of the chunk at p0 into input buffer b
        // (positions outside the loadable range, or rows outside the box, get
        // the benign state); completes at the next wait_stage
        auto issue = [&](int p0, int b) {
            T* buf = sin + b * (NC * 32 * kStageW);
            const int c = lane & 3;
            const bool pin = p0 + c >= plo && p0 + c <= phi;
            // the fab this lane's position lies in: a halo position of a
            // box with a neighbour there reads the neighbour's own cell
            const T* base = gin + p0;
            long long ns = inns;
            int so = 0;
            if (xlo && p0 + c < B.lo[0]) {
                base = xlo + (p0 + c);
                ns = xlo_ns;
                so = 64;
            } else if (xhi && p0 + c > B.hi[0]) {
                base = xhi + (p0 + c);
                ns = xhi_ns;
                so = 96;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = (lane >> 2) + 8 * i;
                if (pin && r < rows_left) {
                    const T* src = base + srow[so + r];
#pragma unroll
                    for (int n = 0; n < NC; ++n) cp_async_elem(&buf[stage_slot(n * 32 + r, c)], src + n * ns);
                } else {
                    T u[NC];
                    benign(u);
#pragma unroll
                    for (int n = 0; n < NC; ++n) buf[stage_slot(n * 32 + r, c)] = u[n];
                }
            }
            cp_async_commit();
        };
        auto wait_stage = [&]() {
            cp_async_wait_all();
            __syncwarp();
        };
        auto flush = [&](int count) {
            __syncwarp();
            const int c = lane & 3;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = (lane >> 2) + 8 * i;
                if (c < count && r < rows_left) {
                    T* dst = gout + srow[32 + r] + obase;
#pragma unroll
                    for (int n = 0; n < NC; ++n) dst[n * ons] = sout[stage_slot(n * 32 + r, c)];
                }
            }
            __syncwarp();
        };
        if constexpr (DIR == 0) {
            extern __shared__ __align__(16) unsigned char bamrex_stage_smem[];
            const int wib = threadIdx.x >> 5;
            sin = reinterpret_cast<T*>(bamrex_stage_smem) + wib * stage_elems_per_warp<T, NC>();
            sout = sin + 2 * NC * 32 * kStageW;
            srow = reinterpret_cast<long long*>(bamrex_stage_smem + (size_t)(kSweepThreads / 32) *
                                                                          stage_elems_per_warp<T, NC>() * sizeof(T)) +
                   wib * 128;
            // lane (r0 = lane / 4, c = lane % 4) moves rows r0 + 8 i, cell c
            gin = B.in.ptr<T>() + (lane & 3);
            gout = B.out.ptr<T>() + (lane & 3);
            pbase = s0 - 2;
            pnext = s0 - 2;
            wait_stage();  // the previous item's copies have landed and its reads are done
            srow[lane] = inoff;        // this lane's row: cell (i, lp, tr) at inoff + i
            srow[32 + lane] = outoff;
            if (a.xnb_on) {
                // a neighbour's fab covers the box's whole halo on that side
                // (lanes past the box's rows keep in-range offsets of row 0)
                if (B.xnb[0].p && s0 - H < B.lo[0]) {
                    long long o, st;
                    column(B.xnb[0], o, st);
                    srow[64 + lane] = o;
                    xlo = B.xnb[0].ptr<T>();
                    xlo_ns = B.xnb[0].ns;
                }
                if (B.xnb[1].p && s1 - 1 + H > B.hi[0]) {
                    long long o, st;
                    column(B.xnb[1], o, st);
                    srow[96 + lane] = o;
                    xhi = B.xnb[1].ptr<T>();
                    xhi_ns = B.xnb[1].ns;
                }
            }
            __syncwarp();
            issue(pbase, 0);
            wait_stage();
            issue(pbase + kStageW, 1);
        }
        auto load = [&](int pos, T (&u)[NC]) {
            if constexpr (DIR == 0) {
                if (pnext == pbase + kStageW) {
                    // the next chunk has landed; the one just read takes the
                    // chunk after it
                    pbase += kStageW;
                    cur ^= 1;
                    wait_stage();
                    issue(pbase + kStageW, cur ^ 1);
                }
                const int c = pnext - pbase;
                const T* buf = sin + cur * (NC * 32 * kStageW);
#pragma unroll
                for (int n = 0; n < NC; ++n) u[n] = buf[stage_slot(n * 32 + lane, c)];
                ++pnext;
                (void)pos;
            } else {
                if (active && pos >= plo && pos <= phi) ld_state(in + (long long)pos * ins, inns, u);
                else benign(u);
            }
        };

        // warm-up: cell stages of cells s0-1 and s0
        T U0[NC], Ua[NC], Ub[NC], Nx[NC], Xm2[NC];
        load(s0 - 2, Xm2);
        load(s0 - 1, U0);
        load(s0, Ua);
        load(s0 + 1, Ub);
        load(s0 + 2, Nx);
        T URa[NC], URb[NC], ULb[NC], Fo[NC], tmp[NC];
        S::cell(Xm2, U0, Ua, k, f.hdtdx, tmp, URa);   // cell s0-1 -> UR(s0-1)
        S::cell(U0, Ua, Ub, k, f.hdtdx, ULb, URb);    // cell s0   -> UL(s0), UR(s0)
#pragma unroll
        for (int n = 0; n < NC; ++n) Fo[n] = T(0);

        // invariant at iteration o: U0 = U(o), Ua = U(o+1), Ub = U(o+2),
        // Nx = U(o+3), URa = UR(o), URb = UR(o+1), ULb = UL(o+1), Fo = F(o)
#pragma unroll kMarchUnroll
        for (int o = s0 - 1; o < s1; ++o) {
            T U3[NC];
            copy_state(Nx, U3);
            load(o + 4, Nx);
            T UL2[NC], UR2[NC];
            S::cell(Ua, Ub, U3, k, f.hdtdx, UL2, UR2);   // cell o+2
            T F1[NC];
            S::face(URa, ULb, k, f.half_dx_dt, f.dt_2dx, F1);  // face o+1
            const bool upd = o >= s0 && do_update && active;
            T Un[NC];
#pragma unroll
            for (int n = 0; n < NC; ++n) Un[n] = U0[n] - f.dtdx * (F1[n] - Fo[n]);
            if constexpr (DIR == 0) {
                if (o >= s0 && do_update) {
#pragma unroll
                    for (int n = 0; n < NC; ++n) sout[stage_slot(n * 32 + lane, o - obase)] = Un[n];
                    if (o - obase == kStageW - 1 || o == s1 - 1) {
                        flush(o - obase + 1);
                        obase += kStageW;
                    }
                }
            } else if (upd) {
                T* po = out + (long long)o * outs;
#pragma unroll
                for (int n = 0; n < NC; ++n) po[n * ons] = Un[n];
            }
            if (ws_on) {
                const double w = (double)S::speed(Un, k);
                track_ws(upd ? w : 0.0, wsmax, nan_seen);
            }
            if (fl && active) {
                const int fo = o + 1;
                if (fo >= s0 && (fo < s1 || (fo == s1 && last_seg))) {
                    T* pf = fl + (long long)fo * fls;
#pragma unroll
                    for (int n = 0; n < NC; ++n) pf[n * fns] = F1[n];
                }
            }
            copy_state(F1, Fo);
            copy_state(Ua, U0);
            copy_state(Ub, Ua);
            copy_state(U3, Ub);
            copy_state(URb, URa);
            copy_state(UR2, URb);
            copy_state(UL2, ULb);
        }
    }
    if constexpr (DIR == 0) cp_async_wait_all();  // no copy outlives the kernel
    if (a.ws_max) reduce_ws(wsmax, nan_seen, a.ws_max);
}

}  // namespace bamrex
