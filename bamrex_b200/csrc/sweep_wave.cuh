// Wavefront sweep of the fast MUSCL-Hancock/HLLC path (energy limiting,
// gamma with 1/z = 7), D = 2, 3: the fused flux + conservative update of one
// direction over every box of a level (compute_MUSCL_hancock_flux + the
// update lambda of AmrLevelAdv::advance_explicit,
// Source/AmrLevelAdv_advance.cpp:290-341), with no per-thread stencil state.
//
// A block of 8 warps takes a work item (box, group of lines, segment) and
// walks the segment in passes of PW positions.  In a pass each thread owns
// one position p of one line:
//   A. reads U(p-1), U(p), U(p+1) from the staged tile, computes the cell
//      stage of p (limiter + half step) and publishes UR(p) in a ring;
//   B. computes the HLLC face between p-1 and p from UR(p-1) (ring) and its
//      own UL(p), and publishes the face flux in a second ring;
//   C. updates cell p-1 from that flux and the flux of the face below
//      (ring) and stores it.
// Two block barriers separate A, B and C (the first also tells every thread
// whether one of them gave up waiting for a tile).  Each position's cell stage and
// face are computed once (the segment's first position and the pass
// rounding are the only extra work), and a thread holds one cell's values
// at a time, so the kernel runs with far fewer registers per thread than a
// march and keeps more warps resident.
//
// Lines and positions: for the y and z sweeps the 32 lanes are 32 lines
// (wa adjacent along the faster transverse direction x wb = 32 / wa) and the
// 8 warps 8 consecutive positions (PW = 8); for the x sweep the lanes are 32
// consecutive positions of a row (PW = 32) and the warps 8 rows.  Either
// way a warp reads and writes shared memory and global memory at
// consecutive addresses.
//
// Staging: the input arrives by TMA in stages of PW positions x all lines x
// NC components (cp.async.bulk.tensor, no multicast, from the box's own
// fab), NST stages in a ring on per-stage mbarriers; a pass reads its own
// stage and the first two positions of the next, and the stage it leaves
// behind is refilled at once.
#pragma once

#include "common.cuh"
#include "euler.cuh"
#include "sweep.cuh"
#include "tma.cuh"

namespace bamrex {

constexpr int kWaveThreads = 256;
constexpr int kWaveWarps = kWaveThreads / 32;

template <typename T, int D, int DIR>
struct WaveShape {
    static constexpr int NC = D + 2;
    static constexpr int PW = DIR == 0 ? 32 : kWaveWarps;   // positions per pass
    static constexpr int NL = DIR == 0 ? kWaveWarps : 32;   // lines per item
    static constexpr int NST = D == 2 ? 4 : 3;              // stages in the ring
    static constexpr int kStageElems = PW * NL * NC;
    static constexpr int kStageBytes = kStageElems * (int)sizeof(T);
    static constexpr int kRingElems = 2 * PW * NC * NL;     // UR or F ring
    static constexpr int kBytes = NST * kStageBytes + 2 * kRingElems * (int)sizeof(T);
};

template <typename T, int D, int DIR>
constexpr int wave_smem_bytes()
{
    return 1024 + WaveShape<T, D, DIR>::kBytes + WaveShape<T, D, DIR>::NST * 8;
}

#ifndef BAMREX_WAVE_MIN_BLOCKS
#define BAMREX_WAVE_MIN_BLOCKS 2
#endif
#ifndef BAMREX_WAVE_MIN_BLOCKS_F32
#define BAMREX_WAVE_MIN_BLOCKS_F32 3
#endif
template <typename T>
constexpr int wave_min_blocks() { return sizeof(T) == 4 ? BAMREX_WAVE_MIN_BLOCKS_F32 : BAMREX_WAVE_MIN_BLOCKS; }

template <typename T, int D, int DIR, int LIM, bool WS>
__global__ void __launch_bounds__(kWaveThreads, wave_min_blocks<T>()) sweep_wave_kernel(const SweepArgs a)
{
    using Sc = Scheme<T, D, DIR, M_MUSCL, LIM>;
    using Sh = WaveShape<T, D, DIR>;
    constexpr int NC = D + 2;
    constexpr int PW = Sh::PW, NL = Sh::NL, NST = Sh::NST;
    constexpr int A = DIR == 0 ? 1 : 0, B_ = DIR == 2 ? 1 : 2;

    StepFactors<T> f;
    if (!step_factors(a, f)) return;
    const K<T> k(a.k);

    extern __shared__ unsigned char bamrex_wave_smem[];
    const uint32_t raw = smem_u32(bamrex_wave_smem);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* sbase = bamrex_wave_smem + (base - raw);
    T* ring_ur = reinterpret_cast<T*>(sbase + NST * Sh::kStageBytes);
    T* ring_f = ring_ur + Sh::kRingElems;
    const uint32_t bars = base + (uint32_t)Sh::kBytes;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int o = DIR == 0 ? lane : warp;       // position offset in a pass
    const int line = DIR == 0 ? warp : lane;    // line of the item
    if (tid == 0) {
#pragma unroll
        for (int b = 0; b < NST; ++b) mbar_init(bars + 8 * b, 1);
        fence_mbar_init();
    }
    __syncthreads();
    uint32_t phase = 0;
    double wsmax = 0.0;
    bool nan_seen = false;
    bool failed = false;

    // ring slot s of component n for this thread's line
    auto ring = [&](T* r, int s, int n) -> T& {
        if constexpr (DIR == 0) return r[(line * NC + n) * (2 * PW) + s];
        else return r[(s * NC + n) * NL + line];
    };

    for (long long it = blockIdx.x; it < a.total_items && !failed; it += gridDim.x) {
        const int b = find_box(a.boxes, a.nboxes, it);
        const SweepBox& Bx = a.boxes[b];
        const long long local = it - Bx.item_begin;
        const int seg = (int)(local % Bx.nseg);
        const int grp = (int)(local / Bx.nseg);
        const int wa = (D == 2) ? NL : Bx.wa, wb = NL / wa;
        const int ngA = (Bx.hi[A] - Bx.lo[A] + wa) / wa;
        const int ga = grp % ngA, gb = grp / ngA;
        const int la = line % wa, lb = line / wa;
        const int a0 = Bx.lo[A] + ga * wa, b0 = Bx.lo[B_] + gb * wb;
        const int ca = a0 + la, cb = b0 + lb;
        const bool active = ca <= Bx.hi[A] && (D == 2 || cb <= Bx.hi[B_]);
        const int s0 = Bx.lo[DIR] + seg * Bx.seglen;
        const int s1 = min(s0 + Bx.seglen, Bx.hi[DIR] + 1);
        constexpr int q16 = 16 / (int)sizeof(T);
        const int pad = DIR == 0 ? ((s0 - 2 - Bx.lo[0]) & (q16 - 1)) : 0;
        const int Q0 = s0 - 2 - pad;                     // first position of stage 0
        const int npass = (s1 - Q0 + PW - 1) / PW;       // cell stages Q0+1 .. Q0+npass*PW
        const int nstage = npass + 1;
        const void* tmap = Bx.tmap;

        const FabDev& O = Bx.out;
        const int ob[3] = { O.b0, O.b1, O.b2 };
        const long long ostr[3] = { 1, O.js, O.ks };
        const int cca = active ? ca : Bx.lo[A], ccb = active ? cb : Bx.lo[B_];
        T* __restrict__ ocol = O.ptr<T>() + (long long)(cca - ob[A]) * ostr[A] +
                               (D == 3 ? (long long)(ccb - ob[B_]) * ostr[B_] : 0) - (long long)ob[DIR] * ostr[DIR];
        const long long ostep = ostr[DIR], ons = O.ns;
        const FabDev& I = Bx.in;
        const int ib[3] = { I.b0 - Bx.xoff, I.b1, I.b2 };

        auto issue = [&](int st) {
            const int slot = st % NST;
            const uint32_t bar = bars + 8 * slot;
            const uint32_t dst = base + (uint32_t)(slot * Sh::kStageBytes);
            mbar_expect_tx(bar, (uint32_t)Sh::kStageBytes);
            int c[3];
            c[DIR] = Q0 + st * PW - ib[DIR];
            c[A] = a0 - ib[A];
            c[B_] = b0 - ib[B_];
            if constexpr (D == 2) tma_load_3d(dst, tmap, c[0], c[1], 0, bar);
            else tma_load_4d(dst, tmap, c[0], c[1], c[2], 0, bar);
        };
        // this thread's elements of a stage: position q of its line at
        // qoff(q) + n * PW * NL (the positions o, o + 1, o + 2 it reads, the
        // last two in the next stage past PW - 1)
        const int pstride = DIR == 0 ? 1 : (D == 3 && DIR == 1 ? wa : NL);
        const int lbase = DIR == 0 ? line * PW : (D == 3 && DIR == 1 ? lb * PW * wa + la : line);
        const int q1 = o + 1 < PW ? o + 1 : o + 1 - PW, q2 = o + 2 < PW ? o + 2 : o + 2 - PW;
        const bool w1 = o + 1 >= PW, w2 = o + 2 >= PW;
        const int off0 = lbase + o * pstride, off1 = lbase + q1 * pstride, off2 = lbase + q2 * pstride;
        if (tid == 0) {
            // the previous item's reads of these buffers ended at its last
            // barrier
            fence_proxy_async_smem();
            for (int s = 0; s < NST && s < nstage; ++s) issue(s);
        }

        int waited = -1;  // stages this thread has seen land
        int issued = min(NST, nstage);
        for (int kp = 0; kp < npass; ++kp) {
            // stages kp and kp + 1 must have landed
            bool ok = true;
            for (int s = waited + 1; s <= kp + 1 && ok; ++s) {
                const int sl = s % NST;
                ok = mbar_wait_bounded(bars + 8 * sl, (phase >> sl) & 1u, kTmaWaitCycles);
                if (ok) {
                    phase ^= 1u << sl;
                    waited = s;
                }
            }
            const int p = Q0 + 1 + kp * PW + o;
            const T* cur = reinterpret_cast<const T*>(sbase + (kp % NST) * Sh::kStageBytes);
            const T* nxt = reinterpret_cast<const T*>(sbase + ((kp + 1) % NST) * Sh::kStageBytes);
            const T* t0 = cur + off0;
            const T* t1 = (w1 ? nxt : cur) + off1;
            const T* t2 = (w2 ? nxt : cur) + off2;
            // A: cell stage of p
            T Um[NC], U0[NC], Up[NC];
#pragma unroll
            for (int n = 0; n < NC; ++n) {
                Um[n] = t0[n * PW * NL];
                U0[n] = t1[n * PW * NL];
                Up[n] = t2[n * PW * NL];
            }
            T UL[NC], UR[NC];
            Sc::cell(Um, U0, Up, k, f.hdtdx, UL, UR);
            // ring slots of positions p and p - 1: (p - Q0) and (p - Q0 - 1)
            // modulo 2 PW, i.e. o + 1 and o, plus PW on odd passes
            const int par = (kp & 1) * PW;
            const int slot = ((o + 1) & (2 * PW - 1)) ^ par;
            const int slot_m = o ^ par;
#pragma unroll
            for (int n = 0; n < NC; ++n) ring(ring_ur, slot, n) = UR[n];
            if (__syncthreads_or(!ok)) {
                failed = true;
                break;
            }
            // the stage left behind is free: refill it
            if (kp + NST < nstage) {
                if (tid == 0) {
                    fence_proxy_async_smem();
                    issue(kp + NST);
                }
                issued = kp + NST + 1;
            }
            // B: face between p-1 and p
            T URm[NC];
#pragma unroll
            for (int n = 0; n < NC; ++n) URm[n] = ring(ring_ur, slot_m, n);
            T Fp[NC];
            Sc::face(URm, UL, k, f.half_dx_dt, f.dt_2dx, Fp);
#pragma unroll
            for (int n = 0; n < NC; ++n) ring(ring_f, slot, n) = Fp[n];
            __syncthreads();
            // C: update of cell p - 1 from the faces below and above it
            T Un[NC];
#pragma unroll
            for (int n = 0; n < NC; ++n) Un[n] = Um[n] - f.dtdx * (Fp[n] - ring(ring_f, slot_m, n));
            const int c = p - 1;
            const bool upd = active && c >= s0 && c < s1;
            T* po = ocol + (long long)c * ostep;
#pragma unroll
            for (int n = 0; n < NC; ++n) st_global_if(po + n * ons, Un[n], upd);
            if constexpr (WS) {
                const double w = (double)Sc::speed(Un, k);
                track_ws(upd ? w : 0.0, wsmax, nan_seen);
            }
        }
        if (failed) {
            // let every stage still in flight land (each wait bounded):
            // those issued that thread 0 has not seen land
            if (tid == 0) {
                for (int s = waited + 1; s < issued; ++s) {
                    const int sl = s % NST;
                    if (mbar_wait_bounded(bars + 8 * sl, (phase >> sl) & 1u, kTmaWaitCycles)) phase ^= 1u << sl;
                }
                if (a.status) atomicExch(a.status, 4 /* BAMREX_ERR_TIMEOUT */);
            }
            __syncthreads();
        }
    }
    if constexpr (WS) {
        if (!failed) reduce_ws(wsmax, nan_seen, a.ws_max);
    }
}

}  // namespace bamrex
