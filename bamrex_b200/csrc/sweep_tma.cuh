// TMA-staged marching sweep of the fast MUSCL-Hancock/HLLC path (energy
// limiting, gamma with 1/z = 7), D = 2, 3: the fused flux + conservative
// update of one direction over every box of a level
// (compute_MUSCL_hancock_flux + the update lambda of
// AmrLevelAdv::advance_explicit, Source/AmrLevelAdv_advance.cpp:290-341).
//
// Work decomposition.  A work item is (box, lane group, segment): the 32
// lanes of a warp take 32 lines along the sweep direction DIR (wa adjacent
// lines along the faster transverse direction A times wb = 32 / wa along the
// slower one B) and march them together over one segment [s0, s1) of the
// box, each lane keeping its line's stencil in registers.
//
// Staging.  The warp's input arrives by TMA: stage k of an item is the
// tile of S consecutive positions x 32 lines x NC components, one tiled
// tensor load (cp.async.bulk.tensor, no multicast) from the box's own fab
// into one of NST shared-memory buffers of the warp, completed on that
// buffer's mbarrier.  While the warp marches through stage k, the loads of
// stages k+1 .. k+NST-1 are in flight.  A lane reads its line from the
// buffer with no address arithmetic beyond a per-lane base (x sweep: the
// tile is stored with the TMA's 32/64/128-byte swizzle so that the 32 lines,
// one per lane, fall into different banks).
//
// March.  Step q (the newest position loaded) does, for every lane: load
// U(q); face q-2 (HLLC between the half-stepped states UR(q-3), UL(q-2) of
// earlier steps); update of cell q-3 from faces q-3 and q-2; cell stage of
// cell q-1 (limiter + half step from U(q-2), U(q-1), U(q)).  The face and
// the cell stage of a step are independent instruction streams.  Register
// slots rotate with the step index within the stage (S is a multiple of 4),
// so the unrolled stage needs no register moves.  Positions run from
// s0 - 2 to s1 + 2 (the last without a load); updates are stored for
// s0 <= q - 3 < s1.
#pragma once

#include "common.cuh"
#include "euler.cuh"
#include "sweep.cuh"
#include "tma.cuh"

namespace bamrex {

constexpr int kTmaThreads = 128;
constexpr int kTmaWarps = kTmaThreads / 32;
// Longest wait for a stage (SM clock cycles, ~1 s) before the warp reports
// BAMREX_ERR_TIMEOUT and stops.
constexpr long long kTmaWaitCycles = 2000000000LL;

// The transverse directions of a sweep: A (the faster in memory, across
// the lanes first) and B.
__host__ __device__ constexpr int tma_dir_a(int DIR) { return DIR == 0 ? 1 : 0; }
__host__ __device__ constexpr int tma_dir_b(int DIR) { return DIR == 2 ? 1 : 2; }

// Stage positions and buffers per warp: S positions of 32 bytes per line
// (4 doubles or 8 floats; the x sweep's stages use the TMA's 32-byte
// swizzle), NST buffers in flight.
// The x sweep also gathers its updates in one output stage of the same
// shape (one line per lane), written out in 32-byte row pieces.
template <typename T, int D, int DIR>
struct TmaShape {
    static constexpr int S = 32 / (int)sizeof(T);
    static constexpr int NST = DIR == 0 ? 2 : 3;
    static constexpr int NOUT = DIR == 0 ? 1 : 0;
    static constexpr int NC = D + 2;
    static constexpr int kStageElems = S * 32 * NC;
    static constexpr int kStageBytes = kStageElems * (int)sizeof(T);
    static constexpr int kWarpBytes = (NST + NOUT) * kStageBytes;
    // x sweep: bytes of one line's S positions = the swizzle span
    static constexpr int kSpan = S * (int)sizeof(T);
};

template <typename T, int D, int DIR>
constexpr int tma_smem_bytes()
{
    return 1024 + kTmaWarps * TmaShape<T, D, DIR>::kWarpBytes + kTmaWarps * TmaShape<T, D, DIR>::NST * 8;
}

// Resident 128-thread blocks per SM the kernels are compiled for.
#ifndef BAMREX_TMA_MIN_BLOCKS
#define BAMREX_TMA_MIN_BLOCKS 3
#endif
#ifndef BAMREX_TMA_MIN_BLOCKS_F32
#define BAMREX_TMA_MIN_BLOCKS_F32 4
#endif
template <typename T>
constexpr int tma_min_blocks() { return sizeof(T) == 4 ? BAMREX_TMA_MIN_BLOCKS_F32 : BAMREX_TMA_MIN_BLOCKS; }

template <typename T, int D, int DIR, int LIM, bool WS>
__global__ void __launch_bounds__(kTmaThreads, tma_min_blocks<T>()) sweep_tma_kernel(const SweepArgs a)
{
    using Sc = Scheme<T, D, DIR, M_MUSCL, LIM>;
    using Sh = TmaShape<T, D, DIR>;
    constexpr int NC = D + 2;
    constexpr int S = Sh::S;
    constexpr int NST = Sh::NST;
    constexpr int A = tma_dir_a(DIR), B_ = tma_dir_b(DIR);
    static_assert(S % 4 == 0, "register slots rotate with period 4");
    static_assert(Sh::kSpan == 32 || Sh::kSpan == 64 || Sh::kSpan == 128, "x-sweep swizzle span");

    StepFactors<T> f;
    if (!step_factors(a, f)) return;
    const K<T> k(a.k);

    extern __shared__ unsigned char bamrex_tma_smem[];
    const uint32_t raw = smem_u32(bamrex_tma_smem);
    const uint32_t base = (raw + 1023u) & ~1023u;  // stage buffers 1024-byte aligned (swizzle pattern)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t wbuf = base + (uint32_t)(warp * Sh::kWarpBytes);
    unsigned char* wbuf_p = bamrex_tma_smem + (base - raw) + warp * Sh::kWarpBytes;
    unsigned char* osb = wbuf_p + NST * Sh::kStageBytes;  // x sweep: the output stage
    const uint32_t bars = base + (uint32_t)(kTmaWarps * Sh::kWarpBytes + warp * NST * 8);
    if (lane == 0) {
#pragma unroll
        for (int b = 0; b < NST; ++b) mbar_init(bars + 8 * b, 1);
        fence_mbar_init();
    }
    __syncwarp();
    uint32_t phase = 0;  // bit b: the parity the next wait on buffer b expects

    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    double wsmax = 0.0;
    bool nan_seen = false;
    bool failed = false;

    // x sweep: the XOR of this lane's line in the swizzled stage (the TMA
    // swizzle of span bytes permutes the 16-byte chunks of each 128-byte row
    // by bits 7.. of the offset)
    constexpr int kSpan = Sh::kSpan;
    const uint32_t xl = (uint32_t)((((lane * kSpan) >> 7) & (kSpan / 16 - 1)) << 4);

    for (long long it = gw; it < a.total_items && !failed; it += nw) {
        const int b = find_box(a.boxes, a.nboxes, it);
        const SweepBox& Bx = a.boxes[b];
        const long long local = it - Bx.item_begin;
        const int seg = (int)(local % Bx.nseg);
        const int grp = (int)(local / Bx.nseg);
        const int wa = D == 2 ? 32 : Bx.wa, wb = 32 / wa;
        const int ngA = (Bx.hi[A] - Bx.lo[A] + wa) / wa;
        const int ga = grp % ngA, gb = grp / ngA;
        const int la = lane % wa, lb = lane / wa;
        const int a0 = Bx.lo[A] + ga * wa, b0 = Bx.lo[B_] + gb * wb;
        const int ca = a0 + la, cb = b0 + lb;
        const bool active = ca <= Bx.hi[A] && (D == 2 || cb <= Bx.hi[B_]);
        const int s0 = Bx.lo[DIR] + seg * Bx.seglen;
        const int s1 = min(s0 + Bx.seglen, Bx.hi[DIR] + 1);
        // first position of stage 0: s0 - 2, lowered in the x sweep to a
        // 16-byte boundary of the row (the TMA's innermost coordinate rule)
        constexpr int q16 = 16 / (int)sizeof(T);
        const int pad = DIR == 0 ? ((s0 - 2 - Bx.lo[0]) & (q16 - 1)) : 0;
        const int P0 = s0 - 2 - pad;
        const int Pend = s1 + 2;
        const int nstage = (Pend - P0) / S + 1;
        const void* tmap = Bx.tmap;

        // output line of this lane: cell (pos along DIR, ca, cb) at ocol + pos * ostr + n * ons
        const FabDev& O = Bx.out;
        const int ob[3] = { O.b0, O.b1, O.b2 };
        const long long ostr[3] = { 1, O.js, O.ks };
        const int cca = active ? ca : Bx.lo[A], ccb = active ? cb : Bx.lo[B_];
        T* __restrict__ ocol = O.ptr<T>() + (long long)(cca - ob[A]) * ostr[A] +
                               (D == 3 ? (long long)(ccb - ob[B_]) * ostr[B_] : 0) - (long long)ob[DIR] * ostr[DIR];
        const long long ostep = ostr[DIR], ons = O.ns;
        // TMA coordinates of the tile origin (tensor map origin: the fab's
        // padded row start, x offset Bx.xoff)
        const FabDev& I = Bx.in;
        const int ib[3] = { I.b0 - Bx.xoff, I.b1, I.b2 };

        auto issue = [&](int st, int buf) {
            const uint32_t bar = bars + 8 * buf;
            const uint32_t dst = wbuf + (uint32_t)(buf * Sh::kStageBytes);
            mbar_expect_tx(bar, (uint32_t)Sh::kStageBytes);
            const int P = P0 + st * S;
            int c[3];
            c[DIR] = P - ib[DIR];
            c[A] = a0 - ib[A];
            c[B_] = b0 - ib[B_];
            if constexpr (D == 2) tma_load_3d(dst, tmap, c[0], c[1], 0, bar);
            else tma_load_4d(dst, tmap, c[0], c[1], c[2], 0, bar);
        };
        if (lane == 0) {
            fence_proxy_async_smem();
#pragma unroll
            for (int s = 0; s < NST; ++s)
                if (s < nstage) issue(s, s);
        }

        // lane's element (component n, position j) of a stage buffer
        auto elem = [&](const unsigned char* sb, int n, int j) -> T {
            if constexpr (DIR == 0) {
                const uint32_t off = (uint32_t)((n * 32 + lane) * kSpan) + (((uint32_t)(j * (int)sizeof(T))) ^ xl);
                return *reinterpret_cast<const T*>(sb + off);
            } else if constexpr (DIR == 1 && D == 2) {
                return reinterpret_cast<const T*>(sb)[(n * S + j) * 32 + lane];
            } else if constexpr (DIR == 1) {
                // box (wa, S, wb, NC): ((n wb + lb) S + j) wa + la
                return reinterpret_cast<const T*>(sb)[(n * wb + lb) * S * wa + j * wa + la];
            } else {
                return reinterpret_cast<const T*>(sb)[(n * S + j) * 32 + lane];
            }
        };

        // x sweep: out-stage kk (positions P0 + kk S ..) to the fab, lanes
        // on 16-byte pieces of 16 rows per instruction (whole 32-byte
        // sectors of each row); rows outside the box and positions outside
        // [s0, s1) are not written
        auto flush = [&](int kk) {
            if constexpr (DIR == 0) {
                __syncwarp();
                constexpr int V = 16 / (int)sizeof(T);  // elements per 16 bytes
                struct alignas(16) V16 {
                    T v[V];
                };
                const int P = P0 + kk * S + (lane & 1) * V;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int r = (lane >> 1) + 16 * i;
                    const int ra = a0 + r % wa, rb = b0 + r / wa;
                    const bool row_ok = ra <= Bx.hi[A] && (D == 2 || rb <= Bx.hi[B_]);
                    const uint32_t xr = (uint32_t)((((r * kSpan) >> 7) & (kSpan / 16 - 1)) << 4);
                    T* grow = O.ptr<T>() + (long long)(row_ok ? ra - O.b1 : 0) * O.js +
                              (D == 3 ? (long long)(row_ok ? rb - O.b2 : 0) * O.ks : 0) - O.b0;
#pragma unroll
                    for (int n = 0; n < NC; ++n) {
                        const V16 v = *reinterpret_cast<const V16*>(osb + (n * 32 + r) * kSpan +
                                                                    (((uint32_t)((lane & 1) * 16)) ^ xr));
                        if (!row_ok) continue;
                        T* dst = grow + P + n * ons;
                        if (P >= s0 && P + V <= s1) {
                            *reinterpret_cast<V16*>(dst) = v;
                        } else {
#pragma unroll
                            for (int e = 0; e < V; ++e)
                                if (P + e >= s0 && P + e < s1) dst[e] = v.v[e];
                        }
                    }
                }
                __syncwarp();
            }
        };
        int flushed = -1;  // x sweep: out-stages written out so far

        T U[4][NC], UL[2][NC], UR[2][NC], F[2][NC];
#pragma unroll
        for (int s = 0; s < 4; ++s) benign(U[s]);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            benign(UL[s]);
            benign(UR[s]);
#pragma unroll
            for (int n = 0; n < NC; ++n) F[s][n] = T(0);
        }

        int st_fail = -1;
        for (int st = 0; st < nstage; ++st) {
            const int buf = st % NST;
            const bool ok = mbar_wait_bounded(bars + 8 * buf, (phase >> buf) & 1u, kTmaWaitCycles);
            if (!__all_sync(0xffffffffu, ok)) {
                failed = true;
                st_fail = st;
                break;
            }
            phase ^= 1u << buf;
            const unsigned char* sb = wbuf_p + buf * Sh::kStageBytes;
            const int qbase = P0 + st * S;
            T* orow = ocol + (long long)(qbase - 3) * ostep;
#pragma unroll
            for (int j = 0; j < S; ++j) {
                const int q = qbase + j;
                if (q > Pend) break;
                // U(q) -> slot j % 4 (U(q-1): (j+3)%4, U(q-2): (j+2)%4, U(q-3): (j+1)%4)
#pragma unroll
                for (int n = 0; n < NC; ++n) U[j % 4][n] = elem(sb, n, j);
                // face q-2 from UR(q-3) (slot (j+1)%2) and UL(q-2) (slot j%2)
                T Fn[NC];
                Sc::face(UR[(j + 1) % 2], UL[j % 2], k, f.half_dx_dt, f.dt_2dx, Fn);
                // update of cell q-3 from faces q-3 (slot (j+1)%2) and q-2
                T Un[NC];
#pragma unroll
                for (int n = 0; n < NC; ++n) Un[n] = U[(j + 1) % 4][n] - f.dtdx * (Fn[n] - F[(j + 1) % 2][n]);
                const int o = q - 3;
                const bool upd = active && o >= s0 && o < s1;
                if constexpr (DIR == 0) {
                    // position o is slot (j + S - 3) % S of out-stage st (j >= 3)
                    // or st - 1 (j < 3); that one is complete after step 2
                    const int pj = (j + S - 3) % S;
#pragma unroll
                    for (int n = 0; n < NC; ++n)
                        *reinterpret_cast<T*>(osb + (n * 32 + lane) * kSpan + (((uint32_t)(pj * (int)sizeof(T))) ^ xl)) =
                            Un[n];
                    if (j == 2 && st >= 1) {
                        flush(st - 1);
                        flushed = st - 1;
                    }
                } else if (upd) {
                    T* po = orow + (long long)j * ostep;
#pragma unroll
                    for (int n = 0; n < NC; ++n) po[n * ons] = Un[n];
                }
                if constexpr (WS) {
                    const double w = (double)Sc::speed(Un, k);
                    track_ws(upd ? w : 0.0, wsmax, nan_seen);
                }
#pragma unroll
                for (int n = 0; n < NC; ++n) F[j % 2][n] = Fn[n];
                // cell stage of cell q-1 -> slot (j+1)%2
                Sc::cell(U[(j + 2) % 4], U[(j + 3) % 4], U[j % 4], k, f.hdtdx, UL[(j + 1) % 2], UR[(j + 1) % 2]);
            }
            // every lane is done with this buffer: refill it with stage st + NST
            __syncwarp();
            if (lane == 0 && st + NST < nstage) {
                fence_proxy_async_smem();
                issue(st + NST, buf);
            }
        }
        if constexpr (DIR == 0) {
            // the out-stage holding the segment's last cell s1 - 1
            const int klast = (s1 - 1 - P0) / S;
            if (!failed && flushed < klast) flush(klast);
        }
        if (failed) {
            // let the copies still in flight (stages st_fail .. st_fail +
            // NST - 1) land, each wait bounded, before leaving
            if (lane == 0) {
                for (int s = st_fail; s < st_fail + NST && s < nstage; ++s)
                    mbar_wait_bounded(bars + 8 * (s % NST), (phase >> (s % NST)) & 1u, kTmaWaitCycles);
                if (a.status) atomicExch(a.status, 4 /* BAMREX_ERR_TIMEOUT */);
            }
            __syncwarp();
        }
    }
    if constexpr (WS) {
        if (!failed) reduce_ws(wsmax, nan_seen, a.ws_max);
    }
}

}  // namespace bamrex
