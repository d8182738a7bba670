// C ABI of libbamrex_cuda.so and the level driver (the host side of
// AmrLevelAdv::advance / advance_explicit / estTimeStep / computeNewDt for
// the explicit methods).  No C++ exception crosses the ABI: every entry point
// returns a BAMREX_* status and records a message for bamrex_last_error().
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <functional>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "bamrex_cuda.h"
#include "launch.h"
#include "level_impl.h"

using namespace bamrex;

namespace {
thread_local std::string g_last_error;
}  // namespace

namespace bamrex {

int fail(int code, const std::string& msg)
{
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char* what)
{
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return BAMREX_ERR_CUDA;
}

const char* last_error_text() { return g_last_error.c_str(); }

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

}  // namespace bamrex

int bamrex_level::set_err(int code)
{
    err = g_last_error;
    return code;
}

namespace {

bool method_supported(int m)
{
    return m == BAMREX_MUSCL_HANCOCK || m == BAMREX_HLLC || m == BAMREX_SLIC || m == BAMREX_FORCE ||
           m == BAMREX_LAX_FRIEDRICHS;
}

int method_halo(int m) { return (m == BAMREX_MUSCL_HANCOCK || m == BAMREX_SLIC) ? 2 : 1; }

// Physical constants in the reference's own expressions (HLLC.H:269-280).
int make_consts(const bamrex_parm* p, int D, Consts& k)
{
    if (!p) return fail(BAMREX_ERR_ARG, "parm is NULL");
    const double g = p->adiabatic, eps = p->epsilon;
    if (!(g > 1.0) || !std::isfinite(g)) return fail(BAMREX_ERR_ARG, "adiabatic index must be > 1");
    if (!(eps > 0.0) || !std::isfinite(eps)) return fail(BAMREX_ERR_ARG, "epsilon must be > 0");
    if (p->limiter < BAMREX_MINBEE || p->limiter > BAMREX_SUPERBEE) return fail(BAMREX_ERR_ARG, "unknown limiter");
    std::memset(&k, 0, sizeof(k));
    k.gamma = g;
    k.eps = eps;
    k.inv_eps = 1.0 / eps;
    k.gm1 = g - 1;
    k.half_gm1 = (g - 1) / 2;
    k.z = (g - 1) / (2 * g);
    k.neg_z = -k.z;
    k.inv_z = 1 / k.z;
    k.gp1_2g = (g + 1) / (2 * g);
    k.gamma_inv_eps = g / eps;
    const double kr = std::nearbyint(k.inv_z);
    if (kr >= 2 && kr <= 16 && std::fabs(k.inv_z - kr) <= 1e-12 * kr) {
        k.root_k = (int)kr;
        k.root_dpos = k.inv_z - kr;
        k.root_dneg = (double)(1.0L / (long double)kr - (long double)k.z);
        k.root_dneg_l2 = (double)((1.0L / (long double)kr - (long double)k.z) * 0.69314718055994530942L);
        k.root_dpos_l2 = (double)(((long double)k.inv_z - (long double)kr) * 0.69314718055994530942L);
    }
    k.half_eps = 0.5 * eps;
    k.limiter = p->limiter;
    const int NC = D + 2;
    bool uniform = true, need_prim = false;
    for (int n = 0; n < NC; ++n) {
        const unsigned idx = p->limiter_indices[n];
        if (idx >= (unsigned)NC)
            return fail(BAMREX_ERR_UNSUPPORTED, "limiting variable index outside the state / primitive vector");
        k.lim_var[n] = (int)idx;
        k.lim_prim[n] = p->limit_on_primv[n] ? 1 : 0;
        need_prim = need_prim || k.lim_prim[n];
        if (idx != p->limiter_indices[0] || k.lim_prim[n]) uniform = false;
    }
    k.uniform_var = uniform ? (int)p->limiter_indices[0] : -1;
    k.need_prim = need_prim ? 1 : 0;
    return BAMREX_OK;
}

FabDev to_fab(const bamrex_array4& a)
{
    FabDev f;
    f.p = a.p;
    f.js = a.jstride;
    f.ks = a.kstride;
    f.ns = a.nstride;
    f.b0 = a.begin[0];
    f.b1 = a.begin[1];
    f.b2 = a.begin[2];
    return f;
}

bool valid_box(const bamrex_box* b, int D)
{
    if (!b) return false;
    for (int d = 0; d < 3; ++d) {
        if (d < D && b->hi[d] < b->lo[d]) return false;
        if (d >= D && (b->lo[d] != 0 || b->hi[d] != 0)) return false;
    }
    return true;
}

// a covers [lo - grow_lo, hi + grow_hi] (per direction) with >= NC components
bool covers(const bamrex_array4& a, const int* lo, const int* hi, const int* glo, const int* ghi, int NC)
{
    if (!a.p || a.ncomp < NC) return false;
    for (int d = 0; d < 3; ++d)
        if (a.begin[d] > lo[d] - glo[d] || a.end[d] <= hi[d] + ghi[d]) return false;
    return true;
}

std::pair<uintptr_t, uintptr_t> byte_range(const bamrex_array4& a, int NC)
{
    const long long span = (long long)(a.end[0] - a.begin[0] - 1) + (long long)(a.end[1] - a.begin[1] - 1) * a.jstride +
                           (long long)(a.end[2] - a.begin[2] - 1) * a.kstride + (long long)(NC - 1) * a.nstride;
    const uintptr_t b = (uintptr_t)a.p;
    return { b, b + (uintptr_t)(span + 1) * sizeof(double) };
}

bool overlaps(const bamrex_array4& a, const bamrex_array4& b, int NC)
{
    auto ra = byte_range(a, NC), rb = byte_range(b, NC);
    return ra.first < rb.second && rb.first < ra.second;
}

// Work items of one box in one sweep direction.
// Work items of one box for the sweep of direction dir: warp-per-row-segment
// items for the x sweep (march = false), else segments of 32 adjacent
// columns (rows for the marching x sweep).
// The box's segments have equal lengths (at most seglen; multiples of 32
// for the row kernel), returned in box_seglen.
void box_items(int dir, const int* lo, const int* hi, int seglen, long long& items, int& nseg, int& ngroup,
               bool march = false, int* box_seglen = nullptr)
{
    const int n[3] = { hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1 };
    nseg = (n[dir] + seglen - 1) / seglen;
    int bl = (n[dir] + nseg - 1) / nseg;
    if (dir == 0 && !march) bl = std::min(seglen, (bl + 31) / 32 * 32);
    if (box_seglen) *box_seglen = bl;
    if (dir == 0 && !march) {
        ngroup = 1;
        items = (long long)n[1] * n[2] * nseg;
    } else {
        // 32 columns of the plane across dir per group (boxes narrower than
        // 32 cells fill the lanes from the next plane)
        const long long cols = (long long)(dir == 0 ? n[1] : n[0]) * (dir == 2 ? n[1] : n[2]);
        ngroup = (int)((cols + 31) / 32);
        items = (long long)ngroup * nseg;
    }
}

// Segment length: the longest that still gives every resident warp several
// items (few partial waves); x segments of the row kernel are multiples of 32.
int choose_seglen(int dir, const std::vector<bamrex_box>& boxes, long long resident_warps, bool march = false)
{
    static const int xs[] = { 2048, 1024, 512, 256, 128, 64, 32 };
    static const int ss[] = { 256, 128, 96, 64, 48, 32, 24, 16 };
    const bool rows = dir == 0 && !march;
    const int* cand = rows ? xs : ss;
    const int ncand = rows ? 7 : 8;
    const long long want = std::max(1LL, resident_warps) * 6;
    for (int c = 0; c < ncand; ++c) {
        long long tot = 0;
        int nseg, ngroup;
        long long it;
        for (const auto& b : boxes) {
            box_items(dir, b.lo, b.hi, cand[c], it, nseg, ngroup, march);
            tot += it;
        }
        if (tot >= want) return cand[c];
    }
    return cand[ncand - 1];
}

// Lane-cell slots of the two x-sweep kernels over a set of boxes: the row
// kernel spends two extra 32-cell chunks on every row segment (its
// software pipeline), the marching kernel four extra cells per segment and
// idle lanes in its last group of 32 rows; its per-cell cost
// carries a 30% allowance for staging rows through shared memory (measured
// on 4096^2 in boxes of 32 to 4096 cells).
bool prefer_x_march(int D, const std::vector<bamrex_box>& boxes, int seg_rows, int seg_march)
{
    if (D < 2) return false;
    double rows = 0, march = 0;
    for (const auto& b : boxes) {
        const long long n0 = b.hi[0] - b.lo[0] + 1, n1 = b.hi[1] - b.lo[1] + 1, n2 = b.hi[2] - b.lo[2] + 1;
        long long items;
        int nseg, ngroup, bl;
        box_items(0, b.lo, b.hi, seg_rows, items, nseg, ngroup, false, &bl);
        for (long long x = 0; x < n0; x += bl) {
            const long long len = std::min<long long>(bl, n0 - x);
            rows += (double)(n1 * n2) * 32.0 * (double)((len + 64 + 31) / 32);
        }
        box_items(0, b.lo, b.hi, seg_march, items, nseg, ngroup, true, &bl);
        for (long long x = 0; x < n0; x += bl) {
            const long long len = std::min<long long>(bl, n0 - x);
            march += 1.3 * (double)((n1 * n2 + 31) / 32 * 32) * (double)(len + 4);
        }
    }
    return march < rows;
}

// ---- TMA-staged sweeps (sweep_tma.cuh, sweep_wave.cuh): lane groups and
// segments.  An item takes NL lines (tma_item_lines): wa along the faster
// transverse direction A times NL / wa along B.
// The choice of wa among NL, NL/2, NL/4 with the fewest line slots on the
// box (2D: always NL).
int tma_wa(int D, int dir, const int* lo, const int* hi, int NL)
{
    if (D == 2) return NL;
    const int A = dir == 0 ? 1 : 0, B = dir == 2 ? 1 : 2;
    const long long nA = hi[A] - lo[A] + 1, nB = hi[B] - lo[B] + 1;
    int best = NL;
    long long bslots = -1;
    for (int wa : { NL, NL / 2, NL / 4 }) {
        const int wb = NL / wa;
        const long long slots = (nA + wa - 1) / wa * wa * ((nB + wb - 1) / wb * wb);
        if (bslots < 0 || slots < bslots) {
            best = wa;
            bslots = slots;
        }
    }
    return best;
}

// Work items of one box for a TMA-staged sweep: line groups x segments of
// equal length bl (at most seglen).  wa_in > 0 imposes the group shape (a
// part of a box swept with the box's tensor maps takes the box's).
void tma_box_items(int D, int dir, const int* lo, const int* hi, int seglen, int NL, long long& items, int& nseg,
                   int& ngroup, int& wa, int& bl, int wa_in = 0)
{
    wa = wa_in > 0 ? wa_in : tma_wa(D, dir, lo, hi, NL);
    const int wb = NL / wa;
    const int A = dir == 0 ? 1 : 0, B = dir == 2 ? 1 : 2;
    const int n[3] = { hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1 };
    nseg = (n[dir] + seglen - 1) / seglen;
    bl = (n[dir] + nseg - 1) / nseg;
    const long long ngA = (n[A] + wa - 1) / wa, ngB = D == 3 ? (n[B] + wb - 1) / wb : 1;
    ngroup = (int)(ngA * ngB);
    items = (long long)ngroup * nseg;
}

// Steps one unit (a warp of the march, a block of the wavefront) spends on
// a segment of len cells: the march's len + about 8 (warm-up, drain, first
// tile); the wavefront's passes of pw positions over len + 2, plus one for
// the first tile.
long long tma_item_cost(bool wave, int pw, int len)
{
    return wave ? ((long long)(len + 3 + pw - 1) / pw + 1) * pw : (long long)len + 8;
}

// Segment length of a TMA-staged sweep: the candidate with the shortest
// makespan when the resident units take the items round robin.
int choose_tma_seglen(int D, int dir, const std::vector<bamrex_box>& boxes, long long resident_units, bool wave)
{
    const int NL = tma_item_lines(wave, dir), pw = tma_pass_positions(wave, dir);
    // the usual lengths, and the widest box's extent split into 1 .. 24
    // equal segments
    std::vector<int> cand = { 4096, 2048, 1024, 768, 512, 384, 256, 192, 128, 96, 64, 48, 32 };
    int nmax = 1;
    for (const auto& b : boxes) nmax = std::max(nmax, b.hi[dir] - b.lo[dir] + 1);
    for (int m = 1; m <= 24; ++m)
        if ((nmax + m - 1) / m >= 32) cand.push_back((nmax + m - 1) / m);
    std::sort(cand.begin(), cand.end(), std::greater<int>());
    cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
    // every candidate >= the widest extent cuts each box into one segment:
    // the largest of them stands for all (it would win their ties)
    while (cand.size() > 1 && cand[1] >= nmax) cand.erase(cand.begin() + 1);
    const long long W = std::max(1LL, resident_units);
    // the span of each candidate, candidates on host threads when the level
    // has many boxes; the first of the smallest spans wins, as in order
    std::vector<long long> spans(cand.size(), 0);
    auto span_of = [&](int c) {
        std::vector<long long> load;
        long long total = 0;
        for (const auto& b : boxes) {
            long long it;
            int nseg, ng, wa, bl;
            tma_box_items(D, dir, b.lo, b.hi, c, NL, it, nseg, ng, wa, bl);
            total += it;
        }
        const long long nw = std::min(W, total);
        load.assign((size_t)nw, 0);
        long long idx = 0;
        for (const auto& b : boxes) {
            long long it;
            int nseg, ng, wa, bl;
            tma_box_items(D, dir, b.lo, b.hi, c, NL, it, nseg, ng, wa, bl);
            const int n = b.hi[dir] - b.lo[dir] + 1;
            for (int g = 0; g < ng; ++g)
                for (int sg = 0; sg < nseg; ++sg, ++idx)
                    load[(size_t)(idx % nw)] += tma_item_cost(wave, pw, std::min(bl, n - sg * bl));
        }
        return *std::max_element(load.begin(), load.end());
    };
    const int nth = boxes.size() >= 256 ? (int)std::min<size_t>(cand.size(), std::max(1u, std::thread::hardware_concurrency()))
                                        : 1;
    if (nth > 1) {
        std::vector<std::thread> th;
        for (int t = 0; t < nth; ++t)
            th.emplace_back([&, t] {
                for (size_t i = (size_t)t; i < cand.size(); i += (size_t)nth) spans[i] = span_of(cand[i]);
            });
        for (auto& x : th) x.join();
    } else {
        for (size_t i = 0; i < cand.size(); ++i) spans[i] = span_of(cand[i]);
    }
    int best = cand[0];
    long long best_span = -1;
    for (size_t i = 0; i < cand.size(); ++i)
        if (best_span < 0 || spans[i] < best_span) {
            best = cand[i];
            best_span = spans[i];
        }
    return best;
}

// Kernel of a sweep direction when the level leaves the choice to the
// library: the kind with the least estimated time, from the slot-steps each
// spends on the level's boxes (idle lanes, warm-up, pass rounding included,
// at the segment lengths each would choose) times a measured time per
// slot-step (B200, 4096^2 2D and 256^3 3D, per direction and storage type;
// the FP64 3D y / z march and TMA figures refitted on 256^3 levels in 16^3,
// 32^3 and 64^3 boxes, where the TMA march was the fastest y / z kernel).
// rows / march: the two L2-loading x kernels.
int auto_sweep_kind(int D, int d, bool fp32, const std::vector<bamrex_box>& boxes, int seg_rows, int seg_march,
                    int seg_tma, int seg_wave, bool allow_tma)
{
    // picoseconds per slot-step: [fp32][D - 2][d] x {rows, march, TMA, wave}
    static const double ps[2][2][3][4] = {
        { { { 28, 37, 53, 27 }, { 0, 30, 29, 29 }, { 0, 0, 0, 0 } },
          { { 39, 47, 70, 27.5 }, { 0, 31.5, 25, 28 }, { 0, 35, 27.5, 31 } } },
        { { { 12.6, 16, 18.5, 13.5 }, { 0, 15, 11, 15 }, { 0, 0, 0, 0 } },
          { { 16, 20, 23, 17 }, { 0, 19, 14, 19 }, { 0, 21, 15, 20 } } },
    };
    const double* c = ps[fp32 ? 1 : 0][D - 2][d];
    double rows = 0, march = 0, tma = 0, wave = 0;
    const int pw = tma_pass_positions(true, d), nlw = tma_item_lines(true, d);
    for (const auto& b : boxes) {
        const int n[3] = { b.hi[0] - b.lo[0] + 1, b.hi[1] - b.lo[1] + 1, b.hi[2] - b.lo[2] + 1 };
        const int A = d == 0 ? 1 : 0, B = d == 2 ? 1 : 2;
        const long long lines = (long long)n[A] * n[B];
        auto segs = [&](int seglen, auto&& per) {
            const int nseg = (n[d] + seglen - 1) / seglen, bl = (n[d] + nseg - 1) / nseg;
            for (int x = 0; x < n[d]; x += bl) per(std::min(bl, n[d] - x));
        };
        if (d == 0) segs(seg_rows, [&](int len) { rows += (double)lines * 32.0 * ((len + 64 + 31) / 32); });
        segs(seg_march, [&](int len) { march += (double)((lines + 31) / 32 * 32) * (len + 4); });
        long long it;
        int nseg, ng, wa, bl;
        tma_box_items(D, d, b.lo, b.hi, seg_tma, 32, it, nseg, ng, wa, bl);
        segs(seg_tma, [&](int len) { tma += (double)ng * 32 * (len + 8); });
        tma_box_items(D, d, b.lo, b.hi, seg_wave, nlw, it, nseg, ng, wa, bl);
        segs(seg_wave, [&](int len) { wave += (double)ng * nlw * ((len + 3 + pw - 1) / pw + 1) * pw; });
    }
    double best = d == 0 ? std::min(rows * c[0], march * c[1]) : march * c[1];
    int kind = BAMREX_STAGING_REGISTERS;
    if (allow_tma && tma * c[2] < best) {
        best = tma * c[2];
        kind = BAMREX_STAGING_TMA;
    }
    if (allow_tma && wave * c[3] < best) kind = BAMREX_STAGING_WAVE;
    return kind;
}

}  // namespace

// ======================================================================
// library identity, errors, Parm
// ======================================================================
extern "C" int bamrex_abi_version(void) { return BAMREX_ABI_VERSION; }

extern "C" const char* bamrex_last_error(void) { return g_last_error.c_str(); }

extern "C" int bamrex_release_memory(void)
{
    const int e = release_pooled();
    return e ? cuda_fail((cudaError_t)e, "release_memory") : BAMREX_OK;
}

extern "C" const char* bamrex_status_string(int status)
{
    switch (status) {
    case BAMREX_OK: return "ok";
    case BAMREX_ERR_ARG: return "invalid argument";
    case BAMREX_ERR_OOM: return "out of memory";
    case BAMREX_ERR_NAN: return "non-finite wave speed or time step";
    case BAMREX_ERR_TIMEOUT: return "device wait timed out";
    case BAMREX_ERR_CUDA: return "CUDA runtime error";
    case BAMREX_ERR_UNSUPPORTED: return "unsupported method or option";
    case BAMREX_ERR_NOT_CONVERGED: return "iterative solve did not converge";
    default: return "unknown status";
    }
}

extern "C" int bamrex_parm_set_defaults(bamrex_parm* parm, int spacedim)
{
    if (!parm) return fail(BAMREX_ERR_ARG, "parm is NULL");
    if (spacedim < 1 || spacedim > 3) return fail(BAMREX_ERR_ARG, "spacedim must be 1, 2 or 3");
    std::memset(parm, 0, sizeof(*parm));
    parm->adiabatic = -1;
    parm->eos_mu = 28.96;
    parm->Pr = 0.71;
    parm->beta = 1.5;
    parm->eta_prime = 1.716e-5;
    parm->T_prime = 273;
    parm->S_eta = 111;
    parm->epsilon = 1;
    parm->Re = 1;
    parm->limiter = BAMREX_VAN_LEER;
    for (int i = 0; i < BAMREX_MAX_NCOMP; ++i) {
        parm->limiter_indices[i] = (unsigned)(1 + spacedim);  // UInd::E
        parm->limit_on_primv[i] = 0;
    }
    parm->need_primitive_for_limiting = 0;
    return BAMREX_OK;
}

extern "C" int bamrex_parm_init(bamrex_parm* parm)
{
    if (!parm) return fail(BAMREX_ERR_ARG, "parm is NULL");
    const double a = parm->adiabatic;
    parm->adia[0] = a;
    parm->adia[1] = a + 1;
    parm->adia[2] = a - 1;
    parm->adia[3] = 1.0 / (a + 1);
    parm->adia[4] = 1.0 / (a - 1);
    parm->adia[5] = (a + 1) / (2 * a);
    parm->adia[6] = (a - 1) / (2 * a);
    parm->adia[7] = a / (a + 1);
    parm->adia[8] = a / (a - 1);
    const double Ru = 8.3145;
    parm->R_spec = Ru / (parm->eos_mu * 1e-3);
    parm->cv = parm->R_spec * parm->adia[4];
    parm->cp = a * parm->cv;
    parm->Reinv = 1.0 / parm->Re;
    unsigned char need = 0;
    for (int n = 0; n < BAMREX_MAX_NCOMP; ++n) need = need || parm->limit_on_primv[n];
    parm->need_primitive_for_limiting = need;
    return BAMREX_OK;
}

// ======================================================================
// per-box entry points (Fluxes.H / Update.H surface)
// ======================================================================
static int per_box_sweep(int method, int dir, int D, const bamrex_box* bx, const bamrex_array4* Uout,
                         const bamrex_array4& Uin, const bamrex_array4* flux, const double dx[3], double dt,
                         const bamrex_parm* parm, void* stream)
{
    if (D < 1 || D > 3) return fail(BAMREX_ERR_ARG, "spacedim must be 1, 2 or 3");
    if (dir < 0 || dir >= D) return fail(BAMREX_ERR_ARG, "dir out of range");
    if (!method_supported(method)) return fail(BAMREX_ERR_UNSUPPORTED, "method not on the explicit path");
    if (!valid_box(bx, D)) return fail(BAMREX_ERR_ARG, "invalid box");
    if (!dx || !(dx[dir] > 0)) return fail(BAMREX_ERR_ARG, "dx must be positive");
    if (!(dt > 0) || !std::isfinite(dt)) return fail(BAMREX_ERR_ARG, "dt must be positive and finite");
    Consts k;
    BX_TRY(make_consts(parm, D, k));
    const int NC = D + 2;
    const int H = method_halo(method);
    int g[3] = { 0, 0, 0 }, z3[3] = { 0, 0, 0 }, f1[3] = { 0, 0, 0 };
    g[dir] = H;
    f1[dir] = 1;
    if (!covers(Uin, bx->lo, bx->hi, g, g, NC))
        return fail(BAMREX_ERR_ARG, "consv must cover the box grown by the stencil halo in dir");
    if (Uout) {
        if (!covers(*Uout, bx->lo, bx->hi, z3, z3, NC)) return fail(BAMREX_ERR_ARG, "Uout must cover the box");
        if (overlaps(*Uout, Uin, NC)) return fail(BAMREX_ERR_ARG, "Uout and Uin must not overlap");
    }
    if (flux && flux->p) {
        if (!covers(*flux, bx->lo, bx->hi, z3, f1, NC))
            return fail(BAMREX_ERR_ARG, "flux must cover surroundingNodes(bx, dir)");
        if (overlaps(*flux, Uin, NC)) return fail(BAMREX_ERR_ARG, "flux and consv must not overlap");
    }
    SweepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.boxes = nullptr;
    a.nboxes = 1;
    SweepBox& B = a.one;
    for (int d = 0; d < 3; ++d) {
        B.lo[d] = bx->lo[d];
        B.hi[d] = bx->hi[d];
    }
    B.in = to_fab(Uin);
    if (Uout) B.out = to_fab(*Uout);
    if (flux && flux->p) B.flux = to_fab(*flux);
    const std::vector<bamrex_box> one(1, *bx);
    const bool march = dir == 0 && prefer_x_march(D, one, 512, 64);
    a.seglen = (dir == 0 && !march) ? 512 : 64;
    long long items;
    box_items(dir, B.lo, B.hi, a.seglen, items, B.nseg, B.ngroup, march, &B.seglen);
    B.item_begin = 0;
    a.total_items = items;
    a.halo = H;
    a.dt_host = dt;
    a.scal = nullptr;
    a.dx = dx[dir];
    a.k = k;
    a.ws_max = nullptr;
    a.do_update = Uout ? 1 : 0;
    BX_CK(launch_sweep(D, dir, method, false, a, (cudaStream_t)stream, march));
    return BAMREX_OK;
}

extern "C" int bamrex_compute_flux(int method, int dir, int spacedim, double time, const bamrex_box* bx,
                                   bamrex_array4 flux, bamrex_array4 consv, const double dx[3], double dt,
                                   const bamrex_parm* parm, void* stream)
{
    (void)time;
    if (!flux.p) return fail(BAMREX_ERR_ARG, "flux.p is NULL");
    return per_box_sweep(method, dir, spacedim, bx, nullptr, consv, &flux, dx, dt, parm, stream);
}

extern "C" int bamrex_sweep_box(int method, int dir, int spacedim, const bamrex_box* bx, bamrex_array4 Uout,
                                bamrex_array4 Uin, bamrex_array4 flux, const double dx[3], double dt,
                                const bamrex_parm* parm, void* stream)
{
    if (!Uout.p) return fail(BAMREX_ERR_ARG, "Uout.p is NULL");
    return per_box_sweep(method, dir, spacedim, bx, &Uout, Uin, flux.p ? &flux : nullptr, dx, dt, parm, stream);
}

extern "C" int bamrex_compute_flux_LR(int kind, int dir, int spacedim, double time, const bamrex_box* bx,
                                      bamrex_array4 flux, bamrex_array4 consv_L, bamrex_array4 consv_R,
                                      const double dx[3], double dt, const bamrex_parm* parm, void* stream)
{
    (void)time;
    const int D = spacedim;
    if (D < 1 || D > 3) return fail(BAMREX_ERR_ARG, "spacedim must be 1, 2 or 3");
    if (dir < 0 || dir >= D) return fail(BAMREX_ERR_ARG, "dir out of range");
    if (kind != BAMREX_HLLC && kind != BAMREX_FORCE) return fail(BAMREX_ERR_UNSUPPORTED, "kind must be HLLC or FORCE");
    if (!valid_box(bx, D)) return fail(BAMREX_ERR_ARG, "invalid box");
    if (!dx || !(dx[dir] > 0)) return fail(BAMREX_ERR_ARG, "dx must be positive");
    if (kind == BAMREX_FORCE && (!(dt > 0) || !std::isfinite(dt))) return fail(BAMREX_ERR_ARG, "dt must be positive");
    Consts k;
    BX_TRY(make_consts(parm, D, k));
    const int NC = D + 2;
    int z3[3] = { 0, 0, 0 }, f1[3] = { 0, 0, 0 };
    f1[dir] = 1;
    if (!flux.p || !covers(flux, bx->lo, bx->hi, z3, f1, NC))
        return fail(BAMREX_ERR_ARG, "flux must cover surroundingNodes(bx, dir)");
    if (!covers(consv_L, bx->lo, bx->hi, f1, z3, NC)) return fail(BAMREX_ERR_ARG, "consv_L must cover bx grown low by 1");
    if (!covers(consv_R, bx->lo, bx->hi, z3, f1, NC)) return fail(BAMREX_ERR_ARG, "consv_R must cover bx grown high by 1");
    BX_CK(launch_flux_LR(D, dir, kind, bx->lo, bx->hi, to_fab(flux), to_fab(consv_L),
                         to_fab(consv_R), k, dx[dir], kind == BAMREX_FORCE ? dt : 1.0, (cudaStream_t)stream));
    return BAMREX_OK;
}

extern "C" int bamrex_sweep_update(int dir, int spacedim, const bamrex_box* bx, bamrex_array4 Uout, bamrex_array4 Uin,
                                   bamrex_array4 flux, const double dx[3], double dt, void* stream)
{
    const int D = spacedim;
    if (D < 1 || D > 3) return fail(BAMREX_ERR_ARG, "spacedim must be 1, 2 or 3");
    if (dir < 0 || dir >= D) return fail(BAMREX_ERR_ARG, "dir out of range");
    if (!valid_box(bx, D)) return fail(BAMREX_ERR_ARG, "invalid box");
    if (!dx || !(dx[dir] > 0)) return fail(BAMREX_ERR_ARG, "dx must be positive");
    const int NC = D + 2;
    int z3[3] = { 0, 0, 0 }, f1[3] = { 0, 0, 0 };
    f1[dir] = 1;
    if (!covers(Uout, bx->lo, bx->hi, z3, z3, NC) || !covers(Uin, bx->lo, bx->hi, z3, z3, NC))
        return fail(BAMREX_ERR_ARG, "Uin/Uout must cover the box");
    if (!covers(flux, bx->lo, bx->hi, z3, f1, NC)) return fail(BAMREX_ERR_ARG, "flux must cover surroundingNodes(bx, dir)");
    UpdateArgs u;
    std::memset(&u, 0, sizeof(u));
    for (int d = 0; d < 3; ++d) {
        u.lo[d] = bx->lo[d];
        u.hi[d] = bx->hi[d];
    }
    u.out = to_fab(Uout);
    u.in = to_fab(Uin);
    u.flux[0] = to_fab(flux);
    u.dtdx[0] = dt / dx[dir];
    BX_CK(launch_sweep_update(D, dir, u, (cudaStream_t)stream));
    return BAMREX_OK;
}

extern "C" int bamrex_conservative_update(int spacedim, const bamrex_box* bx, bamrex_array4 out, bamrex_array4 in,
                                          const bamrex_array4* fluxes, double dt, const double idx[3], void* stream)
{
    const int D = spacedim;
    if (D < 1 || D > 3) return fail(BAMREX_ERR_ARG, "spacedim must be 1, 2 or 3");
    if (!valid_box(bx, D) || !fluxes || !idx) return fail(BAMREX_ERR_ARG, "invalid argument");
    const int NC = D + 2;
    int z3[3] = { 0, 0, 0 };
    if (!covers(out, bx->lo, bx->hi, z3, z3, NC) || !covers(in, bx->lo, bx->hi, z3, z3, NC))
        return fail(BAMREX_ERR_ARG, "in/out must cover the box");
    UpdateArgs u;
    std::memset(&u, 0, sizeof(u));
    for (int d = 0; d < 3; ++d) {
        u.lo[d] = bx->lo[d];
        u.hi[d] = bx->hi[d];
    }
    u.out = to_fab(out);
    u.in = to_fab(in);
    for (int d = 0; d < D; ++d) {
        int f1[3] = { 0, 0, 0 };
        f1[d] = 1;
        if (!covers(fluxes[d], bx->lo, bx->hi, z3, f1, NC)) return fail(BAMREX_ERR_ARG, "flux must cover surroundingNodes");
        u.flux[d] = to_fab(fluxes[d]);
        u.dtdx[d] = dt * idx[d];
    }
    BX_CK(launch_conservative_update(D, u, (cudaStream_t)stream));
    return BAMREX_OK;
}

// ======================================================================
// level
// ======================================================================
namespace bamrex {

void BoxIndex::build(const bamrex_box& dom, const std::vector<bamrex_box>& bxs, int D_)
{
    D = D_;
    boxes = &bxs;
    for (int d = 0; d < 3; ++d) {
        lo[d] = dom.lo[d];
        int mx = 1;
        for (const auto& b : bxs) mx = std::max(mx, b.hi[d] - b.lo[d] + 1);
        bs[d] = mx;
        nb[d] = (dom.hi[d] - dom.lo[d] + 1 + mx - 1) / mx;
        if (nb[d] < 1) nb[d] = 1;
    }
    buckets.assign((size_t)nb[0] * nb[1] * nb[2], {});
    for (int i = 0; i < (int)bxs.size(); ++i) {
        int a[3], c[3];
        for (int d = 0; d < 3; ++d) {
            a[d] = std::max(0, (bxs[i].lo[d] - lo[d]) / bs[d]);
            c[d] = std::min(nb[d] - 1, (bxs[i].hi[d] - lo[d]) / bs[d]);
        }
        for (int z = a[2]; z <= c[2]; ++z)
            for (int y = a[1]; y <= c[1]; ++y)
                for (int x = a[0]; x <= c[0]; ++x) buckets[((size_t)z * nb[1] + y) * nb[0] + x].push_back(i);
    }
}

void BoxIndex::query(const int* rlo, const int* rhi, std::vector<int>& out) const
{
    out.clear();
    int a[3], c[3];
    for (int d = 0; d < 3; ++d) {
        if (rhi[d] < lo[d] || rhi[d] < rlo[d]) return;
        a[d] = std::max(0, (rlo[d] - lo[d]) / bs[d]);
        c[d] = std::min(nb[d] - 1, (rhi[d] - lo[d]) / bs[d]);
        if (a[d] > c[d]) return;
    }
    for (int z = a[2]; z <= c[2]; ++z)
        for (int y = a[1]; y <= c[1]; ++y)
            for (int x = a[0]; x <= c[0]; ++x)
                for (int i : buckets[((size_t)z * nb[1] + y) * nb[0] + x]) {
                    const auto& b = (*boxes)[i];
                    bool hit = true;
                    for (int d = 0; d < 3; ++d) hit = hit && b.lo[d] <= rhi[d] && rlo[d] <= b.hi[d];
                    if (hit && std::find(out.begin(), out.end(), i) == out.end()) out.push_back(i);
                }
}

}  // namespace bamrex

namespace {

// Ghost-fill ops of direction d for every box: the two ghost slabs of
// width ngrow across the box's valid extent in the other directions.
void build_ghost_ops(const bamrex_level* L, int d, const BoxIndex& idx, std::vector<GhostOp>& ops)
{
    const int g = L->ngrow;
    const int dlo = L->domain.lo[d], dhi = L->domain.hi[d], len = dhi - dlo + 1;
    std::vector<int> hits;
    for (int b = 0; b < (int)L->boxes.size(); ++b) {
        const bamrex_box& B = L->boxes[b];
        for (int side = 0; side < 2; ++side) {
            int rlo[3], rhi[3];
            for (int q = 0; q < 3; ++q) {
                rlo[q] = B.lo[q];
                rhi[q] = B.hi[q];
            }
            if (side == 0) {
                rlo[d] = B.lo[d] - g;
                rhi[d] = B.lo[d] - 1;
            } else {
                rlo[d] = B.hi[d] + 1;
                rhi[d] = B.hi[d] + g;
            }
            // split the slab into the part inside the domain and the part outside
            int in_lo = std::max(rlo[d], dlo), in_hi = std::min(rhi[d], dhi);
            if (in_lo <= in_hi) {
                int qlo[3] = { rlo[0], rlo[1], rlo[2] }, qhi[3] = { rhi[0], rhi[1], rhi[2] };
                qlo[d] = in_lo;
                qhi[d] = in_hi;
                idx.query(qlo, qhi, hits);
                for (int s : hits) {
                    if (s == b) continue;
                    GhostOp op;
                    std::memset(&op, 0, sizeof(op));
                    op.dst = b;
                    op.src = s;
                    for (int q = 0; q < 3; ++q) {
                        op.lo[q] = std::max(qlo[q], L->boxes[s].lo[q]);
                        op.hi[q] = std::min(qhi[q], L->boxes[s].hi[q]);
                        op.mul[q] = 1;
                        op.off[q] = 0;
                    }
                    ops.push_back(op);
                }
            }
            int out_lo = rlo[d], out_hi = rhi[d];
            if (side == 0) out_hi = std::min(rhi[d], dlo - 1);
            else out_lo = std::max(rlo[d], dhi + 1);
            if (out_lo > out_hi) continue;
            const int bc = side == 0 ? L->bc_lo[d] : L->bc_hi[d];
            // ghost region outside the domain: dst cells [out_lo, out_hi] in d
            int glo[3] = { rlo[0], rlo[1], rlo[2] }, ghi[3] = { rhi[0], rhi[1], rhi[2] };
            glo[d] = out_lo;
            ghi[d] = out_hi;
            // the source region in d and the map src = off + mul * dst
            int slo[3] = { glo[0], glo[1], glo[2] }, shi[3] = { ghi[0], ghi[1], ghi[2] };
            int off = 0, mul = 1, neg = 0;
            if (bc == BAMREX_BC_PERIODIC) {
                off = side == 0 ? len : -len;
                mul = 1;
                slo[d] = glo[d] + off;
                shi[d] = ghi[d] + off;
            } else if (bc == BAMREX_BC_REFLECTIVE) {
                off = side == 0 ? 2 * dlo - 1 : 2 * dhi + 1;
                mul = -1;
                slo[d] = off - ghi[d];
                shi[d] = off - glo[d];
                neg = 1 << (1 + d);
            } else {  // transmissive: first-order extrapolation
                off = side == 0 ? dlo : dhi;
                mul = 0;
                slo[d] = off;
                shi[d] = off;
            }
            idx.query(slo, shi, hits);
            for (int s : hits) {
                const bamrex_box& S = L->boxes[s];
                GhostOp op;
                std::memset(&op, 0, sizeof(op));
                op.dst = b;
                op.src = s;
                op.negmask = neg;
                bool empty = false;
                for (int q = 0; q < 3; ++q) {
                    op.mul[q] = 1;
                    op.off[q] = 0;
                    if (q != d) {
                        op.lo[q] = std::max(glo[q], S.lo[q]);
                        op.hi[q] = std::min(ghi[q], S.hi[q]);
                    }
                    if (q != d && op.lo[q] > op.hi[q]) empty = true;
                }
                // dst range in d whose source lies in S
                int ilo = std::max(slo[d], S.lo[d]), ihi = std::min(shi[d], S.hi[d]);
                if (ilo > ihi) empty = true;
                if (empty) continue;
                op.mul[d] = mul;
                op.off[d] = off;
                if (mul == 1) {
                    op.lo[d] = ilo - off;
                    op.hi[d] = ihi - off;
                } else if (mul == -1) {
                    op.lo[d] = off - ihi;
                    op.hi[d] = off - ilo;
                } else {
                    op.lo[d] = glo[d];
                    op.hi[d] = ghi[d];
                }
                ops.push_back(op);
            }
        }
    }
}


}  // namespace

namespace bamrex {

int level_launch(bamrex_level* L, cudaError_t e, const char* what)
{
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, what));
    L->launches++;
    return BAMREX_OK;
}

int level_fill(bamrex_level* L, int d, int parity, const StepScalars* scal)
{
    if (L->nghost[d] == 0) return BAMREX_OK;
    return level_launch(L, launch_ghost_fill(L->NC, L->fp32, L->d_ghost[d], L->nghost[d], L->ghost_chunks[d], L->d_fab[parity], scal,
                                             L->stream),
                        "ghost fill");
}

// The x ghost fill of a step: without the slabs the x sweep (and the x
// flux-register faces) read from the neighbouring boxes.
int level_fill_step_x(bamrex_level* L, int parity, const StepScalars* scal)
{
    if (!x_halos_fused(L)) return level_fill(L, 0, parity, scal);
    if (L->nghost_x == 0) return BAMREX_OK;
    return level_launch(L, launch_ghost_fill(L->NC, L->fp32, L->d_ghost_x, L->nghost_x, L->ghost_chunks_x, L->d_fab[parity],
                                             scal, L->stream),
                        "ghost fill");
}

int level_sweep(bamrex_level* L, int d, int parity, double dt_host, const StepScalars* scal, bool reduce_ws,
                bool allow_timing, int part)
{
    SweepArgs a;
    std::memset(&a, 0, sizeof(a));
    a.boxes = L->d_sweep[d][parity];
    a.nboxes = (int)L->boxes.size();
    a.total_items = L->items[d];
    if (part >= 0) {
        // one part of a split sweep (its own box table)
        a.boxes = L->d_split[d][parity][part];
        a.nboxes = L->split_nboxes[d][part];
        a.total_items = L->split_items[d][part];
        if (a.total_items == 0) return BAMREX_OK;
    }
    a.seglen = L->seglen[d];
    a.halo = method_halo(L->method);
    a.dt_host = dt_host;
    a.scal = scal;
    a.dx = L->dx[d];
    a.k = L->k;
    a.ws_max = reduce_ws ? &L->d_scal->ws_bits : nullptr;
    a.do_update = 1;
    a.xnb_on = d == 0 && x_halos_fused(L) ? 1 : 0;
    const bool t = allow_timing && L->timing && L->ev_used < L->events.size();
    if (t) cudaEventRecord(L->events[L->ev_used].first, L->stream);
    int rc;
    if (L->tma(d)) {
        a.status = &L->d_scal->status;
        rc = level_launch(L, launch_sweep_tma(L->D, d, L->fp32, fast_limiter(L->D, L->method, L->k), L->wave(d), a, L->stream),
                          "TMA-staged sweep");
    } else {
        rc = level_launch(L, launch_sweep(L->D, d, L->method, L->fp32, a, L->stream, d == 0 && L->x_march), "sweep");
    }
    if (rc != BAMREX_OK) return rc;
    if (t) {
        cudaEventRecord(L->events[L->ev_used].second, L->stream);
        L->event_dir[L->ev_used] = d;
        L->ev_used++;
    }
    return BAMREX_OK;
}

int level_step(bamrex_level* L, int parity, double dt_host, StepScalars* scal, bool allow_timing, bool next_dt)
{
    // with a rigid body: FillPatch, fill_ghost_rb and fill_consv_boundary
    // (AmrLevelAdv_advance.cpp:108-116) fill every ghost cell first
    if (L->body) BX_TRY(body_fill(L, parity, scal));
    else BX_TRY(level_fill_step_x(L, parity, scal));
    int p = parity;
    for (int d = 0; d < L->D; ++d) {
        BX_TRY(level_sweep(L, d, p, dt_host, scal, d == L->D - 1, allow_timing));
        if (!L->reg_tasks[d].empty()) {
            // Flux-register faces of this sweep, from its input (buffer p,
            // which the next sweep overwrites).  The flux is scaled by dt and
            // the face area as AmrLevelAdv::advance does before
            // FineAdd/CrseInit (Source/AmrLevelAdv_advance.cpp:192-210).
            // With dt on the device the kernel forms the same product there.
            double scale = dt_host, area[2] = { 1.0, 1.0 };
            int na = 0;
            for (int e = 0; e < L->D; ++e)
                if (e != d) {
                    scale *= L->dx[e];
                    area[na++] = L->dx[e];
                }
            for (const RegisterTask& t : L->reg_tasks[d])
                BX_TRY(level_launch(L, launch_register_faces(L->D, d, L->method, L->fp32, L->k, L->d_fab[p], t, L->NC,
                                                             dt_host, L->dx[d], scale, scal, area[0], area[1],
                                                             L->stream,
                                                             d == 0 && x_halos_fused(L) ? L->d_sweep[0][p] : nullptr),
                                    "flux register faces"));
        }
        p ^= 1;
        if (d + 1 < L->D) BX_TRY(level_fill(L, d + 1, p, scal));
    }
    if (scal && next_dt)
        BX_TRY(level_launch(L, launch_step_dt(scal, L->D, L->dx[0], L->dx[1], L->dx[2], L->cfl, 1, L->stream), "step dt"));
    return BAMREX_OK;
}

}  // namespace bamrex

extern "C" int bamrex_level_create(bamrex_level** out, const bamrex_level_desc* desc, void* stream)
{
    if (!out || !desc) return fail(BAMREX_ERR_ARG, "NULL argument");
    *out = nullptr;
    const int D = desc->spacedim;
    if (D < 1 || D > 3) return fail(BAMREX_ERR_ARG, "spacedim must be 1, 2 or 3");
    if (!method_supported(desc->method)) return fail(BAMREX_ERR_UNSUPPORTED, "method not on the explicit path");
    if (desc->ngrow < 2 || desc->ngrow > 16) return fail(BAMREX_ERR_ARG, "ngrow must be in [2, 16]");
    if (desc->nboxes < 1 || !desc->boxes) return fail(BAMREX_ERR_ARG, "no boxes");
    if (!valid_box(&desc->domain, D)) return fail(BAMREX_ERR_ARG, "invalid domain");
    if (!(desc->cfl > 0)) return fail(BAMREX_ERR_ARG, "cfl must be positive");
    for (int d = 0; d < D; ++d) {
        if (!(desc->prob_hi[d] > desc->prob_lo[d])) return fail(BAMREX_ERR_ARG, "prob_hi must exceed prob_lo");
        for (int s = 0; s < 2; ++s) {
            const int bc = s ? desc->bc_hi[d] : desc->bc_lo[d];
            if (bc < BAMREX_BC_TRANSMISSIVE || bc > BAMREX_BC_REFLECTIVE) return fail(BAMREX_ERR_ARG, "unknown boundary kind");
        }
        if ((desc->bc_lo[d] == BAMREX_BC_PERIODIC) != (desc->bc_hi[d] == BAMREX_BC_PERIODIC))
            return fail(BAMREX_ERR_ARG, "periodic boundaries must be set on both sides");
    }
    BX_PROFILE("bamrex_level_create");
    ProfPhases phase("level_create:validate");
    long long covered = 0;
    for (int b = 0; b < desc->nboxes; ++b) {
        const bamrex_box& B = desc->boxes[b];
        if (!valid_box(&B, D)) return fail(BAMREX_ERR_ARG, "invalid box in box array");
        long long n = 1;
        for (int d = 0; d < 3; ++d) {
            if (B.lo[d] < desc->domain.lo[d] || B.hi[d] > desc->domain.hi[d]) return fail(BAMREX_ERR_ARG, "box outside the domain");
            n *= (long long)(B.hi[d] - B.lo[d] + 1);
        }
        covered += n;
    }
    {
        // a level's boxes are disjoint
        const std::vector<bamrex_box> bv(desc->boxes, desc->boxes + desc->nboxes);
        BoxIndex oidx;
        oidx.build(desc->domain, bv, D);
        std::vector<int> hits;
        for (int b = 0; b < desc->nboxes; ++b) {
            oidx.query(bv[b].lo, bv[b].hi, hits);
            for (int h : hits)
                if (h != b) return fail(BAMREX_ERR_ARG, "boxes of a level overlap");
        }
    }

    bamrex_level* L = new (std::nothrow) bamrex_level();
    if (!L) return fail(BAMREX_ERR_OOM, "host allocation failed");
    L->D = D;
    L->NC = D + 2;
    L->ngrow = desc->ngrow;
    L->method = desc->method;
    L->cfl = desc->cfl;
    L->parm = desc->parm;
    L->domain = desc->domain;
    for (int d = 0; d < 3; ++d) {
        L->bc_lo[d] = desc->bc_lo[d];
        L->bc_hi[d] = desc->bc_hi[d];
        L->dx[d] = d < D ? (desc->prob_hi[d] - desc->prob_lo[d]) / (double)(desc->domain.hi[d] - desc->domain.lo[d] + 1) : 1.0;
        L->prob_lo[d] = d < D ? desc->prob_lo[d] : 0.0;
    }
    L->boxes.assign(desc->boxes, desc->boxes + desc->nboxes);
    L->ncells = covered;
    if (desc->x_mode < BAMREX_XSWEEP_AUTO || desc->x_mode > BAMREX_XSWEEP_MARCH) {
        delete L;
        return fail(BAMREX_ERR_ARG, "x_mode must be BAMREX_XSWEEP_AUTO, _ROWS or _MARCH");
    }
    if (desc->precision != BAMREX_FP64 && desc->precision != BAMREX_FP32_STORAGE) {
        delete L;
        return fail(BAMREX_ERR_ARG, "precision must be BAMREX_FP64 or BAMREX_FP32_STORAGE");
    }
    L->fp32 = desc->precision == BAMREX_FP32_STORAGE;
    L->esize = L->fp32 ? 4 : 8;
    int rc = make_consts(&L->parm, D, L->k);
    if (rc != BAMREX_OK) {
        delete L;
        return rc;
    }
    cudaGetDevice(&L->device);
    if (stream) {
        L->stream = (cudaStream_t)stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete L;
            return cuda_fail(e, "cudaStreamCreateWithFlags");
        }
        L->own_stream = true;
    }

    phase.next("level_create:layout");
    // ---- layout of the state fabs: rows padded to 256 bytes, first valid
    // cell of each row 256-byte aligned.
    const int nb = desc->nboxes;
    const int g = L->ngrow;
    const int al = (int)(256 / L->esize);  // elements per 256 bytes
    const int front = (al - g % al) % al;
    L->xoff = front;
    std::vector<long long> fab_off(nb);
    long long per_buf = 0;
    for (int b = 0; b < nb; ++b) {
        const bamrex_box& B = L->boxes[b];
        const int nxg = B.hi[0] - B.lo[0] + 1 + 2 * g;
        const int nyg = D > 1 ? B.hi[1] - B.lo[1] + 1 + 2 * g : 1;
        const int nzg = D > 2 ? B.hi[2] - B.lo[2] + 1 + 2 * g : 1;
        FabDev f;
        f.js = (long long)align_up((size_t)(front + nxg), al);
        f.ks = f.js * nyg;
        f.ns = f.ks * nzg;
        f.b0 = B.lo[0] - g;
        f.b1 = D > 1 ? B.lo[1] - g : B.lo[1];
        f.b2 = D > 2 ? B.lo[2] - g : B.lo[2];
        f.p = nullptr;
        fab_off[b] = per_buf + front;
        per_buf += (long long)align_up((size_t)(f.ns * L->NC), al);
        L->fab[0].push_back(f);
        L->fab[1].push_back(f);
    }

    phase.next("level_create:sweep_tables");
    // ---- staging of each direction's sweep
    if (desc->staging < BAMREX_STAGING_AUTO || desc->staging > BAMREX_STAGING_WAVE) {
        delete L;
        return fail(BAMREX_ERR_ARG, "staging must be BAMREX_STAGING_AUTO, _REGISTERS, _TMA or _WAVE");
    }
    {
        const bool ok = tma_supported(D, L->method, L->k);
        if ((desc->staging == BAMREX_STAGING_TMA || desc->staging == BAMREX_STAGING_WAVE) && !ok) {
            delete L;
            return fail(BAMREX_ERR_UNSUPPORTED, "TMA staging needs the fast MUSCL-Hancock path (energy limiting, "
                                                "gamma 1.4) in 2D or 3D");
        }
        for (int d = 0; d < D; ++d) {
            const int want = desc->staging_dir[d] != BAMREX_STAGING_AUTO ? desc->staging_dir[d] : desc->staging;
            if (want < BAMREX_STAGING_AUTO || want > BAMREX_STAGING_WAVE) {
                delete L;
                return fail(BAMREX_ERR_ARG, "staging_dir must hold BAMREX_STAGING_* values");
            }
            if ((want == BAMREX_STAGING_TMA || want == BAMREX_STAGING_WAVE) && !ok) {
                delete L;
                return fail(BAMREX_ERR_UNSUPPORTED, "TMA staging needs the fast MUSCL-Hancock path (energy limiting, "
                                                    "gamma 1.4) in 2D or 3D");
            }
            L->sweep_kind[d] = want == BAMREX_STAGING_AUTO ? -1 : want;  // -1: decided below by the cost model
        }
    }

    // ---- items and segment lengths (each choice computed once)
    int memo_reg[3][2], memo_tma[3][2];
    for (int d = 0; d < 3; ++d)
        for (int w = 0; w < 2; ++w) memo_reg[d][w] = memo_tma[d][w] = -1;
    auto reg_seg = [&](int d, bool march) {
        int& m = memo_reg[d][march ? 1 : 0];
        if (m < 0) m = choose_seglen(d, L->boxes, sweep_resident_warps(D, d, L->method, L->fp32, L->k, march), march);
        return m;
    };
    auto tma_seg = [&](int d, bool wave) {
        int& m = memo_tma[d][wave ? 1 : 0];
        if (m < 0) {
            const int lim = fast_limiter(D, L->method, L->k);
            m = choose_tma_seglen(D, d, L->boxes, sweep_tma_resident_units(D, d, L->fp32, lim, wave), wave);
        }
        return m;
    };
    std::vector<SweepBox> sweep_host[3];
    // x-sweep kernel: one warp per row segment, or one thread per row
    // (levels of narrow boxes); automatic by the lane-slot estimate
    if (desc->x_mode == BAMREX_XSWEEP_MARCH) L->x_march = D >= 2;
    else if (desc->x_mode == BAMREX_XSWEEP_ROWS) L->x_march = false;
    else {
        const int sr = desc->x_segment > 0 ? (int)align_up((size_t)desc->x_segment, 32) : reg_seg(0, false);
        const int sm = desc->x_segment > 0 ? desc->x_segment : reg_seg(0, true);
        L->x_march = prefer_x_march(D, L->boxes, sr, sm);
    }
    for (int d = 0; d < D; ++d) {
        if (L->sweep_kind[d] >= 0) continue;
        if (!tma_supported(D, L->method, L->k)) {
            L->sweep_kind[d] = BAMREX_STAGING_REGISTERS;
            continue;
        }
        auto seg_for = [&](bool tma_kind, bool wave, bool march) {
            const int user = d == 0 ? desc->x_segment : desc->s_segment;
            if (user > 0) return user;
            return tma_kind ? tma_seg(d, wave) : reg_seg(d, march);
        };
        const int sr = d == 0 ? (int)align_up((size_t)seg_for(false, false, false), 32) : 0;
        const int sm = seg_for(false, false, d == 0);
        L->sweep_kind[d] = auto_sweep_kind(D, d, L->fp32, L->boxes, sr, sm, seg_for(true, false, false),
                                           seg_for(true, true, false), true);
    }
    for (int d = 0; d < D; ++d) {
        const bool march = d == 0 && L->x_march;
        L->seglen[d] = d == 0 ? desc->x_segment : desc->s_segment;
        if (L->seglen[d] <= 0) L->seglen[d] = L->tma(d) ? tma_seg(d, L->wave(d)) : reg_seg(d, march);
        if (d == 0 && !march && !L->tma(d)) L->seglen[d] = (int)align_up((size_t)L->seglen[d], 32);
        long long acc = 0;
        for (int b = 0; b < nb; ++b) {
            SweepBox sb;
            std::memset(&sb, 0, sizeof(sb));
            for (int q = 0; q < 3; ++q) {
                sb.lo[q] = L->boxes[b].lo[q];
                sb.hi[q] = L->boxes[b].hi[q];
            }
            long long it;
            if (L->tma(d)) {
                tma_box_items(D, d, sb.lo, sb.hi, L->seglen[d], tma_item_lines(L->wave(d), d), it, sb.nseg, sb.ngroup, sb.wa,
                              sb.seglen);
                sb.xoff = front;
            } else {
                box_items(d, sb.lo, sb.hi, L->seglen[d], it, sb.nseg, sb.ngroup, march, &sb.seglen);
            }
            sb.item_begin = acc;
            acc += it;
            sweep_host[d].push_back(sb);
        }
        L->items[d] = acc;
    }

    phase.next("level_create:ghost_ops");
    // ---- ghost ops
    BoxIndex bidx;
    bidx.build(L->domain, L->boxes, D);
    std::vector<GhostOp> ghost_host[3];
    {
        // the directions on host threads for levels of many boxes
        auto one_dir = [&](int d) {
            build_ghost_ops(L, d, bidx, ghost_host[d]);
            L->nghost[d] = (int)ghost_host[d].size();
            L->ghost_chunks[d] = number_ghost_ops(ghost_host[d]);
        };
        if (nb >= 256 && D > 1) {
            std::vector<std::thread> th;
            for (int d = 1; d < D; ++d) th.emplace_back(one_dir, d);
            one_dir(0);
            for (auto& x : th) x.join();
        } else {
            for (int d = 0; d < D; ++d) one_dir(d);
        }
    }

    // ---- x halos read in place by the marching x sweep: per box and side,
    // the same-level box that holds the box's whole x ghost slab (inside the
    // domain); the step's x fill then leaves those slabs out
    std::vector<int> xnb[2];
    std::vector<GhostOp> ghost_x;
    if (D >= 2 && L->x_march && !L->tma(0)) {
        for (int side = 0; side < 2; ++side) xnb[side].assign((size_t)nb, -1);
        std::vector<int> hits;
        int nfused = 0;
        for (int b = 0; b < nb; ++b)
            for (int side = 0; side < 2; ++side) {
                bamrex_box slab = L->boxes[b];
                if (side == 0) {
                    slab.hi[0] = slab.lo[0] - 1;
                    slab.lo[0] -= g;
                } else {
                    slab.lo[0] = slab.hi[0] + 1;
                    slab.hi[0] += g;
                }
                if (slab.lo[0] < L->domain.lo[0] || slab.hi[0] > L->domain.hi[0]) continue;
                bidx.query(slab.lo, slab.hi, hits);
                for (int q : hits) {
                    const bamrex_box& Q = L->boxes[q];
                    bool in = q != b;
                    for (int e = 0; e < 3 && in; ++e) in = Q.lo[e] <= slab.lo[e] && slab.hi[e] <= Q.hi[e];
                    if (in) {
                        xnb[side][(size_t)b] = q;
                        ++nfused;
                        break;
                    }
                }
            }
        if (nfused) {
            L->x_fused = true;
            for (const GhostOp& op : ghost_host[0]) {
                bool plain = op.src != op.dst && op.negmask == 0;
                for (int e = 0; e < 3; ++e) plain = plain && op.mul[e] == 1 && op.off[e] == 0;
                const bamrex_box& Bd = L->boxes[op.dst];
                const bool below = plain && op.src == xnb[0][(size_t)op.dst] && op.hi[0] < Bd.lo[0];
                const bool above = plain && op.src == xnb[1][(size_t)op.dst] && op.lo[0] > Bd.hi[0];
                if (!below && !above) ghost_x.push_back(op);
            }
            L->nghost_x = (int)ghost_x.size();
            L->ghost_chunks_x = number_ghost_ops(ghost_x);
        }
    }

    // ---- pack boxes
    std::vector<PackBox> pack_host(nb);
    {
        long long acc = 0;
        for (int b = 0; b < nb; ++b) {
            for (int q = 0; q < 3; ++q) {
                pack_host[b].lo[q] = L->boxes[b].lo[q];
                pack_host[b].hi[q] = L->boxes[b].hi[q];
            }
            pack_host[b].cell_begin = acc;
            acc += (long long)(L->boxes[b].hi[0] - L->boxes[b].lo[0] + 1) * (L->boxes[b].hi[1] - L->boxes[b].lo[1] + 1) *
                   (L->boxes[b].hi[2] - L->boxes[b].lo[2] + 1);
        }
    }

    phase.next("level_create:arena");
    // ---- one arena
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    L->state_bytes = (size_t)per_buf * L->esize;
    const size_t o_state0 = take((size_t)per_buf * L->esize);
    const size_t o_state1 = take((size_t)per_buf * L->esize);
    const size_t o_sums = take(sizeof(double) * nb * L->NC);
    const size_t o_fab0 = take(sizeof(FabDev) * nb);
    const size_t o_fab1 = take(sizeof(FabDev) * nb);
    size_t o_sweep[3][2] = {};
    for (int d = 0; d < D; ++d)
        for (int p = 0; p < 2; ++p) o_sweep[d][p] = take(sizeof(SweepBox) * nb);
    size_t o_ghost[3] = {};
    for (int d = 0; d < D; ++d) o_ghost[d] = take(std::max<size_t>(1, ghost_table_bytes(ghost_host[d].size(), L->ghost_chunks[d])));
    const size_t o_ghost_x = take(std::max<size_t>(1, ghost_table_bytes(ghost_x.size(), L->ghost_chunks_x)));
    // tensor maps of the TMA-staged directions: per direction and parity,
    // one 128-byte map per box (64-byte aligned, as the TMA unit requires)
    constexpr size_t kMapBytes = 128;
    size_t o_tmap[3][2] = {};
    for (int d = 0; d < D; ++d)
        if (L->tma(d))
            for (int p = 0; p < 2; ++p) o_tmap[d][p] = take(kMapBytes * nb);
    const size_t o_pack = take(sizeof(PackBox) * nb);
    const size_t o_scal = take(sizeof(StepScalars));
    cudaError_t e = dev_alloc((void**)&L->arena, off, L->stream);
    if (e != cudaSuccess) {
        if (L->own_stream) cudaStreamDestroy(L->stream);
        delete L;
        return fail(BAMREX_ERR_OOM, std::string("allocation of the level arena failed: ") + cudaGetErrorString(e));
    }
    e = pinned_small_alloc((void**)&L->h_scal, sizeof(StepScalars));
    if (e != cudaSuccess) {
        dev_free(L->arena, L->stream);
        if (L->own_stream) cudaStreamDestroy(L->stream);
        delete L;
        return fail(BAMREX_ERR_OOM, "pinned host allocation failed");
    }
    L->state[0] = L->arena + o_state0;
    L->state[1] = L->arena + o_state1;
    L->d_box_sums = (double*)(L->arena + o_sums);
    for (int p = 0; p < 2; ++p)
        for (int b = 0; b < nb; ++b) L->fab[p][b].p = L->state[p] + (size_t)fab_off[b] * L->esize;
    L->d_fab[0] = (FabDev*)(L->arena + o_fab0);
    L->d_fab[1] = (FabDev*)(L->arena + o_fab1);
    for (int d = 0; d < D; ++d) {
        for (int p = 0; p < 2; ++p) L->d_sweep[d][p] = (SweepBox*)(L->arena + o_sweep[d][p]);
        L->d_ghost[d] = (GhostOp*)(L->arena + o_ghost[d]);
    }
    L->d_ghost_x = (GhostOp*)(L->arena + o_ghost_x);
    L->d_pack = (PackBox*)(L->arena + o_pack);
    L->d_scal = (StepScalars*)(L->arena + o_scal);

    phase.next("level_create:upload");
    // upload tables on the level's stream (ordered before its kernels),
    // then wait for them: setup only
    auto up = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
        if (!bytes) return cudaSuccess;
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, L->stream);
    };
    cudaError_t ue = cudaSuccess;
    for (int p = 0; p < 2 && ue == cudaSuccess; ++p) ue = up(L->d_fab[p], L->fab[p].data(), sizeof(FabDev) * nb);
    for (int d = 0; d < D && ue == cudaSuccess; ++d) {
        for (int p = 0; p < 2 && ue == cudaSuccess; ++p) {
            std::vector<SweepBox> t = sweep_host[d];
            for (int b = 0; b < nb; ++b) {
                t[b].in = L->fab[p][b];
                t[b].out = L->fab[p ^ 1][b];
                t[b].flux.p = nullptr;
                if (d == 0 && L->x_fused)
                    for (int side = 0; side < 2; ++side)
                        if (xnb[side][(size_t)b] >= 0) t[b].xnb[side] = L->fab[p][(size_t)xnb[side][(size_t)b]];
            }
            if (L->tma(d)) {
                struct alignas(64) Map {
                    unsigned char b[kMapBytes];
                };
                std::vector<Map> maps((size_t)nb);
                char* dmaps = L->arena + o_tmap[d][p];
                L->d_tmap[d][p] = dmaps;
                for (int b = 0; b < nb && ue == cudaSuccess; ++b) {
                    const FabDev& f = L->fab[p][b];
                    const bamrex_box& Bb = L->boxes[b];
                    const int nyg = D > 1 ? Bb.hi[1] - Bb.lo[1] + 1 + 2 * g : 1;
                    const int nzg = D > 2 ? Bb.hi[2] - Bb.lo[2] + 1 + 2 * g : 1;
                    const char* row0 = static_cast<const char*>(f.p) - (size_t)front * L->esize;
                    ue = encode_sweep_tmap(maps[(size_t)b].b, L->fp32, D, L->NC, d, L->wave(d), t[b].wa, row0, f.js, f.ks,
                                           f.ns, nyg, nzg);
                    t[b].tmap = dmaps + (size_t)b * kMapBytes;
                }
                if (ue == cudaSuccess) ue = up(dmaps, maps.data(), kMapBytes * nb);
            }
            if (ue == cudaSuccess) ue = up(L->d_sweep[d][p], t.data(), sizeof(SweepBox) * nb);
        }
        if (ue == cudaSuccess) ue = up(L->d_ghost[d], ghost_host[d].data(), sizeof(GhostOp) * ghost_host[d].size());
        if (ue == cudaSuccess) {
            const std::vector<int> ct = ghost_chunk_table(ghost_host[d], L->ghost_chunks[d]);
            ue = up(L->d_ghost[d] + ghost_host[d].size(), ct.data(), sizeof(int) * ct.size());
        }
    }
    if (ue == cudaSuccess && L->x_fused) {
        ue = up(L->d_ghost_x, ghost_x.data(), sizeof(GhostOp) * ghost_x.size());
        if (ue == cudaSuccess) {
            const std::vector<int> ct = ghost_chunk_table(ghost_x, L->ghost_chunks_x);
            ue = up(L->d_ghost_x + ghost_x.size(), ct.data(), sizeof(int) * ct.size());
        }
    }
    if (ue == cudaSuccess) ue = up(L->d_pack, pack_host.data(), sizeof(PackBox) * nb);
    if (ue == cudaSuccess) ue = cudaMemsetAsync(L->arena + o_state0, 0, (size_t)(o_state1 - o_state0) * 2, L->stream);
    if (ue == cudaSuccess) ue = cudaMemsetAsync(L->d_scal, 0, sizeof(StepScalars), L->stream);
    if (ue == cudaSuccess) ue = cudaStreamSynchronize(L->stream);
    if (ue != cudaSuccess) {
        const int r = cuda_fail(ue, "level table upload");
        bamrex_level_destroy(L);
        return r;
    }
    *out = L;
    return BAMREX_OK;
}

extern "C" int bamrex_level_destroy(bamrex_level* L)
{
    if (!L) return BAMREX_OK;
    if (L->stream) cudaStreamSynchronize(L->stream);
    body_destroy(L);
    if (L->hs) {
        if (L->hs->h2d) cudaStreamSynchronize(L->hs->h2d);
        if (L->hs->d2h) cudaStreamSynchronize(L->hs->d2h);
        for (cudaEvent_t e : L->hs->in) cudaEventDestroy(e);
        for (cudaEvent_t e : L->hs->out) cudaEventDestroy(e);
        for (cudaEvent_t e : L->hs->done) cudaEventDestroy(e);
        if (L->hs->start) cudaEventDestroy(L->hs->start);
        if (L->hs->h2d) cudaStreamDestroy(L->hs->h2d);
        if (L->hs->d2h) cudaStreamDestroy(L->hs->d2h);
        dev_free(L->hs->staging_out, L->stream);
        dev_free(L->hs->slab_tab, L->stream);
        delete L->hs;
        L->hs = nullptr;
    }
    for (int p = 0; p < 2; ++p)
        if (L->graph[p]) cudaGraphExecDestroy(L->graph[p]);
    for (auto& ev : L->events) {
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    dev_free(L->arena, L->stream);
    dev_free(L->staging, L->stream);
    dev_free(L->tag_buf, L->stream);
    for (int d = 0; d < 3; ++d) dev_free(L->halo_mem[d], L->stream);
    for (int d = 0; d < 3; ++d) dev_free(L->split_mem[d], L->stream);
    pinned_small_free(L->h_scal);
    if (L->own_stream && L->stream) cudaStreamDestroy(L->stream);
    delete L;
    return BAMREX_OK;
}

extern "C" const char* bamrex_level_last_error(const bamrex_level* L) { return L ? L->err.c_str() : ""; }

extern "C" long long bamrex_level_num_cells(const bamrex_level* L) { return L ? L->ncells : 0; }

extern "C" void* bamrex_level_stream(const bamrex_level* L) { return L ? (void*)L->stream : nullptr; }

extern "C" int bamrex_level_fab(const bamrex_level* L, int box, bamrex_array4* out)
{
    if (!L || !out || box < 0 || box >= (int)L->boxes.size()) return fail(BAMREX_ERR_ARG, "bad level/box");
    // bamrex_array4 describes doubles only: a float fab handed out as one
    // would let an Array4 consumer read twice as far as the buffer goes
    if (L->fp32)
        return fail(BAMREX_ERR_UNSUPPORTED,
                    "bamrex_level_fab: an FP32-storage level holds floats, which bamrex_array4 cannot describe");
    const FabDev& f = L->fab[L->cur][box];
    const bamrex_box& B = L->boxes[box];
    out->p = static_cast<double*>(f.p);
    out->jstride = f.js;
    out->kstride = f.ks;
    out->nstride = f.ns;
    out->begin[0] = f.b0;
    out->begin[1] = f.b1;
    out->begin[2] = f.b2;
    const int g = L->ngrow;
    out->end[0] = B.hi[0] + g + 1;
    out->end[1] = L->D > 1 ? B.hi[1] + g + 1 : B.hi[1] + 1;
    out->end[2] = L->D > 2 ? B.hi[2] + g + 1 : B.hi[2] + 1;
    out->ncomp = L->NC;
    return BAMREX_OK;
}

extern "C" int bamrex_level_x_mode(const bamrex_level* L)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    return L->x_march ? BAMREX_XSWEEP_MARCH : BAMREX_XSWEEP_ROWS;
}

extern "C" int bamrex_level_staging(const bamrex_level* L, int dir)
{
    if (!L || dir < 0 || dir >= L->D) return -fail(BAMREX_ERR_ARG, "bad level/direction");
    return L->sweep_kind[dir];
}

namespace bamrex {

int level_staging_ready(bamrex_level* L)
{
    if (L->staging) return BAMREX_OK;
    void* p = nullptr;
    const cudaError_t e = dev_alloc(&p, (size_t)L->ncells * L->NC * 8, L->stream);
    if (e != cudaSuccess)
        return L->set_err(fail(BAMREX_ERR_OOM, std::string("allocation of the level's host staging buffer failed: ") +
                                                   cudaGetErrorString(e)));
    L->staging = static_cast<double*>(p);
    return BAMREX_OK;
}

}  // namespace bamrex

extern "C" int bamrex_level_copy_in(bamrex_level* L, const double* src)
{
    if (!L || !src) return fail(BAMREX_ERR_ARG, "NULL argument");
    cudaPointerAttributes at;
    const double* from = src;
    if (cudaPointerGetAttributes(&at, src) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        BX_TRY(level_staging_ready(L));
        const cudaError_t e = cudaMemcpyAsync(L->staging, src, (size_t)L->ncells * L->NC * 8, cudaMemcpyDefault, L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "copy_in memcpy"));
        from = L->staging;
    }
    BX_TRY(level_launch(L, launch_pack(L->NC, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(), L->ncells,
                                       const_cast<double*>(from), 0, L->stream),
                        "unpack"));
    L->ws_valid = false;
    return BAMREX_OK;
}

extern "C" int bamrex_level_copy_out(bamrex_level* L, double* dst)
{
    if (!L || !dst) return fail(BAMREX_ERR_ARG, "NULL argument");
    cudaPointerAttributes at;
    const bool dev = cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    if (!dev) BX_TRY(level_staging_ready(L));
    double* to = dev ? dst : L->staging;
    BX_TRY(level_launch(L, launch_pack(L->NC, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(), L->ncells, to, 1, L->stream),
                        "pack"));
    if (!dev) {
        const cudaError_t e = cudaMemcpyAsync(dst, L->staging, (size_t)L->ncells * L->NC * 8, cudaMemcpyDefault, L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "copy_out memcpy"));
    }
    return BAMREX_OK;
}

namespace {

// Slabs of a streamed host step (0: the level cannot be streamed): single
// box, 2D/3D, no flux registers or rigid body, not periodic in the last
// direction, at least 4 layers a slab.
int host_slabs(const bamrex_level* L, int nslabs)
{
    const int D = L->D, a = D - 1;
    bool reg = false;
    for (int d = 0; d < 3; ++d) reg = reg || !L->reg_tasks[d].empty();
    if (L->boxes.size() != 1 || D < 2 || reg || L->body || L->bc_lo[a] == BAMREX_BC_PERIODIC) return 0;
    const int rows = L->boxes[0].hi[a] - L->boxes[0].lo[a] + 1;
    if (nslabs <= 0) {
        // automatic: slabs of at least 16 MiB per component (smaller copies
        // lose PCIe bandwidth when both directions run), 2 to 64 of them
        const long long comp_bytes = (long long)sizeof(double) * L->ncells;
        nslabs = (int)std::max(2LL, std::min(64LL, comp_bytes / (16LL << 20)));
    }
    const int C = std::max(1, std::min(nslabs, rows / 4));
    return C >= 2 ? C : 0;
}

int host_stream_setup(bamrex_level* L, int C)
{
    BX_TRY(level_staging_ready(L));
    cudaError_t e = cudaSuccess;
    if (!L->hs) {
        L->hs = new (std::nothrow) bamrex_level::HostStream();
        if (!L->hs) return L->set_err(fail(BAMREX_ERR_OOM, "host allocation failed"));
        e = cudaStreamCreateWithFlags(&L->hs->h2d, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&L->hs->d2h, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&L->hs->start, cudaEventDisableTiming);
        if (e == cudaSuccess) e = dev_alloc((void**)&L->hs->staging_out, (size_t)L->ncells * L->NC * 8, L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "host-stream set-up"));
    }
    bamrex_level::HostStream& H = *L->hs;
    bool any_tma = false;
    for (int d = 0; d < L->D; ++d) any_tma = any_tma || L->tma(d);
    if (any_tma && H.slabs != C) {
        // the slabs' box-table entries of the TMA-staged directions (the
        // whole fab's tensor maps serve every slab)
        const int D = L->D, a = D - 1;
        const bamrex_box B = L->boxes[0];
        const int rows = B.hi[a] - B.lo[a] + 1;
        std::vector<SweepBox> tab((size_t)3 * 2 * C);
        H.slab_items.assign((size_t)3 * 2 * C, 0);
        for (int d = 0; d < D; ++d) {
            if (!L->tma(d)) continue;
            for (int p = 0; p < 2; ++p)
                for (int c = 0; c < C; ++c) {
                    SweepBox& sb = tab[((size_t)d * 2 + p) * C + c];
                    std::memset(&sb, 0, sizeof(sb));
                    for (int q = 0; q < 3; ++q) {
                        sb.lo[q] = B.lo[q];
                        sb.hi[q] = B.hi[q];
                    }
                    sb.lo[a] = B.lo[a] + (int)((long long)rows * c / C);
                    sb.hi[a] = B.lo[a] + (int)((long long)rows * (c + 1) / C) - 1;
                    sb.in = L->fab[p][0];
                    sb.out = L->fab[p ^ 1][0];
                    sb.flux.p = nullptr;
                    // the group shape of the whole box, which its tensor
                    // maps' boxes are cut to
                    const int NL = tma_item_lines(L->wave(d), d);
                    long long it = 0;
                    tma_box_items(D, d, sb.lo, sb.hi, L->seglen[d], NL, it, sb.nseg, sb.ngroup, sb.wa, sb.seglen,
                                  tma_wa(D, d, B.lo, B.hi, NL));
                    sb.item_begin = 0;
                    sb.tmap = L->d_tmap[d][p];
                    sb.xoff = L->xoff;
                    H.slab_items[((size_t)d * 2 + p) * C + c] = it;
                }
        }
        dev_free(H.slab_tab, L->stream);
        H.slab_tab = nullptr;
        H.slabs = 0;
        e = dev_alloc((void**)&H.slab_tab, sizeof(SweepBox) * tab.size(), L->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(H.slab_tab, tab.data(), sizeof(SweepBox) * tab.size(), cudaMemcpyHostToDevice, L->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "slab box tables"));
        H.slabs = C;
    }
    while ((int)H.in.size() < C) {
        cudaEvent_t ev[3] = { nullptr, nullptr, nullptr };
        for (int q = 0; q < 3 && e == cudaSuccess; ++q) e = cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "host-stream events"));
        H.in.push_back(ev[0]);
        H.out.push_back(ev[1]);
        H.done.push_back(ev[2]);
    }
    return BAMREX_OK;
}

// Enqueue one step of a host-resident state streamed in C slabs along the
// last direction: the upload of slab c, the sweeps of the other directions
// on slab c, the last direction's sweep on slab c - 1 (its stencil reaches
// two cells into slab c) and the download of slab c - 1 run on three
// streams at once.  Every ghost fill covers the whole box and a slab's
// cells are swept only after the cells their stencils read are final, so
// the result is the plain step's.  device_dt: dt from the step scalars and
// the next dt computed at the end of the step (time, steps advanced);
// chained: slab c's upload waits for the previous step's download of slab c
// (the host buffer is read and written in place).
int host_step_enqueue(bamrex_level* L, const double* host_in, double* host_out, int C, double dt_host, bool device_dt,
                      bool chained)
{
    bamrex_level::HostStream& H = *L->hs;
    const int D = L->D, a = D - 1;
    const bamrex_box B = L->boxes[0];
    const int rows = B.hi[a] - B.lo[a] + 1;
    long long plane = 1;  // cells of one layer across the last direction
    for (int d = 0; d < D - 1; ++d) plane *= (long long)(B.hi[d] - B.lo[d] + 1);
    auto lo_of = [&](int c) { return B.lo[a] + (int)((long long)rows * c / C); };
    auto slab_box = [&](int c) {
        PackBox pb;
        for (int d = 0; d < 3; ++d) {
            pb.lo[d] = B.lo[d];
            pb.hi[d] = B.hi[d];
        }
        pb.lo[a] = lo_of(c);
        pb.hi[a] = lo_of(c + 1) - 1;
        pb.cell_begin = 0;
        return pb;
    };
    // staging (in) and staging_out hold the packed layout of the whole box
    // ([n][cells], x fastest); a slab is one range inside every component,
    // moved by one strided copy (NC rows, a component apart) where the pitch
    // allows: PCIe keeps both directions at full rate with few large copies,
    // not with one small copy per component
    auto copies = [&](int c, bool to_host, cudaStream_t s) -> cudaError_t {
        const long long first = (long long)(lo_of(c) - B.lo[a]) * plane, cells = (long long)(lo_of(c + 1) - lo_of(c)) * plane;
        const size_t pitch = sizeof(double) * (size_t)L->ncells;
        if (pitch <= (size_t)INT_MAX) {
            const size_t off = (size_t)first;
            return to_host ? cudaMemcpy2DAsync(host_out + off, pitch, H.staging_out + off, pitch, sizeof(double) * cells,
                                               L->NC, cudaMemcpyDeviceToHost, s)
                           : cudaMemcpy2DAsync(L->staging + off, pitch, host_in + off, pitch, sizeof(double) * cells, L->NC,
                                               cudaMemcpyHostToDevice, s);
        }
        for (int n = 0; n < L->NC; ++n) {
            const size_t off = (size_t)(n * L->ncells + first);
            const cudaError_t r = to_host
                ? cudaMemcpyAsync(host_out + off, H.staging_out + off, sizeof(double) * cells, cudaMemcpyDeviceToHost, s)
                : cudaMemcpyAsync(L->staging + off, host_in + off, sizeof(double) * cells, cudaMemcpyHostToDevice, s);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    };
    PackBox whole;
    for (int d = 0; d < 3; ++d) {
        whole.lo[d] = B.lo[d];
        whole.hi[d] = B.hi[d];
    }
    whole.cell_begin = 0;
    const int cur = L->cur;
    const int p_lag = cur ^ ((D - 1) & 1), p_out = cur ^ (D & 1);
    cudaError_t e = cudaSuccess;
    if (!device_dt) e = cudaMemsetAsync(&L->d_scal->ws_bits, 0, sizeof(unsigned long long), L->stream);
    if (!chained) {
        // the first step waits for everything queued on the level before it;
        // a chained step's dependencies on its predecessor are per slab
        if (e == cudaSuccess) e = cudaEventRecord(H.start, L->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(H.h2d, H.start, 0);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(H.d2h, H.start, 0);
    }
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "host-stream start"));
    auto slab_sweep = [&](int dir, int c, int pin, bool ws) -> int {
        SweepArgs sa;
        std::memset(&sa, 0, sizeof(sa));
        if (L->tma(dir)) {
            // the level's own kernel for this direction, on the slab's entry
            // of the slab box table: the same arithmetic as the plain step
            const size_t idx = ((size_t)dir * 2 + pin) * C + c;
            sa.boxes = H.slab_tab + idx;
            sa.nboxes = 1;
            sa.total_items = H.slab_items[idx];
            sa.seglen = L->seglen[dir];
            sa.halo = method_halo(L->method);
            sa.dt_host = dt_host;
            sa.scal = device_dt ? L->d_scal : nullptr;
            sa.dx = L->dx[dir];
            sa.k = L->k;
            sa.ws_max = ws ? &L->d_scal->ws_bits : nullptr;
            sa.do_update = 1;
            sa.status = &L->d_scal->status;
            return level_launch(L, launch_sweep_tma(D, dir, L->fp32, fast_limiter(D, L->method, L->k), L->wave(dir), sa,
                                                    L->stream),
                                "slab sweep");
        }
        sa.boxes = nullptr;
        sa.nboxes = 1;
        SweepBox& sb = sa.one;
        const PackBox pb = slab_box(c);
        for (int d = 0; d < 3; ++d) {
            sb.lo[d] = pb.lo[d];
            sb.hi[d] = pb.hi[d];
        }
        sb.in = L->fab[pin][0];
        sb.out = L->fab[pin ^ 1][0];
        sb.flux.p = nullptr;
        const bool march = dir == 0 && L->x_march;
        long long items;
        box_items(dir, sb.lo, sb.hi, L->seglen[dir], items, sb.nseg, sb.ngroup, march, &sb.seglen);
        sb.item_begin = 0;
        sa.total_items = items;
        sa.seglen = L->seglen[dir];
        sa.halo = method_halo(L->method);
        sa.dt_host = dt_host;
        sa.scal = device_dt ? L->d_scal : nullptr;
        sa.dx = L->dx[dir];
        sa.k = L->k;
        sa.ws_max = ws ? &L->d_scal->ws_bits : nullptr;
        sa.do_update = 1;
        return level_launch(L, launch_sweep(D, dir, L->method, L->fp32, sa, L->stream, march), "slab sweep");
    };
    const StepScalars* gate = device_dt ? L->d_scal : nullptr;
    auto lagged = [&](int c) -> int {
        BX_TRY(level_fill(L, a, p_lag, gate));
        BX_TRY(slab_sweep(a, c, p_lag, true));
        BX_TRY(level_launch(L, launch_pack_slab(L->NC, L->fp32, L->fab[p_out][0], whole, slab_box(c), H.staging_out, 1,
                                                L->stream),
                            "slab pack"));
        cudaError_t r = cudaEventRecord(H.out[c], L->stream);
        if (r == cudaSuccess) r = cudaStreamWaitEvent(H.d2h, H.out[c], 0);
        if (r == cudaSuccess) r = copies(c, true, H.d2h);
        if (r == cudaSuccess) r = cudaEventRecord(H.done[c], H.d2h);
        return r == cudaSuccess ? BAMREX_OK : L->set_err(cuda_fail(r, "slab download"));
    };
    for (int c = 0; c < C; ++c) {
        // the previous step has read this slab's device rows (packed) and
        // written its host rows (downloaded) once its download is done
        if (chained) e = cudaStreamWaitEvent(H.h2d, H.done[c], 0);
        if (e == cudaSuccess) e = copies(c, false, H.h2d);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "slab upload"));
        BX_TRY(level_launch(L, launch_pack_slab(L->NC, L->fp32, L->fab[cur][0], whole, slab_box(c), L->staging, 0, H.h2d),
                            "slab unpack"));
        e = cudaEventRecord(H.in[c], H.h2d);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(L->stream, H.in[c], 0);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "slab event"));
        int p = cur;
        for (int d = 0; d < D - 1; ++d) {
            BX_TRY(level_fill(L, d, p, gate));
            BX_TRY(slab_sweep(d, c, p, false));
            p ^= 1;
        }
        if (c > 0) BX_TRY(lagged(c - 1));
    }
    BX_TRY(lagged(C - 1));
    if (device_dt)
        BX_TRY(level_launch(L, launch_step_dt(L->d_scal, D, L->dx[0], L->dx[1], L->dx[2], L->cfl, 1, L->stream), "step dt"));
    L->cur = p_out;
    L->ws_valid = !device_dt;
    return BAMREX_OK;
}

}  // namespace

extern "C" int bamrex_level_step_host(bamrex_level* L, const double* host_in, double* host_out, double dt,
                                      int nslabs, double* dt_next)
{
    if (!L || !host_in || !host_out) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (!(dt > 0) || !std::isfinite(dt)) return L->set_err(fail(BAMREX_ERR_ARG, "dt must be positive and finite"));
    const int C = host_slabs(L, nslabs);
    if (!C) {
        // not streamable: the plain sequence
        BX_TRY(bamrex_level_copy_in(L, host_in));
        BX_TRY(bamrex_level_advance(L, 0.0, dt, 1, 1, nullptr));
        if (dt_next) BX_TRY(bamrex_level_est_time_step(L, dt_next));
        BX_TRY(bamrex_level_copy_out(L, host_out));
        return bamrex_level_sync(L);
    }
    BX_TRY(host_stream_setup(L, C));
    BX_TRY(host_step_enqueue(L, host_in, host_out, C, dt, false, false));
    cudaError_t e = cudaStreamSynchronize(L->hs->d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "host step"));
    if (dt_next) BX_TRY(bamrex_level_est_time_step(L, dt_next));
    return BAMREX_OK;
}

extern "C" int bamrex_level_run_host(bamrex_level* L, double* host, int nsteps, double dt0, int nslabs, double* time_io,
                                     double* dt_next)
{
    if (!L || !host || !time_io) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (nsteps < 0) return L->set_err(fail(BAMREX_ERR_ARG, "nsteps must be >= 0"));
    if (!(dt0 > 0) || !std::isfinite(dt0)) return L->set_err(fail(BAMREX_ERR_ARG, "dt0 must be positive and finite"));
    const int C = host_slabs(L, nslabs);
    if (!C) {
        // not streamable: one plain host step after the other
        double t = *time_io, dt = dt0;
        for (int st = 0; st < nsteps; ++st) {
            double nxt = 0.0;
            BX_TRY(bamrex_level_step_host(L, host, host, dt, nslabs, &nxt));
            t += dt;
            dt = nxt;
        }
        *time_io = t;
        if (dt_next) *dt_next = dt;
        return BAMREX_OK;
    }
    BX_TRY(host_stream_setup(L, C));
    StepScalars* h = L->h_scal;
    std::memset(h, 0, sizeof(*h));
    h->time = *time_io;
    h->dt = dt0;
    h->stop_time = -1.0;
    cudaError_t e = cudaMemcpyAsync(L->d_scal, h, sizeof(StepScalars), cudaMemcpyHostToDevice, L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "scalars upload"));
    for (int s = 0; s < nsteps; ++s) BX_TRY(host_step_enqueue(L, host, host, C, 0.0, true, s > 0));
    e = cudaMemcpyAsync(h, L->d_scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->hs->d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "host run"));
    if (h->status != 0)
        return L->set_err(fail(h->status, h->status == BAMREX_ERR_TIMEOUT ? "a sweep gave up waiting for its staged input"
                                                                          : "non-finite time step during the run"));
    *time_io = h->time;
    if (dt_next) *dt_next = h->dt;
    return BAMREX_OK;
}

extern "C" int bamrex_level_host_slabs(const bamrex_level* L, int nslabs, int* slabs)
{
    if (!L || !slabs) return fail(BAMREX_ERR_ARG, "NULL argument");
    *slabs = host_slabs(L, nslabs);
    return BAMREX_OK;
}

extern "C" int bamrex_level_sync(bamrex_level* L)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    const cudaError_t e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "cudaStreamSynchronize"));
    return BAMREX_OK;
}

extern "C" int bamrex_level_conserved_sums(bamrex_level* L, double* totals)
{
    if (!L || !totals) return fail(BAMREX_ERR_ARG, "NULL argument");
    const int nb = (int)L->boxes.size();
    BX_TRY(level_launch(L, launch_box_sums(L->NC, L->fp32, L->d_fab[L->cur], L->d_pack, nb, L->d_box_sums, L->stream),
                        "box sums"));
    std::vector<double> h((size_t)nb * L->NC);
    cudaError_t e = cudaMemcpyAsync(h.data(), L->d_box_sums, h.size() * sizeof(double), cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "conserved sums"));
    double vol = 1.0;
    for (int d = 0; d < L->D; ++d) vol *= L->dx[d];
    for (int n = 0; n < L->NC; ++n) {
        double s = 0.0;
        for (int b = 0; b < nb; ++b) s += h[(size_t)b * L->NC + n];  // fixed box order
        totals[n] = s * vol;
    }
    return BAMREX_OK;
}

extern "C" int bamrex_level_fill_boundary(bamrex_level* L)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    for (int d = 0; d < L->D; ++d) BX_TRY(level_fill(L, d, L->cur, nullptr));
    return BAMREX_OK;
}

extern "C" int bamrex_level_advance(bamrex_level* L, double time, double dt, int iteration, int ncycle, double* dt_out)
{
    (void)time;
    (void)iteration;
    (void)ncycle;
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (!(dt > 0) || !std::isfinite(dt)) return L->set_err(fail(BAMREX_ERR_ARG, "dt must be positive and finite"));
    {
        const cudaError_t e = cudaMemsetAsync(&L->d_scal->ws_bits, 0, sizeof(unsigned long long), L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "memset"));
    }
    BX_TRY(level_step(L, L->cur, dt, nullptr, true));
    L->cur ^= (L->D & 1);
    L->ws_valid = true;
    if (dt_out) *dt_out = dt;
    return BAMREX_OK;
}

extern "C" int bamrex_level_est_time_step(bamrex_level* L, double* dt_est)
{
    if (!L || !dt_est) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (!L->ws_valid) {
        cudaError_t e = cudaMemsetAsync(&L->d_scal->ws_bits, 0, sizeof(unsigned long long), L->stream);
        if (e != cudaSuccess) return L->set_err(cuda_fail(e, "memset"));
        BX_TRY(level_launch(L, launch_max_wave_speed(L->D, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(), L->ncells, L->k,
                                                     &L->d_scal->ws_bits, nullptr, L->stream),
                            "max wave speed"));
    }
    cudaError_t e = cudaMemcpyAsync(L->h_scal, L->d_scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "est_time_step"));
    if (L->h_scal->status == BAMREX_ERR_ARG)
        return L->set_err(fail(BAMREX_ERR_ARG, "a rigid-body interpolation stencil left the fab: raise ngrow"));
    if (L->h_scal->status == BAMREX_ERR_NOT_CONVERGED)
        return L->set_err(fail(BAMREX_ERR_NOT_CONVERGED, "an exact Riemann solve at a rigid-body interface did not converge"));
    if (L->h_scal->status == BAMREX_ERR_TIMEOUT)
        return L->set_err(fail(BAMREX_ERR_TIMEOUT, "a sweep gave up waiting for its staged input"));
    L->ws_valid = true;
    const double ms = [&] {
        double v;
        std::memcpy(&v, &L->h_scal->ws_bits, sizeof(double));
        return v;
    }();
    double dt = 1.0e20;
    for (int d = 0; d < L->D; ++d) dt = std::min(dt, L->dx[d] / ms);
    dt *= L->cfl;
    if (!std::isfinite(dt) || !(dt > 0)) return L->set_err(fail(BAMREX_ERR_NAN, "non-finite time step estimate"));
    *dt_est = dt;
    return BAMREX_OK;
}

extern "C" int bamrex_level_run_async(bamrex_level* L, int nsteps, double stop_time, int use_graph, double start_time)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (nsteps < 0) return L->set_err(fail(BAMREX_ERR_ARG, "nsteps must be >= 0"));
    if (L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "a run is pending: call bamrex_level_run_wait"));
    StepScalars* h = L->h_scal;
    std::memset(h, 0, sizeof(*h));
    h->time = start_time;
    h->stop_time = stop_time;
    cudaError_t e = cudaMemcpyAsync(L->d_scal, h, sizeof(StepScalars), cudaMemcpyHostToDevice, L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "scalars upload"));
    // computeInitialDt from the current state
    BX_TRY(level_launch(L, launch_max_wave_speed(L->D, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(), L->ncells, L->k,
                                                 &L->d_scal->ws_bits, L->d_scal, L->stream),
                        "max wave speed"));
    BX_TRY(level_launch(L, launch_step_dt(L->d_scal, L->D, L->dx[0], L->dx[1], L->dx[2], L->cfl, 0, L->stream), "step dt"));
    const int start = L->cur;
    int p = start;
    for (int s = 0; s < nsteps; ++s) {
        if (use_graph) {
            if (!L->graph[p]) {
                cudaGraph_t gr = nullptr;
                e = cudaStreamBeginCapture(L->stream, cudaStreamCaptureModeThreadLocal);
                if (e != cudaSuccess) return L->set_err(cuda_fail(e, "begin capture"));
                const long long before = L->launches;
                const int rc = level_step(L, p, 0.0, L->d_scal, false);
                e = cudaStreamEndCapture(L->stream, &gr);
                if (rc != BAMREX_OK) {
                    if (gr) cudaGraphDestroy(gr);
                    return rc;
                }
                if (e != cudaSuccess) return L->set_err(cuda_fail(e, "end capture"));
                L->launches = before;  // counted per replay below
                e = cudaGraphInstantiate(&L->graph[p], gr, 0);
                cudaGraphDestroy(gr);
                if (e != cudaSuccess) return L->set_err(cuda_fail(e, "graph instantiate"));
            }
            e = cudaGraphLaunch(L->graph[p], L->stream);
            if (e != cudaSuccess) return L->set_err(cuda_fail(e, "graph launch"));
            L->launches += 2 * L->D + 1;
        } else {
            BX_TRY(level_step(L, p, 0.0, L->d_scal, true));
        }
        p ^= (L->D & 1);
    }
    e = cudaMemcpyAsync(h, L->d_scal, sizeof(StepScalars), cudaMemcpyDeviceToHost, L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "scalars readback"));
    L->run_pending = true;
    L->run_start_parity = start;
    return BAMREX_OK;
}

extern "C" int bamrex_level_run_wait(bamrex_level* L, double* time_out, int* steps_done)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (!L->run_pending) return L->set_err(fail(BAMREX_ERR_ARG, "no run pending"));
    const cudaError_t e = cudaStreamSynchronize(L->stream);
    L->run_pending = false;
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "run"));
    const StepScalars* h = L->h_scal;
    L->cur = L->run_start_parity ^ ((h->steps * L->D) & 1);
    L->ws_valid = false;
    if (time_out) *time_out = h->time;
    if (steps_done) *steps_done = h->steps;
    if (h->status != 0)
        return L->set_err(fail(h->status, h->status == BAMREX_ERR_TIMEOUT ? "a sweep gave up waiting for its staged input"
                                                                          : "non-finite time step during the run"));
    return BAMREX_OK;
}

extern "C" int bamrex_level_run(bamrex_level* L, int nsteps, double stop_time, int use_graph, double* time_io,
                                int* steps_done)
{
    if (!L || !time_io) return fail(BAMREX_ERR_ARG, "NULL argument");
    BX_TRY(bamrex_level_run_async(L, nsteps, stop_time, use_graph, *time_io));
    return bamrex_level_run_wait(L, time_io, steps_done);
}

extern "C" int bamrex_level_set_timing(bamrex_level* L, int enable)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    L->timing = enable != 0;
    if (L->timing && L->events.empty()) {
        L->events.resize(8192);
        L->event_dir.assign(8192, 0);
        for (auto& ev : L->events) {
            if (cudaEventCreate(&ev.first) != cudaSuccess || cudaEventCreate(&ev.second) != cudaSuccess)
                return L->set_err(fail(BAMREX_ERR_CUDA, "cudaEventCreate failed"));
        }
    }
    L->ev_used = 0;
    return BAMREX_OK;
}

static int collect_events(bamrex_level* L)
{
    if (!L->ev_used) return BAMREX_OK;
    const cudaError_t e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "sync"));
    for (size_t i = 0; i < L->ev_used; ++i) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, L->events[i].first, L->events[i].second);
        L->sweep_ms += ms;
        L->dir_ms[L->event_dir[i]] += ms;
        L->dir_launches[L->event_dir[i]] += 1;
    }
    L->sweep_launches += (long long)L->ev_used;
    L->ev_used = 0;
    return BAMREX_OK;
}

extern "C" int bamrex_level_counters(bamrex_level* L, long long* launches, double* sweep_ms, long long* sweep_launches)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    BX_TRY(collect_events(L));
    if (launches) *launches = L->launches;
    if (sweep_ms) *sweep_ms = L->sweep_ms;
    if (sweep_launches) *sweep_launches = L->sweep_launches;
    return BAMREX_OK;
}

extern "C" int bamrex_level_sweep_times(bamrex_level* L, double* ms_by_dir, long long* launches_by_dir)
{
    if (!L || !ms_by_dir || !launches_by_dir) return fail(BAMREX_ERR_ARG, "NULL argument");
    BX_TRY(collect_events(L));
    for (int d = 0; d < 3; ++d) {
        ms_by_dir[d] = L->dir_ms[d];
        launches_by_dir[d] = L->dir_launches[d];
    }
    return BAMREX_OK;
}

extern "C" int bamrex_level_reset_counters(bamrex_level* L)
{
    if (!L) return fail(BAMREX_ERR_ARG, "NULL level");
    if (L->ev_used) cudaStreamSynchronize(L->stream);
    L->launches = 0;
    L->ev_used = 0;
    L->sweep_ms = 0.0;
    L->sweep_launches = 0;
    for (int d = 0; d < 3; ++d) {
        L->dir_ms[d] = 0.0;
        L->dir_launches[d] = 0;
    }
    return BAMREX_OK;
}
