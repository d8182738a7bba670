// Host side of the AMR glue: the coarse/fine coupling of two levels (flux
// register faces, coarse patches for fine ghost interpolation, average_down
// and reflux tables), error-estimation tagging, Berger-Rigoutsos grid
// generation and the subcycled hierarchy time step.  Tables are built once
// per grid configuration; every step then runs a fixed set of kernels on the
// levels' stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <thread>
#include <tuple>
#include <utility>
#include <vector>

#include "amr.h"
#include "bamrex_cuda.h"
#include "level_impl.h"

using namespace bamrex;

namespace {

int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

long long box_volume(const bamrex_box& b)
{
    return (long long)(b.hi[0] - b.lo[0] + 1) * (b.hi[1] - b.lo[1] + 1) * (b.hi[2] - b.lo[2] + 1);
}

bool box_empty(const bamrex_box& b) { return b.hi[0] < b.lo[0] || b.hi[1] < b.lo[1] || b.hi[2] < b.lo[2]; }

bamrex_box intersect(const bamrex_box& a, const bamrex_box& b)
{
    bamrex_box r;
    for (int d = 0; d < 3; ++d) {
        r.lo[d] = std::max(a.lo[d], b.lo[d]);
        r.hi[d] = std::min(a.hi[d], b.hi[d]);
    }
    return r;
}

bamrex_box coarsen(const bamrex_box& b, int r, int D)
{
    bamrex_box c = b;
    for (int d = 0; d < D; ++d) {
        c.lo[d] = floor_div(b.lo[d], r);
        c.hi[d] = floor_div(b.hi[d], r);
    }
    return c;
}

bamrex_box refine(const bamrex_box& b, int r, int D)
{
    bamrex_box c = b;
    for (int d = 0; d < D; ++d) {
        c.lo[d] = b.lo[d] * r;
        c.hi[d] = (b.hi[d] + 1) * r - 1;
    }
    return c;
}

// a minus b as disjoint boxes
void subtract(const bamrex_box& a, const bamrex_box& b, std::vector<bamrex_box>& out)
{
    const bamrex_box x = intersect(a, b);
    if (box_empty(x)) {
        out.push_back(a);
        return;
    }
    bamrex_box rest = a;
    for (int d = 0; d < 3; ++d) {
        if (rest.lo[d] < x.lo[d]) {
            bamrex_box p = rest;
            p.hi[d] = x.lo[d] - 1;
            out.push_back(p);
            rest.lo[d] = x.lo[d];
        }
        if (rest.hi[d] > x.hi[d]) {
            bamrex_box p = rest;
            p.lo[d] = x.hi[d] + 1;
            out.push_back(p);
            rest.hi[d] = x.hi[d];
        }
    }
}

// region minus every box of the index
void subtract_boxes(const bamrex_box& region, const BoxIndex& idx, const std::vector<bamrex_box>& boxes,
                    std::vector<bamrex_box>& out)
{
    std::vector<int> hits;
    idx.query(region.lo, region.hi, hits);
    std::sort(hits.begin(), hits.end());
    std::vector<bamrex_box> cur{ region }, next;
    for (int h : hits) {
        next.clear();
        for (const auto& p : cur) subtract(p, boxes[h], next);
        cur.swap(next);
        if (cur.empty()) break;
    }
    out.insert(out.end(), cur.begin(), cur.end());
}

// The box containing each cell of q (x fastest), -1 where none; a level's
// boxes are disjoint, so the owner is unique.
void cell_owners(const BoxIndex& idx, const std::vector<bamrex_box>& boxes, const bamrex_box& q, std::vector<int>& own,
                 std::vector<int>& hits)
{
    const int nx = q.hi[0] - q.lo[0] + 1, ny = q.hi[1] - q.lo[1] + 1;
    own.assign((size_t)box_volume(q), -1);
    idx.query(q.lo, q.hi, hits);
    for (int h : hits) {
        const bamrex_box x = intersect(q, boxes[h]);
        if (box_empty(x)) continue;
        for (int k = x.lo[2]; k <= x.hi[2]; ++k)
            for (int j = x.lo[1]; j <= x.hi[1]; ++j) {
                int* row = own.data() + ((size_t)(k - q.lo[2]) * ny + (j - q.lo[1])) * nx - q.lo[0];
                for (int i = x.lo[0]; i <= x.hi[0]; ++i) row[i] = h;
            }
    }
}

}  // namespace

struct bamrex_coupling {
    bamrex_level* crse = nullptr;
    bamrex_level* fine = nullptr;
    int r = 2, D = 0, NC = 0;
    char* arena = nullptr;
    // coarse old time level: the coarse values of the ghost patch cells
    // (set 0) at t_old, the only old data a fill reads
    double* d_patch_old = nullptr;
    bool old_valid = false;
    double t_old = 0, t_new = 0;
    // interpolation: [0] coarse/fine ghosts, [1] whole fine boxes (FillCoarsePatch)
    // (the patch values of set [1] live only while fill_coarse_patch runs)
    CfRegion* d_reg_set[2] = { nullptr, nullptr };
    int nreg_set[2] = { 0, 0 };
    long long ncell_set[2] = { 0, 0 };
    long long npatch_set[2] = { 0, 0 };
    double* d_patch_set[2] = { nullptr, nullptr };
    OwnerMap own;         // owners of the coarse level's cells
    CoarseDomain cdom;
    // flux registers
    int nslots[3] = { 0, 0, 0 };
    FaceRec* d_cfaces[3] = { nullptr, nullptr, nullptr };
    FaceRec* d_ffaces[3] = { nullptr, nullptr, nullptr };
    RefluxRec* d_rr[3] = { nullptr, nullptr, nullptr };
    double* d_reg[3] = { nullptr, nullptr, nullptr };
    // average_down and covered sums
    AvgOp* d_avg = nullptr;
    int navg = 0;
    long long navg_cells = 0;
    PackBox* d_cov_box = nullptr;
    FabDev* d_cov_fab[2] = { nullptr, nullptr };
    double* d_cov_sums = nullptr;
};

namespace {

// Map a coarse cell into the domain by the boundary rules (periodic shift,
// reflection with the normal momentum negated, or extrapolation).
void map_into_domain(const bamrex_level* L, int* c, int& negmask)
{
    for (int d = 0; d < L->D; ++d) {
        const int lo = L->domain.lo[d], hi = L->domain.hi[d], len = hi - lo + 1;
        if (c[d] >= lo && c[d] <= hi) continue;
        const int bc = c[d] < lo ? L->bc_lo[d] : L->bc_hi[d];
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

// Gather arguments of patch set `set` (mode as CfGatherArgs) into `patch`.
CfGatherArgs gather_args(const bamrex_coupling* C, int set, int mode, double a_old, double a_new, double* patch)
{
    CfGatherArgs a;
    a.regions = C->d_reg_set[set];
    a.nregions = C->nreg_set[set];
    a.npatch = C->npatch_set[set];
    a.own = C->own;
    a.dom = C->cdom;
    a.patch_old = C->d_patch_old;
    a.crse_new = C->crse->d_fab[C->crse->cur];
    a.NC = C->NC;
    a.mode = mode;
    a.a_old = a_old;
    a.a_new = a_new;
    a.patch = patch;
    a.bad = nullptr;
    a.amr = nullptr;
    a.lc = 0;
    return a;
}

// "coarse cell (i,j,k) is not a valid coarse cell" for patch cell idx of
// a region set.
std::string describe_patch_cell(const bamrex_coupling* C, const std::vector<CfRegion>& R, long long idx)
{
    size_t n = 0;
    while (n + 1 < R.size() && R[n + 1].patch_begin <= idx) ++n;
    const long long local = idx - R[n].patch_begin, row = local / R[n].pn[0];
    int c[3] = { R[n].plo[0] + (int)(local - row * R[n].pn[0]), R[n].plo[1] + (int)(row % R[n].pn[1]),
                 R[n].plo[2] + (int)(row / R[n].pn[1]) };
    int neg = 0;
    map_into_domain(C->crse, c, neg);
    return "coarse cell (" + std::to_string(c[0]) + "," + std::to_string(c[1]) + "," + std::to_string(c[2]) +
           ") is not a valid coarse cell";
}

// Host worker threads for a table build of `work` records: about 64k
// records a thread, at most the machine's threads (and 32).
int table_threads(long long work)
{
    const long long hw = std::max(1u, std::thread::hardware_concurrency());
    return (int)std::max(1LL, std::min({ hw, 32LL, work / 65536 + 1 }));
}

// fn(item, scratch) over items [0, n) on `nthreads` threads taking chunks of
// `chunk` items in turn; each thread owns one Scratch. The first failure in
// item order wins: fn returns an empty string on success, else the message.
template <class Scratch, class F>
int parallel_items(int n, int nthreads, int chunk, F&& fn)
{
    std::atomic<int> next(0);
    std::mutex mu;
    int bad_item = n;
    std::string bad_msg;
    auto worker = [&] {
        Scratch scratch;
        for (;;) {
            const int b = next.fetch_add(chunk);
            if (b >= n) return;
            for (int it = b; it < std::min(n, b + chunk); ++it) {
                std::string msg = fn(it, scratch);
                if (msg.empty()) continue;
                std::lock_guard<std::mutex> g(mu);
                if (it < bad_item) {
                    bad_item = it;
                    bad_msg = std::move(msg);
                }
                break;
            }
        }
    };
    nthreads = std::max(1, std::min(nthreads, (n + chunk - 1) / std::max(1, chunk)));
    if (nthreads == 1) {
        worker();
    } else {
        std::vector<std::thread> th;
        for (int t = 0; t < nthreads; ++t) th.emplace_back(worker);
        for (auto& x : th) x.join();
    }
    return bad_item < n ? fail(BAMREX_ERR_ARG, bad_msg) : BAMREX_OK;
}

struct OwnerScratch {
    std::vector<int> own, hits;
};

// Coarse patches (coarsened region grown by one coarse cell) of a set of
// fine regions: each region's patch box and its place in the patch and cell
// numbering.  The owners of the patch cells are looked up on the device.
long long build_patches(const bamrex_coupling* C, std::vector<CfRegion>& regs)
{
    long long pacc = 0, cacc = 0;
    for (size_t n = 0; n < regs.size(); ++n) {
        CfRegion& R = regs[n];
        bamrex_box w;
        for (int d = 0; d < 3; ++d) {
            w.lo[d] = R.lo[d] + R.shift[d];
            w.hi[d] = R.hi[d] + R.shift[d];
        }
        bamrex_box p = coarsen(w, C->r, C->D);
        for (int d = 0; d < C->D; ++d) {
            p.lo[d] -= 1;
            p.hi[d] += 1;
        }
        for (int d = 0; d < 3; ++d) {
            R.plo[d] = p.lo[d];
            R.pn[d] = p.hi[d] - p.lo[d] + 1;
        }
        R.patch_begin = pacc;
        R.cell_begin = cacc;
        pacc += box_volume(p);
        cacc += (long long)(R.hi[0] - R.lo[0] + 1) * (R.hi[1] - R.lo[1] + 1) * (R.hi[2] - R.lo[2] + 1);
    }
    return pacc;
}

// Owner map of a level (OwnerMap): blocks as large as the greatest common
// divisor of the box corners' offsets from the domain corner and of the
// domain's extent, per direction.
int build_owner_map(const bamrex_level* L, std::vector<int>& owner, int* g, int* nb)
{
    long long total = 1;
    for (int d = 0; d < 3; ++d) {
        const int n = L->domain.hi[d] - L->domain.lo[d] + 1;
        int gg = n;
        for (const auto& b : L->boxes) {
            gg = std::gcd(gg, b.lo[d] - L->domain.lo[d]);
            gg = std::gcd(gg, b.hi[d] + 1 - L->domain.lo[d]);
        }
        g[d] = std::max(1, gg);
        nb[d] = n / g[d];
        total *= nb[d];
    }
    if (total > (1LL << 28))
        return fail(BAMREX_ERR_UNSUPPORTED, "coarse level boxes too finely aligned for its owner map (more than 2^28 blocks)");
    owner.assign((size_t)total, -1);
    for (int b = 0; b < (int)L->boxes.size(); ++b) {
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            lo[d] = (L->boxes[b].lo[d] - L->domain.lo[d]) / g[d];
            hi[d] = (L->boxes[b].hi[d] + 1 - L->domain.lo[d]) / g[d] - 1;
        }
        for (int K = lo[2]; K <= hi[2]; ++K)
            for (int J = lo[1]; J <= hi[1]; ++J)
                for (int I = lo[0]; I <= hi[0]; ++I) owner[((size_t)K * nb[1] + J) * nb[0] + I] = b;
    }
    return BAMREX_OK;
}

CfRegion make_region(int dst, const bamrex_box& b, const int* shift)
{
    CfRegion R;
    std::memset(&R, 0, sizeof(R));
    R.dst = dst;
    for (int d = 0; d < 3; ++d) {
        R.lo[d] = b.lo[d] - shift[d];
        R.hi[d] = b.hi[d] - shift[d];
        R.shift[d] = shift[d];
    }
    return R;
}

// The fine ghost regions to interpolate: face slabs of depth ngrow of every
// fine box, inside the domain (or the periodic image outside it), minus the
// fine boxes.  Boxes on host threads, their regions joined in box order.
void build_ghost_regions(const bamrex_level* Lf, const BoxIndex& fidx, std::vector<CfRegion>& regs)
{
    const int g = Lf->ngrow;
    const int nbf = (int)Lf->boxes.size();
    std::vector<std::vector<CfRegion>> per(nbf);
    auto one_box = [&](int b, int&) -> std::string {
        std::vector<CfRegion>& regs = per[(size_t)b];
        const bamrex_box& B = Lf->boxes[b];
        for (int d = 0; d < Lf->D; ++d) {
            const int dlo = Lf->domain.lo[d], dhi = Lf->domain.hi[d], len = dhi - dlo + 1;
            for (int side = 0; side < 2; ++side) {
                bamrex_box slab = B;
                if (side == 0) {
                    slab.lo[d] = B.lo[d] - g;
                    slab.hi[d] = B.lo[d] - 1;
                } else {
                    slab.lo[d] = B.hi[d] + 1;
                    slab.hi[d] = B.hi[d] + g;
                }
                bamrex_box in = slab;
                in.lo[d] = std::max(slab.lo[d], dlo);
                in.hi[d] = std::min(slab.hi[d], dhi);
                const int zero[3] = { 0, 0, 0 };
                if (in.lo[d] <= in.hi[d]) {
                    std::vector<bamrex_box> pieces;
                    subtract_boxes(in, fidx, Lf->boxes, pieces);
                    for (const auto& p : pieces) regs.push_back(make_region(b, p, zero));
                }
                const int bc = side == 0 ? Lf->bc_lo[d] : Lf->bc_hi[d];
                if (bc != BAMREX_BC_PERIODIC) continue;  // physical ghosts: the level's own boundary fill
                bamrex_box out = slab;
                if (side == 0) out.hi[d] = std::min(slab.hi[d], dlo - 1);
                else out.lo[d] = std::max(slab.lo[d], dhi + 1);
                if (out.lo[d] > out.hi[d]) continue;
                int shift[3] = { 0, 0, 0 };
                shift[d] = side == 0 ? len : -len;
                bamrex_box img = out;
                img.lo[d] += shift[d];
                img.hi[d] += shift[d];
                std::vector<bamrex_box> pieces;
                subtract_boxes(img, fidx, Lf->boxes, pieces);
                for (const auto& p : pieces) regs.push_back(make_region(b, p, shift));
            }
        }
        return std::string();
    };
    parallel_items<int>(nbf, table_threads((long long)nbf * 4096), 16, one_box);
    size_t n = 0;
    for (const auto& v : per) n += v.size();
    regs.reserve(regs.size() + n);
    for (const auto& v : per) regs.insert(regs.end(), v.begin(), v.end());
}

// A table of records in a buffer the caller owns (the coupling's pinned
// staging buffer, or host memory where that cannot be had).
template <class T>
struct RecSpan {
    T* p = nullptr;
    size_t n = 0;
    size_t size() const { return n; }
    T* data() const { return p; }
    T& operator[](size_t i) const { return p[i]; }
};
using FaceRecs = RecSpan<FaceRec>;
using RefluxRecs = RecSpan<RefluxRec>;

// One direction's flux-register records per fine box, before the join.
struct RegParts {
    std::vector<std::vector<FaceRec>> cfb, ffb;
    std::vector<std::vector<RefluxRec>> rrb;
    std::vector<size_t> at;  // first slot of each box
    size_t n = 0;            // slots
    size_t per_rec = 1;      // fine faces per slot
};

// The bit map of a coarse domain for the duplicate-slot check, one per host
// thread that builds couplings, kept between calls and left all zero.
std::vector<unsigned long long>& slot_bitmap(size_t words)
{
    thread_local std::vector<unsigned long long> bits;
    if (bits.size() < words) bits.assign(words, 0ULL);
    return bits;
}

// Flux-register slots of direction d, per fine box: the fine boxes run on
// host threads, each filling its own record lists (register_join then
// joins them in box order).
int register_parts(const bamrex_coupling* C, int d, const BoxIndex& fidx, const BoxIndex& cidx, RegParts& P)
{
    const bamrex_level* Lf = C->fine;
    const bamrex_level* Lc = C->crse;
    const int r = C->r, D = C->D;
    const int dlo = Lf->domain.lo[d], dhi = Lf->domain.hi[d], len = dhi - dlo + 1;
    const int nbf = (int)Lf->boxes.size();
    P.cfb.assign((size_t)nbf, {});
    P.ffb.assign((size_t)nbf, {});
    P.rrb.assign((size_t)nbf, {});
    auto& cfb = P.cfb;
    auto& ffb = P.ffb;
    auto& rrb = P.rrb;
    // the r^(D-1) fine faces under a coarse face, transverse index fastest
    // in x, then y, then z
    const int tz = (D > 2 && d != 2) ? r : 1;
    const int ty = (D > 1 && d != 1) ? r : 1;
    const int tx = (d != 0) ? r : 1;
    auto box = [&](int b, OwnerScratch& S) -> std::string {
        const bamrex_box& B = Lf->boxes[b];
        for (int side = 0; side < 2; ++side) {
            bamrex_box layer = B;
            layer.lo[d] = layer.hi[d] = side == 0 ? B.lo[d] - 1 : B.hi[d] + 1;
            int shift = 0;
            if (layer.lo[d] < dlo || layer.lo[d] > dhi) {
                const int bc = side == 0 ? Lf->bc_lo[d] : Lf->bc_hi[d];
                if (bc != BAMREX_BC_PERIODIC) continue;  // domain face: no coarse neighbour
                shift = side == 0 ? len : -len;
                layer.lo[d] += shift;
                layer.hi[d] += shift;
            }
            std::vector<bamrex_box> pieces;
            subtract_boxes(layer, fidx, Lf->boxes, pieces);
            const int fface = side == 0 ? B.lo[d] : B.hi[d] + 1;
            for (const auto& p : pieces) {
                const bamrex_box cp = coarsen(p, r, D);
                cell_owners(cidx, Lc->boxes, cp, S.own, S.hits);
                size_t oq = 0;
                for (int k = cp.lo[2]; k <= cp.hi[2]; ++k)
                    for (int j = cp.lo[1]; j <= cp.hi[1]; ++j)
                        for (int i = cp.lo[0]; i <= cp.hi[0]; ++i, ++oq) {
                            const int c[3] = { i, j, k };
                            const int cb = S.own[oq];
                            if (cb < 0) return "fine level not properly nested (flux register)";
                            rrb[b].push_back(RefluxRec{ cb, i, j, k, side == 0 ? -1 : 1 });
                            FaceRec f{ cb, i, j, k };
                            const int cface = c[d] + (side == 0 ? 1 : 0);
                            if (d == 0) f.i = cface;
                            else if (d == 1) f.j = cface;
                            else f.k = cface;
                            cfb[b].push_back(f);
                            for (int a2 = 0; a2 < tz; ++a2)
                                for (int a1 = 0; a1 < ty; ++a1)
                                    for (int a0 = 0; a0 < tx; ++a0)
                                        ffb[b].push_back(FaceRec{ b, d == 0 ? fface : c[0] * r + a0,
                                                                  d == 1 ? fface : (D > 1 ? c[1] * r + a1 : 0),
                                                                  d == 2 ? fface : (D > 2 ? c[2] * r + a2 : 0) });
                        }
            }
        }
        return std::string();
    };
    long long work = 0;
    for (const auto& B : Lf->boxes) work += box_volume(B) / std::max(1, B.hi[d] - B.lo[d] + 1);
    ProfPhases phase("registers:boxes");
    BX_TRY(parallel_items<OwnerScratch>(nbf, table_threads(work), 4, box));
    P.at.assign((size_t)nbf + 1, 0);
    for (int b = 0; b < nbf; ++b) P.at[(size_t)b + 1] = P.at[(size_t)b] + rrb[(size_t)b].size();
    P.n = P.at[(size_t)nbf];
    P.per_rec = (size_t)tx * ty * tz;
    return BAMREX_OK;
}

// The records of register_parts joined in box order into the tables cf, ff
// and rr (their buffers sized by the caller: P.n, P.n * P.per_rec, P.n),
// the boxes' lists copied on host threads; then the check that no coarse
// cell borders the fine region on both sides.
int register_join(const bamrex_coupling* C, const RegParts& P, FaceRecs& cf, FaceRecs& ff, RefluxRecs& rr)
{
    const bamrex_level* Lc = C->crse;
    const int nbf = (int)P.rrb.size();
    const size_t n = P.n, per_rec = P.per_rec;
    ProfPhases phase("registers:join");
    const int jt = table_threads((long long)n);
    parallel_items<int>(nbf, jt, 16, [&](int b, int&) -> std::string {
        std::copy(P.rrb[(size_t)b].begin(), P.rrb[(size_t)b].end(), rr.data() + P.at[(size_t)b]);
        std::copy(P.cfb[(size_t)b].begin(), P.cfb[(size_t)b].end(), cf.data() + P.at[(size_t)b]);
        std::copy(P.ffb[(size_t)b].begin(), P.ffb[(size_t)b].end(), ff.data() + P.at[(size_t)b] * per_rec);
        return std::string();
    });
    phase.next("registers:dup");
    // a coarse cell may border the fine region on one side only: mark each
    // slot's cell in a bit map of the coarse domain (sorted keys where the
    // domain is too large for one); marks by atomic OR on host threads
    const int* cl = Lc->domain.lo;
    const unsigned long long nx = Lc->domain.hi[0] - cl[0] + 1, ny = Lc->domain.hi[1] - cl[1] + 1,
                             nz = Lc->domain.hi[2] - cl[2] + 1;
    bool dup = false;
    if (nx * ny * nz <= (1ULL << 27)) {
        std::vector<unsigned long long>& seen = slot_bitmap((nx * ny * nz + 63) / 64);
        std::atomic<bool> any(false);
        constexpr size_t kChunk = 65536;
        const int nchunk = (int)((n + kChunk - 1) / kChunk);
        auto key_of = [&](size_t q) {
            return ((unsigned long long)(rr[q].k - cl[2]) * ny + (rr[q].j - cl[1])) * nx + (rr[q].i - cl[0]);
        };
        parallel_items<int>(nchunk, jt, 1, [&](int c, int&) -> std::string {
            const size_t q1 = std::min(n, (size_t)(c + 1) * kChunk);
            for (size_t q = (size_t)c * kChunk; q < q1; ++q) {
                const unsigned long long key = key_of(q), bit = 1ULL << (key & 63);
                if (__atomic_fetch_or(&seen[key >> 6], bit, __ATOMIC_RELAXED) & bit) any.store(true, std::memory_order_relaxed);
            }
            return std::string();
        });
        // back to all zero: only the words the slots touched
        parallel_items<int>(nchunk, jt, 1, [&](int c, int&) -> std::string {
            const size_t q1 = std::min(n, (size_t)(c + 1) * kChunk);
            for (size_t q = (size_t)c * kChunk; q < q1; ++q) __atomic_store_n(&seen[key_of(q) >> 6], 0ULL, __ATOMIC_RELAXED);
            return std::string();
        });
        dup = any.load();
    } else {
        std::vector<unsigned long long> keys(rr.size());
        for (size_t q = 0; q < rr.size(); ++q)
            keys[q] = ((unsigned long long)(rr[q].k - cl[2]) << 42) | ((unsigned long long)(rr[q].j - cl[1]) << 21) |
                      (unsigned long long)(rr[q].i - cl[0]);
        std::sort(keys.begin(), keys.end());
        dup = std::adjacent_find(keys.begin(), keys.end()) != keys.end();
    }
    if (dup)
        return fail(BAMREX_ERR_ARG,
                    "fine boxes closer than two coarse cells: a coarse cell borders the fine region on both sides");
    return BAMREX_OK;
}

void drop_tasks(bamrex_level* L, const double* reg)
{
    if (!L) return;
    for (int d = 0; d < 3; ++d) {
        auto& v = L->reg_tasks[d];
        v.erase(std::remove_if(v.begin(), v.end(), [&](const RegisterTask& t) { return t.reg == reg; }), v.end());
    }
}

int cpl_launch(bamrex_coupling* C, cudaError_t e, const char* what)
{
    if (e != cudaSuccess) return cuda_fail(e, what);
    C->fine->launches++;
    return BAMREX_OK;
}

}  // namespace

extern "C" int bamrex_coupling_create(bamrex_coupling** out, bamrex_level* crse, bamrex_level* fine, int ref_ratio)
{
    if (!out || !crse || !fine) return fail(BAMREX_ERR_ARG, "NULL argument");
    *out = nullptr;
    const int D = crse->D, r = ref_ratio;
    if (r != 2 && r != 4) return fail(BAMREX_ERR_ARG, "ref_ratio must be 2 or 4");
    if (fine->D != D || fine->fp32 != crse->fp32 || fine->method != crse->method)
        return fail(BAMREX_ERR_ARG, "coarse and fine levels differ in dimension, precision or method");
    if (fine->stream != crse->stream) return fail(BAMREX_ERR_ARG, "coarse and fine levels must share a stream");
    if (fine->ngrow < 2) return fail(BAMREX_ERR_ARG, "fine ngrow must be >= 2");
    for (int d = 0; d < D; ++d) {
        if (fine->domain.lo[d] != crse->domain.lo[d] * r || fine->domain.hi[d] != (crse->domain.hi[d] + 1) * r - 1)
            return fail(BAMREX_ERR_ARG, "fine domain is not the refined coarse domain");
        if (fine->bc_lo[d] != crse->bc_lo[d] || fine->bc_hi[d] != crse->bc_hi[d])
            return fail(BAMREX_ERR_ARG, "coarse and fine boundary conditions differ");
    }
    for (const auto& B : fine->boxes)
        for (int d = 0; d < D; ++d)
            if (B.lo[d] % r != 0 || (B.hi[d] + 1) % r != 0)
                return fail(BAMREX_ERR_ARG, "fine boxes must be aligned to the refinement ratio");
    for (int d = 0; d < 3; ++d)
        if (crse->domain.hi[d] - crse->domain.lo[d] >= (1 << 21))
            return fail(BAMREX_ERR_ARG, "coarse domain wider than 2^21 cells");

    BX_PROFILE("bamrex_coupling_create");
    ProfPhases phase("coupling_create:index");
    std::unique_ptr<bamrex_coupling> C(new (std::nothrow) bamrex_coupling());
    if (!C) return fail(BAMREX_ERR_OOM, "host allocation failed");
    C->crse = crse;
    C->fine = fine;
    C->r = r;
    C->D = D;
    C->NC = crse->NC;

    BoxIndex fidx, cidx;
    fidx.build(fine->domain, fine->boxes, D);
    cidx.build(crse->domain, crse->boxes, D);

    phase.next("coupling_create:patches");
    // interpolation regions and their coarse patches
    std::vector<CfRegion> regs[2];
    build_ghost_regions(fine, fidx, regs[0]);
    const int zero[3] = { 0, 0, 0 };
    for (int b = 0; b < (int)fine->boxes.size(); ++b) regs[1].push_back(make_region(b, fine->boxes[b], zero));
    long long npatch[2];
    for (int s = 0; s < 2; ++s) npatch[s] = build_patches(C.get(), regs[s]);
    std::vector<int> owner;
    int og[3], onb[3];
    BX_TRY(build_owner_map(crse, owner, og, onb));

    phase.next("coupling_create:registers");
    // flux registers
    RegParts parts[3];
    for (int d = 0; d < D; ++d) BX_TRY(register_parts(C.get(), d, fidx, cidx, parts[d]));
    // every direction's records in one pinned staging buffer, written once
    // by the joining threads and uploaded from there (held to the end of
    // this function, after the upload has completed)
    size_t so[3][3] = {}, stage_bytes = 0;
    for (int d = 0; d < D; ++d) {
        const size_t sz[3] = { sizeof(RefluxRec) * parts[d].n, sizeof(FaceRec) * parts[d].n,
                               sizeof(FaceRec) * parts[d].n * parts[d].per_rec };
        for (int t = 0; t < 3; ++t) {
            so[d][t] = stage_bytes;
            stage_bytes = align_up(stage_bytes + sz[t], 64);
        }
    }
    PinnedStage stage(stage_bytes);
    std::vector<char> heap_stage;
    char* sb = stage.data();
    if (!sb && stage_bytes) {
        heap_stage.resize(stage_bytes);
        sb = heap_stage.data();
    }
    FaceRecs cf[3], ff[3];
    RefluxRecs rr[3];
    for (int d = 0; d < D; ++d) {
        rr[d] = RefluxRecs{ reinterpret_cast<RefluxRec*>(sb + so[d][0]), parts[d].n };
        cf[d] = FaceRecs{ reinterpret_cast<FaceRec*>(sb + so[d][1]), parts[d].n };
        ff[d] = FaceRecs{ reinterpret_cast<FaceRec*>(sb + so[d][2]), parts[d].n * parts[d].per_rec };
        BX_TRY(register_join(C.get(), parts[d], cf[d], ff[d], rr[d]));
        parts[d] = RegParts();
    }

    phase.next("coupling_create:avg_down");
    // average_down
    std::vector<AvgOp> avg;
    {
        long long acc = 0;
        std::vector<int> hits;
        for (int b = 0; b < (int)fine->boxes.size(); ++b) {
            const bamrex_box cb = coarsen(fine->boxes[b], r, D);
            cidx.query(cb.lo, cb.hi, hits);
            std::sort(hits.begin(), hits.end());
            long long covered = 0;
            for (int h : hits) {
                const bamrex_box x = intersect(cb, crse->boxes[h]);
                if (box_empty(x)) continue;
                AvgOp op;
                std::memset(&op, 0, sizeof(op));
                op.crse = h;
                op.fine = b;
                for (int d = 0; d < 3; ++d) {
                    op.lo[d] = x.lo[d];
                    op.hi[d] = x.hi[d];
                }
                op.cell_begin = acc;
                acc += box_volume(x);
                covered += box_volume(x);
                avg.push_back(op);
            }
            if (covered != box_volume(cb)) return fail(BAMREX_ERR_ARG, "fine level not covered by the coarse level");
        }
        C->navg = (int)avg.size();
        C->navg_cells = acc;
    }
    std::vector<PackBox> cov(avg.size());
    std::vector<FabDev> covfab[2];
    for (size_t i = 0; i < avg.size(); ++i) {
        for (int d = 0; d < 3; ++d) {
            cov[i].lo[d] = avg[i].lo[d];
            cov[i].hi[d] = avg[i].hi[d];
        }
        cov[i].cell_begin = avg[i].cell_begin;
        for (int p = 0; p < 2; ++p) covfab[p].push_back(crse->fab[p][avg[i].crse]);
    }

    phase.next("coupling_create:upload");
    // one arena
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align_up(off + std::max<size_t>(bytes, 1), 256);
        return o;
    };
    const size_t o_old = take(sizeof(double) * C->NC * npatch[0]);
    size_t o_reg[2];
    for (int s = 0; s < 2; ++s) o_reg[s] = take(sizeof(CfRegion) * regs[s].size());
    const size_t o_patch0 = take(sizeof(double) * C->NC * npatch[0]);
    const size_t o_owner = take(sizeof(int) * owner.size());
    const size_t o_bad = take(2 * sizeof(unsigned long long));
    size_t o_cf[3] = {}, o_ff[3] = {}, o_rr[3] = {}, o_rg[3] = {};
    for (int d = 0; d < D; ++d) {
        o_cf[d] = take(sizeof(FaceRec) * cf[d].size());
        o_ff[d] = take(sizeof(FaceRec) * ff[d].size());
        o_rr[d] = take(sizeof(RefluxRec) * rr[d].size());
        o_rg[d] = take(sizeof(double) * C->NC * rr[d].size());
    }
    const size_t o_avg = take(sizeof(AvgOp) * avg.size());
    const size_t o_cov = take(sizeof(PackBox) * cov.size());
    const size_t o_covf0 = take(sizeof(FabDev) * cov.size());
    const size_t o_covf1 = take(sizeof(FabDev) * cov.size());
    const size_t o_covs = take(sizeof(double) * C->NC * std::max<size_t>(1, cov.size()));
    cudaError_t e = dev_alloc((void**)&C->arena, off, crse->stream);
    if (e != cudaSuccess) return fail(BAMREX_ERR_OOM, std::string("allocation of the coupling failed: ") + cudaGetErrorString(e));
    char* A = C->arena;
    C->d_patch_old = (double*)(A + o_old);
    for (int s = 0; s < 2; ++s) {
        C->d_reg_set[s] = (CfRegion*)(A + o_reg[s]);
        C->nreg_set[s] = (int)regs[s].size();
        C->ncell_set[s] = regs[s].empty() ? 0
                                          : regs[s].back().cell_begin + (long long)(regs[s].back().hi[0] - regs[s].back().lo[0] + 1) *
                                                                          (regs[s].back().hi[1] - regs[s].back().lo[1] + 1) *
                                                                          (regs[s].back().hi[2] - regs[s].back().lo[2] + 1);
        C->npatch_set[s] = npatch[s];
    }
    C->d_patch_set[0] = (double*)(A + o_patch0);
    C->own.owner = (const int*)(A + o_owner);
    for (int d = 0; d < 3; ++d) {
        C->own.lo[d] = crse->domain.lo[d];
        C->own.g[d] = og[d];
        C->own.nb[d] = onb[d];
        C->cdom.lo[d] = crse->domain.lo[d];
        C->cdom.hi[d] = crse->domain.hi[d];
        C->cdom.bc_lo[d] = crse->bc_lo[d];
        C->cdom.bc_hi[d] = crse->bc_hi[d];
    }
    C->cdom.D = D;
    unsigned long long* d_bad = (unsigned long long*)(A + o_bad);
    for (int d = 0; d < D; ++d) {
        C->nslots[d] = (int)rr[d].size();
        C->d_cfaces[d] = (FaceRec*)(A + o_cf[d]);
        C->d_ffaces[d] = (FaceRec*)(A + o_ff[d]);
        C->d_rr[d] = (RefluxRec*)(A + o_rr[d]);
        C->d_reg[d] = (double*)(A + o_rg[d]);
    }
    C->d_avg = (AvgOp*)(A + o_avg);
    C->d_cov_box = (PackBox*)(A + o_cov);
    C->d_cov_fab[0] = (FabDev*)(A + o_covf0);
    C->d_cov_fab[1] = (FabDev*)(A + o_covf1);
    C->d_cov_sums = (double*)(A + o_covs);

    auto up = [&](void* dst, const void* src, size_t bytes) -> cudaError_t {
        return bytes ? cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, crse->stream) : cudaSuccess;
    };
    for (int s = 0; s < 2 && e == cudaSuccess; ++s) {
        e = up(C->d_reg_set[s], regs[s].data(), sizeof(CfRegion) * regs[s].size());
    }
    if (e == cudaSuccess) e = up((void*)C->own.owner, owner.data(), sizeof(int) * owner.size());
    // every patch cell of both sets must be a valid coarse cell (proper
    // nesting): checked once here on the device
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0xff, 2 * sizeof(unsigned long long), crse->stream);
    for (int s = 0; s < 2 && e == cudaSuccess; ++s) {
        CfGatherArgs ga = gather_args(C.get(), s, 3, 0.0, 1.0, nullptr);
        ga.bad = d_bad + s;
        e = launch_cf_gather(crse->fp32, ga, crse->stream);
    }
    unsigned long long bad[2] = { ~0ULL, ~0ULL };
    if (e == cudaSuccess) e = cudaMemcpyAsync(bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, crse->stream);
    for (int d = 0; d < D && e == cudaSuccess; ++d) {
        e = up(C->d_cfaces[d], cf[d].data(), sizeof(FaceRec) * cf[d].size());
        if (e == cudaSuccess) e = up(C->d_ffaces[d], ff[d].data(), sizeof(FaceRec) * ff[d].size());
        if (e == cudaSuccess) e = up(C->d_rr[d], rr[d].data(), sizeof(RefluxRec) * rr[d].size());
        if (e == cudaSuccess) e = cudaMemsetAsync(C->d_reg[d], 0, sizeof(double) * C->NC * rr[d].size(), crse->stream);
    }
    if (e == cudaSuccess) e = up(C->d_avg, avg.data(), sizeof(AvgOp) * avg.size());
    if (e == cudaSuccess) e = up(C->d_cov_box, cov.data(), sizeof(PackBox) * cov.size());
    for (int p = 0; p < 2 && e == cudaSuccess; ++p) e = up(C->d_cov_fab[p], covfab[p].data(), sizeof(FabDev) * cov.size());
    if (e == cudaSuccess) e = cudaStreamSynchronize(crse->stream);
    if (e != cudaSuccess) {
        dev_free(C->arena, crse->stream);
        return cuda_fail(e, "coupling table upload");
    }
    for (int s = 0; s < 2; ++s)
        if (bad[s] != ~0ULL) {
            const std::string where = describe_patch_cell(C.get(), regs[s], (long long)bad[s]);
            dev_free(C->arena, crse->stream);
            return fail(BAMREX_ERR_ARG, "fine level not properly nested: " + where);
        }
    const int per_slot = D == 1 ? 1 : (D == 2 ? r : r * r);
    for (int d = 0; d < D; ++d) {
        if (!C->nslots[d]) continue;
        RegisterTask tc;
        tc.faces = C->d_cfaces[d];
        tc.nslots = C->nslots[d];
        tc.per_slot = 1;
        tc.reg = C->d_reg[d];
        tc.mode = 0;
        crse->reg_tasks[d].push_back(tc);
        RegisterTask tf = tc;
        tf.faces = C->d_ffaces[d];
        tf.per_slot = per_slot;
        tf.mode = 1;
        fine->reg_tasks[d].push_back(tf);
    }
    *out = C.release();
    return BAMREX_OK;
}

extern "C" int bamrex_coupling_destroy(bamrex_coupling* C)
{
    if (!C) return BAMREX_OK;
    if (C->crse && C->crse->stream) cudaStreamSynchronize(C->crse->stream);
    for (int d = 0; d < 3; ++d) {
        if (!C->d_reg[d]) continue;
        drop_tasks(C->crse, C->d_reg[d]);
        drop_tasks(C->fine, C->d_reg[d]);
    }
    dev_free(C->arena, C->crse ? C->crse->stream : nullptr);
    delete C;
    return BAMREX_OK;
}

// The coarse values the fine level's ghost patches read, kept for t_old
// (AMReX keeps the whole old MultiFab; only these cells are ever read).
static int save_patch_old(bamrex_coupling* C)
{
    bamrex_level* Lc = C->crse;
    return cpl_launch(C, launch_cf_gather(Lc->fp32, gather_args(C, 0, 4, 0.0, 1.0, C->d_patch_old), Lc->stream),
                      "coarse old patch");
}

extern "C" int bamrex_coupling_save_coarse_old(bamrex_coupling* C, double t_old, double t_new)
{
    if (!C) return fail(BAMREX_ERR_ARG, "NULL coupling");
    if (!(t_new > t_old)) return fail(BAMREX_ERR_ARG, "t_new must exceed t_old");
    BX_TRY(save_patch_old(C));
    C->old_valid = true;
    C->t_old = t_old;
    C->t_new = t_new;
    return BAMREX_OK;
}

static int run_interp(bamrex_coupling* C, int set, int mode, double a_old, double a_new, const AmrDev* amr = nullptr,
                      int lc = 0)
{
    bamrex_level* Lc = C->crse;
    bamrex_level* Lf = C->fine;
    if (!C->ncell_set[set]) return BAMREX_OK;
    double* patch = C->d_patch_set[set];
    if (set == 1) {
        cudaError_t e = dev_alloc((void**)&patch, sizeof(double) * C->NC * C->npatch_set[1], Lc->stream);
        if (e != cudaSuccess) return fail(BAMREX_ERR_OOM, std::string("coarse patch allocation failed: ") + cudaGetErrorString(e));
    }
    struct Release {
        double* p;
        cudaStream_t s;
        ~Release()
        {
            if (p) dev_free(p, s);
        }
    } release{ set == 1 ? patch : nullptr, Lc->stream };
    CfGatherArgs ga = gather_args(C, set, mode, a_old, a_new, patch);
    ga.amr = amr;
    ga.lc = lc;
    BX_TRY(cpl_launch(C, launch_cf_gather(Lc->fp32, ga, Lc->stream), "coarse patch gather"));
    CfInterpArgs a;
    a.regions = C->d_reg_set[set];
    a.nregions = C->nreg_set[set];
    a.ncells = C->ncell_set[set];
    a.patch = patch;
    a.npatch = C->npatch_set[set];
    a.fine0 = Lf->d_fab[0];
    a.fine1 = Lf->d_fab[1];
    a.D = C->D;
    a.NC = C->NC;
    a.ratio = C->r;
    BX_TRY(cpl_launch(C, launch_cf_interp(Lc->fp32, a, Lc->stream), "coarse/fine interpolation"));
    Lf->ws_valid = false;
    return BAMREX_OK;
}

extern "C" int bamrex_coupling_fill_patch(bamrex_coupling* C, double time)
{
    if (!C) return fail(BAMREX_ERR_ARG, "NULL coupling");
    int mode = 1;
    double a_old = 0.0, a_new = 1.0;
    if (C->old_valid) {
        const double span = C->t_new - C->t_old;
        const double teps = 1e-3 * span;
        if (time < C->t_old - teps || time > C->t_new + teps)
            return fail(BAMREX_ERR_ARG, "fill_patch time outside the coarse old/new interval");
        if (std::fabs(time - C->t_old) < teps) {
            mode = 0;
        } else if (std::fabs(time - C->t_new) < teps) {
            mode = 1;
        } else {
            mode = 2;
            a_old = (C->t_new - time) / span;
            a_new = (time - C->t_old) / span;
        }
    }
    return run_interp(C, 0, mode, a_old, a_new);
}

extern "C" int bamrex_coupling_fill_coarse_patch(bamrex_coupling* C)
{
    if (!C) return fail(BAMREX_ERR_ARG, "NULL coupling");
    return run_interp(C, 1, 1, 0.0, 1.0);
}

extern "C" int bamrex_coupling_reflux(bamrex_coupling* C)
{
    if (!C) return fail(BAMREX_ERR_ARG, "NULL coupling");
    bamrex_level* Lc = C->crse;
    double vol = 1.0;
    for (int d = 0; d < C->D; ++d) vol *= Lc->dx[d];
    for (int d = 0; d < C->D; ++d)
        BX_TRY(cpl_launch(C, launch_reflux(C->NC, Lc->fp32, C->d_rr[d], C->nslots[d], C->d_reg[d], vol, Lc->d_fab[Lc->cur],
                                           Lc->stream),
                          "reflux"));
    Lc->ws_valid = false;
    return BAMREX_OK;
}

extern "C" int bamrex_coupling_avg_down(bamrex_coupling* C)
{
    if (!C) return fail(BAMREX_ERR_ARG, "NULL coupling");
    bamrex_level* Lc = C->crse;
    bamrex_level* Lf = C->fine;
    BX_TRY(cpl_launch(C, launch_avg_down(C->D, C->NC, C->r, Lc->fp32, C->d_avg, C->navg, C->navg_cells, Lc->d_fab[Lc->cur],
                                         Lf->d_fab[Lf->cur], Lc->stream),
                      "average_down"));
    Lc->ws_valid = false;
    return BAMREX_OK;
}

extern "C" int bamrex_coupling_covered_sums(bamrex_coupling* C, double* sums)
{
    if (!C || !sums) return fail(BAMREX_ERR_ARG, "NULL argument");
    bamrex_level* Lc = C->crse;
    const int n = C->navg;
    for (int m = 0; m < C->NC; ++m) sums[m] = 0.0;
    if (!n) return BAMREX_OK;
    BX_TRY(cpl_launch(C, launch_box_sums(C->NC, Lc->fp32, C->d_cov_fab[Lc->cur], C->d_cov_box, n, C->d_cov_sums, Lc->stream),
                      "covered sums"));
    std::vector<double> h((size_t)n * C->NC);
    BX_CK(cudaMemcpyAsync(h.data(), C->d_cov_sums, h.size() * sizeof(double), cudaMemcpyDeviceToHost, Lc->stream));
    BX_CK(cudaStreamSynchronize(Lc->stream));
    double vol = 1.0;
    for (int d = 0; d < C->D; ++d) vol *= Lc->dx[d];
    for (int m = 0; m < C->NC; ++m) {
        double s = 0.0;
        for (int b = 0; b < n; ++b) s += h[(size_t)b * C->NC + m];
        sums[m] = s * vol;
    }
    return BAMREX_OK;
}

extern "C" int bamrex_coupling_register(bamrex_coupling* C, int dir, double* reg, int* nslots)
{
    if (!C || !nslots || dir < 0 || dir >= C->D) return fail(BAMREX_ERR_ARG, "bad argument");
    *nslots = C->nslots[dir];
    if (!reg || !C->nslots[dir]) return BAMREX_OK;
    BX_CK(cudaMemcpyAsync(reg, C->d_reg[dir], sizeof(double) * C->NC * C->nslots[dir], cudaMemcpyDeviceToHost,
                          C->crse->stream));
    BX_CK(cudaStreamSynchronize(C->crse->stream));
    return BAMREX_OK;
}

static int level_tag_spec(bamrex_level* L, const bamrex_tag_desc& t, char* tags)
{
    if (!L || !tags) return fail(BAMREX_ERR_ARG, "NULL argument");
    const bool do_grad = t.do_grad && t.phigrad > 0;
    if ((do_grad && (t.grad_var < 0 || t.grad_var >= L->NC)) || (t.do_err && (t.err_var < 0 || t.err_var >= L->NC)))
        return L->set_err(fail(BAMREX_ERR_ARG, "tagging variable index outside the state vector"));
    for (int d = 0; d < L->D; ++d) BX_TRY(level_fill(L, d, L->cur, nullptr));
    TagSpec spec;
    std::memset(&spec, 0, sizeof(spec));
    spec.do_err = t.do_err ? 1 : 0;
    spec.err_var = t.err_var;
    spec.err_primv = t.err_var_is_primv ? 1 : 0;
    spec.err_thr = t.phierr;
    spec.do_grad = do_grad ? 1 : 0;
    spec.grad_var = t.grad_var;
    spec.grad_primv = t.grad_var_is_primv ? 1 : 0;
    spec.grad_thr = t.phigrad;
    spec.do_box = t.do_box ? 1 : 0;
    for (int d = 0; d < 3; ++d) {
        spec.box_lo[d] = t.box_lo[d];
        spec.box_hi[d] = t.box_hi[d];
        spec.dx[d] = L->dx[d];
        spec.prob_lo[d] = L->prob_lo[d];
    }
    if (body_tag_tables(L, &spec.ls_tab, &spec.flag_tab)) {
        spec.do_iface = t.do_interface ? 1 : 0;
        spec.lstol = t.lstol;
    }
    if (!L->tag_buf) {
        const cudaError_t ea = dev_alloc((void**)&L->tag_buf, (size_t)std::max(1LL, L->ncells), L->stream);
        if (ea != cudaSuccess) return L->set_err(cuda_fail(ea, "tag buffer allocation"));
    }
    char* dtags = L->tag_buf;
    BX_TRY(level_launch(L, launch_tag(L->D, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(), L->ncells, L->k,
                                      spec, dtags, L->stream),
                        "tagging"));
    cudaError_t e = cudaMemcpyAsync(tags, dtags, (size_t)L->ncells, cudaMemcpyDeviceToHost, L->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "tag readback"));
    return BAMREX_OK;
}

extern "C" int bamrex_level_tag(bamrex_level* L, int grad_var, int grad_var_is_primv, double grad_threshold,
                                int do_err, int err_var, int err_var_is_primv, double phierr, char* tags)
{
    bamrex_tag_desc t;
    std::memset(&t, 0, sizeof(t));
    t.do_grad = grad_threshold > 0;
    t.grad_var = grad_var;
    t.grad_var_is_primv = grad_var_is_primv;
    t.phigrad = grad_threshold;
    t.do_err = do_err;
    t.err_var = err_var;
    t.err_var_is_primv = err_var_is_primv;
    t.phierr = phierr;
    return level_tag_spec(L, t, tags);
}

extern "C" int bamrex_level_tag_ex(bamrex_level* L, const bamrex_tag_desc* desc, char* tags)
{
    if (!desc) return fail(BAMREX_ERR_ARG, "NULL argument");
    return level_tag_spec(L, *desc, tags);
}

// ======================================================================
// grid generation
// ======================================================================
namespace {

struct Mask3 {
    int n[3] = { 1, 1, 1 };
    std::vector<unsigned char> v;
    void init(const int* nn, unsigned char x)
    {
        for (int d = 0; d < 3; ++d) n[d] = nn[d];
        v.assign((size_t)n[0] * n[1] * n[2], x);
    }
    unsigned char& at(int i, int j, int k) { return v[((size_t)k * n[1] + j) * n[0] + i]; }
    unsigned char at(int i, int j, int k) const { return v[((size_t)k * n[1] + j) * n[0] + i]; }
};

// Blocked-space tags and the proper-nesting test of grid generation, built
// from the level's boxes without a cell mask over the whole domain.  A
// blocked cell (c level-l cells per side) is tagged when a tagged cell lies
// within n_error_buf cells of its footprint, and allowed when every cell
// within n_proper cells of its footprint is covered by the level's boxes
// (across a non-periodic domain side every cell counts as covered, a
// periodic side wraps).  A blocked cell refines when it is both.  This is
// the same as buffering the tags cell by cell, dropping buffered tags
// outside the n_proper-eroded coverage and then blocking, because every
// footprint cell of an allowed blocked cell lies in the eroded coverage.
struct BlockedSpace {
    int D = 0, c = 1, nbuf = 0, nprop = 0;
    int n[3] = { 1, 1, 1 }, nt[3] = { 1, 1, 1 }, dl[3] = { 0, 0, 0 }, per[3] = { 0, 0, 0 };
    const std::vector<bamrex_box>* boxes = nullptr;
    BoxIndex idx;
    Mask3 near_tag;   // a tag within n_error_buf of the footprint
    Mask3 allowed;    // 0 / 1, 2 = not evaluated yet

    int cell(int d) const { return d < D ? c : 1; }

    // the blocked indices [a, b] of dimension d wrapped (periodic) or
    // clipped into range; returns the number of pieces written to lo/hi
    int pieces(int d, int a, int b, int* lo, int* hi, int N) const
    {
        if (per[d]) {
            if (b - a + 1 >= N) {
                lo[0] = 0;
                hi[0] = N - 1;
                return 1;
            }
            const int a2 = ((a % N) + N) % N, b2 = a2 + (b - a);
            if (b2 < N) {
                lo[0] = a2;
                hi[0] = b2;
                return 1;
            }
            lo[0] = a2;
            hi[0] = N - 1;
            lo[1] = 0;
            hi[1] = b2 - N;
            return 2;
        }
        lo[0] = std::max(a, 0);
        hi[0] = std::min(b, N - 1);
        return lo[0] <= hi[0] ? 1 : 0;
    }

    void mark_run(int x0, int x1, int y, int z)
    {
        const int cl[3] = { x0, y, z }, ch[3] = { x1, y, z };
        int lo[3][2], hi[3][2], np[3];
        for (int d = 0; d < 3; ++d) {
            const int nb = d < D ? nbuf : 0, cc = cell(d);
            np[d] = pieces(d, floor_div(cl[d] - nb, cc), floor_div(ch[d] + nb, cc), lo[d], hi[d], nt[d]);
        }
        for (int pz = 0; pz < np[2]; ++pz)
            for (int K = lo[2][pz]; K <= hi[2][pz]; ++K)
                for (int py = 0; py < np[1]; ++py)
                    for (int J = lo[1][py]; J <= hi[1][py]; ++J)
                        for (int px = 0; px < np[0]; ++px)
                            for (int I = lo[0][px]; I <= hi[0][px]; ++I)
                                __atomic_store_n(&near_tag.at(I, J, K), (unsigned char)1, __ATOMIC_RELAXED);
    }

    // the cache entry of (I, J, K) is written by its caller only; hits:
    // the caller's scratch
    bool is_allowed(int I, int J, int K, std::vector<int>& hits)
    {
        unsigned char& v = allowed.at(I, J, K);
        if (v != 2) return v != 0;
        const int B[3] = { I, J, K };
        int lo[3][2], hi[3][2], np[3];
        for (int d = 0; d < 3; ++d) {
            const int pr = d < D ? nprop : 0, cc = cell(d);
            np[d] = pieces(d, B[d] * cc - pr, B[d] * cc + cc - 1 + pr, lo[d], hi[d], n[d]);
        }
        bool ok = true;
        for (int pz = 0; pz < np[2] && ok; ++pz)
            for (int py = 0; py < np[1] && ok; ++py)
                for (int px = 0; px < np[0] && ok; ++px) {
                    bamrex_box q;
                    q.lo[0] = lo[0][px] + dl[0];
                    q.hi[0] = hi[0][px] + dl[0];
                    q.lo[1] = lo[1][py] + dl[1];
                    q.hi[1] = hi[1][py] + dl[1];
                    q.lo[2] = lo[2][pz] + dl[2];
                    q.hi[2] = hi[2][pz] + dl[2];
                    idx.query(q.lo, q.hi, hits);
                    long long got = 0;
                    for (int h : hits) got += box_volume(intersect(q, (*boxes)[h]));
                    ok = got == box_volume(q);  // the level's boxes are disjoint
                }
        v = ok ? 1 : 0;
        return ok;
    }
};

struct Cluster {
    const Mask3* tags;
    double eff;
    int D;
    std::vector<bamrex_box> out;

    // One pass over b: the tag signatures along each direction, from which
    // the tight bounding box (the first and last non-zero entries) and the
    // tag count follow; the signatures of the tight box are the non-zero
    // range of these, as no tag lies outside it.
    void run(bamrex_box b, int depth)
    {
        std::vector<long long> sig[3];
        for (int d = 0; d < D; ++d) sig[d].assign(b.hi[d] - b.lo[d] + 1, 0);
        long long nt = 0;
        for (int k = b.lo[2]; k <= b.hi[2]; ++k)
            for (int j = b.lo[1]; j <= b.hi[1]; ++j)
                for (int i = b.lo[0]; i <= b.hi[0]; ++i)
                    if (tags->at(i, j, k)) {
                        const int c[3] = { i, j, k };
                        for (int d = 0; d < D; ++d) sig[d][c[d] - b.lo[d]]++;
                        ++nt;
                    }
        if (nt == 0) return;
        for (int d = 0; d < D; ++d) {
            int f = 0, l = (int)sig[d].size() - 1;
            while (sig[d][f] == 0) ++f;
            while (sig[d][l] == 0) --l;
            sig[d].erase(sig[d].begin() + l + 1, sig[d].end());
            sig[d].erase(sig[d].begin(), sig[d].begin() + f);
            b.hi[d] = b.lo[d] + l;
            b.lo[d] += f;
        }
        const long long vol = box_volume(b);
        bool all_unit = true;
        for (int d = 0; d < D; ++d) all_unit = all_unit && b.hi[d] == b.lo[d];
        if ((double)nt >= eff * (double)vol || all_unit || depth > 64) {
            out.push_back(b);
            return;
        }
        int best_d = -1, best_cut = 0;
        // 1) a hole (zero signature) closest to the middle
        long long best_score = -1;
        for (int d = 0; d < D; ++d) {
            const int n = (int)sig[d].size();
            for (int x = 1; x < n - 1; ++x)
                if (sig[d][x] == 0) {
                    const long long score = (long long)n * 4 - std::abs(2 * x - n);
                    if (score > best_score) {
                        best_score = score;
                        best_d = d;
                        best_cut = x;
                    }
                }
        }
        if (best_d < 0) {
            // 2) the strongest inflection of the signature (sign change of
            // its second difference)
            long long best_jump = 0;
            for (int d = 0; d < D; ++d) {
                const int n = (int)sig[d].size();
                if (n < 4) continue;
                std::vector<long long> lap(n, 0);
                for (int x = 1; x < n - 1; ++x) lap[x] = sig[d][x - 1] - 2 * sig[d][x] + sig[d][x + 1];
                for (int x = 1; x < n - 2; ++x) {
                    if ((lap[x] > 0 && lap[x + 1] < 0) || (lap[x] < 0 && lap[x + 1] > 0)) {
                        const long long jump = std::llabs(lap[x] - lap[x + 1]);
                        if (jump > best_jump) {
                            best_jump = jump;
                            best_d = d;
                            best_cut = x + 1;
                        }
                    }
                }
            }
        }
        if (best_d < 0) {
            // 3) halve the longest side
            int len = 0;
            for (int d = 0; d < D; ++d)
                if (b.hi[d] - b.lo[d] + 1 > len) {
                    len = b.hi[d] - b.lo[d] + 1;
                    best_d = d;
                }
            best_cut = len / 2;
        }
        bamrex_box a = b, c = b;
        a.hi[best_d] = b.lo[best_d] + best_cut - 1;
        c.lo[best_d] = b.lo[best_d] + best_cut;
        run(a, depth + 1);
        run(c, depth + 1);
    }
};

// Split b until every piece lies inside the allowed blocked cells (pieces
// with no allowed cell are dropped).
void clip_to_allowed(BlockedSpace& bs, const bamrex_box& b, int D, std::vector<bamrex_box>& out,
                     std::vector<int>& hits)
{
    long long nin = 0;
    for (int k = b.lo[2]; k <= b.hi[2]; ++k)
        for (int j = b.lo[1]; j <= b.hi[1]; ++j)
            for (int i = b.lo[0]; i <= b.hi[0]; ++i) nin += bs.is_allowed(i, j, k, hits) ? 1 : 0;
    if (nin == 0) return;
    if (nin == box_volume(b)) {
        out.push_back(b);
        return;
    }
    int best_d = 0, len = 0;
    for (int d = 0; d < D; ++d)
        if (b.hi[d] - b.lo[d] + 1 > len) {
            len = b.hi[d] - b.lo[d] + 1;
            best_d = d;
        }
    bamrex_box a = b, c = b;
    a.hi[best_d] = b.lo[best_d] + len / 2 - 1;
    c.lo[best_d] = b.lo[best_d] + len / 2;
    clip_to_allowed(bs, a, D, out, hits);
    clip_to_allowed(bs, c, D, out, hits);
}

void chop(const bamrex_box& b, int D, int mgs, std::vector<bamrex_box>& out)
{
    for (int d = 0; d < D; ++d) {
        const int len = b.hi[d] - b.lo[d] + 1;
        if (len > mgs) {
            const int pieces = (len + mgs - 1) / mgs;
            const int base = len / pieces, extra = len % pieces;
            int lo = b.lo[d];
            for (int p = 0; p < pieces; ++p) {
                bamrex_box q = b;
                q.lo[d] = lo;
                q.hi[d] = lo + base + (p < extra ? 1 : 0) - 1;
                lo = q.hi[d] + 1;
                chop(q, D, mgs, out);
            }
            return;
        }
    }
    out.push_back(b);
}

}  // namespace

extern "C" int bamrex_cluster_tags(int D, const bamrex_box* domain, const int* periodic, const bamrex_box* boxes,
                                   int nboxes, const char* tags, int ref_ratio, int blocking_factor,
                                   int max_grid_size, int n_error_buf, int n_proper, double grid_eff,
                                   bamrex_box* out, int max_out, int* nout)
{
    BX_PROFILE("bamrex_cluster_tags");
    if (!domain || !boxes || !tags || !nout || D < 1 || D > 3 || nboxes < 1) return fail(BAMREX_ERR_ARG, "bad argument");
    if (ref_ratio != 2 && ref_ratio != 4) return fail(BAMREX_ERR_ARG, "ref_ratio must be 2 or 4");
    if (blocking_factor < 2 * ref_ratio || blocking_factor % (2 * ref_ratio) != 0)
        return fail(BAMREX_ERR_ARG, "blocking_factor must be a multiple of 2 * ref_ratio");
    if (max_grid_size < blocking_factor || max_grid_size % blocking_factor != 0)
        return fail(BAMREX_ERR_ARG, "max_grid_size must be a multiple of blocking_factor");
    if (n_error_buf < 0 || n_proper < 0 || !(grid_eff > 0 && grid_eff <= 1))
        return fail(BAMREX_ERR_ARG, "bad n_error_buf / n_proper / grid_eff");
    const int c = blocking_factor / ref_ratio;  // level-l cells per blocked cell
    int n[3] = { 1, 1, 1 }, nt[3] = { 1, 1, 1 };
    for (int d = 0; d < D; ++d) {
        n[d] = domain->hi[d] - domain->lo[d] + 1;
        if (n[d] % c != 0) return fail(BAMREX_ERR_ARG, "domain not divisible by blocking_factor / ref_ratio");
        nt[d] = n[d] / c;
    }
    const int dl[3] = { domain->lo[0], domain->lo[1], domain->lo[2] };
    std::vector<bamrex_box> bxs(boxes, boxes + nboxes);
    for (const auto& B : bxs)
        for (int d = 0; d < 3; ++d)
            if (B.lo[d] < dl[d] || B.hi[d] >= dl[d] + n[d] || B.hi[d] < B.lo[d])
                return fail(BAMREX_ERR_ARG, "box outside the domain");
    ProfPhases phase("cluster_tags:mark");
    BlockedSpace bs;
    bs.D = D;
    bs.c = c;
    bs.nbuf = n_error_buf;
    bs.nprop = n_proper;
    for (int d = 0; d < 3; ++d) {
        bs.n[d] = n[d];
        bs.nt[d] = nt[d];
        bs.dl[d] = dl[d];
        bs.per[d] = (periodic && d < D) ? (periodic[d] != 0) : 0;
    }
    bs.boxes = &bxs;
    bs.idx.build(*domain, bxs, D);
    bs.near_tag.init(nt, 0);
    bs.allowed.init(nt, 2);
    // runs of tagged cells along x, box by box in packed order, boxes on
    // host threads (marks are idempotent stores of 1); zero words of eight
    // tags are skipped whole
    std::vector<long long> boff(bxs.size() + 1, 0);
    for (size_t b = 0; b < bxs.size(); ++b) boff[b + 1] = boff[b] + box_volume(bxs[b]);
    auto scan_box = [&](int b, int&) -> std::string {
        const bamrex_box& B = bxs[(size_t)b];
        const int len = B.hi[0] - B.lo[0] + 1;
        long long off = boff[(size_t)b];
        for (int k = B.lo[2]; k <= B.hi[2]; ++k)
            for (int j = B.lo[1]; j <= B.hi[1]; ++j) {
                const char* row = tags + off;
                off += len;
                for (int i = 0; i < len;) {
                    if (i + 8 <= len) {
                        unsigned long long w;
                        std::memcpy(&w, row + i, 8);
                        if (!w) {
                            i += 8;
                            continue;
                        }
                    }
                    if (!row[i]) {
                        ++i;
                        continue;
                    }
                    int e = i;
                    while (e + 1 < len && row[e + 1]) ++e;
                    bs.mark_run(B.lo[0] + i - dl[0], B.lo[0] + e - dl[0], j - dl[1], k - dl[2]);
                    i = e + 1;
                }
            }
        return std::string();
    };
    BX_TRY(parallel_items<int>((int)bxs.size(), table_threads(boff.back() / 8), 8, scan_box));
    phase.next("cluster_tags:allowed");
    // blocked cells near a tag and allowed, planes of K on host threads
    Mask3 btag;
    btag.init(nt, 0);
    auto plane = [&](int K, std::vector<int>& hits) -> std::string {
        for (int J = 0; J < nt[1]; ++J)
            for (int I = 0; I < nt[0]; ++I)
                if (bs.near_tag.at(I, J, K) && bs.is_allowed(I, J, K, hits)) btag.at(I, J, K) = 1;
        return std::string();
    };
    BX_TRY(parallel_items<std::vector<int>>(nt[2], table_threads((long long)nt[0] * nt[1] * nt[2] / 4), 1, plane));
    phase.next("cluster_tags:cluster");
    Cluster cl;
    cl.tags = &btag;
    cl.eff = grid_eff;
    cl.D = D;
    bamrex_box all;
    for (int d = 0; d < 3; ++d) {
        all.lo[d] = 0;
        all.hi[d] = nt[d] - 1;
    }
    cl.run(all, 0);
    phase.next("cluster_tags:clip_chop");
    // the clusters are disjoint, so each blocked cell's cache entry is
    // evaluated by one thread; pieces joined in cluster order
    std::vector<std::vector<bamrex_box>> pieces(cl.out.size());
    long long cvol = 0;
    for (const auto& b : cl.out) cvol += box_volume(b);
    BX_TRY(parallel_items<std::vector<int>>((int)cl.out.size(), table_threads(cvol / 4), 4,
                                            [&](int q, std::vector<int>& hits) -> std::string {
                                                clip_to_allowed(bs, cl.out[(size_t)q], D, pieces[(size_t)q], hits);
                                                return std::string();
                                            }));
    std::vector<bamrex_box> clipped, chopped;
    for (const auto& p : pieces) clipped.insert(clipped.end(), p.begin(), p.end());
    const int mgs_t = max_grid_size / blocking_factor;
    for (const auto& b : clipped) chop(b, D, mgs_t, chopped);
    std::sort(chopped.begin(), chopped.end(), [](const bamrex_box& a, const bamrex_box& b) {
        return std::make_tuple(a.lo[2], a.lo[1], a.lo[0]) < std::make_tuple(b.lo[2], b.lo[1], b.lo[0]);
    });
    *nout = (int)chopped.size();
    if ((int)chopped.size() > max_out) return fail(BAMREX_ERR_ARG, "output box array too small");
    for (size_t q = 0; q < chopped.size(); ++q) {
        bamrex_box f;
        for (int d = 0; d < 3; ++d) {
            if (d < D) {
                f.lo[d] = (chopped[q].lo[d] * c + dl[d]) * ref_ratio;
                f.hi[d] = ((chopped[q].hi[d] + 1) * c + dl[d]) * ref_ratio - 1;
            } else {
                f.lo[d] = f.hi[d] = 0;
            }
        }
        out[q] = f;
    }
    return BAMREX_OK;
}

// ======================================================================
// hierarchy
// ======================================================================
struct bamrex_amr {
    bamrex_amr_desc desc;
    int D = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<bamrex_level*> levels;
    std::vector<bamrex_coupling*> cpl;  // cpl[l] couples l-1 and l
    std::vector<double> dt_level;
    int steps = 0;
    bool have_dt = false;
    bool has_body = false;     // a rigid body on every level (bamrex_amr_set_body)
    bamrex_body_desc body;
    // coarse steps as CUDA graphs (time steps computed on the device): one
    // graph per level-state key, all dropped when the levels change
    bool use_graph = true;
    unsigned generation = 0;
    AmrDev* d_amr = nullptr;
    AmrDev* h_amr = nullptr;   // pinned: the step's dt and status, read back
    double* h_up = nullptr;    // pinned: {time, stop_time} uploaded per step
    struct StepGraph {
        unsigned gen = 0;
        std::vector<int> key;   // per level: current buffer, CFL estimate valid
        cudaGraphExec_t exec = nullptr;
        std::vector<int> post;  // the key after the step
        long long kernels = 0;  // kernel launches inside the graph
    };
    std::vector<StepGraph> graphs;
    int graph_captures = 0;
    long long graph_replays = 0;
    int gen_steps = 0;  // coarse steps since the levels last changed
    std::string err;
    int set_err(int code)
    {
        err = last_error_text();
        return code;
    }
};

namespace {

int amr_fail(bamrex_amr* A, int code, const std::string& msg) { return A->set_err(fail(code, msg)); }

#define AMR_TRY(A, call)                           \
    do {                                           \
        int rc_ = (call);                          \
        if (rc_ != BAMREX_OK) return (A)->set_err(rc_); \
    } while (0)

int make_level(bamrex_amr* A, int lev, const std::vector<bamrex_box>& boxes, bamrex_level** out)
{
    bamrex_level_desc d = A->desc.base;
    int f = 1;
    for (int l = 0; l < lev; ++l) f *= A->desc.ref_ratio;
    for (int q = 0; q < A->D; ++q) {
        d.domain.lo[q] = A->desc.base.domain.lo[q] * f;
        d.domain.hi[q] = (A->desc.base.domain.hi[q] + 1) * f - 1;
    }
    d.boxes = boxes.data();
    d.nboxes = (int)boxes.size();
    BX_TRY(bamrex_level_create(out, &d, A->stream));
    if (A->has_body) {
        const int rc = bamrex_level_set_body(*out, &A->body);
        if (rc != BAMREX_OK) {
            bamrex_level_destroy(*out);
            *out = nullptr;
            return rc;
        }
    }
    return BAMREX_OK;
}

void drop_step_graphs(bamrex_amr* A)
{
    for (auto& g : A->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    A->graphs.clear();
    A->generation++;
    A->gen_steps = 0;
}

void drop_levels_above(bamrex_amr* A, int lev)
{
    if ((int)A->levels.size() > lev + 1) drop_step_graphs(A);
    while ((int)A->levels.size() > lev + 1) {
        const int l = (int)A->levels.size() - 1;
        bamrex_coupling_destroy(A->cpl[l]);
        bamrex_level_destroy(A->levels[l]);
        A->cpl.pop_back();
        A->levels.pop_back();
    }
    A->dt_level.resize(A->levels.size(), A->dt_level.empty() ? 0.0 : A->dt_level.back());
}

bool same_boxes(const std::vector<bamrex_box>& a, const std::vector<bamrex_box>& b)
{
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
        for (int d = 0; d < 3; ++d)
            if (a[i].lo[d] != b[i].lo[d] || a[i].hi[d] != b[i].hi[d]) return false;
    return true;
}

// defer_finer: leave the next finer level uncoupled (cpl[lev + 1] null) for
// couple_missing, as a regrid about to replace that level would throw the
// coupling away
int set_level(bamrex_amr* A, int lev, const std::vector<bamrex_box>& boxes, bool defer_finer = false)
{
    const int finest = (int)A->levels.size() - 1;
    if (lev < 1 || lev > finest + 1 || lev > A->desc.max_level) return amr_fail(A, BAMREX_ERR_ARG, "level out of range");
    const int bf = A->desc.blocking_factor;
    for (const auto& b : boxes)
        for (int d = 0; d < A->D; ++d)
            if (b.lo[d] % bf != 0 || (b.hi[d] + 1) % bf != 0)
                return amr_fail(A, BAMREX_ERR_ARG, "fine boxes must be aligned to blocking_factor");
    if (lev <= finest && same_boxes(boxes, A->levels[lev]->boxes)) return BAMREX_OK;
    BX_PROFILE("amr_set_level");
    drop_step_graphs(A);
    ProfPhases phase("amr_set_level:make_level");
    bamrex_level* L = nullptr;
    AMR_TRY(A, make_level(A, lev, boxes, &L));
    phase.next("amr_set_level:coupling");
    bamrex_coupling* C = nullptr;
    int rc = bamrex_coupling_create(&C, A->levels[lev - 1], L, A->desc.ref_ratio);
    if (rc != BAMREX_OK) {
        bamrex_level_destroy(L);
        return A->set_err(rc);
    }
    phase.next("amr_set_level:fill_coarse_patch");
    rc = bamrex_coupling_fill_coarse_patch(C);
    phase.next("amr_set_level:copy_old");
    if (rc == BAMREX_OK && lev <= finest) {
        // old data of this level where the new boxes overlap it
        bamrex_level* O = A->levels[lev];
        std::vector<GhostOp> ops;
        const int nnew = (int)L->boxes.size();
        BoxIndex oidx;
        oidx.build(O->domain, O->boxes, A->D);
        std::vector<int> hits;
        for (int b = 0; b < nnew; ++b) {
            oidx.query(L->boxes[b].lo, L->boxes[b].hi, hits);
            std::sort(hits.begin(), hits.end());
            for (int s : hits) {
                const bamrex_box x = intersect(L->boxes[b], O->boxes[s]);
                if (box_empty(x)) continue;
                GhostOp op;
                std::memset(&op, 0, sizeof(op));
                op.dst = b;
                op.src = nnew + s;
                for (int d = 0; d < 3; ++d) {
                    op.lo[d] = x.lo[d];
                    op.hi[d] = x.hi[d];
                    op.mul[d] = 1;
                }
                ops.push_back(op);
            }
        }
        const int nchunks = number_ghost_ops(ops);
        if (!ops.empty()) {
            std::vector<FabDev> tab = L->fab[L->cur];
            tab.insert(tab.end(), O->fab[O->cur].begin(), O->fab[O->cur].end());
            void* dmem = nullptr;
            const size_t tb = sizeof(FabDev) * tab.size(), ob = sizeof(GhostOp) * ops.size();
            const std::vector<int> ct = ghost_chunk_table(ops, nchunks);
            cudaError_t e = dev_alloc(&dmem, align_up(tb, 256) + ghost_table_bytes(ops.size(), nchunks), A->stream);
            if (e == cudaSuccess) e = cudaMemcpyAsync(dmem, tab.data(), tb, cudaMemcpyHostToDevice, A->stream);
            GhostOp* dops = (GhostOp*)((char*)dmem + align_up(tb, 256));
            if (e == cudaSuccess) e = cudaMemcpyAsync(dops, ops.data(), ob, cudaMemcpyHostToDevice, A->stream);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(dops + ops.size(), ct.data(), sizeof(int) * ct.size(), cudaMemcpyHostToDevice, A->stream);
            if (e == cudaSuccess)
                e = launch_ghost_fill(L->NC, L->fp32, dops, (int)ops.size(), nchunks, (const FabDev*)dmem, nullptr, A->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
            dev_free(dmem, A->stream);
            if (e != cudaSuccess) rc = cuda_fail(e, "regrid copy");
        }
    }
    if (rc == BAMREX_OK) rc = bamrex_level_sync(L);
    if (rc != BAMREX_OK) {
        bamrex_coupling_destroy(C);
        bamrex_level_destroy(L);
        return A->set_err(rc);
    }
    phase.next("amr_set_level:recouple_finer");
    // the next finer level stays if it is still properly nested in the new
    // boxes (coupled afresh), else it and everything above it go
    bamrex_coupling* C2 = nullptr;
    bool keep_finer = false;
    if (lev + 1 <= finest) {
        bamrex_coupling_destroy(A->cpl[lev + 1]);
        A->cpl[lev + 1] = nullptr;
        keep_finer = defer_finer || bamrex_coupling_create(&C2, L, A->levels[lev + 1], A->desc.ref_ratio) == BAMREX_OK;
    }
    phase.next("amr_set_level:destroy_old");
    if (lev <= finest) {
        bamrex_coupling_destroy(A->cpl[lev]);
        bamrex_level_destroy(A->levels[lev]);
        A->levels[lev] = L;
        A->cpl[lev] = C;
    } else {
        A->levels.push_back(L);
        A->cpl.push_back(C);
        A->dt_level.resize(A->levels.size(), A->dt_level.empty() ? 0.0 : A->dt_level.back() / A->desc.ref_ratio);
    }
    if (lev + 1 <= finest) {
        if (keep_finer) A->cpl[lev + 1] = C2;
        else drop_levels_above(A, lev);
    }
    return BAMREX_OK;
}

// Couple every level from 1 to upto (at most the finest) that a deferred
// set_level left uncoupled; a level that is not properly nested in the one
// below goes, with everything above it.
int couple_missing(bamrex_amr* A, int upto)
{
    for (int l = 1; l <= upto && l < (int)A->levels.size(); ++l) {
        if (A->cpl[l]) continue;
        bamrex_coupling* C = nullptr;
        if (bamrex_coupling_create(&C, A->levels[l - 1], A->levels[l], A->desc.ref_ratio) == BAMREX_OK) {
            A->cpl[l] = C;
        } else {
            drop_levels_above(A, l - 1);
            break;
        }
    }
    return BAMREX_OK;
}

int level_tags(bamrex_amr* A, int l, double time, std::vector<char>& tags)
{
    BX_PROFILE("amr_regrid:tags");
    bamrex_level* L = A->levels[l];
    if (l > 0) AMR_TRY(A, bamrex_coupling_fill_patch(A->cpl[l], time));
    const bamrex_amr_desc& d = A->desc;
    bamrex_tag_desc t;
    std::memset(&t, 0, sizeof(t));
    t.do_grad = l < d.max_phigrad_lev;
    t.phigrad = t.do_grad ? d.phigrad[l] : 0.0;
    t.grad_var = d.phigrad_var;
    t.grad_var_is_primv = d.phigrad_var_is_primv;
    t.do_err = l < d.max_phierr_lev;
    t.phierr = t.do_err ? d.phierr[l] : 0.0;
    t.err_var = d.phierr_var;
    t.err_var_is_primv = d.phierr_var_is_primv;
    t.do_box = l < d.max_box_lev;
    for (int q = 0; q < 3; ++q) {
        t.box_lo[q] = d.box_lo[q];
        t.box_hi[q] = d.box_hi[q];
    }
    t.do_interface = A->has_body && l < d.max_int_lev;
    t.lstol = (t.do_interface && l < BAMREX_MAX_LEVELS) ? d.lstol[l] : 0.0;
    tags.assign((size_t)L->ncells, 0);
    AMR_TRY(A, bamrex_level_tag_ex(L, &t, tags.data()));
    return BAMREX_OK;
}

int regrid_levels(bamrex_amr* A, int lbase, double time)
{
    const bamrex_amr_desc& d = A->desc;
    for (int l = lbase; l < d.max_level && l < (int)A->levels.size(); ++l) {
        BX_TRY(couple_missing(A, l));  // level l's ghost fill needs its coupling
        if (l >= (int)A->levels.size()) break;
        std::vector<char> tags;
        BX_TRY(level_tags(A, l, time, tags));
        bamrex_level* L = A->levels[l];
        int periodic[3] = { 0, 0, 0 };
        for (int q = 0; q < A->D; ++q) periodic[q] = L->bc_lo[q] == BAMREX_BC_PERIODIC;
        // at most one new box per blocked cell
        const int cb = d.blocking_factor / d.ref_ratio;
        long long nblk = 1;
        for (int q = 0; q < A->D; ++q) nblk *= (L->domain.hi[q] - L->domain.lo[q] + 1) / cb;
        std::vector<bamrex_box> nb((size_t)std::max<long long>(1, nblk));
        int n = 0;
        AMR_TRY(A, bamrex_cluster_tags(A->D, &L->domain, periodic, L->boxes.data(), (int)L->boxes.size(), tags.data(),
                                       d.ref_ratio, d.blocking_factor, d.max_grid_size, d.n_error_buf, d.n_proper,
                                       d.grid_eff, nb.data(), (int)nb.size(), &n));
        nb.resize(n);
        if (n == 0) {
            drop_levels_above(A, l);
            break;
        }
        BX_TRY(set_level(A, l + 1, nb, true));
    }
    return BAMREX_OK;
}

// Regrid levels lbase+1 and up: every level replaced defers the coupling of
// the one above it, which the next round of the loop usually replaces too;
// what is left uncoupled is coupled at the end, on every path.
int regrid(bamrex_amr* A, int lbase, double time)
{
    BX_PROFILE("amr_regrid");
    const int rc = regrid_levels(A, lbase, time);
    const int rc2 = couple_missing(A, (int)A->levels.size() - 1);
    return rc != BAMREX_OK ? rc : rc2;
}

int compute_dt(bamrex_amr* A, double time, double stop_time, bool initial, bool post_regrid)
{
    const int nl = (int)A->levels.size();
    std::vector<double> dt_min(nl);
    for (int l = 0; l < nl; ++l) {
        double e = 0;
        AMR_TRY(A, bamrex_level_est_time_step(A->levels[l], &e));
        dt_min[l] = e;
        if (!initial && post_regrid && l < (int)A->dt_level.size() && A->dt_level[l] > 0)
            dt_min[l] = std::min(dt_min[l], A->dt_level[l]);
    }
    double dt0 = 1.0e100;
    long long nf = 1;
    for (int l = 0; l < nl; ++l) {
        if (l > 0) nf *= A->desc.ref_ratio;
        dt0 = std::min(dt0, (double)nf * dt_min[l]);
    }
    const double eps = 0.001 * dt0;
    if (stop_time >= 0.0 && (time + dt0) > (stop_time - eps)) dt0 = stop_time - time;
    A->dt_level.assign(nl, 0.0);
    nf = 1;
    for (int l = 0; l < nl; ++l) {
        if (l > 0) nf *= A->desc.ref_ratio;
        A->dt_level[l] = dt0 / (double)nf;
    }
    A->have_dt = true;
    return BAMREX_OK;
}

int time_step(bamrex_amr* A, int l, double time)
{
    const int finest = (int)A->levels.size() - 1;
    const double dt = A->dt_level[l];
    bamrex_level* L = A->levels[l];
    if (l < finest) AMR_TRY(A, bamrex_coupling_save_coarse_old(A->cpl[l + 1], time, time + dt));
    if (l > 0) AMR_TRY(A, bamrex_coupling_fill_patch(A->cpl[l], time));
    double used = 0;
    AMR_TRY(A, bamrex_level_advance(L, time, dt, 1, 1, &used));
    if (l < finest) {
        const double dtf = A->dt_level[l + 1];
        for (int i = 0; i < A->desc.ref_ratio; ++i) BX_TRY(time_step(A, l + 1, time + i * dtf));
        if (A->desc.do_reflux) AMR_TRY(A, bamrex_coupling_reflux(A->cpl[l + 1]));
        AMR_TRY(A, bamrex_coupling_avg_down(A->cpl[l + 1]));
    }
    return BAMREX_OK;
}

// ---------------------------------------------------------------------
// A coarse step with the time steps on the device, replayed as one graph.
//
// The host path above reads every level's CFL estimate back, forms the
// coarse dt and enqueues the subcycled recursion with host values.  Here
// the estimates, the coarse dt (amr_dt_kernel: the same operations) and
// the substeps' start times (amr_substep_kernel: parent start + i * dt)
// stay on the device; the levels' sweeps and flux registers read their dt
// from their step scalars and the coarse/fine fills pick their time weights
// from the device times.  The recursion does not depend on the values, so
// it is captured once per level-state key and replayed every coarse step.
// ---------------------------------------------------------------------

// bamrex_level_advance with the level's device dt (set by amr_dt_kernel).
int level_advance_dev(bamrex_level* L)
{
    const cudaError_t e = cudaMemsetAsync(&L->d_scal->ws_bits, 0, sizeof(unsigned long long), L->stream);
    if (e != cudaSuccess) return L->set_err(cuda_fail(e, "memset"));
    BX_TRY(level_step(L, L->cur, 0.0, L->d_scal, false, false));
    L->cur ^= (L->D & 1);
    L->ws_valid = true;
    return BAMREX_OK;
}

// time_step on device times: substep i of level l within its parent's step.
int time_step_dev(bamrex_amr* A, int l, int i)
{
    const int finest = (int)A->levels.size() - 1;
    bamrex_level* L = A->levels[l];
    if (l > 0) BX_CK(launch_amr_substep(A->d_amr, l, i, A->stream));
    if (l < finest) {
        // bamrex_coupling_save_coarse_old; its times are set on the host
        // after the step (host_step_times)
        bamrex_coupling* C = A->cpl[l + 1];
        AMR_TRY(A, save_patch_old(C));
        C->old_valid = true;
    }
    if (l > 0) AMR_TRY(A, run_interp(A->cpl[l], 0, 2, 0.0, 1.0, A->d_amr, l - 1));
    AMR_TRY(A, level_advance_dev(L));
    if (l < finest) {
        for (int j = 0; j < A->desc.ref_ratio; ++j) BX_TRY(time_step_dev(A, l + 1, j));
        if (A->desc.do_reflux) AMR_TRY(A, bamrex_coupling_reflux(A->cpl[l + 1]));
        AMR_TRY(A, bamrex_coupling_avg_down(A->cpl[l + 1]));
    }
    return BAMREX_OK;
}

// The couplings' coarse old/new times the host recursion leaves (time_step).
void host_step_times(bamrex_amr* A, int l, double time)
{
    if (l + 1 >= (int)A->levels.size()) return;
    bamrex_coupling* C = A->cpl[l + 1];
    C->old_valid = true;
    C->t_old = time;
    C->t_new = time + A->dt_level[l];
    const double dtf = A->dt_level[l + 1];
    for (int i = 0; i < A->desc.ref_ratio; ++i) host_step_times(A, l + 1, time + i * dtf);
}

std::vector<int> step_key(const bamrex_amr* A)
{
    std::vector<int> k;
    for (const bamrex_level* L : A->levels) {
        k.push_back(L->cur);
        k.push_back(L->ws_valid ? 1 : 0);
    }
    return k;
}

void set_step_key(bamrex_amr* A, const std::vector<int>& k)
{
    for (size_t l = 0; l < A->levels.size(); ++l) {
        A->levels[l]->cur = k[2 * l];
        A->levels[l]->ws_valid = k[2 * l + 1] != 0;
    }
}

AmrLevelsArg levels_arg(const bamrex_amr* A)
{
    AmrLevelsArg a;
    std::memset(&a, 0, sizeof(a));
    a.nl = (int)A->levels.size();
    a.D = A->D;
    a.ratio = A->desc.ref_ratio;
    for (int l = 0; l < a.nl; ++l) {
        const bamrex_level* L = A->levels[l];
        a.scal[l] = L->d_scal;
        a.cfl[l] = L->cfl;
        for (int d = 0; d < 3; ++d) a.dx[l][d] = L->dx[d];
    }
    return a;
}

int coarse_step_graph(bamrex_amr* A, double stop_time, double time)
{
    cudaError_t e = cudaSuccess;
    if (!A->d_amr) {
        e = dev_alloc((void**)&A->d_amr, sizeof(AmrDev), A->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(A->d_amr, 0, sizeof(AmrDev), A->stream);
        if (e == cudaSuccess) e = pinned_small_alloc((void**)&A->h_amr, sizeof(AmrDev));
        if (e == cudaSuccess) e = pinned_small_alloc((void**)&A->h_up, 4 * sizeof(double));
        if (e != cudaSuccess) return amr_fail(A, BAMREX_ERR_CUDA, std::string("step block: ") + cudaGetErrorString(e));
    }
    // the estimates the host path reads (bamrex_level_est_time_step): the
    // max wave speed of every level whose fused value is stale
    {
        BX_PROFILE("amr_coarse_step:dt");
        for (bamrex_level* L : A->levels) {
            if (L->ws_valid) continue;
            e = cudaMemsetAsync(&L->d_scal->ws_bits, 0, sizeof(unsigned long long), L->stream);
            if (e == cudaSuccess)
                e = launch_max_wave_speed(L->D, L->fp32, L->d_fab[L->cur], L->d_pack, (int)L->boxes.size(), L->ncells,
                                          L->k, &L->d_scal->ws_bits, nullptr, L->stream);
            if (e != cudaSuccess) return amr_fail(A, BAMREX_ERR_CUDA, std::string("max wave speed: ") + cudaGetErrorString(e));
            L->launches++;
            L->ws_valid = true;
        }
        // {time, stop_time, dt0, status} of the step
        A->h_up[0] = time;
        A->h_up[1] = stop_time;
        A->h_up[2] = 0.0;
        A->h_up[3] = 0.0;
        e = cudaMemcpyAsync(A->d_amr, A->h_up, 4 * sizeof(double), cudaMemcpyHostToDevice, A->stream);
        if (e == cudaSuccess) e = launch_amr_dt(A->d_amr, levels_arg(A), A->stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(A->h_amr, A->d_amr, sizeof(AmrDev), cudaMemcpyDeviceToHost, A->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
        if (e != cudaSuccess) return amr_fail(A, BAMREX_ERR_CUDA, std::string("coarse time step: ") + cudaGetErrorString(e));
    }
    const AmrDev& h = *A->h_amr;
    if (h.status == BAMREX_ERR_ARG)
        return amr_fail(A, BAMREX_ERR_ARG, "a rigid-body interpolation stencil left the fab: raise ngrow");
    if (h.status == BAMREX_ERR_NOT_CONVERGED)
        return amr_fail(A, BAMREX_ERR_NOT_CONVERGED, "an exact Riemann solve at a rigid-body interface did not converge");
    if (h.status == BAMREX_ERR_TIMEOUT)
        return amr_fail(A, BAMREX_ERR_TIMEOUT, "a sweep gave up waiting for its staged input");
    if (h.status != 0 || !(h.dt0 > 0) || !std::isfinite(h.dt0))
        return amr_fail(A, BAMREX_ERR_NAN, "non-positive or non-finite coarse time step");
    A->dt_level.assign(A->levels.size(), 0.0);
    for (size_t l = 0; l < A->levels.size(); ++l) A->dt_level[l] = h.dt[l];
    A->have_dt = true;

    const std::vector<int> key = step_key(A);
    bamrex_amr::StepGraph* G = nullptr;
    for (auto& g : A->graphs)
        if (g.gen == A->generation && g.key == key) G = &g;
    if (!G) {
        BX_PROFILE("amr_coarse_step:capture");
        bamrex_amr::StepGraph g;
        g.gen = A->generation;
        g.key = key;
        cudaGraph_t gr = nullptr;
        e = cudaStreamBeginCapture(A->stream, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return amr_fail(A, BAMREX_ERR_CUDA, std::string("begin capture: ") + cudaGetErrorString(e));
        const int rc = time_step_dev(A, 0, 0);
        e = cudaStreamEndCapture(A->stream, &gr);
        if (rc != BAMREX_OK || e != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            set_step_key(A, key);
            if (rc != BAMREX_OK) return A->set_err(rc);
            return amr_fail(A, BAMREX_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(e));
        }
        g.post = step_key(A);
        size_t nn = 0;
        if (cudaGraphGetNodes(gr, nullptr, &nn) == cudaSuccess && nn) {
            std::vector<cudaGraphNode_t> nodes(nn);
            if (cudaGraphGetNodes(gr, nodes.data(), &nn) == cudaSuccess)
                for (size_t q = 0; q < nn; ++q) {
                    cudaGraphNodeType t;
                    if (cudaGraphNodeGetType(nodes[q], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) g.kernels++;
                }
        }
        e = cudaGraphInstantiate(&g.exec, gr, 0);
        cudaGraphDestroy(gr);
        if (e != cudaSuccess) {
            set_step_key(A, key);
            return amr_fail(A, BAMREX_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
        }
        A->graphs.push_back(std::move(g));
        G = &A->graphs.back();
        A->graph_captures++;
    }
    {
        BX_PROFILE("amr_coarse_step:replay");
        e = cudaGraphLaunch(G->exec, A->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(A->stream);
        if (e != cudaSuccess) return amr_fail(A, BAMREX_ERR_CUDA, std::string("coarse step graph: ") + cudaGetErrorString(e));
    }
    A->graph_replays++;
    set_step_key(A, G->post);
    host_step_times(A, 0, time);
    return BAMREX_OK;
}

}  // namespace

extern "C" int bamrex_amr_create(bamrex_amr** out, const bamrex_amr_desc* desc, void* stream)
{
    if (!out || !desc) return fail(BAMREX_ERR_ARG, "NULL argument");
    *out = nullptr;
    const int D = desc->base.spacedim;
    if (desc->max_level < 0 || desc->max_level >= BAMREX_MAX_LEVELS) return fail(BAMREX_ERR_ARG, "max_level out of range");
    if (desc->ref_ratio != 2 && desc->ref_ratio != 4) return fail(BAMREX_ERR_ARG, "ref_ratio must be 2 or 4");
    if (desc->max_level > 0) {
        if (desc->blocking_factor < 2 * desc->ref_ratio || desc->blocking_factor % (2 * desc->ref_ratio) != 0)
            return fail(BAMREX_ERR_ARG, "blocking_factor must be a multiple of 2 * ref_ratio");
        if (desc->max_grid_size < desc->blocking_factor || desc->max_grid_size % desc->blocking_factor != 0)
            return fail(BAMREX_ERR_ARG, "max_grid_size must be a multiple of blocking_factor");
    }
    std::unique_ptr<bamrex_amr> A(new (std::nothrow) bamrex_amr());
    if (!A) return fail(BAMREX_ERR_OOM, "host allocation failed");
    A->desc = *desc;
    A->D = D;
    if (stream) {
        A->stream = (cudaStream_t)stream;
    } else {
        BX_CK(cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking));
        A->own_stream = true;
    }
    bamrex_level* L0 = nullptr;
    const int rc = bamrex_level_create(&L0, &desc->base, A->stream);
    if (rc != BAMREX_OK) {
        if (A->own_stream) cudaStreamDestroy(A->stream);
        return rc;
    }
    A->levels.push_back(L0);
    A->cpl.push_back(nullptr);
    A->dt_level.push_back(0.0);
    *out = A.release();
    return BAMREX_OK;
}

extern "C" int bamrex_amr_destroy(bamrex_amr* A)
{
    if (!A) return BAMREX_OK;
    drop_step_graphs(A);
    if (A->d_amr) dev_free(A->d_amr, A->stream);
    pinned_small_free(A->h_amr);
    pinned_small_free(A->h_up);
    drop_levels_above(A, 0);
    if (!A->levels.empty()) bamrex_level_destroy(A->levels[0]);
    if (A->own_stream) cudaStreamDestroy(A->stream);
    delete A;
    return BAMREX_OK;
}

extern "C" const char* bamrex_amr_last_error(const bamrex_amr* A) { return A ? A->err.c_str() : ""; }

extern "C" int bamrex_amr_finest_level(const bamrex_amr* A) { return A ? (int)A->levels.size() - 1 : -1; }

extern "C" bamrex_level* bamrex_amr_level(bamrex_amr* A, int lev)
{
    if (!A || lev < 0 || lev >= (int)A->levels.size()) return nullptr;
    return A->levels[lev];
}

extern "C" int bamrex_amr_boxes(const bamrex_amr* A, int lev, bamrex_box* out, int max_out, int* nout)
{
    if (!A || !nout || lev < 0 || lev >= (int)A->levels.size()) return fail(BAMREX_ERR_ARG, "bad argument");
    const auto& b = A->levels[lev]->boxes;
    *nout = (int)b.size();
    if (!out) return BAMREX_OK;
    if ((int)b.size() > max_out) return fail(BAMREX_ERR_ARG, "output array too small");
    std::copy(b.begin(), b.end(), out);
    return BAMREX_OK;
}

extern "C" int bamrex_amr_set_level_boxes(bamrex_amr* A, int lev, const bamrex_box* boxes, int nboxes)
{
    if (!A || !boxes || nboxes < 1) return fail(BAMREX_ERR_ARG, "bad argument");
    std::vector<bamrex_box> b(boxes, boxes + nboxes);
    return set_level(A, lev, b);
}

extern "C" int bamrex_amr_regrid(bamrex_amr* A, int lbase, double time)
{
    if (!A || lbase < 0 || lbase >= (int)A->levels.size()) return fail(BAMREX_ERR_ARG, "bad argument");
    return regrid(A, lbase, time);
}

extern "C" int bamrex_amr_avg_down_all(bamrex_amr* A)
{
    if (!A) return fail(BAMREX_ERR_ARG, "NULL hierarchy");
    for (int l = (int)A->levels.size() - 1; l >= 1; --l) AMR_TRY(A, bamrex_coupling_avg_down(A->cpl[l]));
    return BAMREX_OK;
}

extern "C" int bamrex_amr_coarse_step(bamrex_amr* A, double stop_time, double* time_io, double* dt_out)
{
    if (!A || !time_io) return fail(BAMREX_ERR_ARG, "NULL argument");
    const double time = *time_io;
    bool regridded = false;
    if (A->steps > 0 && A->desc.regrid_int > 0 && A->desc.max_level > 0 && A->steps % A->desc.regrid_int == 0) {
        BX_TRY(regrid(A, 0, time));
        regridded = true;
    }
    BX_PROFILE("amr_coarse_step");
    // Graphs once the levels have taken a step as they are and will keep
    // them for a few steps (a graph captured for one replay costs more than
    // it saves); the first step after a regrid takes the host path, whose
    // dt rule also differs there.
    const bool graph = A->use_graph && !regridded && A->steps > 0 && A->have_dt && A->gen_steps > 0 &&
                       (A->desc.regrid_int <= 0 || A->desc.regrid_int >= 4 || A->desc.max_level == 0) &&
                       (int)A->levels.size() <= kAmrMaxLevels;
    if (graph) {
        BX_TRY(coarse_step_graph(A, stop_time, time));
        A->steps++;
        A->gen_steps++;
        *time_io = time + A->dt_level[0];
        if (dt_out) *dt_out = A->dt_level[0];
        return BAMREX_OK;
    }
    ProfPhases phase("amr_coarse_step:dt");
    BX_TRY(compute_dt(A, time, stop_time, A->steps == 0, regridded));
    if (!(A->dt_level[0] > 0) || !std::isfinite(A->dt_level[0]))
        return amr_fail(A, BAMREX_ERR_NAN, "non-positive or non-finite coarse time step");
    phase.next("amr_coarse_step:enqueue");
    BX_TRY(time_step(A, 0, time));
    phase.next("amr_coarse_step:sync");
    AMR_TRY(A, bamrex_level_sync(A->levels[0]));
    A->steps++;
    A->gen_steps++;
    *time_io = time + A->dt_level[0];
    if (dt_out) *dt_out = A->dt_level[0];
    return BAMREX_OK;
}

extern "C" int bamrex_amr_set_graph(bamrex_amr* A, int use_graph)
{
    if (!A) return fail(BAMREX_ERR_ARG, "NULL hierarchy");
    A->use_graph = use_graph != 0;
    if (!A->use_graph) drop_step_graphs(A);
    return BAMREX_OK;
}

extern "C" int bamrex_amr_graph_stats(const bamrex_amr* A, int* captures, long long* replays, long long* kernels)
{
    if (!A) return fail(BAMREX_ERR_ARG, "NULL hierarchy");
    if (captures) *captures = A->graph_captures;
    if (replays) *replays = A->graph_replays;
    if (kernels) {
        *kernels = 0;
        for (const auto& g : A->graphs)
            if (g.gen == A->generation) *kernels = std::max(*kernels, g.kernels);
    }
    return BAMREX_OK;
}

extern "C" int bamrex_amr_set_body(bamrex_amr* A, const bamrex_body_desc* desc)
{
    if (!A) return fail(BAMREX_ERR_ARG, "NULL hierarchy");
    drop_step_graphs(A);
    for (bamrex_level* L : A->levels) AMR_TRY(A, bamrex_level_set_body(L, desc));
    A->has_body = desc != nullptr;
    if (desc) A->body = *desc;
    return BAMREX_OK;
}

extern "C" int bamrex_amr_set_regrid_int(bamrex_amr* A, int regrid_int)
{
    if (!A || regrid_int < 0) return fail(BAMREX_ERR_ARG, "bad argument");
    A->desc.regrid_int = regrid_int;
    return BAMREX_OK;
}

extern "C" int bamrex_amr_dt_level(const bamrex_amr* A, double* dt_level)
{
    if (!A || !dt_level) return fail(BAMREX_ERR_ARG, "NULL argument");
    for (size_t l = 0; l < A->dt_level.size(); ++l) dt_level[l] = A->dt_level[l];
    return BAMREX_OK;
}

extern "C" int bamrex_amr_get_stepping(const bamrex_amr* A, bamrex_amr_stepping* out)
{
    if (!A || !out) return fail(BAMREX_ERR_ARG, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    out->coarse_steps = A->steps;
    out->have_dt = A->have_dt ? 1 : 0;
    out->nlevels = (int)std::min<size_t>(A->dt_level.size(), BAMREX_MAX_LEVELS);
    for (int l = 0; l < out->nlevels; ++l) out->dt_level[l] = A->dt_level[(size_t)l];
    return BAMREX_OK;
}

extern "C" int bamrex_amr_set_stepping(bamrex_amr* A, const bamrex_amr_stepping* in)
{
    if (!A || !in) return fail(BAMREX_ERR_ARG, "NULL argument");
    if (in->coarse_steps < 0 || in->nlevels < 0 || in->nlevels > BAMREX_MAX_LEVELS)
        return amr_fail(A, BAMREX_ERR_ARG, "stepping state out of range");
    A->steps = in->coarse_steps;
    A->have_dt = in->have_dt != 0;
    A->dt_level.assign(in->dt_level, in->dt_level + in->nlevels);
    return BAMREX_OK;
}

extern "C" int bamrex_amr_conserved_sums(bamrex_amr* A, double* totals)
{
    if (!A || !totals) return fail(BAMREX_ERR_ARG, "NULL argument");
    const int NC = A->D + 2;
    for (int m = 0; m < NC; ++m) totals[m] = 0.0;
    double s[BAMREX_MAX_NCOMP], c[BAMREX_MAX_NCOMP];
    for (int l = 0; l < (int)A->levels.size(); ++l) {
        AMR_TRY(A, bamrex_level_conserved_sums(A->levels[l], s));
        for (int m = 0; m < NC; ++m) c[m] = 0.0;
        if (l + 1 < (int)A->levels.size()) AMR_TRY(A, bamrex_coupling_covered_sums(A->cpl[l + 1], c));
        for (int m = 0; m < NC; ++m) totals[m] += s[m] - c[m];
    }
    return BAMREX_OK;
}
