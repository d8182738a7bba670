// Pooled device blocks and small pinned blocks (declarations and rationale
// in devmem.h).
#include "devmem.h"

#include <chrono>
#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "profiler.h"

namespace bamrex {
namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kPinnedBlock = 4096;
constexpr size_t kPinnedSlab = 64 * kPinnedBlock;

// Blocks of kCacheMin bytes and more keep their pages and addresses after
// dev_free: up to kCacheBlocks per device wait here, whole, for a request
// of their size class or a little below (kCacheSlack).  Handing a large
// range back to the pool and taking it out again costs the pool about as
// much as mapping it afresh (a third of a second for a 10 GB level arena,
// measured), where reusing a kept block costs nothing.
constexpr size_t kCacheMin = size_t(64) << 20;
constexpr int kCacheBlocks = 16;
constexpr size_t kCacheSlack = 4;  // a kept block serves requests down to 3/4 of its size

struct Block {
    int dev = -1;
    size_t bytes = 0;
};

struct Kept {
    void* p;
    size_t bytes;
    unsigned long long stamp;  // order of keeping: the oldest goes first
};

struct Pools {
    std::mutex mu;
    cudaMemPool_t pool[kMaxDevices] = {};
    long long live[kMaxDevices] = {};
    std::unordered_map<void*, Block> owner;  // block -> device and size
    std::vector<Kept> kept[kMaxDevices];
    unsigned long long stamp = 0;
    std::vector<void*> pinned_free;
};

Pools& pools()
{
    static Pools* P = new Pools();  // never destroyed: blocks may outlive static destruction order
    return *P;
}

cudaError_t device_pool(Pools& P, int dev, cudaMemPool_t* out)
{
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    if (!P.pool[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        P.pool[dev] = pool;
    }
    *out = P.pool[dev];
    return cudaSuccess;
}

// Requests of 64 MiB and more are rounded up to a size class (eight per
// doubling, at most 12.5% more): a level that grows a little at every
// regrid then fits the block its predecessor freed, where an exact size
// would make the pool map fresh pages (about a second for a 10 GB arena).
size_t size_class(size_t bytes)
{
    constexpr size_t kMin = size_t(64) << 20;
    if (bytes < kMin) return bytes;
    int e = 63;
    while (!(bytes >> e)) --e;  // 2^e <= bytes < 2^(e+1)
    const size_t step = size_t(1) << (e - 3);
    return (bytes + step - 1) / step * step;
}

// Kept blocks of device `dev` back to its pool (they are idle: dev_free
// synchronised the device before keeping them); called with P.mu held.
void release_kept(Pools& P, int dev)
{
    if (P.kept[dev].empty()) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    for (const Kept& k : P.kept[dev]) cudaFreeAsync(k.p, 0);
    P.kept[dev].clear();
    cudaStreamSynchronize(0);
    if (cur != dev && cur >= 0) cudaSetDevice(cur);
}

}  // namespace

cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t s)
{
    // a kept block is looked for at the request's size class; a large block
    // taken from the pool is made one eighth larger, so that the kept block
    // of a level that grows a little at every regrid still fits the level
    // two regrids on
    bytes = size_class(bytes);
    const size_t alloc = bytes >= kCacheMin ? size_class(bytes + bytes / 8) : bytes;
    *p = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    Pools& P = pools();
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> g(P.mu);
        e = device_pool(P, dev, &pool);
        if (e != cudaSuccess) return e;
        if (bytes >= kCacheMin) {
            // the smallest kept block that fits and is not much larger
            std::vector<Kept>& K = P.kept[dev];
            int best = -1;
            for (int i = 0; i < (int)K.size(); ++i)
                if (K[i].bytes >= bytes && K[i].bytes - K[i].bytes / kCacheSlack <= bytes &&
                    (best < 0 || K[i].bytes < K[best].bytes))
                    best = i;
            if (best >= 0) {
                BX_PROFILE("dev_alloc:kept");
                *p = K[best].p;
                P.owner[*p] = Block{ dev, K[best].bytes };
                K.erase(K.begin() + best);
                ++P.live[dev];
                return cudaSuccess;
            }
        }
    }
    // profiled: whether the pool had to map pages for the block (grow) or
    // handed out pages it kept (reuse), and the wait for the stream
    const bool prof = g_profile_on.load(std::memory_order_relaxed) != 0;
    uint64_t res0 = 0, res1 = 0;
    std::chrono::steady_clock::time_point t0;
    if (prof) {
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &res0);
        t0 = std::chrono::steady_clock::now();
    }
    size_t got = alloc ? alloc : 1;
    e = cudaMallocFromPoolAsync(p, got, pool, s);
    if (e == cudaErrorMemoryAllocation) {
        // the kept blocks' pages may be what is missing: give them to the
        // pool and try once more, then without the extra eighth
        cudaGetLastError();
        bool had = false;
        {
            std::lock_guard<std::mutex> g(P.mu);
            had = !P.kept[dev].empty();
            release_kept(P, dev);
        }
        if (had) e = cudaMallocFromPoolAsync(p, got, pool, s);
        if (e == cudaErrorMemoryAllocation && alloc > bytes) {
            cudaGetLastError();
            got = bytes ? bytes : 1;
            e = cudaMallocFromPoolAsync(p, got, pool, s);
        }
    }
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
    }
    if (prof) {
        const auto t1 = std::chrono::steady_clock::now();
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &res1);
        profile_record(res1 > res0 ? "dev_alloc:pool_grow" : "dev_alloc:pool_reuse",
                       std::chrono::duration<double>(t1 - t0).count());
    }
    // the tables are uploaded with copies outside `s`: the block must be
    // ready for every stream when this returns
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFreeAsync(*p, s);
        *p = nullptr;
        return e;
    }
    std::lock_guard<std::mutex> g(P.mu);
    P.owner[*p] = Block{ dev, got };
    ++P.live[dev];
    return cudaSuccess;
}

void dev_free(void* p, cudaStream_t s)
{
    if (!p) return;
    Pools& P = pools();
    Block b;
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.owner.find(p);
        if (it != P.owner.end()) {
            b = it->second;
            P.owner.erase(it);
        }
    }
    if (b.dev < 0) return;  // not a pooled block
    // as cudaFree: every stream's work on the block (table uploads and
    // memsets on the default stream, copies on helper streams) is finished
    // before the block can be handed out again or its pages released
    cudaDeviceSynchronize();
    std::lock_guard<std::mutex> g(P.mu);
    --P.live[b.dev];
    if (b.bytes >= kCacheMin) {
        std::vector<Kept>& K = P.kept[b.dev];
        K.push_back(Kept{ p, b.bytes, ++P.stamp });
        if ((int)K.size() > kCacheBlocks) {
            // the block kept longest goes back to the pool
            int old = 0;
            for (int i = 1; i < (int)K.size(); ++i)
                if (K[i].stamp < K[old].stamp) old = i;
            cudaFreeAsync(K[old].p, s);
            K.erase(K.begin() + old);
        }
        return;
    }
    cudaFreeAsync(p, s);
}

namespace {

struct Stage {
    std::mutex mu;
    char* p = nullptr;
    size_t cap = 0;
};

Stage& stage()
{
    static Stage* S = new Stage();  // never destroyed, as the pools
    return *S;
}

}  // namespace

PinnedStage::PinnedStage(size_t bytes) : lock_(stage().mu)
{
    Stage& S = stage();
    if (bytes == 0) return;
    if (S.cap < bytes) {
        if (S.p) cudaFreeHost(S.p);
        S.p = nullptr;
        S.cap = 0;
        const size_t want = bytes + bytes / 4;  // room for a level that grows
        if (cudaMallocHost((void**)&S.p, want) == cudaSuccess) {
            S.cap = want;
        } else {
            cudaGetLastError();
            S.p = nullptr;
        }
    }
    p_ = S.p;
}

int release_pooled()
{
    {
        // the staging buffer first, under its own lock only (a holder of
        // the stage may take the pools' lock, never the other way round)
        Stage& S = stage();
        std::lock_guard<std::mutex> sg(S.mu);
        if (S.p) cudaFreeHost(S.p);
        S.p = nullptr;
        S.cap = 0;
    }
    Pools& P = pools();
    std::lock_guard<std::mutex> g(P.mu);
    cudaError_t e = cudaDeviceSynchronize();
    for (int d = 0; d < kMaxDevices && e == cudaSuccess; ++d) {
        if (!P.pool[d]) continue;
        release_kept(P, d);
        e = cudaMemPoolTrimTo(P.pool[d], 0);
    }
    return e == cudaSuccess ? 0 : (int)e;
}

cudaError_t pinned_small_alloc(void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes > kPinnedBlock) return cudaErrorInvalidValue;
    Pools& P = pools();
    std::lock_guard<std::mutex> g(P.mu);
    if (P.pinned_free.empty()) {
        char* slab = nullptr;
        const cudaError_t e = cudaMallocHost((void**)&slab, kPinnedSlab);
        if (e != cudaSuccess) return e;
        for (size_t o = kPinnedSlab; o > 0; o -= kPinnedBlock) P.pinned_free.push_back(slab + o - kPinnedBlock);
    }
    *p = P.pinned_free.back();
    P.pinned_free.pop_back();
    return cudaSuccess;
}

void pinned_small_free(void* p)
{
    if (!p) return;
    Pools& P = pools();
    std::lock_guard<std::mutex> g(P.mu);
    P.pinned_free.push_back(p);
}

}  // namespace bamrex
