// Pooled device blocks and small pinned blocks (declarations and rationale
// in devmem.h).
#include "devmem.h"

#include <cstdint>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace bamrex {
namespace {

constexpr int kMaxDevices = 64;
constexpr size_t kPinnedBlock = 4096;
constexpr size_t kPinnedSlab = 64 * kPinnedBlock;

struct Pools {
    std::mutex mu;
    cudaMemPool_t pool[kMaxDevices] = {};
    long long live[kMaxDevices] = {};
    std::unordered_map<void*, int> owner;  // block -> device
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

}  // namespace

cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t s)
{
    bytes = size_class(bytes);
    *p = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    Pools& P = pools();
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> g(P.mu);
        e = device_pool(P, dev, &pool);
    }
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync(p, bytes ? bytes : 1, pool, s);
    if (e != cudaSuccess) {
        *p = nullptr;
        return e;
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
    P.owner[*p] = dev;
    ++P.live[dev];
    return cudaSuccess;
}

void dev_free(void* p, cudaStream_t s)
{
    if (!p) return;
    Pools& P = pools();
    int dev = -1;
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.owner.find(p);
        if (it != P.owner.end()) {
            dev = it->second;
            P.owner.erase(it);
        }
    }
    if (dev < 0) return;  // not a pooled block
    // as cudaFree: every stream's work on the block (table uploads and
    // memsets on the default stream, copies on helper streams) is finished
    // before the block can be handed out again or its pages released
    cudaDeviceSynchronize();
    cudaFreeAsync(p, s);
    std::lock_guard<std::mutex> g(P.mu);
    --P.live[dev];
}

int release_pooled()
{
    Pools& P = pools();
    std::lock_guard<std::mutex> g(P.mu);
    cudaError_t e = cudaDeviceSynchronize();
    for (int d = 0; d < kMaxDevices && e == cudaSuccess; ++d)
        if (P.pool[d]) e = cudaMemPoolTrimTo(P.pool[d], 0);
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
