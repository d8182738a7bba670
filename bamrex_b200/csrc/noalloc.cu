// bamrex_conserved_sums_noalloc: conserved totals of caller-owned fabs
// without any device allocation.
//
// Some callers cannot let a library allocate device memory on their behalf.
// A host code built on an AMReX-style arena hands most of the GPU to its own
// pool at start-up, so a cudaMalloc from inside a library call can fail or
// fragment memory the pool expects to own; a checker run in an error or
// shutdown path may no longer trust the allocator at all.  This entry point
// therefore keeps all of its scratch (the box table, per-box partial sums,
// the totals and a completion counter) in one file-scope device array of
// fixed size, reached through cudaGetSymbolAddress.
//
// Limits: at most kMaxBoxes boxes and BAMREX_MAX_NCOMP components per call.
// The scratch is shared by every call on a device: calls that overlap in
// time (different streams or host threads) race on it and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "bamrex_cuda.h"
#include "level_impl.h"

namespace {

constexpr int kMaxBoxes = 4096;
constexpr int kMaxComp = BAMREX_MAX_NCOMP;
constexpr int kThreads = 256;

struct NaBox {
    const double* p;
    long long js, ks, ns;
    int begin[3];
    int lo[3], hi[3];
};

// Scratch layout (bytes, each part 256-byte aligned).
constexpr size_t align256(size_t v) { return (v + 255) / 256 * 256; }
constexpr size_t kOffBoxes = 0;
constexpr size_t kOffPartial = kOffBoxes + align256(sizeof(NaBox) * kMaxBoxes);
constexpr size_t kOffTotal = kOffPartial + align256(sizeof(double) * kMaxBoxes * kMaxComp);
constexpr size_t kOffCounter = kOffTotal + align256(sizeof(double) * kMaxComp);
constexpr size_t kScratchBytes = kOffCounter + 256;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// One block per box: the per-box sum of every component over the valid
// cells in the same order as the level's conserved-sums reduction (strided
// accumulation per thread, then a fixed-shape tree), then the last block to
// finish adds the partials box by box and scales by the cell volume.
__global__ void __launch_bounds__(kThreads) sums_noalloc_kernel(int NC, int nboxes, double vol,
                                                                unsigned char* __restrict__ scratch)
{
    __shared__ double red[kThreads];
    __shared__ bool last;
    const NaBox* boxes = reinterpret_cast<const NaBox*>(scratch + kOffBoxes);
    double* partial = reinterpret_cast<double*>(scratch + kOffPartial);
    double* total = reinterpret_cast<double*>(scratch + kOffTotal);
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kOffCounter);

    const int b = blockIdx.x;
    const NaBox B = boxes[b];
    const int nx = B.hi[0] - B.lo[0] + 1, ny = B.hi[1] - B.lo[1] + 1, nz = B.hi[2] - B.lo[2] + 1;
    const long long ncell = (long long)nx * ny * nz;
    for (int n = 0; n < NC; ++n) {
        double acc = 0.0;
        for (long long c = threadIdx.x; c < ncell; c += blockDim.x) {
            const int i = B.lo[0] + (int)(c % nx);
            const int j = B.lo[1] + (int)((c / nx) % ny);
            const int k = B.lo[2] + (int)(c / ((long long)nx * ny));
            acc += B.p[(long long)(i - B.begin[0]) + (long long)(j - B.begin[1]) * B.js +
                       (long long)(k - B.begin[2]) * B.ks + n * B.ns];
        }
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[(long long)b * NC + n] = red[0];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(counter, 1u) == (unsigned int)(nboxes - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        for (int n = 0; n < NC; ++n) {
            double s = 0.0;
            for (int q = 0; q < nboxes; ++q) s += ((volatile double*)partial)[(long long)q * NC + n];
            total[n] = s * vol;
        }
    }
}

std::mutex g_mu;
void* g_addr[64] = {};

// The scratch address on the current device, looked up once per device and
// kept for the life of the process.  A cudaDeviceReset unloads the module,
// after which the array may sit elsewhere: the entry point's documentation
// rules out calls after a reset of the device.
int scratch_address(unsigned char** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return bamrex::cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= 64) return bamrex::fail(BAMREX_ERR_UNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return bamrex::cuda_fail(e, "cudaGetSymbolAddress of the static scratch");
        g_addr[dev] = p;
    }
    *out = static_cast<unsigned char*>(g_addr[dev]);
    return BAMREX_OK;
}

}  // namespace

extern "C" int bamrex_conserved_sums_noalloc(int spacedim, const bamrex_box* boxes, const bamrex_array4* fabs,
                                             int nboxes, const double dx[3], double* totals, void* stream)
{
    if (spacedim < 1 || spacedim > 3) return bamrex::fail(BAMREX_ERR_ARG, "spacedim must be 1, 2 or 3");
    if (!boxes || !fabs || !dx || !totals) return bamrex::fail(BAMREX_ERR_ARG, "NULL argument");
    if (nboxes < 1 || nboxes > kMaxBoxes)
        return bamrex::fail(BAMREX_ERR_ARG, "nboxes must be in [1, " + std::to_string(kMaxBoxes) +
                                                "]: bamrex_conserved_sums_noalloc has a fixed scratch of that many boxes");
    const int NC = spacedim + 2;
    std::vector<NaBox> tab((size_t)nboxes);
    for (int b = 0; b < nboxes; ++b) {
        const bamrex_box& B = boxes[b];
        const bamrex_array4& a = fabs[b];
        for (int d = 0; d < 3; ++d) {
            if (B.hi[d] < B.lo[d] || (d >= spacedim && (B.lo[d] != 0 || B.hi[d] != 0)))
                return bamrex::fail(BAMREX_ERR_ARG, "invalid box " + std::to_string(b));
            if (a.begin[d] > B.lo[d] || a.end[d] <= B.hi[d])
                return bamrex::fail(BAMREX_ERR_ARG, "fab " + std::to_string(b) + " does not cover its box");
        }
        if (!a.p || a.ncomp < NC) return bamrex::fail(BAMREX_ERR_ARG, "fab " + std::to_string(b) + " has too few components");
        NaBox& t = tab[(size_t)b];
        t.p = a.p;
        t.js = a.jstride;
        t.ks = a.kstride;
        t.ns = a.nstride;
        for (int d = 0; d < 3; ++d) {
            t.begin[d] = a.begin[d];
            t.lo[d] = B.lo[d];
            t.hi[d] = B.hi[d];
        }
    }
    unsigned char* scratch = nullptr;
    const int rc = scratch_address(&scratch);
    if (rc != BAMREX_OK) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double vol = 1.0;
    for (int d = 0; d < spacedim; ++d) vol *= dx[d];
    // the completion counter must start at zero
    cudaError_t e = cudaMemsetAsync(scratch + kOffCounter, 0, sizeof(unsigned int), s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scratch + kOffBoxes, tab.data(), sizeof(NaBox) * tab.size(), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return bamrex::cuda_fail(e, "scratch set-up");
    sums_noalloc_kernel<<<nboxes, kThreads, 0, s>>>(NC, nboxes, vol, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return bamrex::cuda_fail(e, "conserved sums kernel");
    e = cudaMemcpyAsync(totals, scratch + kOffTotal, sizeof(double) * NC, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bamrex::cuda_fail(e, "conserved sums readback");
    return BAMREX_OK;
}
