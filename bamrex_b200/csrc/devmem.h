// Device and pinned memory for the tables and states that levels, halo
// plans and AMR couplings own.
//
// A regrid frees one level and its coupling and makes the next one of about
// the same size. Plain cudaMalloc/cudaFree there maps and unmaps pages in the
// driver on every call (and cudaFree synchronises the device), which costs
// from a millisecond to, on a loaded host, hundreds. These helpers take the
// blocks from a stream-ordered pool per device that keeps freed blocks
// (release threshold = unlimited), so the next level reuses the same pages,
// also across hierarchies created one after the other.  Freed blocks of
// 64 MiB and more are kept whole (a few per device) and handed out again
// as they are, which spares the pool re-dealing a large range.  The pages
// go back to the driver at process exit or when release_pooled() is called.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>

namespace bamrex {

// A block of `bytes` on the current device, ordered after the work already
// queued on `s` and usable from every stream when the call returns.
cudaError_t dev_alloc(void** p, size_t bytes, cudaStream_t s);

// Give a block back (after a device-wide synchronisation, as cudaFree).
void dev_free(void* p, cudaStream_t s);

// Hand every page the pools keep but no block uses back to the driver
// (0 or a cudaError_t).
int release_pooled();

// The process's pinned host staging buffer, at least `bytes` long, held with
// its lock while the object lives: large table uploads are written there by
// host threads and copied to the device in one DMA each, instead of going
// through the driver's pageable path.  Grows (never shrinks) on demand;
// data() is null if pinned memory could not be had.  The holder must let
// its copies out of the buffer finish before the object goes.
class PinnedStage {
public:
    explicit PinnedStage(size_t bytes);
    char* data() const { return p_; }
    PinnedStage(const PinnedStage&) = delete;
    PinnedStage& operator=(const PinnedStage&) = delete;

private:
    std::unique_lock<std::mutex> lock_;
    char* p_ = nullptr;
};

// Small pinned host blocks (up to 4 KB) for the scalars a step reads back,
// cut from pinned slabs that are kept for the life of the process.
cudaError_t pinned_small_alloc(void** p, size_t bytes);
void pinned_small_free(void* p);

}  // namespace bamrex
