// pinned.h -- page-locked host memory for large staging buffers.
//
// cudaMallocHost page-locks memory one 4 KB page at a time in one thread, which
// for the volume-sized buffers of the streaming memory modes costs seconds (about
// 0.45 s per GB on a B200 host).  Large buffers are therefore mapped anonymously
// with transparent huge pages requested, faulted in by several threads (the
// kernel zeroes the pages, which is the bulk of the cost) and then registered with
// the driver; small ones still come from cudaMallocHost.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace xpr {

// Buffers at or above this size take the mapped path.
constexpr uint64_t kPinnedMapThreshold = 32ull << 20;

// Page-locked host memory of at least `bytes` bytes, zero-filled on the mapped path.
cudaError_t pinned_alloc(void **ptr, uint64_t bytes);
// Releases memory from pinned_alloc (either path); nullptr is ignored.
cudaError_t pinned_free(void *ptr);

}  // namespace xpr
