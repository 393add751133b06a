// hostcopy.h -- host memory copies split over a few threads: one thread copies at well
// under the host memory bandwidth, which would otherwise bound the transfers between
// caller memory and page-locked staging.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstring>

namespace xpr {

inline void par_memcpy(void *dst, const void *src, size_t n)
{
    constexpr size_t kTask = 4u << 20;
    const int64_t tasks = (int64_t)((n + kTask - 1) / kTask);
#pragma omp parallel for schedule(static) num_threads(8) if (tasks > 1)
    for (int64_t t = 0; t < tasks; ++t) {
        const size_t o = (size_t)t * kTask;
        std::memcpy((char *)dst + o, (const char *)src + o, std::min(kTask, n - o));
    }
}

}  // namespace xpr
