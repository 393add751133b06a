// pinned.cpp -- page-locked host memory (see pinned.h).
#include "pinned.h"

#include <sys/mman.h>
#include <unistd.h>

#include <algorithm>
#include <mutex>
#include <unordered_map>

#include <omp.h>

namespace xpr {
namespace {

constexpr uint64_t kHugePage = 2ull << 20;

struct Mapping {
    void *base;
    uint64_t length;
};

std::mutex g_mu;
std::unordered_map<void *, Mapping> g_maps;  // registered pointer -> its mapping

uint64_t round_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

}  // namespace

cudaError_t pinned_alloc(void **ptr, uint64_t bytes)
{
    *ptr = nullptr;
    if (bytes < kPinnedMapThreshold) return cudaMallocHost(ptr, bytes ? bytes : 4);
    // one spare huge page so the buffer can start on a huge-page boundary
    const uint64_t size = round_up(bytes, kHugePage);
    const uint64_t length = size + kHugePage;
    void *base = mmap(nullptr, length, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (base == MAP_FAILED) return cudaMallocHost(ptr, bytes);
    char *p = reinterpret_cast<char *>(round_up(reinterpret_cast<uintptr_t>(base), kHugePage));
    madvise(p, size, MADV_HUGEPAGE);  // a request: without huge pages the path still works
    // fault every page in from several threads before the driver pins them
    const long page = std::max(4096L, sysconf(_SC_PAGESIZE));
    const int64_t pages = (int64_t)(size / (uint64_t)page);
    const int threads = std::max(1, std::min(16, omp_get_num_procs()));
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t i = 0; i < pages; ++i) reinterpret_cast<volatile char *>(p)[i * page] = 0;
    cudaError_t e = cudaHostRegister(p, size, cudaHostRegisterDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        munmap(base, length);
        return cudaMallocHost(ptr, bytes);
    }
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_maps[p] = Mapping{base, length};
    }
    *ptr = p;
    return cudaSuccess;
}

cudaError_t pinned_free(void *ptr)
{
    if (!ptr) return cudaSuccess;
    Mapping m{nullptr, 0};
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_maps.find(ptr);
        if (it != g_maps.end()) {
            m = it->second;
            g_maps.erase(it);
        }
    }
    if (!m.base) return cudaFreeHost(ptr);
    const cudaError_t e = cudaHostUnregister(ptr);
    munmap(m.base, m.length);
    return e;
}

}  // namespace xpr
