// Host buffers for results (svdb_rec u / s / vt on the host).
//
// Device-to-host copies into freshly malloc'd memory run at pageable speed
// and fault in every page on first touch: about 20 ms for the 52 MB of a
// 100,000 x 30,000 rank-50 randomized_svd result.  Buffers of 64 KB and more
// therefore come from page-locked memory that the library keeps for reuse:
// svdb_rec_free hands them back, a later result of a similar size takes them
// again, and svdb_release_cached_memory returns them to the driver.  Smaller
// buffers are plain malloc.
#include <cstdlib>
#include <map>
#include <mutex>
#include <unordered_map>

#include "svdb_internal.h"

namespace svdb {
namespace {

constexpr size_t kPinnedMin = 64 << 10;             // smaller results use malloc
constexpr size_t kPinnedGrain = 2 << 20;            // pinned sizes are rounded up to 2 MB
constexpr size_t kPinnedCacheMax = size_t(4) << 30;  // bytes kept for reuse

struct PinnedCache {
    std::mutex mu;
    std::unordered_map<void*, size_t> live;  // handed out: pointer -> capacity
    std::multimap<size_t, void*> idle;       // kept for reuse: capacity -> pointer
    size_t idle_bytes = 0;
};

PinnedCache& cache() {
    static PinnedCache* c = new PinnedCache();  // never destroyed: frees may come during exit
    return *c;
}

}  // namespace

void* host_result_alloc(size_t bytes) {
    if (bytes < kPinnedMin) {
        void* p = std::malloc(bytes ? bytes : 1);
        if (!p) throw std::bad_alloc();
        return p;
    }
    PinnedCache& c = cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.idle.lower_bound(bytes);
        if (it != c.idle.end() && it->first <= 2 * bytes + kPinnedGrain) {  // no more than about twice the size
            void* p = it->second;
            const size_t cap = it->first;
            c.idle.erase(it);
            c.idle_bytes -= cap;
            c.live[p] = cap;
            return p;
        }
    }
    const size_t cap = (bytes + kPinnedGrain - 1) / kPinnedGrain * kPinnedGrain;
    void* p = nullptr;
    if (cudaHostAlloc(&p, cap, cudaHostAllocPortable) != cudaSuccess || !p) {
        cudaGetLastError();  // fall back to pageable memory
        p = std::malloc(bytes);
        if (!p) throw std::bad_alloc();
        return p;
    }
    std::lock_guard<std::mutex> lk(c.mu);
    c.live[p] = cap;
    return p;
}

void host_result_free(void* p) {
    if (!p) return;
    PinnedCache& c = cache();
    std::unique_lock<std::mutex> lk(c.mu);
    auto it = c.live.find(p);
    if (it == c.live.end()) {
        lk.unlock();
        std::free(p);
        return;
    }
    const size_t cap = it->second;
    c.live.erase(it);
    if (c.idle_bytes + cap <= kPinnedCacheMax) {
        c.idle.emplace(cap, p);
        c.idle_bytes += cap;
        return;
    }
    lk.unlock();
    cudaFreeHost(p);
}

void host_result_release() {
    PinnedCache& c = cache();
    std::multimap<size_t, void*> idle;
    {
        std::lock_guard<std::mutex> lk(c.mu);
        idle.swap(c.idle);
        c.idle_bytes = 0;
    }
    for (auto& kv : idle) cudaFreeHost(kv.second);
}

}  // namespace svdb
