// Host-side memory pool and thread helper (declared in internal.h).
#include "internal.h"

#include <algorithm>
#include <cstdlib>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <set>
#include <thread>

namespace ommgpu {

namespace {

constexpr size_t kPoolMin = size_t(1) << 20;   // smaller blocks are not cached
constexpr size_t kPoolCap = size_t(4) << 30;   // bytes kept in the pool at most
constexpr size_t kPinMin = size_t(16) << 20;   // blocks from this size up are page-locked

struct HostPool {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks;     // cached blocks by size
    std::deque<std::pair<void*, size_t>> order;  // the same blocks, oldest first
    std::set<void*> pinned;                       // blocks registered with the CUDA driver
    size_t cached = 0;
};
// never destroyed: vectors of static objects may hand their blocks back during exit
HostPool& pool() {
    static HostPool* p = new HostPool;
    return *p;
}

// A large block is page-locked once, when it is first allocated (the pool hands it out again
// and again), so that the uploads of CSC arrays and column-group blocks made from it run as
// direct DMA transfers.  Only once the library runtime is bound to a device (so that pinning
// never creates a CUDA context on a device the caller has not chosen); before that, without a
// GPU, or when the driver declines, the block stays pageable.
void* new_block(size_t bytes, HostPool& P) {
    if (bytes >= kPinMin && runtime_bound()) {
        const size_t rounded = (bytes + 4095) / 4096 * 4096;
        void* p = std::aligned_alloc(4096, rounded);
        if (!p) throw std::bad_alloc();
        if (cudaHostRegister(p, rounded, cudaHostRegisterPortable) == cudaSuccess) {
            std::lock_guard<std::mutex> lk(P.mu);
            P.pinned.insert(p);
        } else {
            cudaGetLastError();
        }
        return p;
    }
    void* p = std::malloc(bytes);
    if (!p) throw std::bad_alloc();
    return p;
}

void free_block(void* p, HostPool& P) {
    bool pinned = false;
    {
        std::lock_guard<std::mutex> lk(P.mu);
        pinned = P.pinned.erase(p) > 0;
    }
    if (pinned && cudaHostUnregister(p) != cudaSuccess) cudaGetLastError();
    std::free(p);
}

}  // namespace

void* host_pool_get(size_t bytes) {
    bytes = std::max<size_t>(bytes, 1);
    if (bytes >= kPoolMin) {
        HostPool& P = pool();
        std::lock_guard<std::mutex> lk(P.mu);
        auto it = P.free_blocks.find(bytes);
        if (it != P.free_blocks.end()) {
            void* p = it->second;
            P.free_blocks.erase(it);
            for (auto o = P.order.begin(); o != P.order.end(); ++o)
                if (o->first == p) {
                    P.order.erase(o);
                    break;
                }
            P.cached -= bytes;
            return p;
        }
    }
    return new_block(bytes, pool());
}

void host_pool_put(void* p, size_t bytes) {
    if (!p) return;
    bytes = std::max<size_t>(bytes, 1);
    if (bytes < kPoolMin || bytes > kPoolCap) {
        free_block(p, pool());
        return;
    }
    HostPool& P = pool();
    std::vector<void*> drop;
    {
        std::lock_guard<std::mutex> lk(P.mu);
        P.free_blocks.emplace(bytes, p);
        P.order.emplace_back(p, bytes);
        P.cached += bytes;
        while (P.cached > kPoolCap && !P.order.empty()) {
            auto [q, b] = P.order.front();
            P.order.pop_front();
            auto range = P.free_blocks.equal_range(b);
            for (auto it = range.first; it != range.second; ++it)
                if (it->second == q) {
                    P.free_blocks.erase(it);
                    break;
                }
            P.cached -= b;
            drop.push_back(q);
        }
    }
    for (void* q : drop) free_block(q, P);
}

void host_pool_release() {
    HostPool& P = pool();
    std::vector<void*> drop;
    {
        std::lock_guard<std::mutex> lk(P.mu);
        for (auto& kv : P.free_blocks) drop.push_back(kv.second);
        P.free_blocks.clear();
        P.order.clear();
        P.cached = 0;
    }
    for (void* q : drop) free_block(q, P);
}

size_t host_pool_cached_bytes() {
    HostPool& P = pool();
    std::lock_guard<std::mutex> lk(P.mu);
    return P.cached;
}

void host_parallel(long long count, const std::function<void(long long, long long)>& f) {
    long long nt = (long long)std::min<unsigned>(16u, std::max(1u, std::thread::hardware_concurrency()));
    nt = std::max<long long>(1, std::min<long long>(nt, count / 64));
    if (nt <= 1) {
        f(0, count);
        return;
    }
    std::vector<std::thread> th;
    th.reserve((size_t)nt - 1);
    for (long long t = 1; t < nt; ++t) th.emplace_back(f, count * t / nt, count * (t + 1) / nt);
    f(0, count / nt);
    for (auto& x : th) x.join();
}

}  // namespace ommgpu
