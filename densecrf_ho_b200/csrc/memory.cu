// Device memory for DevBuf: a process-wide cache of freed blocks.
//
// Building a model or a lattice allocates some twenty buffers, and a model's
// destruction frees them; cudaMalloc and cudaFree cost tens to hundreds of
// microseconds each (cudaFree also waits for the device).  Blocks are sized
// in classes (powers of two split in quarters, 512 bytes at least), and a
// released block is kept, per device, for the next request of its class, so
// a process that builds one model per image pays for the allocations once.
// A released block first goes to a pending list, without waiting; before a
// pending block is handed out again, its device is synchronised once (as
// cudaFree would wait) and every pending block of that device moves to the
// cache: a block is never reused while a kernel may still read it, and a
// burst of releases (a batch rebuilding its lattices) costs one wait, not one
// per buffer.
#include <algorithm>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace dcrf {
namespace {

struct Block {
    void* p;
    size_t bytes;
    int dev;
};

std::mutex g_mu;
size_t g_live = 0;         // bytes handed out and not yet released (every device)
size_t g_limit = 0;        // cap on g_live; 0 = none (dcrf_set_device_memory_limit)
unsigned long long g_mallocs = 0;  // cudaMalloc calls that succeeded
std::vector<Block>& cache() {
    static auto* c = new std::vector<Block>();  // never destroyed: the process exit frees the memory
    return *c;
}
size_t g_cached = 0;
std::vector<Block>& pending() {
    static auto* c = new std::vector<Block>();  // released, not yet known to be idle
    return *c;
}
size_t g_pending = 0;

// Bytes of released blocks kept for reuse: DCRF_CACHE_MB, else a quarter of
// the (first) device's memory, at least 2 GiB.  A batch that releases and
// rebuilds its lattices between passes (mean-field with lattice recompute)
// then reuses its blocks instead of going back to cudaMalloc each time.
size_t cache_cap() {
    static const size_t cap = [] {
        const char* v = std::getenv("DCRF_CACHE_MB");
        if (v) return (size_t)std::strtoull(v, nullptr, 10) << 20;
        size_t fr = 0, total = 0;
        if (cudaMemGetInfo(&fr, &total) != cudaSuccess) {
            cudaGetLastError();
            total = 0;
        }
        return std::max((size_t)2048 << 20, total / 4);
    }();
    return cap;
}

size_t size_class(size_t b) {
    if (b <= 512) return 512;
    size_t p = 512;
    while (p < b) p <<= 1;
    const size_t q = p >> 2;  // quarters of the next power of two
    return ((b + q - 1) / q) * q;
}

}  // namespace

std::recursive_mutex& capture_mutex() {
    static auto* m = new std::recursive_mutex();  // never destroyed
    return *m;
}

// Waits for device `dev` once and moves its pending blocks to the cache
// (freeing them instead when the wait fails or the cache is full).  Caller
// holds the capture mutex, not g_mu.
void flush_pending(int dev) noexcept {
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (dev != cur) cudaSetDevice(dev);
    const bool ok = cudaDeviceSynchronize() == cudaSuccess;
    if (!ok) cudaGetLastError();
    std::vector<void*> drop;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto& pd = pending();
        for (size_t i = pd.size(); i-- > 0;)
            if (pd[i].dev == dev) {
                g_pending -= pd[i].bytes;
                if (ok && g_cached + pd[i].bytes <= cache_cap()) {
                    cache().push_back(pd[i]);
                    g_cached += pd[i].bytes;
                } else {
                    drop.push_back(pd[i].p);  // a broken context (no reuse), or no room
                }
                pd[i] = pd.back();
                pd.pop_back();
            }
    }
    for (void* q : drop) cudaFree(q);
    if (dev != cur) cudaSetDevice(cur);
}

void* dev_alloc(size_t bytes, size_t* got) {
    const size_t b = size_class(bytes);
    int dev = 0;
    DCRF_CUDA(cudaGetDevice(&dev));
    {
        std::lock_guard<std::mutex> lk(g_mu);
        // A caller-set budget: refused on the host, before any device call.
        if (g_limit && g_live + b > g_limit)
            throw Error(DCRF_E_NOMEM, "device memory limit of " + std::to_string(g_limit) + " bytes reached (" +
                                          std::to_string(g_live) + " in use, " + std::to_string(b) + " requested)");
        g_live += b;
        auto& c = cache();
        for (size_t i = c.size(); i-- > 0;)
            if (c[i].dev == dev && c[i].bytes == b) {
                void* p = c[i].p;
                c[i] = c.back();
                c.pop_back();
                g_cached -= b;
                *got = b;
                return p;
            }
    }
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    bool in_pending = false;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (const Block& q : pending())
            if (q.dev == dev && q.bytes == b) {
                in_pending = true;
                break;
            }
    }
    if (in_pending) {  // one wait makes every pending block of the device reusable
        flush_pending(dev);
        std::lock_guard<std::mutex> lk(g_mu);
        auto& c = cache();
        for (size_t i = c.size(); i-- > 0;)
            if (c[i].dev == dev && c[i].bytes == b) {
                void* p = c[i].p;
                c[i] = c.back();
                c.pop_back();
                g_cached -= b;
                *got = b;
                return p;
            }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaErrorMemoryAllocation) {  // give the cached blocks back and try once more
        cudaGetLastError();
        dev_trim(false);
        e = cudaMalloc(&p, b);
    }
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_live -= b;
    }
    DCRF_CUDA(e);
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_mallocs++;
    }
    *got = b;
    return p;
}

void set_device_memory_limit(size_t bytes) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_limit = bytes;
}

void device_memory_stats(size_t* live, size_t* cached, unsigned long long* mallocs) {
    std::lock_guard<std::mutex> lk(g_mu);
    *live = g_live;
    *cached = g_cached + g_pending;  // held for reuse, whether or not yet known to be idle
    *mallocs = g_mallocs;
}

void dev_release(void* p, size_t bytes) noexcept {
    if (!p) return;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_live -= bytes;
    }
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    // the block's own device (the caller's current device may be another)
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return;
    }
    bool over = false;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        pending().push_back(Block{p, bytes, a.device});
        g_pending += bytes;
        over = g_cached + g_pending > cache_cap();
    }
    if (over) flush_pending(a.device);  // keeps what fits, frees the rest
}

void dev_trim(bool all_devices) noexcept {
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    {
        std::vector<int> devs;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            for (const Block& q : pending())
                if ((all_devices || q.dev == dev) &&
                    std::find(devs.begin(), devs.end(), q.dev) == devs.end())
                    devs.push_back(q.dev);
        }
        for (int dv : devs) flush_pending(dv);
    }
    std::vector<void*> drop;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto& c = cache();
        for (size_t i = c.size(); i-- > 0;)
            if (all_devices || c[i].dev == dev) {
                drop.push_back(c[i].p);
                g_cached -= c[i].bytes;
                c[i] = c.back();
                c.pop_back();
            }
    }
    for (void* p : drop) cudaFree(p);
}

}  // namespace dcrf
