// Device memory for DevBuf: a process-wide cache of freed blocks.
//
// Building a model or a lattice allocates some twenty buffers, and a model's
// destruction frees them; cudaMalloc and cudaFree cost tens to hundreds of
// microseconds each (cudaFree also waits for the device).  Blocks are sized
// in classes (powers of two split in quarters, 512 bytes at least), and a
// released block is kept, per device, for the next request of its class, so
// a process that builds one model per image pays for the allocations once.
// A release waits for the device first, as cudaFree would: a cached block is
// never handed out while a kernel may still read it.
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

size_t cache_cap() {
    static const size_t cap = [] {
        const char* v = std::getenv("DCRF_CACHE_MB");
        return (size_t)(v ? std::strtoull(v, nullptr, 10) : 2048ull) << 20;
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
    *cached = g_cached;
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
    int cur = 0, dev = 0;
    cudaPointerAttributes a;
    if (cudaGetDevice(&cur) != cudaSuccess || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(p);
        return;
    }
    dev = a.device;
    if (dev != cur) cudaSetDevice(dev);
    const bool ok = cudaDeviceSynchronize() == cudaSuccess;
    if (dev != cur) cudaSetDevice(cur);
    if (!ok) {
        cudaGetLastError();
        cudaFree(p);  // a broken context: no reuse
        return;
    }
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (g_cached + bytes <= cache_cap()) {
            cache().push_back(Block{p, bytes, dev});
            g_cached += bytes;
            return;
        }
    }
    cudaFree(p);
}

void dev_trim(bool all_devices) noexcept {
    std::lock_guard<std::recursive_mutex> cap(capture_mutex());
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
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
