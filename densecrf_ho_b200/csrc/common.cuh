// Shared helpers of libdcrf_cuda: status plumbing, device buffers, and the
// exact-rounding arithmetic the reference's SSE2 build performs.
#pragma once
#include <cstdlib>
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>

#include "dcrf.h"

namespace dcrf {

// Thrown inside the library, converted to a dcrf_status at the C boundary.
struct Error : public std::runtime_error {
    dcrf_status code;
    Error(dcrf_status c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define DCRF_CUDA(call)                                                              \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                       \
            throw ::dcrf::Error(e_ == cudaErrorMemoryAllocation ? DCRF_E_NOMEM       \
                                                                : DCRF_E_CUDA,       \
                                std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define DCRF_LAUNCH_CHECK() DCRF_CUDA(cudaGetLastError())

inline void require(bool ok, dcrf_status code, const std::string& msg) {
    if (!ok) throw Error(code, msg);
}

// Device memory through a process-wide cache of freed blocks (memory.cu):
// dev_alloc returns a block of at least `bytes` (its size class in *got),
// from the cache or cudaMalloc; dev_release waits for the device, as
// cudaFree does, then keeps the block for reuse up to DCRF_CACHE_MB
// (default 2048) MiB of cached memory per process, beyond which it frees it.
void* dev_alloc(size_t bytes, size_t* got);
// Held while a solver loop is captured into a CUDA graph, and by dev_alloc /
// dev_release around cudaMalloc, cudaFree and the device-wide wait: a thread
// that frees or allocates waits until another thread's capture has ended.
std::recursive_mutex& capture_mutex();
void dev_release(void* p, size_t bytes) noexcept;
// Frees the cached blocks of the current device, or of every device
// (dcrf_release_cached_memory).
void dev_trim(bool all_devices) noexcept;
// A budget on the bytes held by live DevBufs (0 = none): a request beyond it
// fails with DCRF_E_NOMEM on the host, before any device call.
void set_device_memory_limit(size_t bytes);
// Bytes held by live DevBufs, bytes kept in the cache, cudaMalloc calls made.
void device_memory_stats(size_t* live, size_t* cached, unsigned long long* mallocs);

// Owning device allocation; grows, never shrinks.
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    size_t bytes = 0;  // size of the block behind p
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) dev_release(p, bytes);
        p = nullptr;
        n = 0;
        bytes = 0;
    }
    T* ensure(size_t count) {
        if (count > n) {
            release();
            p = static_cast<T*>(dev_alloc((count ? count : 1) * sizeof(T), &bytes));
            n = count;
        }
        return p;
    }
    T* get() const { return p; }
};

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// The solver loops run as CUDA graphs with device-side while nodes unless the
// environment sets DCRF_GRAPHS=0 (then every iteration is launched from the
// host, kernel by kernel: for profilers that do not follow conditional graph
// nodes).  Results are the same either way.
inline bool graphs_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("DCRF_GRAPHS");
        return !(v && v[0] == '0');
    }();
    return on;
}

// Process-wide count of kernels this library has launched (benchmarks read
// it through dcrf_kernel_launches()).
extern std::atomic<unsigned long long> g_kernel_launches;

// Every kernel of the library is launched through here.
template <typename... KArgs, typename... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                   Args&&... args) {
    kernel<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
    g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
}

// Number of SMs of the current device (cached per process; one device per
// process is the supported deployment).
int sm_count();

// ------------------------------------------------------------------------
// Exact float arithmetic.  The reference is compiled for x86-64 SSE2, which
// has no fused multiply-add; every product and sum is rounded separately to
// nearest-even.  These wrappers keep nvcc from contracting them (the library
// is additionally built with -fmad=false).
// ------------------------------------------------------------------------
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }

}  // namespace dcrf
