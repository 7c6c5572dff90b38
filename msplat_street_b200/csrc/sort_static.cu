// Radix sort that allocates nothing: its scratch is a fixed array in device memory.
//
// Who needs it: callers that are not allowed to allocate GPU memory at the moment
// they sort. A serving process that has committed its whole HBM budget to resident
// scenes cannot risk an allocation failing or evicting a scene mid-request; a
// latency-bound render loop cannot afford the device-wide synchronisation that
// cudaMalloc / cudaFree imply; a plugin host that owns all device memory forbids
// libraries from allocating behind its back. msplat_cuda_radix_sort grows buffers
// in its context on demand, so none of them can call it; they call
// msplat_cuda_radix_sort_static instead, which uses the array below.
//
// The array is a file-scope __device__ object, so every GPU that loads this library
// holds it (MSPLAT_STATIC_SORT_BYTES) until the process exits. Its name in host code
// is only a host-side stand-in, not a device address: the entry point looks the real
// address up with cudaGetSymbolAddress, once per device, on that device's first call
// (which is why the first call on each device should come before any stream capture
// begins), and passes that address to the kernels. The address is kept per device
// ordinal, so a device reset or a non-primary driver context is not supported.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/msplat_cuda.h"
#include "kernels.h"

namespace msplat {

// keys and values of the second ping-pong buffer, then the radix histogram scratch
constexpr uint32_t STATIC_SORT_MAX_KEYS = MSPLAT_STATIC_SORT_MAX_KEYS;
constexpr size_t STATIC_KEYS_BYTES = (size_t)STATIC_SORT_MAX_KEYS * sizeof(uint64_t);
constexpr size_t STATIC_VALS_BYTES = (size_t)STATIC_SORT_MAX_KEYS * sizeof(uint32_t);
constexpr size_t STATIC_RADIX_BYTES = MSPLAT_STATIC_SORT_BYTES - STATIC_KEYS_BYTES - STATIC_VALS_BYTES;

static __device__ __align__(256) unsigned char g_static_sort_scratch[MSPLAT_STATIC_SORT_BYTES];

namespace {

constexpr int MAX_DEVICES = 64;
std::mutex g_static_mu;
void *g_static_addr[MAX_DEVICES] = {};  // device address of the array, per device ordinal

int static_fail(int code, const std::string &msg) { return report_error(code, msg.c_str()); }

}  // namespace
}  // namespace msplat

using namespace msplat;

extern "C" {

int msplat_cuda_radix_sort_static(void *stream, uint64_t *keys, int32_t *vals, uint32_t n, int key_bits) {
    if (n == 0 || key_bits <= 0) return MSPLAT_CUDA_OK;
    if (!keys || !vals) return static_fail(MSPLAT_CUDA_EINVAL, "msplat_cuda_radix_sort_static: null keys or values");
    if (n > STATIC_SORT_MAX_KEYS)
        return static_fail(MSPLAT_CUDA_ECAPACITY,
                           "msplat_cuda_radix_sort_static: " + std::to_string(n) + " keys exceed the static scratch "
                           "capacity of " + std::to_string(STATIC_SORT_MAX_KEYS) + " keys");
    if (radix_scratch_bytes((int)n) > STATIC_RADIX_BYTES)
        return static_fail(MSPLAT_CUDA_ECAPACITY, "msplat_cuda_radix_sort_static: histogram scratch too small");
    if (key_bits > 64) key_bits = 64;
    // an error left by the caller's own earlier work is not this call's: report it as
    // pending (without clearing it) and enqueue nothing
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess)
        return static_fail(MSPLAT_CUDA_ECUDA, std::string("msplat_cuda_radix_sort_static: pending error before the "
                                                          "call: ") + cudaGetErrorString(e));
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return static_fail(MSPLAT_CUDA_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= MAX_DEVICES) return static_fail(MSPLAT_CUDA_EINVAL, "device ordinal out of range");
    void *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_static_mu);
        if (!g_static_addr[dev]) {
            // first call on this device (which is current): find the array's device address
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_static_sort_scratch);
            if (e != cudaSuccess || !p)
                return static_fail(MSPLAT_CUDA_ECUDA,
                                   std::string("cudaGetSymbolAddress(static sort scratch): ") + cudaGetErrorString(e));
            g_static_addr[dev] = p;
        }
        base = g_static_addr[dev];
    }
    unsigned char *b = static_cast<unsigned char *>(base);
    uint64_t *k1 = reinterpret_cast<uint64_t *>(b);
    uint32_t *v1 = reinterpret_cast<uint32_t *>(b + STATIC_KEYS_BYTES);
    void *radix = b + STATIC_KEYS_BYTES + STATIC_VALS_BYTES;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // Every pass writes its histogram, offsets and scan partials before reading them,
    // so nothing in the array has to start at zero.
    uint64_t *kk[2] = {keys, k1};
    uint32_t *vv[2] = {reinterpret_cast<uint32_t *>(vals), v1};
    const int cur = radix_sort_pairs(kk, vv, (int)n, key_bits, radix, st);
    if (cur == 1) {
        e = cudaMemcpyAsync(keys, k1, (size_t)n * 8, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(vals, v1, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return static_fail(MSPLAT_CUDA_ECUDA, std::string("copy back: ") + cudaGetErrorString(e));
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return static_fail(MSPLAT_CUDA_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
    return MSPLAT_CUDA_OK;
}

}  // extern "C"
