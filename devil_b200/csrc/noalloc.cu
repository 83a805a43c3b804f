// p-value adjustment over device buffers that allocates nothing.
//
// Who needs it: a caller whose device memory is already claimed by another
// allocator (a framework's caching pool holding most of HBM, where a
// cudaMalloc would fail or force that pool to give memory back), or one
// that must not stall the GPU (cudaFree synchronizes the device, so every
// other stream would wait).  Such callers cannot create a devil_ctx, whose
// workspace grows with cudaMalloc, yet still want the BH step of test_de
// on p-values they already hold on the device.
//
// How: the sort keys, indices, CUB's temporary storage and the valid-count
// live in one file-scope __device__ array, part of the module's global
// memory, held by every GPU that loads the library until the process
// exits.  Its size caps the number of p-values (kStaticMaxM).  Host code
// cannot use the array's name as a device address (on the host it names a
// stand-in object), so the address is looked up with cudaGetSymbolAddress
// once per device, on the first call made with that device current; that
// first call should come before any stream capture begins on the caller's
// side.
//
// What must start at zero: the valid-count (NaN p-values are excluded from
// n) is cleared by a cudaMemsetAsync on the caller's stream at the start
// of every call; everything else in the array is written before it is
// read, although it still holds whatever the previous call left there.
//
// Overlapping calls race: every call on a device uses the same array, so
// two calls in flight at the same time on one device (different streams or
// threads without ordering between them) corrupt each other's results.
// Calls must be serialised, e.g. issued on one stream.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>

#include "../../include/devil_b200.h"
#include "internal.h"

namespace {

constexpr int64_t kStaticMaxM = 1 << 16;          // p-values per call
constexpr size_t kStaticBytes = (size_t)4 << 20;  // 4 MiB of device scratch
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_padj_scratch[kStaticBytes];

std::atomic<void*> g_scratch[kMaxDevices];
std::mutex g_setup;

void put_err(char* buf, size_t len, const char* msg) {
    if (buf && len) snprintf(buf, len, "%s", msg);
}

}  // namespace

extern "C" {

DEVIL_API int devil_p_adjust_device_static(int64_t m, const double* p_dev, int method,
                                           double* out_dev, void* stream, char* errbuf,
                                           size_t errlen) {
    if (m < 0 || (m > 0 && (!p_dev || !out_dev))) {
        put_err(errbuf, errlen, "devil_p_adjust_device_static: need m >= 0 and device p / out");
        return DEVIL_ERR_ARG;
    }
    if (method < DEVIL_ADJ_NONE || method > DEVIL_ADJ_HOMMEL) {
        put_err(errbuf, errlen, "devil_p_adjust_device_static: unknown adjustment method");
        return DEVIL_ERR_ARG;
    }
    if (m > kStaticMaxM) {
        char msg[160];
        snprintf(msg, sizeof msg,
                 "devil_p_adjust_device_static: m = %lld exceeds the static limit of %lld "
                 "p-values (use devil_p_adjust_device)", (long long)m, (long long)kStaticMaxM);
        put_err(errbuf, errlen, msg);
        return DEVIL_ERR_ARG;
    }
    if (devil::p_adjust_temp_bytes(m) > kStaticBytes) {
        put_err(errbuf, errlen, "devil_p_adjust_device_static: scratch for this m exceeds 4 MiB");
        return DEVIL_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        put_err(errbuf, errlen, "devil_p_adjust_device_static: no current CUDA device");
        return DEVIL_ERR_CUDA;
    }
    void* scratch = g_scratch[dev].load(std::memory_order_acquire);
    if (!scratch) {
        std::lock_guard<std::mutex> lk(g_setup);
        scratch = g_scratch[dev].load(std::memory_order_relaxed);
        if (!scratch) {
            e = cudaGetSymbolAddress(&scratch, g_padj_scratch);
            if (e != cudaSuccess || !scratch) {
                char msg[200];
                snprintf(msg, sizeof msg,
                         "devil_p_adjust_device_static: cudaGetSymbolAddress failed: %s",
                         cudaGetErrorString(e));
                put_err(errbuf, errlen, msg);
                return DEVIL_ERR_CUDA;
            }
            g_scratch[dev].store(scratch, std::memory_order_release);
        }
    }
    e = devil::launch_p_adjust(m, p_dev, method, out_dev, scratch, kStaticBytes,
                               static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        char msg[200];
        snprintf(msg, sizeof msg, "devil_p_adjust_device_static: %s", cudaGetErrorString(e));
        put_err(errbuf, errlen, msg);
        return DEVIL_ERR_CUDA;
    }
    return DEVIL_OK;
}

}  // extern "C"
