// Shared state of the C ABI: last-error message, version, device properties.
#include <stdarg.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "common.cuh"

namespace bb {

static thread_local char g_last_error[512] = {0};

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

int check_launch(const char* what) {
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        return set_error(BLADE_CUDA_ERROR, "%s failed to launch: %s", what, cudaGetErrorString(e));
    }
    return BLADE_SUCCESS;
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (cached[dev] == 0) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
        cached[dev] = n;
    }
    return cached[dev];
}

int ensure_smem(const void* func, size_t bytes) {
    if (bytes == 0) return BLADE_SUCCESS;
    struct Entry { const void* f; int dev; size_t bytes; };
    static std::mutex mu;
    static std::vector<Entry> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    for (auto& e : done)
        if (e.f == func && e.dev == dev && e.bytes >= bytes) return BLADE_SUCCESS;
    // the 48 KB that need no opt-in cover static and dynamic shared memory together
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, func);
    if (e == cudaSuccess && bytes + fa.sharedSizeBytes > 48 * 1024)
        e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return set_error(BLADE_CUDA_ERROR, "shared memory opt-in (%zu bytes): %s", bytes,
                                           cudaGetErrorString(e));
    done.push_back({func, dev, bytes});
    return BLADE_SUCCESS;
}

}  // namespace bb

extern "C" const char* blade_last_error(void) { return bb::g_last_error; }

extern "C" int blade_version(void) { return 1 * 10000 + 0 * 100 + 0; }
