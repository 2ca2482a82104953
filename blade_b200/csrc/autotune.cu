// Autotuner cache, query and the synthetic inputs the tuning runs use.
#include <string.h>

#include <map>
#include <mutex>

#include "autotune.cuh"

namespace bb {
namespace {

struct TuneKey {
    int family, dev;
    uint64_t shape[8];
    bool operator<(const TuneKey& o) const {
        if (family != o.family) return family < o.family;
        if (dev != o.dev) return dev < o.dev;
        return memcmp(shape, o.shape, sizeof(shape)) < 0;
    }
};

std::mutex g_mu;
std::map<TuneKey, TuneEntry> g_cache;

TuneKey make_key(int family, const uint64_t (&shape)[8]) {
    TuneKey k;
    k.family = family;
    k.dev = 0;
    cudaGetDevice(&k.dev);
    memcpy(k.shape, shape, sizeof(k.shape));
    return k;
}

__device__ __forceinline__ uint32_t mix(uint64_t i) {
    uint64_t z = i * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return (uint32_t)(z ^ (z >> 31));
}

__global__ void fill_ci8_kernel(int8_t* p, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = (int8_t)((int)(mix(i) % 255u) - 127);
}

__global__ void fill_phasor_kernel(float2* p, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        float s, c;
        sincospif((float)(mix(i) & 0xFFFFFFu) * (2.f / 16777216.f), &s, &c);
        p[i] = make_float2(c, s);
    }
}

}  // namespace

bool tune_lookup(int family, const uint64_t (&shape)[8], TuneEntry* out) {
    const TuneKey k = make_key(family, shape);
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_cache.find(k);
    if (it == g_cache.end()) return false;
    if (out) *out = it->second;
    return true;
}

void tune_store(int family, const uint64_t (&shape)[8], const TuneEntry& e) {
    const TuneKey k = make_key(family, shape);
    std::lock_guard<std::mutex> lock(g_mu);
    g_cache[k] = e;
}

int tune_fill_ci8(void* p, uint64_t n, cudaStream_t s) {
    if (n == 0) return BLADE_SUCCESS;
    fill_ci8_kernel<<<grid_for(n, 256), 256, 0, s>>>(static_cast<int8_t*>(p), n);
    return check_launch("autotune input fill");
}

int tune_fill_phasors(void* p, uint64_t n, cudaStream_t s) {
    if (n == 0) return BLADE_SUCCESS;
    fill_phasor_kernel<<<grid_for(n, 256), 256, 0, s>>>(static_cast<float2*>(p), n);
    return check_launch("autotune phasor fill");
}

}  // namespace bb

extern "C" int blade_autotune_clear(void) {
    std::lock_guard<std::mutex> lock(bb::g_mu);
    bb::g_cache.clear();
    return BLADE_SUCCESS;
}

extern "C" int blade_autotune_query(int family, const uint64_t shape[8], uint32_t params[8], float* us, int* tuned) {
    using namespace bb;
    if (!shape || !params || !us || !tuned) return set_error(BLADE_ERROR, "blade_autotune_query: null argument");
    uint64_t key[8];
    for (int i = 0; i < 8; i++) key[i] = shape[i];
    switch (family) {
        case BLADE_TUNE_TC: return tc_query(key, params, us, tuned);
        case BLADE_TUNE_F32: return f32_query(key, params, us, tuned);
        case BLADE_TUNE_SPECTROMETER: return spec_query(key, params, us, tuned);
        default: return set_error(BLADE_ERROR, "blade_autotune_query: unknown family %d", family);
    }
}
