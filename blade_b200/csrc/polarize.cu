// Polarizer: linear (X, Y) -> circular (X + iY, X - iY), no 1/sqrt(2).
//
// Reference: src/modules/polarizer/polarizer.cu:5-25 (one thread per 2 complex
// values, half the launched threads idle) and src/modules/polarizer/base.cc:12-68
// (in place, CF32 and CF16).  Here one 128-bit load/store per thread-iteration:
// one dual-pol CF32 sample, or two dual-pol CF16 samples.  CF16 arithmetic is the
// exact sum rounded once to half, the same value the reference's half add gives.
#include "common.cuh"

namespace bb {
namespace {

__global__ void __launch_bounds__(256) polarize_cf32_kernel(const float4* __restrict__ in, float4* __restrict__ out,
                                                            uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        float4 v = in[i];  // (xr, xi, yr, yi)
        out[i] = make_float4(v.x - v.w, v.y + v.z, v.x + v.w, v.y - v.z);
    }
}

__device__ __forceinline__ uint2 polarize_h(uint2 v) {
    __half2 x = *reinterpret_cast<__half2*>(&v.x);  // (xr, xi)
    __half2 y = *reinterpret_cast<__half2*>(&v.y);  // (yr, yi)
    __half2 iy = __halves2half2(__hneg(__high2half(y)), __low2half(y));  // i*Y = (-yi, yr)
    __half2 l = __hadd2(x, iy), r = __hsub2(x, iy);
    uint2 o;
    o.x = *reinterpret_cast<uint32_t*>(&l);
    o.y = *reinterpret_cast<uint32_t*>(&r);
    return o;
}

__global__ void __launch_bounds__(256) polarize_cf16_kernel(const uint4* __restrict__ in, uint4* __restrict__ out,
                                                            uint64_t n_pairs) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_pairs; i += stride) {
        uint4 v = in[i];
        uint2 a = polarize_h(make_uint2(v.x, v.y)), b = polarize_h(make_uint2(v.z, v.w));
        out[i] = make_uint4(a.x, a.y, b.x, b.y);
    }
}

__global__ void polarize_cf16_tail(const uint2* __restrict__ in, uint2* __restrict__ out, uint64_t i) {
    out[i] = polarize_h(in[i]);
}

}  // namespace
}  // namespace bb

extern "C" int blade_polarize(int type, const void* in, void* out, uint64_t n_samples, blade_stream_t stream) {
    using namespace bb;
    if (n_samples == 0) return BLADE_SUCCESS;
    if (!in || !out) return set_error(BLADE_ERROR, "blade_polarize: null buffer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (type == BLADE_CF32) {
        if (!aligned16(in) || !aligned16(out))
            return set_error(BLADE_ERROR, "blade_polarize: CF32 buffers must be 16-byte aligned");
        polarize_cf32_kernel<<<grid_for(n_samples, 256), 256, 0, s>>>(static_cast<const float4*>(in),
                                                                     static_cast<float4*>(out), n_samples);
    } else if (type == BLADE_CF16) {
        if (!aligned16(in) || !aligned16(out))
            return set_error(BLADE_ERROR, "blade_polarize: CF16 buffers must be 16-byte aligned");
        uint64_t pairs = n_samples / 2;
        if (pairs)
            polarize_cf16_kernel<<<grid_for(pairs, 256), 256, 0, s>>>(static_cast<const uint4*>(in),
                                                                     static_cast<uint4*>(out), pairs);
        if (n_samples & 1)
            polarize_cf16_tail<<<1, 1, 0, s>>>(static_cast<const uint2*>(in), static_cast<uint2*>(out),
                                               n_samples - 1);
    } else {
        return set_error(BLADE_ERROR, "blade_polarize: type must be CF32 or CF16");
    }
    return check_launch("blade_polarize");
}
