// Cast: per-scalar static_cast with 128-bit loads.
//
// Reference: src/modules/cast/cast.cu:5-12 (one scalar per thread, byte loads)
// and src/modules/cast/base.cc:12-66 (N = size * 2 scalars for complex types,
// complex <-> real rejected, same type bypassed).  Here each thread converts a
// 16-byte input vector per iteration of a grid-stride loop; the tail and any
// unaligned buffer fall back to a scalar loop.  Conversions are the ones the
// reference's static_cast compiles to: int8 -> float/half exact, half -> float
// exact, float -> half round-to-nearest-even, float -> int32 round-toward-zero.
#include "common.cuh"

namespace bb {
namespace {

template <typename IT, typename OT> struct Conv;
template <> struct Conv<int8_t, int8_t> { __device__ static int8_t f(int8_t v) { return v; } };
template <> struct Conv<int8_t, float> { __device__ static float f(int8_t v) { return (float)v; } };
template <> struct Conv<int8_t, __half> { __device__ static __half f(int8_t v) { return __int2half_rn((int)v); } };
template <> struct Conv<__half, __half> { __device__ static __half f(__half v) { return v; } };
template <> struct Conv<__half, float> { __device__ static float f(__half v) { return __half2float(v); } };
template <> struct Conv<float, float> { __device__ static float f(float v) { return v; } };
template <> struct Conv<float, __half> { __device__ static __half f(float v) { return __float2half_rn(v); } };
template <> struct Conv<float, int32_t> { __device__ static int32_t f(float v) { return __float2int_rz(v); } };

template <typename IT, typename OT>
__global__ void __launch_bounds__(256) cast_vec_kernel(const IT* __restrict__ in, OT* __restrict__ out,
                                                       uint64_t nvec) {
    constexpr int V = 16 / sizeof(IT);
    constexpr int OB = V * sizeof(OT);  // output bytes per vector: 4..64
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        uint4 raw = ldg_nc_u4(in + i * V);
        const IT* src = reinterpret_cast<const IT*>(&raw);
        alignas(16) OT dst[V];
#pragma unroll
        for (int k = 0; k < V; k++) dst[k] = Conv<IT, OT>::f(src[k]);
        char* o = reinterpret_cast<char*>(out + i * V);
        if constexpr (OB >= 16) {
#pragma unroll
            for (int k = 0; k < OB / 16; k++)
                reinterpret_cast<uint4*>(o)[k] = reinterpret_cast<const uint4*>(dst)[k];
        } else if constexpr (OB == 8) {
            *reinterpret_cast<uint2*>(o) = *reinterpret_cast<const uint2*>(dst);
        } else {
            *reinterpret_cast<uint32_t*>(o) = *reinterpret_cast<const uint32_t*>(dst);
        }
    }
}

// Widening casts (output wider than input): each thread writes one 16-byte output
// vector per step from a 2-, 4- or 8-byte input piece, so both the loads and the
// stores of a warp are contiguous.
template <int BYTES> struct Piece;
template <> struct Piece<2> { using T = uint16_t; };
template <> struct Piece<4> { using T = uint32_t; };
template <> struct Piece<8> { using T = uint2; };

template <typename IT, typename OT>
__global__ void __launch_bounds__(256) cast_widen_kernel(const IT* __restrict__ in, OT* __restrict__ out,
                                                         uint64_t nvec) {
    constexpr int VO = 16 / sizeof(OT);            // elements per output vector
    constexpr int IB = VO * (int)sizeof(IT);       // input bytes per vector: 2, 4 or 8
    using PT = typename Piece<IB>::T;
    const PT* pin = reinterpret_cast<const PT*>(in);
    uint4* pout = reinterpret_cast<uint4*>(out);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        const PT raw = __ldg(pin + i);
        const IT* src = reinterpret_cast<const IT*>(&raw);
        alignas(16) OT dst[VO];
#pragma unroll
        for (int k = 0; k < VO; k++) dst[k] = Conv<IT, OT>::f(src[k]);
        pout[i] = *reinterpret_cast<const uint4*>(dst);
    }
}

template <typename IT, typename OT>
__global__ void cast_scalar_kernel(const IT* __restrict__ in, OT* __restrict__ out, uint64_t begin,
                                   uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = begin + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = Conv<IT, OT>::f(in[i]);
}

template <typename IT, typename OT>
int launch_cast(const void* vin, void* vout, uint64_t n, cudaStream_t s) {
    const IT* in = static_cast<const IT*>(vin);
    OT* out = static_cast<OT*>(vout);
    if (n == 0) return BLADE_SUCCESS;
    constexpr int V = 16 / sizeof(IT);
    uint64_t done = 0;
    if constexpr (sizeof(OT) > sizeof(IT)) {
        constexpr int VO = 16 / sizeof(OT);
        if (aligned16(out) && (reinterpret_cast<uintptr_t>(in) % (VO * sizeof(IT))) == 0) {
            const uint64_t nvec = n / VO;
            if (nvec) {
                cast_widen_kernel<IT, OT><<<grid_for(nvec, 256), 256, 0, s>>>(in, out, nvec);
                done = nvec * VO;
            }
            if (done < n) cast_scalar_kernel<IT, OT><<<grid_for(n - done, 256), 256, 0, s>>>(in, out, done, n);
            return check_launch("blade_cast");
        }
    }
    if (aligned16(in) && (reinterpret_cast<uintptr_t>(out) % (V * sizeof(OT) >= 16 ? 16 : V * sizeof(OT))) == 0) {
        uint64_t nvec = n / V;
        if (nvec) {
            cast_vec_kernel<IT, OT><<<grid_for(nvec, 256), 256, 0, s>>>(in, out, nvec);
            done = nvec * V;
        }
    }
    if (done < n) {
        cast_scalar_kernel<IT, OT><<<grid_for(n - done, 256), 256, 0, s>>>(in, out, done, n);
    }
    return check_launch("blade_cast");
}

enum Scalar { S_I8, S_I32, S_F16, S_F32, S_F64, S_BAD };

Scalar scalar_of(int t) {
    switch (t) {
        case BLADE_I8: case BLADE_CI8: return S_I8;
        case BLADE_I32: return S_I32;
        case BLADE_F16: case BLADE_CF16: return S_F16;
        case BLADE_F32: case BLADE_CF32: return S_F32;
        case BLADE_F64: case BLADE_CF64: return S_F64;
        default: return S_BAD;
    }
}

}  // namespace
}  // namespace bb

extern "C" int blade_cast(int in_type, int out_type, const void* in, void* out, uint64_t n_elements,
                          blade_stream_t stream) {
    using namespace bb;
    if (dtype_bytes(in_type) == 0 || dtype_bytes(out_type) == 0)
        return set_error(BLADE_ERROR, "blade_cast: unknown dtype (%d -> %d)", in_type, out_type);
    if (dtype_is_complex(in_type) != dtype_is_complex(out_type))
        return set_error(BLADE_ERROR, "blade_cast: cannot cast between complex and non-complex types");
    if (n_elements && (!in || !out)) return set_error(BLADE_ERROR, "blade_cast: null buffer");
    const uint64_t n = n_elements * (dtype_is_complex(in_type) ? 2 : 1);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const Scalar si = scalar_of(in_type), so = scalar_of(out_type);
    if (si == so) {
        if (in == out || n == 0) return BLADE_SUCCESS;
        return blade_duplicate(in, out, n_elements * dtype_bytes(in_type), stream);
    }
    if (si == S_I8 && so == S_F32) return launch_cast<int8_t, float>(in, out, n, s);
    if (si == S_I8 && so == S_F16) return launch_cast<int8_t, __half>(in, out, n, s);
    if (si == S_F16 && so == S_F32) return launch_cast<__half, float>(in, out, n, s);
    if (si == S_F32 && so == S_F16) return launch_cast<float, __half>(in, out, n, s);
    if (si == S_F32 && so == S_I32) return launch_cast<float, int32_t>(in, out, n, s);
    return set_error(BLADE_ERROR, "blade_cast: conversion %d -> %d is not provided by the reference", in_type,
                     out_type);
}
