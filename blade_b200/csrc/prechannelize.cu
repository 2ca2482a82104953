// Pre-beamformer stages of the ATA ModeB bundle on CI8 voltages, exact in FP16:
// Cast<CI8,CF32> -> Channelizer(rate R <= 4) -> [Polarizer XY -> LR]
// (include/blade/bundles/ata/mode_b.hh:99-139; src/modules/channelizer/
// base.cc:59-138 + channelizer.cu:5-19, src/modules/polarizer/polarizer.cu:17-23):
//   out[a, f*R + k, s, p] = sum_j (-1)^j x[a, f, s*R + j, p] e^{-2 pi i j k / R}
// (the fftshifted R-point DFT), then (X, Y) -> (X + iY, X - iY) when circular.
// CI8 components are integers in [-128, 127], so every output component is an
// integer of magnitude <= 1024: the FP16 output holds the same values the FP32
// module chain computes, and the tensor-core beamformer reads them exactly.
#include "common.cuh"

namespace bb {
namespace {

// One thread per (a, f, spectrum s): R sample words in, R dual-polarisation
// CF16 samples out (8 bytes each, consecutive threads write consecutive s).
template <int R, bool CIRC>
__global__ void __launch_bounds__(256) prechannelize_kernel(const uint32_t* __restrict__ in,
                                                            uint2* __restrict__ out, uint64_t AF, uint32_t S) {
    const uint64_t n = AF * S;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t af = i / S;
        const uint32_t s = (uint32_t)(i - af * S);
        float xr[2][R], xi[2][R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            const uint32_t w = __ldg(in + af * (uint64_t)S * R + (uint64_t)s * R + j);
            const float sg = (j & 1) ? -1.f : 1.f;  // fftshift pre-multiply (even R)
            xr[0][j] = (R > 1 ? sg : 1.f) * (float)(int8_t)(w & 0xFFu);
            xi[0][j] = (R > 1 ? sg : 1.f) * (float)(int8_t)((w >> 8) & 0xFFu);
            xr[1][j] = (R > 1 ? sg : 1.f) * (float)(int8_t)((w >> 16) & 0xFFu);
            xi[1][j] = (R > 1 ? sg : 1.f) * (float)(int8_t)(w >> 24);
        }
#pragma unroll
        for (int k = 0; k < R; k++) {
            float zr[2], zi[2];
#pragma unroll
            for (int p = 0; p < 2; p++) {
                zr[p] = 0.f;
                zi[p] = 0.f;
#pragma unroll
                for (int j = 0; j < R; j++) {
                    // e^{-2 pi i j k / R} for R <= 4 is one of 1, -i, -1, i
                    const int q = (j * k * (4 / R)) & 3;
                    const float re = xr[p][j], im = xi[p][j];
                    zr[p] += q == 0 ? re : q == 1 ? im : q == 2 ? -re : -im;
                    zi[p] += q == 0 ? im : q == 1 ? -re : q == 2 ? -im : re;
                }
            }
            if (CIRC) {
                const float lr = zr[0] - zi[1], li = zi[0] + zr[1];  // X + iY
                const float rr = zr[0] + zi[1], ri = zi[0] - zr[1];  // X - iY
                zr[0] = lr;
                zi[0] = li;
                zr[1] = rr;
                zi[1] = ri;
            }
            const __half2 h0 = __floats2half2_rn(zr[0], zi[0]), h1 = __floats2half2_rn(zr[1], zi[1]);
            uint2 o;
            o.x = *reinterpret_cast<const uint32_t*>(&h0);
            o.y = *reinterpret_cast<const uint32_t*>(&h1);
            out[(af * R + k) * (uint64_t)S + s] = o;
        }
    }
}

template <int R>
void launch_pre(const uint32_t* in, uint2* out, uint64_t AF, uint32_t S, bool circ, cudaStream_t st) {
    const unsigned grid = grid_for(AF * S, 256);
    if (circ) prechannelize_kernel<R, true><<<grid, 256, 0, st>>>(in, out, AF, S);
    else prechannelize_kernel<R, false><<<grid, 256, 0, st>>>(in, out, AF, S);
}

}  // namespace
}  // namespace bb

extern "C" int blade_prechannelize_cf16(const void* in, void* out, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                        uint64_t rate, int circular, blade_stream_t stream) {
    using namespace bb;
    if (P != 2) return set_error(BLADE_ERROR, "blade_prechannelize_cf16: P must be 2");
    if (rate != 1 && rate != 2 && rate != 4)
        return set_error(BLADE_ERROR, "blade_prechannelize_cf16: rate must be 1, 2 or 4 (got %llu)",
                         (unsigned long long)rate);
    if (T % rate != 0)
        return set_error(BLADE_ERROR, "blade_prechannelize_cf16: the number of time samples (%llu) should be "
                         "divisible by the rate (%llu)", (unsigned long long)T, (unsigned long long)rate);
    if (T / rate > 0xFFFFFFFFull) return set_error(BLADE_ERROR, "blade_prechannelize_cf16: T too large");
    if (A * F * T == 0) return BLADE_SUCCESS;
    if (!in || !out) return set_error(BLADE_ERROR, "blade_prechannelize_cf16: null buffer");
    if ((reinterpret_cast<uintptr_t>(in) & 3) || (reinterpret_cast<uintptr_t>(out) & 7))
        return set_error(BLADE_ERROR, "blade_prechannelize_cf16: input must be 4-byte and output 8-byte aligned");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t* x = static_cast<const uint32_t*>(in);
    uint2* y = static_cast<uint2*>(out);
    const uint32_t S = (uint32_t)(T / rate);
    if (rate == 1) launch_pre<1>(x, y, A * F, S, circular != 0, st);
    else if (rate == 2) launch_pre<2>(x, y, A * F, S, circular != 0, st);
    else launch_pre<4>(x, y, A * F, S, circular != 0, st);
    return check_launch("blade_prechannelize_cf16");
}
