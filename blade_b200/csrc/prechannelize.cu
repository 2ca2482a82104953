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
// CF16 samples out (8 bytes each, consecutive threads write consecutive s).  Each
// thread keeps the loads of kSpt spectra in flight before it computes any of them.
constexpr int kSpt = 4;

template <int R>
__device__ __forceinline__ void load_spectrum(const uint32_t* src, uint32_t (&ws)[R]) {
    if constexpr (R == 4) {
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(src));
        ws[0] = v.x;
        ws[1 % R] = v.y;
        ws[2 % R] = v.z;
        ws[3 % R] = v.w;
    } else if constexpr (R == 2) {
        const uint2 v = __ldg(reinterpret_cast<const uint2*>(src));
        ws[0] = v.x;
        ws[1 % R] = v.y;
    } else {
        ws[0] = __ldg(src);
    }
}

template <int R, bool CIRC>
__device__ __forceinline__ void spectrum_out(const uint32_t (&ws)[R], uint2* __restrict__ out, uint64_t af,
                                             uint32_t S, uint32_t s) {
    float xr[2][R], xi[2][R];
#pragma unroll
    for (int j = 0; j < R; j++) {
        const uint32_t w = ws[j];
        const float sg = (R > 1 && (j & 1)) ? -1.f : 1.f;  // fftshift pre-multiply (even R)
        xr[0][j] = sg * (float)(int8_t)(w & 0xFFu);
        xi[0][j] = sg * (float)(int8_t)((w >> 8) & 0xFFu);
        xr[1][j] = sg * (float)(int8_t)((w >> 16) & 0xFFu);
        xi[1][j] = sg * (float)(int8_t)(w >> 24);
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

template <int R, bool CIRC>
__global__ void __launch_bounds__(256) prechannelize_kernel(const uint32_t* __restrict__ in,
                                                            uint2* __restrict__ out, uint64_t AF, uint32_t S) {
    const uint64_t n = AF * S;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; base < n; base += kSpt * stride) {
        uint32_t ws[kSpt][R];
#pragma unroll
        for (int q = 0; q < kSpt; q++) {
            const uint64_t i = base + q * stride;
            if (i < n) load_spectrum<R>(in + i * R, ws[q]);  // spectrum i = af * S + s starts at word i * R
        }
#pragma unroll
        for (int q = 0; q < kSpt; q++) {
            const uint64_t i = base + q * stride;
            if (i < n) {
                const uint64_t af = i / S;
                spectrum_out<R, CIRC>(ws[q], out, af, S, (uint32_t)(i - af * S));
            }
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
    if ((reinterpret_cast<uintptr_t>(in) & (4 * rate - 1)) || (reinterpret_cast<uintptr_t>(out) & 7))
        return set_error(BLADE_ERROR, "blade_prechannelize_cf16: input must be (4 x rate)-byte and output 8-byte "
                         "aligned");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t* x = static_cast<const uint32_t*>(in);
    uint2* y = static_cast<uint2*>(out);
    const uint32_t S = (uint32_t)(T / rate);
    if (rate == 1) launch_pre<1>(x, y, A * F, S, circular != 0, st);
    else if (rate == 2) launch_pre<2>(x, y, A * F, S, circular != 0, st);
    else launch_pre<4>(x, y, A * F, S, circular != 0, st);
    return check_launch("blade_prechannelize_cf16");
}

// ---- incoherent beam of ModeB with the detector, on the CF16 fine channels ----
// Beamformer::ATA's incoherent beam (src/modules/beamformer/beamformer.cu:64-78:
// sum_a |x * w[0]|^2 per polarisation, square-rooted when the detector follows,
// mode_b.hh:146-147) followed by the Stokes-I detector (detector.cu:34-51), which
// squares the root back: out[f, u] = sum_{t in window u} sum_p sum_a
// |x[a,f,t,p]|^2 |w[0,a,f,0,p]|^2.  One thread per sample (coalesced 8-byte
// loads), the window closed with lane shuffles; I is a power of two <= 32.
namespace bb {
namespace {

__global__ void __launch_bounds__(256) incoherent_detect_cf16_kernel(const uint2* __restrict__ x,
                                                                     const float2* __restrict__ w0, float* out,
                                                                     uint32_t A, uint32_t F, uint32_t T, uint32_t I) {
    extern __shared__ float g2[];  // |w[0, a, f, 0, p]|^2, [a][p]
    const uint32_t f = blockIdx.y;
    for (uint32_t i = threadIdx.x; i < 2 * A; i += blockDim.x) {
        const float2 w = w0[((uint64_t)(i >> 1) * F + f) * 2 + (i & 1)];
        g2[i] = w.x * w.x + w.y * w.y;
    }
    __syncthreads();
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    float acc = 0.f;
    if (t < T) {
        for (uint32_t a = 0; a < A; a++) {
            const uint2 v = __ldg(x + ((uint64_t)a * F + f) * T + t);
            const float2 p0 = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
            const float2 p1 = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
            acc = fmaf(p0.x * p0.x + p0.y * p0.y, g2[2 * a], acc);
            acc = fmaf(p1.x * p1.x + p1.y * p1.y, g2[2 * a + 1], acc);
        }
    }
    for (uint32_t off = 1; off < I; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if (t < T && (t % I) == 0) out[(uint64_t)f * (T / I) + t / I] = acc;
}

}  // namespace
}  // namespace bb

extern "C" int blade_incoherent_detect_cf16(const void* in, const void* phasors, void* out, uint64_t A, uint64_t F,
                                            uint64_t T, uint64_t P, uint64_t integration, blade_stream_t stream) {
    using namespace bb;
    if (P != 2) return set_error(BLADE_ERROR, "blade_incoherent_detect_cf16: P must be 2");
    if (integration == 0 || integration > 32 || (integration & (integration - 1)) != 0 || T % integration != 0)
        return set_error(BLADE_ERROR, "blade_incoherent_detect_cf16: integration must be a power of two <= 32 "
                         "dividing T");
    if (A * F * T == 0) return BLADE_SUCCESS;
    if (F > 65535 || T >= (1ull << 31)) return set_error(BLADE_ERROR, "blade_incoherent_detect_cf16: too large");
    if (!in || !phasors || !out) return set_error(BLADE_ERROR, "blade_incoherent_detect_cf16: null buffer");
    if ((reinterpret_cast<uintptr_t>(in) & 7) || (reinterpret_cast<uintptr_t>(out) & 3))
        return set_error(BLADE_ERROR, "blade_incoherent_detect_cf16: misaligned buffer");
    const size_t smem = 2 * A * sizeof(float);
    if (int rc = ensure_smem(reinterpret_cast<const void*>(incoherent_detect_cf16_kernel), smem)) return rc;
    const dim3 grid((unsigned)((T + 255) / 256), (unsigned)F);
    incoherent_detect_cf16_kernel<<<grid, 256, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const uint2*>(in), static_cast<const float2*>(phasors), static_cast<float*>(out), (uint32_t)A,
        (uint32_t)F, (uint32_t)T, (uint32_t)integration);
    return check_launch("blade_incoherent_detect_cf16");
}
