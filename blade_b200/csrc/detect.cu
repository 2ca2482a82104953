// Detector: time-integrated power products, deterministic (no atomics).
//
// Reference: src/modules/detector/detector.cu:7-51 zeroes the output and then
// atomicAdds one product per input sample (summation order varies run to run, and
// the zeroing races with other blocks' adds); src/modules/detector/base.cc:9-85
// requires P = 2 and T % I == 0, out [A, F, T/I, 1|4].
// Here a CTA stages a chunk of whole windows: its 256 threads load the chunk's
// dual-pol samples with coalesced 128-bit loads, write the per-sample products to
// shared memory, and each window is then summed by one thread in a fixed
// (skewed, bank-conflict-free) order.  Windows longer than 1024 samples are
// summed by one warp each with a fixed shuffle tree.
#include "common.cuh"

namespace bb {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 2048;  // samples staged per CTA iteration

template <int NPOL>
__global__ void __launch_bounds__(kThreads) detect_chunk_kernel(const float4* __restrict__ in, float* __restrict__ out,
                                                                uint64_t n_windows, uint32_t integ,
                                                                uint32_t win_per_chunk) {
    __shared__ float s_prod[NPOL][kChunk];
    const uint64_t n_chunks = ceil_div(n_windows, win_per_chunk);
    const uint32_t chunk_samples = win_per_chunk * integ;
    for (uint64_t c = blockIdx.x; c < n_chunks; c += gridDim.x) {
        const uint64_t w0 = c * win_per_chunk;
        const uint32_t nw = (uint32_t)min((uint64_t)win_per_chunk, n_windows - w0);
        const uint32_t ns = nw * integ;
        const float4* src = in + w0 * integ;
        for (uint32_t i = threadIdx.x; i < ns; i += kThreads) {
            float4 v = ldg_nc_f4(src + i);
            if (NPOL == 1) {
                s_prod[0][i] = v.x * v.x + v.y * v.y + (v.z * v.z + v.w * v.w);
            } else {
                s_prod[0][i] = v.x * v.x + v.y * v.y;                 // |X|^2
                s_prod[NPOL > 1 ? 1 : 0][i] = v.z * v.z + v.w * v.w;  // |Y|^2
                s_prod[NPOL > 2 ? 2 : 0][i] = v.x * v.z + v.y * v.w;  // Re X conj(Y)
                s_prod[NPOL > 3 ? 3 : 0][i] = v.y * v.z - v.x * v.w;  // Im X conj(Y)
            }
        }
        __syncthreads();
        for (uint32_t w = threadIdx.x; w < nw; w += kThreads) {
            const uint32_t base = w * integ;
            float acc[NPOL];
#pragma unroll
            for (int q = 0; q < NPOL; q++) acc[q] = 0.f;
            uint32_t k = w % integ;  // skewed start spreads the threads over banks
            for (uint32_t j = 0; j < integ; j++) {
#pragma unroll
                for (int q = 0; q < NPOL; q++) acc[q] += s_prod[q][base + k];
                k = (k + 1 == integ) ? 0 : k + 1;
            }
            if (NPOL == 1) {
                out[w0 + w] = acc[0];
            } else {
                reinterpret_cast<float4*>(out)[w0 + w] =
                    make_float4(acc[0], acc[NPOL > 1 ? 1 : 0], acc[NPOL > 2 ? 2 : 0], acc[NPOL > 3 ? 3 : 0]);
            }
        }
        __syncthreads();
    }
    (void)chunk_samples;
}

template <int NPOL>
__global__ void __launch_bounds__(kThreads) detect_warp_kernel(const float4* __restrict__ in, float* __restrict__ out,
                                                               uint64_t n_windows, uint64_t integ) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * kThreads + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * kThreads) >> 5;
    for (uint64_t w = warp; w < n_windows; w += nwarps) {
        const float4* src = in + w * integ;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (uint64_t i = lane; i < integ; i += 32) {
            float4 v = ldg_nc_f4(src + i);
            if (NPOL == 1) {
                acc[0] += v.x * v.x + v.y * v.y + (v.z * v.z + v.w * v.w);
            } else {
                acc[0] += v.x * v.x + v.y * v.y;
                acc[1] += v.z * v.z + v.w * v.w;
                acc[2] += v.x * v.z + v.y * v.w;
                acc[3] += v.y * v.z - v.x * v.w;
            }
        }
#pragma unroll
        for (int q = 0; q < NPOL; q++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        }
        if (lane == 0) {
            if (NPOL == 1) out[w] = acc[0];
            else reinterpret_cast<float4*>(out)[w] = make_float4(acc[0], acc[1], acc[2], acc[3]);
        }
    }
}

}  // namespace
}  // namespace bb

extern "C" int blade_detect(const void* in, void* out, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                            uint64_t integration, uint64_t out_pols, blade_stream_t stream) {
    using namespace bb;
    if (integration == 0) return set_error(BLADE_ERROR, "blade_detect: integration size should be more than zero");
    if (T % integration != 0)
        return set_error(BLADE_ERROR, "blade_detect: number of time samples (%llu) should be divisible by the "
                         "integration size (%llu)", (unsigned long long)T, (unsigned long long)integration);
    if (P != 2) return set_error(BLADE_ERROR, "blade_detect: number of polarizations (%llu) should be two (2)",
                                 (unsigned long long)P);
    if (A == 0) return set_error(BLADE_ERROR, "blade_detect: number of aspects should be more than zero");
    if (out_pols != 1 && out_pols != 4)
        return set_error(BLADE_ERROR, "blade_detect: number of output polarizations (%llu) not supported",
                         (unsigned long long)out_pols);
    const uint64_t n_windows = A * F * (T / integration);
    if (n_windows == 0) return BLADE_SUCCESS;
    if (!in || !out) return set_error(BLADE_ERROR, "blade_detect: null buffer");
    if (!aligned16(in) || (out_pols == 4 && !aligned16(out)))
        return set_error(BLADE_ERROR, "blade_detect: buffers must be 16-byte aligned");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const float4* src = static_cast<const float4*>(in);
    float* dst = static_cast<float*>(out);
    if (integration <= 1024) {
        uint32_t wpc = (uint32_t)(kChunk / integration);
        // small inputs: shorter chunks so that at least two CTAs per SM have work
        const uint64_t fill = ceil_div(n_windows, (uint64_t)sm_count() * 2);
        if (fill < wpc) wpc = (uint32_t)(fill > 0 ? fill : 1);
        uint64_t chunks = ceil_div(n_windows, wpc);
        unsigned grid = (unsigned)(chunks < (uint64_t)sm_count() * 8 ? chunks : (uint64_t)sm_count() * 8);
        if (out_pols == 1)
            detect_chunk_kernel<1><<<grid, kThreads, 0, s>>>(src, dst, n_windows, (uint32_t)integration, wpc);
        else
            detect_chunk_kernel<4><<<grid, kThreads, 0, s>>>(src, dst, n_windows, (uint32_t)integration, wpc);
    } else {
        uint64_t warps = n_windows;
        unsigned grid = grid_for(warps * 32, kThreads);
        if (out_pols == 1)
            detect_warp_kernel<1><<<grid, kThreads, 0, s>>>(src, dst, n_windows, integration);
        else
            detect_warp_kernel<4><<<grid, kThreads, 0, s>>>(src, dst, n_windows, integration);
    }
    return check_launch("blade_detect");
}
