// Test-only checker: the reference's own CUDA kernels, compiled from the
// reference sources where they lie (see build.sh), instantiated at the fixed
// shapes of the golden fixtures and exposed through extern "C" launchers.
// Nothing in blade_b200 links or loads this library.
//
// Kernels: src/modules/cast/cast.cu (cast), src/modules/beamformer/beamformer.cu
// (ATA), src/modules/detector/detector.cu (detector_1pol, detector_4pol),
// src/modules/channelizer/channelizer.cu (pre_channelizer) + cuFFT, launched with
// the grids the reference modules compute (cast/base.cc:27-31,
// beamformer/ata.cc:51-53, detector/base.cc:53-69, channelizer/base.cc:59-112).
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include "src/modules/cast/cast.cu"
#include "src/modules/beamformer/beamformer.cu"
#include "src/modules/detector/detector.cu"
#include "src/modules/channelizer/channelizer.cu"

#include "golden_shapes.h"

static int finish() {
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return (int)e;
}

extern "C" int ref_cast_ci8_cf32(const void* in, void* out) {
    constexpr uint64_t N = G_CAST_N * 2;  // scalars
    cast<int8_t, float, N><<<(N + 511) / 512, 512>>>((const int8_t*)in, (float*)out);
    return finish();
}

extern "C" int ref_beamformer(const void* in, const void* ph, void* out) {
    ATA<G_BF_B, G_BF_A, G_BF_F, G_BF_T, 2, G_BF_TBLOCK, true, true>
        <<<dim3(G_BF_F, G_BF_T / G_BF_TBLOCK), G_BF_TBLOCK>>>((const cuFloatComplex*)in,
                                                              (const cuFloatComplex*)ph, (cuFloatComplex*)out);
    return finish();
}

extern "C" int ref_beamformer_plain(const void* in, const void* ph, void* out) {
    ATA<G_BF_B, G_BF_A, G_BF_F, G_BF_T, 2, G_BF_TBLOCK, false, false>
        <<<dim3(G_BF_F, G_BF_T / G_BF_TBLOCK), G_BF_TBLOCK>>>((const cuFloatComplex*)in,
                                                              (const cuFloatComplex*)ph, (cuFloatComplex*)out);
    return finish();
}

extern "C" int ref_detector(const void* in, void* out1, void* out4) {
    constexpr uint64_t N = G_DET_A * G_DET_F * G_DET_T;
    detector_1pol<N, G_DET_I><<<(N + 511) / 512, 512>>>((const cuFloatComplex*)in, (float*)out1);
    int rc = finish();
    if (rc) return rc;
    detector_4pol<N, G_DET_I><<<(N + 511) / 512, 512>>>((const cuFloatComplex*)in, (float*)out4);
    return finish();
}

// Channelizer with rate == T, in place, as Modules::Channelizer::process does.
extern "C" int ref_channelizer(void* buf) {
    constexpr uint64_t P = 2, N = G_CH_A * G_CH_F * G_CH_T * P;
    pre_channelizer<P * 2, P, N><<<(N + 511) / 512, 512>>>((const cuFloatComplex*)buf, (cuFloatComplex*)buf);
    int rc = finish();
    if (rc) return rc;
    cufftHandle plan;
    int n[] = {(int)G_CH_T};
    int inembed[] = {0}, onembed[] = {0};
    int batch = (int)(N / P / G_CH_T);
    if (cufftPlanMany(&plan, 1, n, inembed, (int)P, (int)(G_CH_T * P), onembed, (int)P, (int)(G_CH_T * P),
                      CUFFT_C2C, batch) != CUFFT_SUCCESS)
        return -1;
    for (uint64_t p = 0; p < P; p++) {
        cufftComplex* ptr = reinterpret_cast<cufftComplex*>(buf) + p;
        if (cufftExecC2C(plan, ptr, ptr, CUFFT_FORWARD) != CUFFT_SUCCESS) {
            cufftDestroy(plan);
            return -2;
        }
    }
    rc = finish();
    cufftDestroy(plan);
    return rc;
}
