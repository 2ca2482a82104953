// Phasor generation from delays, FP64 with explicit argument reduction.
//
// Reference: src/modules/phasor/ata.cc:176-208 computes, on the host in FP64 for
// every block, phasor = exp(-i 2 pi tau f_idx chanBW) * exp(-i 2 pi tau (obs -
// totalBW/2)) * cal[a, f, p] and writes CF32 into unified memory.  The fringe
// phase reaches ~2 pi * 6e9 Hz * 5 us ~ 2e5 rad, so the phase is reduced in FP64
// before the sine/cosine: turns = tau * (f_idx chanBW) + tau * fringe, and only
// the fractional turn r = turns - rint(turns), |r| <= 1/2, reaches sincospi.
// One thread per (b, a, f) writes both polarisations.
#include "common.cuh"

namespace bb {
namespace {

__global__ void __launch_bounds__(256) phasor_kernel(const double* __restrict__ delays,
                                                     const double2* __restrict__ cal, float2* __restrict__ out,
                                                     uint64_t B, uint64_t A, uint64_t F, uint64_t P, double fringe,
                                                     double chan_bw, uint64_t start) {
    const uint64_t n = B * A * F;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t f = i % F;
        const uint64_t ba = i / F;
        const uint64_t a = ba % A;
        const double tau = delays[ba];
        const double freq = (double)(f + start) * chan_bw;
        double t1 = tau * freq, t2 = tau * fringe;
        // Reduce each product separately (exact in FP64 for the fractional part
        // magnitudes involved) and then their sum.
        t1 -= rint(t1);
        t2 -= rint(t2);
        double r = t1 + t2;
        r -= rint(r);
        double sn, cs;
        sincospi(-2.0 * r, &sn, &cs);  // exp(-i 2 pi r)
        for (uint64_t p = 0; p < P; p++) {
            double2 c = cal ? cal[(a * F + f) * P + p] : make_double2(1.0, 0.0);
            const double re = cs * c.x - sn * c.y;
            const double im = cs * c.y + sn * c.x;
            out[i * P + p] = make_float2((float)re, (float)im);
        }
    }
}

}  // namespace
}  // namespace bb

extern "C" int blade_phasor_from_delays(const double* delays, const void* calibrations, void* phasors, uint64_t B,
                                        uint64_t A, uint64_t F, uint64_t P, double obs_freq_hz, double chan_bw_hz,
                                        double total_bw_hz, uint64_t freq_start_index, blade_stream_t stream) {
    using namespace bb;
    if (B * A * F * P == 0) return BLADE_SUCCESS;
    if (!delays || !phasors) return set_error(BLADE_ERROR, "blade_phasor_from_delays: null buffer");
    const double fringe = obs_freq_hz - total_bw_hz / 2.0;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    phasor_kernel<<<grid_for(B * A * F, 256), 256, 0, s>>>(delays, static_cast<const double2*>(calibrations),
                                                         static_cast<float2*>(phasors), B, A, F, P, fringe,
                                                         chan_bw_hz, freq_start_index);
    return check_launch("blade_phasor_from_delays");
}
