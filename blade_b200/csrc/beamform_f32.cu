// Plain FP32 CUDA-core beamformer (the drop-in) and the fused FP32 chain
// Cast -> Beamformer -> Channelizer(rate 1|2|4) -> Detector (Stokes-I).
//
// Reference: src/modules/beamformer/beamformer.cu:13-79.  There one thread owns one
// time sample, caches all A x P antenna samples in registers and loops over beams
// with the phasors in a static [B][A][P] shared array (so B x A x P is capped by
// the 48 KB static limit, and A = B = 64 does not compile) and the block size is
// capped by the register file at large A.
//
// Here a CTA owns one channel f, a tile of TT = 4 TG consecutive time samples and
// a tile of BT = 4 (256 / TG) beams.  Thread (tg, bg) accumulates a 4 x 4 register
// tile: 4 consecutive time samples x 4 beams x P polarisations.  Antennas stream
// through double-buffered shared memory in chunks of AC = 256 / TG (voltages stored
// time-interleaved so that the per-thread 4-sample reads are bank-conflict free;
// phasors read as broadcasts); the next chunk's global loads are in flight while
// the current chunk is multiplied.  Any A, B, F, T.
//
// The fused chain keeps the beam voltages in registers: the 4 consecutive samples
// of a thread are one rate-4 spectrum (or two rate-2 spectra, or four rate-1
// samples); the (-1)^t fftshift pre-multiply and the DFT are applied in
// registers (their coefficients are +-1, +-i), |.|^2 is summed over both
// polarisations, and the integration window is closed with warp shuffles over
// adjacent lanes.  Nothing but the Stokes-I output touches HBM.
#include "autotune.cuh"
#include "common.cuh"

namespace bb {
namespace {

enum { IN_CF32 = 0, IN_CI8 = 1 };

// Phasor element strides (float2 units) of beam, antenna, channel and
// polarisation: [B, A, F, 1, P] for ATA, (A, 1, 0, 0) for MeerKAT's [B, A] weights
// shared by every channel and polarisation.
struct PhLayout {
    uint64_t sb, sa, sf, sp;
};

inline PhLayout ata_layout(uint64_t A, uint64_t F, uint64_t P) { return PhLayout{A * F * P, F * P, P, 1}; }

__device__ __forceinline__ void cmac(float2& acc, float2 x, float2 w) {
    acc.x = fmaf(x.x, w.x, acc.x);
    acc.x = fmaf(-x.y, w.y, acc.x);
    acc.y = fmaf(x.x, w.y, acc.y);
    acc.y = fmaf(x.y, w.x, acc.y);
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmuli(float2 a) { return make_float2(-a.y, a.x); }  // i * a
__device__ __forceinline__ float pw(float2 a) { return a.x * a.x + a.y * a.y; }

template <int P, int TG, int IN, int R>
__global__ void __launch_bounds__(256, 2) bf32_kernel(const void* __restrict__ vin, const float2* __restrict__ phasors,
                                                   void* __restrict__ vout, uint32_t B, uint32_t A, uint32_t F,
                                                   uint32_t T, uint32_t integ, const PhLayout ph) {
    constexpr int BGN = 256 / TG;
    constexpr int BT = BGN * 4;
    constexpr int TT = TG * 4;
    constexpr int AC = 256 / TG;
    constexpr int XPT = 4;  // samples loaded per thread per chunk: AC * TT / 256 = 4
    static_assert(AC * TT == 1024, "chunk must hold 1024 samples");

    __shared__ __align__(16) float2 xs[2][AC][4][TG][P];
    __shared__ __align__(16) float2 ws[2][AC][BT][P];

    const int tid = threadIdx.x;
    const int tg = tid % TG, bg = tid / TG;
    const uint32_t t0 = blockIdx.x * TT;
    const uint32_t f = blockIdx.y;
    const uint32_t b0 = blockIdx.z * BT;

    // Prefetch registers.
    float2 xr[XPT][P];
    float2 wr[2];

    auto load_chunk = [&](uint32_t a0) {
#pragma unroll
        for (int m = 0; m < XPT; m++) {
            const int s = tid + 256 * m;
            const int al = s / TT, tl = s % TT;
            const uint32_t a = a0 + al, t = t0 + tl;
            if (a < A && t < T) {
                const uint64_t idx = ((uint64_t)(a * (uint64_t)F + f) * T + t) * P;
                if (IN == IN_CF32) {
                    const float2* x = static_cast<const float2*>(vin) + idx;
                    if (P == 2) {
                        float4 v = ldg_nc_f4(x);
                        xr[m][0] = make_float2(v.x, v.y);
                        xr[m][P - 1] = make_float2(v.z, v.w);
                    } else {
                        xr[m][0] = __ldg(x);
                    }
                } else {
                    const char2* x = static_cast<const char2*>(vin) + idx;
                    if (P == 2) {
                        char4 v = __ldg(reinterpret_cast<const char4*>(x));
                        xr[m][0] = make_float2((float)v.x, (float)v.y);
                        xr[m][P - 1] = make_float2((float)v.z, (float)v.w);
                    } else {
                        char2 v = __ldg(x);
                        xr[m][0] = make_float2((float)v.x, (float)v.y);
                    }
                }
            } else {
#pragma unroll
                for (int p = 0; p < P; p++) xr[m][p] = make_float2(0.f, 0.f);
            }
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const int e = tid + 256 * m;  // over AC * BT * P elements (<= 512)
            wr[m] = make_float2(0.f, 0.f);
            if (e < AC * BT * P) {
                const int p = e % P, j = (e / P) % BT, al = e / (P * BT);
                const uint32_t a = a0 + al, b = b0 + j;
                if (a < A && b < B)
                    wr[m] = __ldg(phasors + b * ph.sb + a * ph.sa + (uint64_t)f * ph.sf + (uint64_t)p * ph.sp);
            }
        }
    };
    auto store_chunk = [&](int buf) {
#pragma unroll
        for (int m = 0; m < XPT; m++) {
            const int s = tid + 256 * m;
            const int al = s / TT, tl = s % TT;
#pragma unroll
            for (int p = 0; p < P; p++) xs[buf][al][tl % 4][tl / 4][p] = xr[m][p];
        }
#pragma unroll
        for (int m = 0; m < 2; m++) {
            const int e = tid + 256 * m;
            if (e < AC * BT * P) {
                const int p = e % P, j = (e / P) % BT, al = e / (P * BT);
                ws[buf][al][j][p] = wr[m];
            }
        }
    };

    float2 acc[4][4][P];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int p = 0; p < P; p++) acc[i][j][p] = make_float2(0.f, 0.f);

    const uint32_t nchunks = (A + AC - 1) / AC;
    load_chunk(0);
    store_chunk(0);
    __syncthreads();
    for (uint32_t c = 0; c < nchunks; c++) {
        const int buf = c & 1;
        if (c + 1 < nchunks) load_chunk((c + 1) * AC);
#pragma unroll
        for (int al = 0; al < AC; al++) {
            float2 xv[4][P], wv[4][P];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                if (P == 2) {
                    float4 v = *reinterpret_cast<const float4*>(&xs[buf][al][i][tg][0]);
                    xv[i][0] = make_float2(v.x, v.y);
                    xv[i][P - 1] = make_float2(v.z, v.w);
                } else {
                    xv[i][0] = xs[buf][al][i][tg][0];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                if (P == 2) {
                    float4 v = *reinterpret_cast<const float4*>(&ws[buf][al][bg * 4 + j][0]);
                    wv[j][0] = make_float2(v.x, v.y);
                    wv[j][P - 1] = make_float2(v.z, v.w);
                } else {
                    wv[j][0] = ws[buf][al][bg * 4 + j][0];
                }
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++)
#pragma unroll
                    for (int p = 0; p < P; p++) cmac(acc[i][j][p], xv[i][p], wv[j][p]);
        }
        if (c + 1 < nchunks) store_chunk(buf ^ 1);
        __syncthreads();
    }

    const uint32_t tb = t0 + tg * 4;  // first of this thread's 4 samples
    if constexpr (R == 0) {
        // Beam voltages, CF32 [B, F, T, P].
        float2* out = static_cast<float2*>(vout);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t b = b0 + bg * 4 + j;
            if (b >= B) continue;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t t = tb + i;
                if (t >= T) continue;
                float2* o = out + ((uint64_t)(b * (uint64_t)F + f) * T + t) * P;
                if (P == 2) stg_f4(o, make_float4(acc[i][j][0].x, acc[i][j][0].y, acc[i][j][P - 1].x,
                                                  acc[i][j][P - 1].y));
                else o[0] = acc[i][j][0];
            }
        }
    } else {
        // Stokes-I of the rate-R channelized beams, integrated over `integ` spectra.
        constexpr int NS = 4 / R;  // spectra held by this thread
        float* out = static_cast<float*>(vout);
        const uint32_t U = T / (R * integ);
        const uint32_t s0 = tb / R;  // first spectrum index of this thread
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const uint32_t b = b0 + bg * 4 + j;
            float S[NS][R];
#pragma unroll
            for (int q = 0; q < NS; q++) {
#pragma unroll
                for (int k = 0; k < R; k++) S[q][k] = 0.f;
#pragma unroll
                for (int p = 0; p < P; p++) {
                    if (R == 1) {
                        S[q][0] += pw(acc[q][j][p]);
                    } else if (R == 2) {
                        const float2 y0 = acc[2 * q][j][p], y1 = acc[2 * q + 1][j][p];
                        S[q][0] += pw(csub(y0, y1));
                        S[q][R - 1] += pw(cadd(y0, y1));
                    } else {
                        const float2 y0 = acc[0][j][p], y1 = acc[1][j][p], y2 = acc[2][j][p], y3 = acc[3][j][p];
                        const float2 e02 = cadd(y0, y2), d02 = csub(y0, y2);
                        const float2 e13 = cadd(y1, y3), d13 = csub(y1, y3);
                        S[q][0] += pw(csub(e02, e13));                 // y0 - y1 + y2 - y3
                        S[q][R > 1 ? 1 : 0] += pw(cadd(d02, cmuli(d13)));  // y0 + i y1 - y2 - i y3
                        S[q][R > 2 ? 2 : 0] += pw(cadd(e02, e13));     // y0 + y1 + y2 + y3
                        S[q][R > 3 ? 3 : 0] += pw(csub(d02, cmuli(d13)));  // y0 - i y1 - y2 + i y3
                    }
                }
            }
            if ((uint32_t)NS >= integ) {
                // Whole windows inside the thread.
                const uint32_t nw = NS / integ;
                for (uint32_t v = 0; v < nw; v++) {
#pragma unroll
                    for (int k = 0; k < R; k++) {
                        float sum = 0.f;
                        for (uint32_t q = v * integ; q < (v + 1) * integ; q++) sum += S[q][k];
                        const uint32_t u = s0 / integ + v;
                        if (b < B && u < U) out[((uint64_t)(b * (uint64_t)F + f) * R + k) * U + u] = sum;
                    }
                }
            } else {
                // Window spans g = integ / NS adjacent lanes (power of two <= 32).
                const uint32_t g = integ / NS;
#pragma unroll
                for (int k = 0; k < R; k++) {
                    float sum = 0.f;
#pragma unroll
                    for (int q = 0; q < NS; q++) sum += S[q][k];
                    for (uint32_t o = 1; o < g; o <<= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
                    const uint32_t u = s0 / integ;
                    if ((tg % g) == 0 && b < B && u < U) out[((uint64_t)(b * (uint64_t)F + f) * R + k) * U + u] = sum;
                }
            }
        }
    }
}

// Incoherent beam: out[B, f, t, p] = ([sqrt] sum_a |x[a,f,t,p] w[0,a,f,0,p]|^2, 0)
// (reference src/modules/beamformer/beamformer.cu:64-78).
template <int P>
__global__ void __launch_bounds__(256) incoherent_kernel(const float2* __restrict__ in,
                                                         const float2* __restrict__ phasors, float2* __restrict__ out,
                                                         uint32_t B, uint32_t A, uint32_t F, uint32_t T, int do_sqrt) {
    const uint64_t n = (uint64_t)F * T;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t f = i / T;
        float acc[P];
#pragma unroll
        for (int p = 0; p < P; p++) acc[p] = 0.f;
        for (uint32_t a = 0; a < A; a++) {
#pragma unroll
            for (int p = 0; p < P; p++) {
                const float2 x = in[((uint64_t)a * F * T + i) * P + p];
                const float2 w = phasors[((uint64_t)a * F + f) * P + p];
                const float re = x.x * w.x - x.y * w.y, im = x.x * w.y + x.y * w.x;
                acc[p] += re * re + im * im;
            }
        }
#pragma unroll
        for (int p = 0; p < P; p++)
            out[((uint64_t)B * F * T + i) * P + p] = make_float2(do_sqrt ? sqrtf(acc[p]) : acc[p], 0.f);
    }
}

// Small blocks (the tiled kernel would leave SMs idle): one thread per
// (beam, channel, sample) and both polarisations, antennas in order; the CTA's
// phasors are the same for all its threads and its voltages come from L2 (every
// beam re-reads them).  Same arithmetic as the tiled kernel per output.
template <int P>
__global__ void __launch_bounds__(256) bf32_small_kernel(const float2* __restrict__ in,
                                                         const float2* __restrict__ phasors, float2* __restrict__ out,
                                                         uint32_t A, uint32_t F, uint32_t T, const PhLayout ph) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x, f = blockIdx.y, b = blockIdx.z;
    if (t >= T) return;
    float2 acc[P];
#pragma unroll
    for (int p = 0; p < P; p++) acc[p] = make_float2(0.f, 0.f);
    const float2* x = in + ((uint64_t)f * T + t) * P;
    const float2* w = phasors + b * ph.sb + (uint64_t)f * ph.sf;
    for (uint32_t a = 0; a < A; a++) {
#pragma unroll
        for (int p = 0; p < P; p++) {
            const float2 xv = __ldg(x + (uint64_t)a * F * T * P + p), wv = __ldg(w + a * ph.sa + p * ph.sp);
            acc[p].x = fmaf(xv.x, wv.x, fmaf(-xv.y, wv.y, acc[p].x));
            acc[p].y = fmaf(xv.x, wv.y, fmaf(xv.y, wv.x, acc[p].y));
        }
    }
    float2* o = out + (((uint64_t)b * F + f) * T + t) * P;
#pragma unroll
    for (int p = 0; p < P; p++) o[p] = acc[p];
}

template <int P, int TG, int IN, int R>
void launch_bf(const void* in, const float2* ph, void* out, uint64_t B, uint64_t A, uint64_t F, uint64_t T,
               uint64_t integ, cudaStream_t s, const PhLayout& lay) {
    constexpr int TT = TG * 4, BT = (256 / TG) * 4;
    dim3 grid((unsigned)ceil_div(T, TT), (unsigned)F, (unsigned)ceil_div(B, BT));
    bf32_kernel<P, TG, IN, R><<<grid, 256, 0, s>>>(in, ph, out, (uint32_t)B, (uint32_t)A, (uint32_t)F, (uint32_t)T,
                                                   (uint32_t)integ, lay);
}

int pick_tg(uint64_t B) { return B <= 4 ? 256 : B <= 8 ? 128 : B <= 16 ? 64 : 32; }

template <int P, int IN, int R>
void dispatch_tg(int tg, const void* in, const float2* ph, void* out, uint64_t B, uint64_t A, uint64_t F, uint64_t T,
                 uint64_t integ, cudaStream_t s, const PhLayout& lay) {
    switch (tg) {
        case 256: launch_bf<P, 256, IN, R>(in, ph, out, B, A, F, T, integ, s, lay); break;
        case 128: launch_bf<P, 128, IN, R>(in, ph, out, B, A, F, T, integ, s, lay); break;
        case 64: launch_bf<P, 64, IN, R>(in, ph, out, B, A, F, T, integ, s, lay); break;
        default: launch_bf<P, 32, IN, R>(in, ph, out, B, A, F, T, integ, s, lay); break;
    }
}

bool dims_ok(uint64_t B, uint64_t A, uint64_t F, uint64_t T) {
    return B < (1u << 31) && A < (1u << 31) && F <= 65535 && T < (1u << 31) && ceil_div(B, 4) <= 65535;
}

}  // namespace
}  // namespace bb

namespace bb {
namespace {

// Beams 0..B-1 of the plain FP32 beamformer for a phasor layout (no incoherent beam).
int beamform_f32_beams(const char* who, const void* in, const float2* ph, void* out, uint64_t B, uint64_t A,
                       uint64_t F, uint64_t T, uint64_t P, const PhLayout& lay, cudaStream_t s) {
    if (B == 0) return BLADE_SUCCESS;
    const int tg = pick_tg(B);
    const uint64_t tiles = ceil_div(T, (uint64_t)tg * 4) * F * ceil_div(B, (uint64_t)(256 / tg) * 4);
    if (tiles < 2ull * sm_count() && B <= 65535) {
        const dim3 grid((unsigned)ceil_div(T, 256), (unsigned)F, (unsigned)B);
        if (P == 2)
            bf32_small_kernel<2><<<grid, 256, 0, s>>>(static_cast<const float2*>(in), ph, static_cast<float2*>(out),
                                                      (uint32_t)A, (uint32_t)F, (uint32_t)T, lay);
        else
            bf32_small_kernel<1><<<grid, 256, 0, s>>>(static_cast<const float2*>(in), ph, static_cast<float2*>(out),
                                                      (uint32_t)A, (uint32_t)F, (uint32_t)T, lay);
    } else if (P == 2) {
        dispatch_tg<2, IN_CF32, 0>(tg, in, ph, out, B, A, F, T, 1, s, lay);
    } else {
        dispatch_tg<1, IN_CF32, 0>(tg, in, ph, out, B, A, F, T, 1, s, lay);
    }
    return check_launch(who);
}

int check_f32_args(const char* who, const void* in, const void* phasors, void* out, uint64_t B, uint64_t A,
                   uint64_t F, uint64_t T, uint64_t P) {
    if (P != 1 && P != 2) return set_error(BLADE_ERROR, "%s: P must be 1 or 2", who);
    if (!in || !phasors || !out) return set_error(BLADE_ERROR, "%s: null buffer", who);
    if (!dims_ok(B, A, F, T)) return set_error(BLADE_ERROR, "%s: dimensions out of range", who);
    if (P == 2 && (!aligned16(in) || !aligned16(out)))
        return set_error(BLADE_ERROR, "%s: dual-pol buffers must be 16-byte aligned", who);
    return BLADE_SUCCESS;
}

}  // namespace
}  // namespace bb

extern "C" int blade_beamform_f32(const void* in, const void* phasors, void* out, uint64_t B, uint64_t A, uint64_t F,
                                  uint64_t T, uint64_t P, int incoherent, int incoherent_sqrt, blade_stream_t stream) {
    using namespace bb;
    if (P != 1 && P != 2) return set_error(BLADE_ERROR, "blade_beamform_f32: P must be 1 or 2");
    if (B == 0 && !incoherent) return BLADE_SUCCESS;
    if (A == 0 || F == 0 || T == 0) return BLADE_SUCCESS;
    if (int rc = check_f32_args("blade_beamform_f32", in, phasors, out, B, A, F, T, P)) return rc;
    if (incoherent && B == 0) return set_error(BLADE_ERROR, "blade_beamform_f32: incoherent beam needs beam 0");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const float2* ph = static_cast<const float2*>(phasors);
    if (int rc = beamform_f32_beams("blade_beamform_f32", in, ph, out, B, A, F, T, P, ata_layout(A, F, P), s))
        return rc;
    if (incoherent) {
        if (P == 2)
            incoherent_kernel<2><<<grid_for(F * T, 256), 256, 0, s>>>(static_cast<const float2*>(in), ph,
                                                                     static_cast<float2*>(out), (uint32_t)B,
                                                                     (uint32_t)A, (uint32_t)F, (uint32_t)T,
                                                                     incoherent_sqrt);
        else
            incoherent_kernel<1><<<grid_for(F * T, 256), 256, 0, s>>>(static_cast<const float2*>(in), ph,
                                                                     static_cast<float2*>(out), (uint32_t)B,
                                                                     (uint32_t)A, (uint32_t)F, (uint32_t)T,
                                                                     incoherent_sqrt);
    }
    return check_launch("blade_beamform_f32");
}

extern "C" int blade_beamform_meerkat_f32(const void* in, const void* phasors, void* out, uint64_t B, uint64_t A,
                                          uint64_t F, uint64_t T, uint64_t P, int incoherent, blade_stream_t stream) {
    using namespace bb;
    if (B == 0 && !incoherent) return BLADE_SUCCESS;
    if (A == 0 || F == 0 || T == 0) return BLADE_SUCCESS;
    if (int rc = check_f32_args("blade_beamform_meerkat_f32", in, phasors, out, B, A, F, T, P)) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (int rc = beamform_f32_beams("blade_beamform_meerkat_f32", in, static_cast<const float2*>(phasors), out, B, A,
                                    F, T, P, PhLayout{A, 1, 0, 0}, s))
        return rc;
    if (incoherent) {
        // the reference sizes the incoherent beam but its MeerKAT kernel never writes it
        const cudaError_t e =
            cudaMemsetAsync(static_cast<float2*>(out) + B * F * T * P, 0, F * T * P * sizeof(float2), s);
        if (e != cudaSuccess) return check_cuda(e, "blade_beamform_meerkat_f32");
    }
    return check_launch("blade_beamform_meerkat_f32");
}

namespace bb {

int f32_default_tg(uint64_t B, uint64_t rate, uint64_t integration) {
    int tg = pick_tg(B);
    // The window (rate * integration samples) must tile the CTA's 4 TG samples and
    // span at most one warp of threads.
    while (tg < 256 && (4ull * tg) % (rate * integration) != 0) tg *= 2;
    return tg;
}

bool f32_tg_ok(uint32_t tg, uint64_t B, uint64_t rate, uint64_t integration) {
    return (tg == 32 || tg == 64 || tg == 128 || tg == 256) && (4ull * tg) % (rate * integration) == 0 &&
           ceil_div(B, 1024 / tg) <= 65535;
}

// TG of a fused FP32 launch: the tuned width for this shape on this device when
// blade_beamform_detect_f32_autotune stored one, else the default.
int f32_tg(uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t rate, uint64_t integration, int in_type,
           bool* tuned = nullptr, TuneEntry* entry = nullptr) {
    int tg = f32_default_tg(B, rate, integration);
    if (tuned) *tuned = false;
    const uint64_t key[8] = {B, A, F, T, 2, rate, integration, (uint64_t)in_type};
    TuneEntry e;
    if (tune_lookup(BLADE_TUNE_F32, key, &e) && f32_tg_ok(e.params[0], B, rate, integration)) {
        tg = (int)e.params[0];
        if (tuned) *tuned = true;
        if (entry) *entry = e;
    }
    return tg;
}

void f32_launch(int in_type, int tg, const void* in, const float2* ph, void* out, uint64_t B, uint64_t A, uint64_t F,
                uint64_t T, uint64_t rate, uint64_t integration, cudaStream_t s) {
    const PhLayout lay = ata_layout(A, F, 2);
    if (in_type == BLADE_CI8) {
        if (rate == 1) dispatch_tg<2, IN_CI8, 1>(tg, in, ph, out, B, A, F, T, integration, s, lay);
        else if (rate == 2) dispatch_tg<2, IN_CI8, 2>(tg, in, ph, out, B, A, F, T, integration, s, lay);
        else dispatch_tg<2, IN_CI8, 4>(tg, in, ph, out, B, A, F, T, integration, s, lay);
    } else {
        if (rate == 1) dispatch_tg<2, IN_CF32, 1>(tg, in, ph, out, B, A, F, T, integration, s, lay);
        else if (rate == 2) dispatch_tg<2, IN_CF32, 2>(tg, in, ph, out, B, A, F, T, integration, s, lay);
        else dispatch_tg<2, IN_CF32, 4>(tg, in, ph, out, B, A, F, T, integration, s, lay);
    }
}

int f32_query(const uint64_t (&shape)[8], uint32_t* params, float* us, int* tuned) {
    bool t = false;
    TuneEntry e;
    const int tg = f32_tg(shape[0], shape[1], shape[2], shape[3], shape[5], shape[6], (int)shape[7], &t, &e);
    for (int i = 0; i < kTuneParams; i++) params[i] = t ? e.params[i] : 0u;
    params[0] = (uint32_t)tg;
    *us = t ? e.us : 0.f;
    *tuned = t ? 1 : 0;
    return BLADE_SUCCESS;
}

}  // namespace bb

extern "C" int blade_beamform_detect_f32(int in_type, const void* in, const void* phasors, void* out, uint64_t B,
                                         uint64_t A, uint64_t F, uint64_t T, uint64_t P, uint64_t rate,
                                         uint64_t integration, blade_stream_t stream) {
    using namespace bb;
    if (P != 2) return set_error(BLADE_ERROR, "blade_beamform_detect_f32: P must be 2 (Stokes-I detector)");
    if (rate != 1 && rate != 2 && rate != 4)
        return set_error(BLADE_ERROR, "blade_beamform_detect_f32: rate must be 1, 2 or 4");
    if (integration == 0) return set_error(BLADE_ERROR, "blade_beamform_detect_f32: integration must be > 0");
    if (T % (rate * integration) != 0)
        return set_error(BLADE_ERROR, "blade_beamform_detect_f32: T must be a multiple of rate * integration");
    if (in_type != BLADE_CF32 && in_type != BLADE_CI8)
        return set_error(BLADE_ERROR, "blade_beamform_detect_f32: input type must be CF32 or CI8");
    if (B == 0 || A == 0 || F == 0 || T == 0) return BLADE_SUCCESS;
    if (!in || !phasors || !out) return set_error(BLADE_ERROR, "blade_beamform_detect_f32: null buffer");
    if (!dims_ok(B, A, F, T)) return set_error(BLADE_ERROR, "blade_beamform_detect_f32: dimensions out of range");
    const uint64_t ns = 4 / rate;  // spectra per thread
    const int tg = f32_tg(B, A, F, T, rate, integration, in_type);
    if ((4ull * tg) % (rate * integration) != 0)
        return set_error(BLADE_ERROR, "blade_beamform_detect_f32: rate * integration must divide %d", 4 * tg);
    if (integration > ns) {
        const uint64_t g = integration / ns;
        if (integration % ns != 0 || (g & (g - 1)) != 0 || g > 32)
            return set_error(BLADE_ERROR, "blade_beamform_detect_f32: integration %llu not supported at rate %llu",
                             (unsigned long long)integration, (unsigned long long)rate);
    } else if (ns % integration != 0) {
        return set_error(BLADE_ERROR, "blade_beamform_detect_f32: integration must divide %llu",
                         (unsigned long long)ns);
    }
    if (in_type == BLADE_CF32 && !aligned16(in))
        return set_error(BLADE_ERROR, "blade_beamform_detect_f32: CF32 input must be 16-byte aligned");
    if (in_type == BLADE_CI8 && (reinterpret_cast<uintptr_t>(in) & 3))
        return set_error(BLADE_ERROR, "blade_beamform_detect_f32: CI8 input must be 4-byte aligned");
    f32_launch(in_type, tg, in, static_cast<const float2*>(phasors), out, B, A, F, T, rate, integration,
               reinterpret_cast<cudaStream_t>(stream));
    return check_launch("blade_beamform_detect_f32");
}

extern "C" int blade_beamform_detect_f32_autotune(int in_type, uint64_t B, uint64_t A, uint64_t F, uint64_t T,
                                                  uint64_t P, uint64_t rate, uint64_t integration,
                                                  blade_stream_t stream) {
    using namespace bb;
    const char* who = "blade_beamform_detect_f32_autotune";
    if (P != 2 || (rate != 1 && rate != 2 && rate != 4) || integration == 0 || T % (rate * integration) != 0 ||
        (in_type != BLADE_CF32 && in_type != BLADE_CI8) || B == 0 || A == 0 || F == 0 || T == 0 ||
        !dims_ok(B, A, F, T))
        return set_error(BLADE_ERROR, "%s: unsupported configuration", who);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const size_t n = (size_t)A * F * T * P;  // complex samples
    const size_t in_bytes = n * (in_type == BLADE_CI8 ? 2 : 8), ph_count = (size_t)B * A * F * P;
    const size_t out_bytes = (size_t)B * F * rate * (T / (rate * integration)) * sizeof(float);
    std::vector<void*> bufs;
    auto get = [&](size_t bytes) {
        void* q = nullptr;
        if (cudaMalloc(&q, bytes < 16 ? 16 : bytes) != cudaSuccess) return (void*)nullptr;
        bufs.push_back(q);
        return q;
    };
    struct Free {
        std::vector<void*>& b;
        ~Free() {
            for (void* q : b) cudaFree(q);
        }
    } release{bufs};
    void* in = get(in_bytes);
    void* ph = get(ph_count * sizeof(float2));
    void* ref = get(out_bytes);
    void* out = get(out_bytes);
    if (!in || !ph || !ref || !out) return set_error(BLADE_CUDA_ERROR, "%s: allocation failed", who);
    if (in_type == BLADE_CI8) {
        if (int rc = tune_fill_ci8(in, in_bytes, st)) return rc;
    } else {
        if (int rc = tune_fill_phasors(in, n, st)) return rc;  // unit-modulus samples serve as CF32 voltages
    }
    if (int rc = tune_fill_phasors(ph, ph_count, st)) return rc;
    // the public entry validates the configuration (window and rate rules)
    if (int rc = blade_beamform_detect_f32(in_type, in, ph, ref, B, A, F, T, P, rate, integration, stream)) return rc;
    const int def = f32_default_tg(B, rate, integration);
    std::vector<int> cands{def};
    for (int tg : {32, 64, 128, 256})
        if (tg != def && f32_tg_ok((uint32_t)tg, B, rate, integration)) cands.push_back(tg);
    int best = -1;
    float best_us = 0.f;
    uint32_t ndiff = 0, ntimed = 0;
    for (size_t i = 0; i < cands.size(); i++) {
        void* dst = i == 0 ? ref : out;
        const float us = tune_time(
            [&]() {
                f32_launch(in_type, cands[i], in, static_cast<const float2*>(ph), dst, B, A, F, T, rate, integration,
                           st);
                return check_launch(who);
            },
            st);
        if (us < 0.f) return set_error(BLADE_CUDA_ERROR, "%s: candidate TG=%d failed: %s", who, cands[i],
                                       blade_last_error());
        ntimed++;
        if (i > 0 && !tune_same(ref, out, out_bytes)) {
            ndiff++;
            continue;
        }
        if (best < 0 || us < best_us) {
            best = (int)i;
            best_us = us;
        }
    }
    TuneEntry e = {};
    e.params[0] = (uint32_t)cands[best];
    e.params[4] = ntimed;
    e.params[5] = ndiff;
    e.us = best_us;
    const uint64_t key[8] = {B, A, F, T, P, rate, integration, (uint64_t)in_type};
    tune_store(BLADE_TUNE_F32, key, e);
    return BLADE_SUCCESS;
}
