// Adjoint of beamform + Stokes-I detect with respect to the complex weights.
// No reference counterpart (the reference has no differentiation).
//
// L = -sum_{b,f,t,p} |y[b,f,t,p]|^2,  y[b,f,t,p] = sum_a x[a,f,t,p] w[b,a,f,0,p]
// dL/d conj(w[b,a,f,0,p]) = -sum_t y[b,f,t,p] conj(x[a,f,t,p])
// (detector integration windows do not change the sum, so they drop out).
//
// Main path (P = 2, B A <= 1024): one CTA owns one channel f and one chunk of the
// time axis (as many chunks as fill the resident CTA slots once), both polarisations.  It walks its
// chunk in tiles of 128 samples: the tile's voltages are staged in shared memory
// with 16-byte loads (all of a thread's loads of a tile in flight together) (both polarisations of a sample at once, rows padded so that
// the per-antenna reads of the gradient pass do not share banks), the beam
// voltages y are recomputed for the tile (never stored to HBM), and each thread
// accumulates y conj(x) for its (beam, antenna) pairs over its slice of every tile
// in registers.  The slices are added in a fixed order at the end, the chunks by a
// second kernel and the loss by a third, so results are deterministic.  HBM traffic
// is one read of the voltages.  One beam (B = 1, A <= 32) takes a kernel without
// shared-memory staging (adjoint_b1_kernel); other shapes the one-CTA-per-(f, p)
// kernel.
#include <mutex>

#include "common.cuh"
#include "tc_ptx.cuh"

namespace bb {
namespace {

constexpr int kT = 256;  // time samples per tile == threads per CTA

__global__ void __launch_bounds__(kT) adjoint_kernel(const float2* __restrict__ x, const float2* __restrict__ w,
                                                     float2* __restrict__ grad, double* __restrict__ loss, uint32_t B,
                                                     uint32_t A, uint32_t F, uint32_t T, uint32_t P) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // Layout: ws[B*A] | xs[A*kT] | ys[B*kT] | gacc[B*A] | red[kT] (float2) | lred[kT] (double)
    float2* ws = reinterpret_cast<float2*>(smem_raw);
    float2* xs = ws + (size_t)B * A;
    float2* ys = xs + (size_t)A * kT;
    float2* gacc = ys + (size_t)B * kT;
    float2* red = gacc + (size_t)B * A;
    double* lred = reinterpret_cast<double*>(red + kT);

    const uint32_t fp = blockIdx.x;
    const uint32_t f = fp / P, p = fp % P;
    const int tid = threadIdx.x;
    const uint32_t Q = B * A;

    for (uint32_t q = tid; q < Q; q += kT) {
        const uint32_t b = q / A, a = q % A;
        ws[q] = w[((uint64_t)(b * (uint64_t)A + a) * F + f) * P + p];
        gacc[q] = make_float2(0.f, 0.f);
    }
    double lsum = 0.0;
    // Thread split of the pair reduction: S slices of the tile per pair.
    const uint32_t S = Q >= kT ? 1 : kT / Q;
    const uint32_t span = (kT + S - 1) / S;  // the S slices cover every sample of the tile
    __syncthreads();

    for (uint32_t t0 = 0; t0 < T; t0 += kT) {
        const uint32_t nt = min((uint32_t)kT, T - t0);
        // Stage x[:, f, t0 + t, p].
        for (uint32_t e = tid; e < A * kT; e += kT) {
            const uint32_t a = e / kT, t = e % kT;
            xs[e] = (t < nt) ? x[(((uint64_t)a * F + f) * T + t0 + t) * P + p] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        // Recompute y for this tile; thread = time sample.
        float lt = 0.f;
        for (uint32_t b = 0; b < B; b++) {
            float2 acc = make_float2(0.f, 0.f);
            for (uint32_t a = 0; a < A; a++) {
                const float2 xv = xs[a * kT + tid], wv = ws[b * A + a];
                acc.x = fmaf(xv.x, wv.x, acc.x);
                acc.x = fmaf(-xv.y, wv.y, acc.x);
                acc.y = fmaf(xv.x, wv.y, acc.y);
                acc.y = fmaf(xv.y, wv.x, acc.y);
            }
            ys[b * kT + tid] = acc;
            lt += acc.x * acc.x + acc.y * acc.y;
        }
        lsum += (double)lt;
        __syncthreads();
        // g[b, a] += sum_t y_b(t) conj(x_a(t)).
        for (uint32_t q0 = 0; q0 < Q; q0 += (Q >= kT ? kT : Q)) {
            const uint32_t q = q0 + (tid % (Q >= kT ? kT : Q));
            const uint32_t sl = (Q >= kT) ? 0 : tid / Q;
            float2 part = make_float2(0.f, 0.f);
            if (q < Q && sl < S) {
                const uint32_t b = q / A, a = q % A;
                const uint32_t t_end = min((sl + 1) * span, (uint32_t)kT);
                for (uint32_t t = sl * span; t < t_end; t++) {
                    const float2 yv = ys[b * kT + t], xv = xs[a * kT + t];
                    part.x = fmaf(yv.x, xv.x, part.x);
                    part.x = fmaf(yv.y, xv.y, part.x);
                    part.y = fmaf(yv.y, xv.x, part.y);
                    part.y = fmaf(-yv.x, xv.y, part.y);
                }
            }
            red[tid] = part;
            __syncthreads();
            if (Q >= kT) {
                if (q < Q) gacc[q] = make_float2(gacc[q].x + red[tid].x, gacc[q].y + red[tid].y);
            } else if (tid < (int)Q) {
                float2 s = gacc[tid];
                for (uint32_t k = 0; k < S; k++) {
                    s.x += red[k * Q + tid].x;
                    s.y += red[k * Q + tid].y;
                }
                gacc[tid] = s;
            }
            __syncthreads();
        }
    }
    for (uint32_t q = tid; q < Q; q += kT) {
        const uint32_t b = q / A, a = q % A;
        const float2 g = gacc[q];
        grad[((uint64_t)(b * (uint64_t)A + a) * F + f) * P + p] = make_float2(-g.x, -g.y);
    }
    if (loss) {
        lred[tid] = lsum;
        __syncthreads();
        for (int s = kT / 2; s > 0; s >>= 1) {
            if (tid < s) lred[tid] += lred[tid + s];
            __syncthreads();
        }
        if (tid == 0) loss[fp] = lred[0];  // partial sum of |y|^2 (loss_sum_kernel negates the total)
    }
}


constexpr int kTA = 128;          // samples per tile == threads per CTA (main path)
constexpr uint32_t kMaxPairs = 1024;

__device__ __forceinline__ float4 cmac2(float4 acc, float4 y, float4 x) {
    // acc += (y0 conj x0, y1 conj x1) for the two polarisations packed in float4
    acc.x = fmaf(y.x, x.x, fmaf(y.y, x.y, acc.x));
    acc.y = fmaf(y.y, x.x, fmaf(-y.x, x.y, acc.y));
    acc.z = fmaf(y.z, x.z, fmaf(y.w, x.w, acc.z));
    acc.w = fmaf(y.w, x.z, fmaf(-y.z, x.w, acc.w));
    return acc;
}

// grid = F * nch; gpart[(f * nch + c) * Q + q] (float4: both polarisations),
// lpart[f * nch + c].  NACC = accumulators per thread when Q > kTA.
template <int NACC>
__global__ void __launch_bounds__(kTA) adjoint_chunk_kernel(const float4* __restrict__ x, const float2* __restrict__ w,
                                                            float4* __restrict__ gpart, double* __restrict__ lpart,
                                                            uint32_t B, uint32_t A, uint32_t F, uint32_t T,
                                                            uint32_t nch, uint32_t tiles_per_chunk) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t Q = B * A, ld = kTA + 1;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);  // tile arrival (bulk copies)
    float4* ws = reinterpret_cast<float4*>(smem_raw + 16);  // [Q] (w pol 0, w pol 1)
    float4* xs = ws + Q;                              // [A][ld]
    float4* ys = xs + (size_t)A * ld;                 // [B][kTA]
    float4* red = ys + (size_t)B * kTA;               // [kTA]
    double* lred = reinterpret_cast<double*>(red + kTA);
    const uint32_t f = blockIdx.x / nch, c = blockIdx.x - f * nch;
    const uint32_t tid = threadIdx.x;
    if (tid == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_mbar_init();
    }
    for (uint32_t q = tid; q < Q; q += kTA) {
        const uint32_t b = q / A, a = q - b * A;
        const uint64_t wi = ((uint64_t)(b * (uint64_t)A + a) * F + f) * 2;
        const float2 w0 = w[wi], w1 = w[wi + 1];
        ws[q] = make_float4(w0.x, w0.y, w1.x, w1.y);
    }
    // Pair / slice ownership: Q < kTA -> S = kTA / Q slices of the tile per pair;
    // else one slice, pairs tid, tid + kTA, ...
    const uint32_t S = Q < kTA ? kTA / Q : 1u;
    const uint32_t span = (kTA + S - 1) / S;  // the S slices cover every sample of the tile
    const uint32_t sl = Q < kTA ? tid / Q : 0u;
    const uint32_t q0 = Q < kTA ? tid - sl * Q : tid;
    const bool sl_ok = sl < S;
    float4 acc[NACC];
#pragma unroll
    for (int k = 0; k < NACC; k++) acc[k] = make_float4(0.f, 0.f, 0.f, 0.f);
    double lsum = 0.0;
    const float4* xf = x + (uint64_t)f * T;  // x[a][f][t] float4 = both polarisations
    const uint32_t tile0 = c * tiles_per_chunk;
    const uint32_t ntiles = (T + kTA - 1) / kTA;
    const uint32_t tile1 = min(ntiles, tile0 + tiles_per_chunk);
    __syncthreads();
    volatile int never = 0;
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = tile0; tile < tile1 && ok; tile++) {
        const uint32_t t0 = tile * kTA;
        const uint32_t nt = min((uint32_t)kTA, T - t0);
        // stage x[a][f][t0 .. t0 + nt) for every antenna with one bulk copy per antenna
        // row (16 bytes per sample, all rows in flight together); samples past T read 0
        if (tid == 0) {
            tc::fence_proxy_async_smem();  // the previous tile's reads of xs come first
            tc::mbar_arrive_expect_tx(bar, A * nt * 16u);
            for (uint32_t a = 0; a < A; a++)
                tc::bulk_g2s(xs + a * ld, xf + (uint64_t)a * F * T + t0, nt * 16u, bar);
        }
        if (nt < (uint32_t)kTA)
            for (uint32_t a = 0; a < A; a++)
                if (tid >= nt) xs[a * ld + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
        ok = tc::mbar_wait(bar, phase, &never, 2000000000ll);
        phase ^= 1u;
        __syncthreads();
        if (!__syncthreads_and(ok)) {
            ok = false;
            break;
        }
        // beam voltages of sample tid, both polarisations
        float lt = 0.f;
        for (uint32_t b = 0; b < B; b++) {
            float4 yv = make_float4(0.f, 0.f, 0.f, 0.f);
            for (uint32_t a = 0; a < A; a++) {
                const float4 xv = xs[a * ld + tid], wv = ws[b * A + a];
                yv.x = fmaf(xv.x, wv.x, fmaf(-xv.y, wv.y, yv.x));
                yv.y = fmaf(xv.x, wv.y, fmaf(xv.y, wv.x, yv.y));
                yv.z = fmaf(xv.z, wv.z, fmaf(-xv.w, wv.w, yv.z));
                yv.w = fmaf(xv.z, wv.w, fmaf(xv.w, wv.z, yv.w));
            }
            ys[b * kTA + tid] = yv;
            lt += yv.x * yv.x + yv.y * yv.y + yv.z * yv.z + yv.w * yv.w;
        }
        lsum += (double)lt;
        __syncthreads();
        // g[b, a] += sum over this thread's slice of y_b conj(x_a)
        if (sl_ok) {
#pragma unroll
            for (int k = 0; k < NACC; k++) {
                const uint32_t q = q0 + k * kTA;
                if (q < Q) {
                    const uint32_t b = q / A, a = q - b * A;
                    const uint32_t t_beg = sl * span, t_end = min(t_beg + span, (uint32_t)kTA);
                    const float4* yr = ys + b * kTA;
                    const float4* xr = xs + a * ld;
                    float4 s4 = acc[k];
                    for (uint32_t t = t_beg; t < t_end; t++) s4 = cmac2(s4, yr[t], xr[t]);
                    acc[k] = s4;
                }
            }
        }
        __syncthreads();
    }
    // slices -> pairs in a fixed order
    if (Q < kTA) {
        red[tid] = acc[0];
        __syncthreads();
        if (tid < Q) {
            float4 g = red[tid];
            for (uint32_t k = 1; k < S; k++) {
                const float4 r = red[k * Q + tid];
                g.x += r.x; g.y += r.y; g.z += r.z; g.w += r.w;
            }
            gpart[(uint64_t)blockIdx.x * Q + tid] = g;
        }
    } else {
#pragma unroll
        for (int k = 0; k < NACC; k++) {
            const uint32_t q = q0 + k * kTA;
            if (q < Q) gpart[(uint64_t)blockIdx.x * Q + q] = acc[k];
        }
    }
    lred[tid] = lsum;
    __syncthreads();
    for (uint32_t s = kTA / 2; s > 0; s >>= 1) {
        if (tid < s) lred[tid] += lred[tid + s];
        __syncthreads();
    }
    if (tid == 0) lpart[blockIdx.x] = lred[0];
}

// grad[b, a, f, 0, p] = -sum_c gpart[f, c, q][p], one thread per (f, q)
__global__ void adjoint_chunks_kernel(const float4* __restrict__ gpart, float2* __restrict__ grad, uint32_t B,
                                      uint32_t A, uint32_t F, uint32_t nch) {
    const uint32_t Q = B * A;
    const uint64_t n = (uint64_t)F * Q;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t f = (uint32_t)(i / Q), q = (uint32_t)(i - (uint64_t)f * Q);
        float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t c = 0; c < nch; c++) {
            const float4 r = gpart[((uint64_t)f * nch + c) * Q + q];
            g.x += r.x; g.y += r.y; g.z += r.z; g.w += r.w;
        }
        const uint32_t b = q / A, a = q - b * A;
        const uint64_t gi = ((uint64_t)(b * (uint64_t)A + a) * F + f) * 2;
        grad[gi] = make_float2(-g.x, -g.y);
        grad[gi + 1] = make_float2(-g.z, -g.w);
    }
}

// loss = -sum of the n partials, fixed-order tree in one CTA
__global__ void __launch_bounds__(256) loss_sum_kernel(const double* __restrict__ part, uint32_t n,
                                                       double* __restrict__ loss) {
    __shared__ double sh[256];
    double v = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += 256) v += part[i];
    sh[threadIdx.x] = v;
    __syncthreads();
    for (uint32_t s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = -sh[0];
}

// ---- one beam (the calibration shape: B = 1, P = 2, A <= 32) -------------------
// No shared-memory staging: four threads share a sample, thread g of the group
// owning antennas a = g + 4 i (i < NA); each loads its voltages with 16-byte loads
// (both polarisations), multiplies them by its phasors (held in registers), the
// group adds its four partial beam voltages with two lane shuffles, and every
// thread accumulates y conj(x_a) for its own antennas in registers across the
// chunk.  The CTA's 64 sample lanes are reduced once at the end (lane shuffles,
// then the eight warps in a fixed order) into the same per-chunk partials as the
// shared-memory kernel above, which the two reduction kernels add in a fixed order.
// One read of the voltages is the only HBM traffic, and no barrier sits between a
// round's loads and its arithmetic.
constexpr int kB1Threads = 256;       // 64 samples x 4 antenna groups
constexpr uint32_t kB1Samples = 512;  // samples per CTA (chunk)

template <int NA>
__global__ void __launch_bounds__(kB1Threads) adjoint_b1_kernel(const float4* __restrict__ x,
                                                                const float2* __restrict__ w,
                                                                float4* __restrict__ gpart, double* __restrict__ lpart,
                                                                uint32_t A, uint32_t F, uint32_t T, uint32_t nch) {
    constexpr uint32_t kWarps = kB1Threads / 32;
    __shared__ float4 red[kWarps][4][NA];
    __shared__ double lred[kB1Threads];
    const uint32_t f = blockIdx.x / nch, c = blockIdx.x - f * nch;
    const uint32_t tid = threadIdx.x, g = tid & 3u, sl = tid >> 2, lane = tid & 31u, warp = tid >> 5;
    float4 wr[NA], acc[NA];
#pragma unroll
    for (int i = 0; i < NA; i++) {
        const uint32_t a = g + 4u * i;
        wr[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (a < A) {
            const float2 w0 = w[((uint64_t)a * F + f) * 2], w1 = w[((uint64_t)a * F + f) * 2 + 1];
            wr[i] = make_float4(w0.x, w0.y, w1.x, w1.y);
        }
        acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    double lsum = 0.0;
    const uint32_t t_beg = c * kB1Samples, t_end = min(T, t_beg + kB1Samples);
    const float4* xf = x + (uint64_t)f * T;  // x[a][f][t] float4 = both polarisations
    const uint64_t astride = (uint64_t)F * T;
    // every lane runs the same number of rounds (the shuffles need the whole warp);
    // samples past the chunk read zeros and contribute nothing
    for (uint32_t t0 = t_beg; t0 < t_end; t0 += kB1Threads / 4) {
        const uint32_t t = t0 + sl;
        float4 xv[NA];
#pragma unroll
        for (int i = 0; i < NA; i++) {
            const uint32_t a = g + 4u * i;
            xv[i] = (t < t_end && a < A) ? __ldg(xf + a * astride + t) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        float4 yv = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int i = 0; i < NA; i++) {
            const float4 xa = xv[i], wv = wr[i];
            yv.x = fmaf(xa.x, wv.x, fmaf(-xa.y, wv.y, yv.x));
            yv.y = fmaf(xa.x, wv.y, fmaf(xa.y, wv.x, yv.y));
            yv.z = fmaf(xa.z, wv.z, fmaf(-xa.w, wv.w, yv.z));
            yv.w = fmaf(xa.z, wv.w, fmaf(xa.w, wv.z, yv.w));
        }
#pragma unroll
        for (uint32_t m = 1; m <= 2; m <<= 1) {
            yv.x += __shfl_xor_sync(0xffffffffu, yv.x, m);
            yv.y += __shfl_xor_sync(0xffffffffu, yv.y, m);
            yv.z += __shfl_xor_sync(0xffffffffu, yv.z, m);
            yv.w += __shfl_xor_sync(0xffffffffu, yv.w, m);
        }
        if (g == 0) lsum += (double)(yv.x * yv.x + yv.y * yv.y + yv.z * yv.z + yv.w * yv.w);
#pragma unroll
        for (int i = 0; i < NA; i++) acc[i] = cmac2(acc[i], yv, xv[i]);
    }
    // the warp's eight sample lanes of each antenna group, then the warps in order
#pragma unroll
    for (int i = 0; i < NA; i++) {
#pragma unroll
        for (uint32_t m = 4; m < 32; m <<= 1) {
            acc[i].x += __shfl_xor_sync(0xffffffffu, acc[i].x, m);
            acc[i].y += __shfl_xor_sync(0xffffffffu, acc[i].y, m);
            acc[i].z += __shfl_xor_sync(0xffffffffu, acc[i].z, m);
            acc[i].w += __shfl_xor_sync(0xffffffffu, acc[i].w, m);
        }
        if (lane < 4) red[warp][g][i] = acc[i];
    }
    lred[tid] = lsum;
    __syncthreads();
    if (tid < A) {
        const uint32_t ga = tid & 3u, ia = tid >> 2;
        float4 s = red[0][ga][ia];
        for (uint32_t k = 1; k < kWarps; k++) {
            const float4 r = red[k][ga][ia];
            s.x += r.x; s.y += r.y; s.z += r.z; s.w += r.w;
        }
        gpart[(uint64_t)blockIdx.x * A + tid] = s;
    }
    for (uint32_t s2 = kB1Threads / 2; s2 > 0; s2 >>= 1) {
        if (tid < s2) lred[tid] += lred[tid + s2];
        __syncthreads();
    }
    if (tid == 0) lpart[blockIdx.x] = lred[0];
}

// ---- tensor-core path (P = 2, A <= 32, B <= 32, T a multiple of 128) ----------
// Per CTA one channel f and one chunk of 128-sample tiles, both polarisations; the
// phases of a tile run in order, separated by barriers:
//  1. every thread converts its voltages (loaded during the previous tile's
//     gradient MMAs) into FP16 hi/lo pairs and stores two operand forms:
//       XF[p][h]  128 rows (sample s) x K = [Re x | Im x] of 32 antennas,
//       XG[h]     128 rows m = 64 p + 2 a + c (c = 0: Re, 1: Im) x K = 128 samples,
//     both K-major with the 128-byte swizzle;
//  2. one thread issues the forward y = x w per polarisation against the hi/lo
//     phasor image of blade_beamform_tc_prepare (its stacked layout: hi and lo
//     products side by side along N) for x hi and for x lo, FP32 accumulators in
//     tensor memory;
//  3. warps 0-3 (lane = sample) read y = hi + lo, add |y|^2 to the loss, split y into
//     FP16 hi/lo and store YG[h]: 4 NB rows n = 2 NB p + NB c + b x K = 128 samples;
//  4. one thread issues G += XG YG^T for the four (x, y) hi/lo combinations: M = 128
//     rows (both polarisations), N = 4 NB, K = 128, accumulated over the chunk in
//     tensor memory (the cross-polarisation blocks are computed and never read).
// At the end lanes 2 a and 2 a + 1 of warp quarter p hold, for every beam, the four
// real products of (Re x_a, Im x_a) with (Re y_b, Im y_b); one lane shuffle gives
//   Re G = Re x . Re y + Im x . Im y,   Im G = Re x . Im y - Im x . Re y,
// and G = sum_t y conj(x) per chunk goes to the partial sums that the two reduction
// kernels above add in a fixed order.  The phases wait on tcgen05 commits with
// bounded waits; on expiry the kernel records a status and returns.
constexpr int kTcThreads = 256;
constexpr uint32_t kTcKA = 32;
constexpr long long kTcBudget = 2000000000ll;

struct AdjTcArgs {
    const float4* x;      // [A][F][T] (p0 re, p0 im, p1 re, p1 im)
    const uint8_t* plan;  // phasor images, img_bytes per channel
    float4* gpart;        // [gridDim.x][B A]
    double* lpart;        // [gridDim.x]
    uint32_t A, B, F, T, NB, img_bytes, nch, tiles_per_chunk;
};

__device__ unsigned int g_adj_status = 0;

__device__ __forceinline__ uint32_t split_pair(float v0, float v1, uint32_t& lo) {
    const __half h0 = __float2half_rn(v0), h1 = __float2half_rn(v1);
    const __half l0 = __float2half_rn(v0 - __half2float(h0)), l1 = __float2half_rn(v1 - __half2float(h1));
    lo = (uint32_t)__half_as_ushort(l0) | ((uint32_t)__half_as_ushort(l1) << 16);
    return (uint32_t)__half_as_ushort(h0) | ((uint32_t)__half_as_ushort(h1) << 16);
}

// Byte offset of K element k (k even for 4-byte pairs) of `row` in a K-major 128-byte-
// swizzled operand whose 64-element K blocks are `block_bytes` apart.
__device__ __forceinline__ uint32_t kmaj_off(uint32_t row, uint32_t k, uint32_t block_bytes) {
    return (k >> 6) * block_bytes + tc::sw128_off(row, (k >> 3) & 7u) + (k & 7u) * 2u;
}

__global__ void __launch_bounds__(kTcThreads, 1) adjoint_tc_kernel(const AdjTcArgs g) {
    using namespace tc;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t NB = g.NB, A = g.A, F = g.F, T = g.T;
    const uint32_t img_pad = (g.img_bytes + 1023u) & ~1023u;
    uint8_t* img = smem;
    uint8_t* xf = img + img_pad;          // [p][h] 16 KB each
    uint8_t* xg = xf + 4 * 16384;         // [h] 32 KB each (two K blocks of 16 KB)
    uint8_t* yg = xg + 2 * 32768;         // [h] 2 K blocks of 4 NB rows x 128 B
    const uint32_t yblk = 4u * NB * 128u, yg_h = 2u * yblk;
    uint64_t* bars = reinterpret_cast<uint64_t*>(yg + 2 * yg_h);  // bar_f, bar_g, bar_end
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 3);
    double* red = reinterpret_cast<double*>(xf);  // loss reduction, after the last MMA has drained
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    volatile int never = 0;

    const uint32_t f = blockIdx.x / g.nch, chunk = blockIdx.x - f * g.nch;
    const uint32_t ntiles = T / 128u;
    const uint32_t tile0 = chunk * g.tiles_per_chunk, tile1 = min(ntiles, tile0 + g.tiles_per_chunk);

    if (tid == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, 512);
        tmem_relinquish();
    }
    // the channel's phasor image and zero voltage operands (padded antennas stay 0)
    {
        const uint4* src = reinterpret_cast<const uint4*>(g.plan + (uint64_t)f * g.img_bytes);
        uint4* dst = reinterpret_cast<uint4*>(img);
        for (uint32_t i = tid; i < g.img_bytes / 16; i += kTcThreads) dst[i] = src[i];
        uint4* z = reinterpret_cast<uint4*>(xf);
        for (uint32_t i = tid; i < (4 * 16384 + 2 * 32768) / 16; i += kTcThreads) z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t d_cols = 4u * NB;           // forward accumulator columns per polarisation
    const uint32_t dg = tmem + 256u;           // gradient accumulator, columns 256 .. 256 + 4 NB
    const uint32_t idesc_f = idesc_f16(128, d_cols), idesc_g = idesc_f16(128, 4u * NB);

    // voltages of this thread's tasks: (antenna pair a2, sample pair s2) = (t / 64, t % 64)
    float4 xv[4][4];  // [task][(a0, s0), (a0, s0 + 1), (a0 + 1, s0), (a0 + 1, s0 + 1)]
    auto load = [&](uint32_t tile) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t tk = tid + kTcThreads * i, a0 = 2u * (tk >> 6), s0 = 2u * (tk & 63u);
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const uint32_t a = a0 + (e >> 1), s = s0 + (e & 1);
                xv[i][e] = a < A ? __ldg(g.x + ((uint64_t)a * F + f) * T + tile * 128u + s)
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
    };
    double lsum = 0.0;
    uint32_t fph = 0, gph = 0;
    bool ok = true;
    if (tile0 < tile1) load(tile0);
    for (uint32_t tile = tile0; tile < tile1 && ok; tile++) {
        // the previous tile's gradient MMAs read XF/XG/YG: wait for them
        if (tile > tile0) {
            const bool w = mbar_wait(&bars[1], gph, &never, kTcBudget);
            gph ^= 1;
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
            tc_fence_after();
        }
        // phase 1: operands
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t tk = tid + kTcThreads * i, a0 = 2u * (tk >> 6), s0 = 2u * (tk & 63u);
            if (a0 >= kTcKA) continue;
#pragma unroll
            for (int p = 0; p < 2; p++) {
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    // component (p, c) of the four samples: v[a][s]
                    float v[2][2];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const float4 q = xv[i][e];
                        v[e >> 1][e & 1] = p ? (c ? q.w : q.z) : (c ? q.y : q.x);
                    }
                    // XF: row s, K = 32 c + a0 (antennas a0, a0 + 1)
#pragma unroll
                    for (int ds = 0; ds < 2; ds++) {
                        uint32_t lo;
                        const uint32_t hi = split_pair(v[0][ds], v[1][ds], lo);
                        const uint32_t off = kmaj_off(s0 + ds, 32u * c + a0, 16384u);
                        *reinterpret_cast<uint32_t*>(xf + (2 * p + 0) * 16384 + off) = hi;
                        *reinterpret_cast<uint32_t*>(xf + (2 * p + 1) * 16384 + off) = lo;
                    }
                    // XG: row 64 p + 2 a + c, K = s0 (samples s0, s0 + 1)
#pragma unroll
                    for (int da = 0; da < 2; da++) {
                        uint32_t lo;
                        const uint32_t hi = split_pair(v[da][0], v[da][1], lo);
                        const uint32_t off = kmaj_off(64u * p + 2u * (a0 + da) + c, s0, 16384u);
                        *reinterpret_cast<uint32_t*>(xg + off) = hi;
                        *reinterpret_cast<uint32_t*>(xg + 32768 + off) = lo;
                    }
                }
            }
        }
        fence_proxy_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // phase 2: forward, x hi and x lo against the stacked hi/lo image
        if (tid == 0) {
            const uint64_t wdesc = smem_desc_sw128(smem_u32(img));
            const uint32_t wpol16 = 4u * NB * 8u;  // one polarisation's column block of 4 NB rows
#pragma unroll 1
            for (uint32_t p = 0; p < 2; p++) {
                const uint32_t d = tmem + p * d_cols;
#pragma unroll 1
                for (uint32_t h = 0; h < 2; h++) {
                    const uint64_t ad = smem_desc_sw128(smem_u32(xf + (2 * p + h) * 16384));
                    for (uint32_t j = 0; j < 4; j++)
                        mma_f16(d, ad + (uint64_t)((j * 32u) >> 4), wdesc + (uint64_t)(p * wpol16 + j * 2u), idesc_f,
                                (h | j) ? 1u : 0u);
                }
            }
            mma_commit(&bars[0]);
        }
        // the next tile's voltages travel while the tensor cores work
        if (tile + 1 < tile1) load(tile + 1);
        {
            const bool w = mbar_wait(&bars[0], fph, &never, kTcBudget);
            fph ^= 1;
            if (!__syncthreads_and(w)) {
                ok = false;
                break;
            }
            tc_fence_after();
        }
        // phase 3: y (lane = sample) -> loss and the YG operand
        if (warp < 4) {
            const uint32_t s = 32u * warp + lane;
            const uint32_t lane_addr = tmem + ((32u * warp) << 16);
            float lt = 0.f;
            for (uint32_t p = 0; p < 2; p++) {
                for (uint32_t b0 = 0; b0 < NB; b0 += 16) {
                    uint32_t hr[16], hi_[16], lr[16], li[16];
                    tmem_ld16(lane_addr + p * d_cols + b0, hr);
                    tmem_ld16(lane_addr + p * d_cols + NB + b0, hi_);
                    tmem_ld16(lane_addr + p * d_cols + 2 * NB + b0, lr);
                    tmem_ld16(lane_addr + p * d_cols + 3 * NB + b0, li);
                    tmem_ld_wait();
#pragma unroll
                    for (int e = 0; e < 16; e++) {
                        const float yr = __uint_as_float(hr[e]) + __uint_as_float(lr[e]);
                        const float yi = __uint_as_float(hi_[e]) + __uint_as_float(li[e]);
                        lt = fmaf(yr, yr, fmaf(yi, yi, lt));
                        const uint32_t b = b0 + e;
#pragma unroll
                        for (int c = 0; c < 2; c++) {
                            const float v = c ? yi : yr;
                            const __half h = __float2half_rn(v);
                            const __half l = __float2half_rn(v - __half2float(h));
                            const uint32_t off = kmaj_off(2u * NB * p + NB * c + b, s, yblk);
                            *reinterpret_cast<__half*>(yg + off) = h;
                            *reinterpret_cast<__half*>(yg + yg_h + off) = l;
                        }
                    }
                }
            }
            lsum += (double)lt;
        }
        fence_proxy_async_smem();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        // phase 4: G += XG YG^T over the four hi/lo combinations, accumulated over the chunk
        if (tid == 0) {
            for (uint32_t hx = 0; hx < 2; hx++)
                for (uint32_t hy = 0; hy < 2; hy++) {
                    const uint64_t ad = smem_desc_sw128(smem_u32(xg + hx * 32768));
                    const uint64_t bd = smem_desc_sw128(smem_u32(yg + hy * yg_h));
                    for (uint32_t j = 0; j < 8; j++) {
                        const uint32_t first = (tile == tile0 && hx == 0 && hy == 0 && j == 0) ? 1u : 0u;
                        mma_f16(dg, ad + (uint64_t)(((j >> 2) * 16384u + (j & 3u) * 32u) >> 4),
                                bd + (uint64_t)(((j >> 2) * yblk + (j & 3u) * 32u) >> 4), idesc_g, first ? 0u : 1u);
                    }
                }
            mma_commit(&bars[1]);
        }
    }
    // drain: every MMA this CTA issued has completed before tensor memory is read or freed
    if (tid == 0) {
        mma_commit(&bars[2]);
        if (!mbar_wait(&bars[2], 0, &never, kTcBudget)) atomicCAS(&g_adj_status, 0u, 2u);
    }
    if (!ok && tid == 0) atomicCAS(&g_adj_status, 0u, 1u);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // final: G of this chunk, lanes (2 a, 2 a + 1) of quarter 2 p + a / 16
    if (warp < 4 && ok && tile0 < tile1) {
        const uint32_t m = 32u * warp + lane, p = m >> 6, a = (m & 63u) >> 1;
        const bool re_lane = (m & 1u) == 0;
        const uint32_t lane_addr = dg + ((32u * warp) << 16);
        const uint32_t Q = g.B * A;
        for (uint32_t b0 = 0; b0 < NB; b0 += 16) {
            uint32_t ur[16], vr[16];
            tmem_ld16(lane_addr + 2u * NB * p + b0, ur);       // x_c . Re y_b
            tmem_ld16(lane_addr + 2u * NB * p + NB + b0, vr);  // x_c . Im y_b
            tmem_ld_wait();
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const float u = __uint_as_float(ur[e]), v = __uint_as_float(vr[e]);
                const float u1 = __shfl_xor_sync(0xffffffffu, u, 1), v1 = __shfl_xor_sync(0xffffffffu, v, 1);
                const uint32_t b = b0 + e;
                if (re_lane && a < A && b < g.B) {
                    // lane 2a: (Re x . Re y, Re x . Im y); lane 2a + 1: (Im x . Re y, Im x . Im y)
                    float2* gp = reinterpret_cast<float2*>(g.gpart + (uint64_t)blockIdx.x * Q + b * A + a);
                    gp[p] = make_float2(u + v1, v - u1);
                }
            }
        }
    } else if (warp < 4 && tile0 >= tile1) {
        // an empty chunk contributes zeros
        const uint32_t m = 32u * warp + lane, p = m >> 6, a = (m & 63u) >> 1;
        if ((m & 1u) == 0 && a < A)
            for (uint32_t b = 0; b < g.B; b++)
                reinterpret_cast<float2*>(g.gpart + (uint64_t)blockIdx.x * g.B * A + b * A + a)[p] = make_float2(0.f, 0.f);
    }
    red[tid] = lsum;
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 512);
    }
    for (uint32_t s = kTcThreads / 2; s > 0; s >>= 1) {
        if (tid < s) red[tid] += red[tid + s];
        __syncthreads();
    }
    if (tid == 0) g.lpart[blockIdx.x] = red[0];
}

size_t adjoint_tc_smem(uint32_t NB, uint32_t img_bytes) {
    const size_t img_pad = (img_bytes + 1023u) & ~1023u;
    return 1024 + img_pad + 4 * 16384 + 2 * 32768 + 2 * (2u * 4u * NB * 128u) + 4 * 8;
}

// Stream-ordered scratch comes from a pool owned by the library, one per device,
// that keeps its memory between calls (release threshold = max): steady-state
// calls reuse it and never reach the driver's allocator, which the default pool
// (threshold 0) does again after every synchronisation.
cudaError_t scratch_alloc(void** p, size_t bytes, cudaStream_t s) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, s);
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!pools[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&pool, &props);
            if (e != cudaSuccess) return e;
            uint64_t keep = ~0ull;
            e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) {
                cudaMemPoolDestroy(pool);
                return e;
            }
            pools[dev] = pool;
        }
        pool = pools[dev];
    }
    return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

}  // namespace
}  // namespace bb

namespace bb {

// Reads and clears the adjoint kernels' device status word (blade_device_status).
int adjoint_status_take(uint32_t* v) {
    unsigned int x = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&x, g_adj_status, sizeof(x));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_adj_status, &zero, sizeof(zero));
    if (e != cudaSuccess) return check_cuda(e, "blade_device_status");
    *v = x;
    return BLADE_SUCCESS;
}

namespace {

bool adjoint_tc_applies(uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P, const void* in) {
    return P == 2 && A >= 1 && A <= kTcKA && B >= 1 && B <= 32 && T > 0 && T % 128 == 0 && T < (1ull << 31) &&
           F > 0 && F < (1ull << 24) && aligned16(in);
}

int adjoint_tensor_cores(const void* in, const void* phasors, void* grad, double* loss, uint64_t B, uint64_t A,
                         uint64_t F, uint64_t T, cudaStream_t s) {
    const char* who = "blade_beamform_detect_adjoint";
    const uint32_t NB = (uint32_t)((B + 15) / 16 * 16);
    const uint32_t img_bytes = 1024u * NB;  // stacked image of 32 antennas (blade_beamform_tc_prepare)
    const uint64_t plan_bytes = blade_beamform_tc_plan_size(B, A, F, 2);
    if (plan_bytes != (uint64_t)F * img_bytes) return set_error(BLADE_ASSERTION_ERROR, "%s: image layout", who);
    const uint64_t ntiles = T / 128, Q = B * A;
    uint64_t nch = (uint64_t)sm_count() / F;  // one CTA per SM (all of tensor memory)
    if (nch < 1) nch = 1;
    if (nch > ntiles) nch = ntiles;
    const uint64_t tpc = (ntiles + nch - 1) / nch;
    nch = (ntiles + tpc - 1) / tpc;
    const size_t smem = adjoint_tc_smem(NB, img_bytes);
    if (int rc = ensure_smem(reinterpret_cast<const void*>(adjoint_tc_kernel), smem)) return rc;
    uint8_t* plan = nullptr;
    float4* gpart = nullptr;
    double* lpart = nullptr;
    cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&plan), plan_bytes, s);
    if (e == cudaSuccess) e = scratch_alloc(reinterpret_cast<void**>(&gpart), F * nch * Q * sizeof(float4), s);
    if (e == cudaSuccess) e = scratch_alloc(reinterpret_cast<void**>(&lpart), F * nch * sizeof(double), s);
    int rc = e == cudaSuccess ? BLADE_SUCCESS : check_cuda(e, "blade_beamform_detect_adjoint (scratch)");
    if (!rc) rc = blade_beamform_tc_prepare(phasors, plan, B, A, F, 2, reinterpret_cast<blade_stream_t>(s));
    if (!rc) {
        AdjTcArgs g;
        g.x = static_cast<const float4*>(in);
        g.plan = plan;
        g.gpart = gpart;
        g.lpart = lpart;
        g.A = (uint32_t)A;
        g.B = (uint32_t)B;
        g.F = (uint32_t)F;
        g.T = (uint32_t)T;
        g.NB = NB;
        g.img_bytes = img_bytes;
        g.nch = (uint32_t)nch;
        g.tiles_per_chunk = (uint32_t)tpc;
        adjoint_tc_kernel<<<(unsigned)(F * nch), kTcThreads, smem, s>>>(g);
        adjoint_chunks_kernel<<<grid_for(F * Q, 256), 256, 0, s>>>(gpart, static_cast<float2*>(grad), (uint32_t)B,
                                                                   (uint32_t)A, (uint32_t)F, (uint32_t)nch);
        if (loss) loss_sum_kernel<<<1, 256, 0, s>>>(lpart, (uint32_t)(F * nch), loss);
        rc = check_launch(who);
    }
    if (plan) cudaFreeAsync(plan, s);
    if (gpart) cudaFreeAsync(gpart, s);
    if (lpart) cudaFreeAsync(lpart, s);
    return rc;
}

}  // namespace
}  // namespace bb

extern "C" int blade_beamform_detect_adjoint(const void* in, const void* phasors, void* grad, double* loss, uint64_t B,
                                             uint64_t A, uint64_t F, uint64_t T, uint64_t P, blade_stream_t stream) {
    using namespace bb;
    if (P != 1 && P != 2) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: P must be 1 or 2");
    if (B == 0 || A == 0 || F == 0) return BLADE_SUCCESS;
    if (!in || !phasors || !grad) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: null buffer");
    if (F * P > 0x7fffffffull || T >= (1ull << 32) || T == 0)
        return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: dimensions out of range");
    // below 8 beams the contraction is GEMV-like and the CUDA-core kernel, bound by the
    // voltage read, is faster (B = 1: 58 us against 222 us on the calibration block)
    if (B >= 8 && adjoint_tc_applies(B, A, F, T, P, in))
        return adjoint_tensor_cores(in, phasors, grad, loss, B, A, F, T, reinterpret_cast<cudaStream_t>(stream));
    return blade_beamform_detect_adjoint_f32(in, phasors, grad, loss, B, A, F, T, P, stream);
}

extern "C" int blade_beamform_detect_adjoint_tc(const void* in, const void* phasors, void* grad, double* loss,
                                                uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                                blade_stream_t stream) {
    using namespace bb;
    if (B == 0 || A == 0 || F == 0) return BLADE_SUCCESS;
    if (!in || !phasors || !grad) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint_tc: null buffer");
    if (!adjoint_tc_applies(B, A, F, T, P, in))
        return set_error(BLADE_ERROR,
                         "blade_beamform_detect_adjoint_tc: needs P = 2, 1 <= A <= 32, 1 <= B <= 32, T %% 128 == 0 "
                         "and 16-byte aligned voltages (B=%llu A=%llu T=%llu P=%llu)",
                         (unsigned long long)B, (unsigned long long)A, (unsigned long long)T, (unsigned long long)P);
    return adjoint_tensor_cores(in, phasors, grad, loss, B, A, F, T, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int blade_beamform_detect_adjoint_f32(const void* in, const void* phasors, void* grad, double* loss,
                                                 uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                                 blade_stream_t stream) {
    using namespace bb;
    if (P != 1 && P != 2) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint_f32: P must be 1 or 2");
    if (B == 0 || A == 0 || F == 0) return BLADE_SUCCESS;
    if (!in || !phasors || !grad) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint_f32: null buffer");
    if (F * P > 0x7fffffffull || T >= (1ull << 32) || T == 0)
        return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint_f32: dimensions out of range");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t Q = B * A;
    if (B == 1 && P == 2 && A <= 32 && aligned16(in)) {
        // one beam: register-resident kernel, chunks of kB1Samples samples
        const uint64_t nch = (T + kB1Samples - 1) / kB1Samples;
        if (F * nch > 0x7fffffffull) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint_f32: too many chunks");
        float4* gpart = nullptr;
        double* lpart = nullptr;
        cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&gpart), F * nch * A * sizeof(float4), s);
        if (e == cudaSuccess) e = scratch_alloc(reinterpret_cast<void**>(&lpart), F * nch * sizeof(double), s);
        if (e != cudaSuccess) {
            if (gpart) cudaFreeAsync(gpart, s);
            return check_cuda(e, "blade_beamform_detect_adjoint (scratch)");
        }
        const unsigned grid = (unsigned)(F * nch);
        const float4* x4 = static_cast<const float4*>(in);
        const float2* w2 = static_cast<const float2*>(phasors);
        const uint32_t a = (uint32_t)A, f = (uint32_t)F, t = (uint32_t)T, c = (uint32_t)nch;
        switch ((A + 3) / 4) {
#define BB_ADJ_B1(NA) \
    case NA: adjoint_b1_kernel<NA><<<grid, kB1Threads, 0, s>>>(x4, w2, gpart, lpart, a, f, t, c); break
            BB_ADJ_B1(1); BB_ADJ_B1(2); BB_ADJ_B1(3); BB_ADJ_B1(4);
            BB_ADJ_B1(5); BB_ADJ_B1(6); BB_ADJ_B1(7); BB_ADJ_B1(8);
#undef BB_ADJ_B1
        }
        adjoint_chunks_kernel<<<grid_for(F * Q, 256), 256, 0, s>>>(gpart, static_cast<float2*>(grad), 1u, a, f, c);
        if (loss) loss_sum_kernel<<<1, 256, 0, s>>>(lpart, (uint32_t)(F * nch), loss);
        const int rc = check_launch("blade_beamform_detect_adjoint");
        cudaFreeAsync(gpart, s);
        cudaFreeAsync(lpart, s);
        return rc;
    }
    const size_t fast_smem = 16 + (Q + A * (kTA + 1) + B * kTA + kTA) * sizeof(float4) + kTA * sizeof(double);
    if (P == 2 && Q <= kMaxPairs && fast_smem <= 227 * 1024 && aligned16(in)) {
        // chunks of the time axis: F * nch CTAs fill the resident slots once (one wave)
        const uint64_t ntiles = (T + kTA - 1) / kTA;
        int per_sm = 1;
        const void* fn0 = reinterpret_cast<const void*>(adjoint_chunk_kernel<1>);
        if (int rc0 = ensure_smem(fn0, fast_smem)) return rc0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn0, kTA, fast_smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        uint64_t nch = (uint64_t)sm_count() * per_sm / F;
        if (nch > ntiles) nch = ntiles;
        if (nch < 1) nch = 1;
        const uint64_t tpc = (ntiles + nch - 1) / nch;
        nch = (ntiles + tpc - 1) / tpc;
        float4* gpart = nullptr;
        double* lpart = nullptr;
        cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&gpart), F * nch * Q * sizeof(float4), s);
        if (e == cudaSuccess) e = scratch_alloc(reinterpret_cast<void**>(&lpart), F * nch * sizeof(double), s);
        if (e != cudaSuccess) {
            if (gpart) cudaFreeAsync(gpart, s);
            return check_cuda(e, "blade_beamform_detect_adjoint (scratch)");
        }
        const int nacc = Q <= (uint64_t)kTA ? 1 : Q <= 2u * kTA ? 2 : Q <= 4u * kTA ? 4 : 8;
        const void* fn = nacc == 1 ? reinterpret_cast<const void*>(adjoint_chunk_kernel<1>)
                         : nacc == 2 ? reinterpret_cast<const void*>(adjoint_chunk_kernel<2>)
                         : nacc == 4 ? reinterpret_cast<const void*>(adjoint_chunk_kernel<4>)
                                     : reinterpret_cast<const void*>(adjoint_chunk_kernel<8>);
        int rc = ensure_smem(fn, fast_smem);
        if (!rc) {
            const unsigned grid = (unsigned)(F * nch);
            const float4* x4 = static_cast<const float4*>(in);
            const float2* w2 = static_cast<const float2*>(phasors);
            const uint32_t b = (uint32_t)B, a = (uint32_t)A, f = (uint32_t)F, t = (uint32_t)T, c = (uint32_t)nch,
                           tp = (uint32_t)tpc;
            if (nacc == 1) adjoint_chunk_kernel<1><<<grid, kTA, fast_smem, s>>>(x4, w2, gpart, lpart, b, a, f, t, c, tp);
            else if (nacc == 2) adjoint_chunk_kernel<2><<<grid, kTA, fast_smem, s>>>(x4, w2, gpart, lpart, b, a, f, t, c, tp);
            else if (nacc == 4) adjoint_chunk_kernel<4><<<grid, kTA, fast_smem, s>>>(x4, w2, gpart, lpart, b, a, f, t, c, tp);
            else adjoint_chunk_kernel<8><<<grid, kTA, fast_smem, s>>>(x4, w2, gpart, lpart, b, a, f, t, c, tp);
            adjoint_chunks_kernel<<<grid_for(F * Q, 256), 256, 0, s>>>(gpart, static_cast<float2*>(grad), b, a, f, c);
            if (loss) loss_sum_kernel<<<1, 256, 0, s>>>(lpart, (uint32_t)(F * nch), loss);
            rc = check_launch("blade_beamform_detect_adjoint");
        }
        cudaFreeAsync(gpart, s);
        cudaFreeAsync(lpart, s);
        return rc;
    }
    // General path: one CTA per (f, p), loss partials per CTA summed by loss_sum_kernel.
    const size_t smem = ((size_t)B * A * 2 + (size_t)A * kT + (size_t)B * kT + kT) * sizeof(float2) +
                        kT * sizeof(double);
    if (smem > 227 * 1024)
        return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: B=%llu x A=%llu exceeds shared memory",
                         (unsigned long long)B, (unsigned long long)A);
    double* lpart = nullptr;
    if (loss) {
        cudaError_t e = scratch_alloc(reinterpret_cast<void**>(&lpart), F * P * sizeof(double), s);
        if (e != cudaSuccess) return check_cuda(e, "blade_beamform_detect_adjoint (scratch)");
    }
    int rc = ensure_smem(reinterpret_cast<const void*>(adjoint_kernel), smem);
    if (!rc) {
        adjoint_kernel<<<(unsigned)(F * P), kT, smem, s>>>(static_cast<const float2*>(in),
                                                           static_cast<const float2*>(phasors),
                                                           static_cast<float2*>(grad), lpart, (uint32_t)B, (uint32_t)A,
                                                           (uint32_t)F, (uint32_t)T, (uint32_t)P);
        if (loss) loss_sum_kernel<<<1, 256, 0, s>>>(lpart, (uint32_t)(F * P), loss);
        rc = check_launch("blade_beamform_detect_adjoint");
    }
    if (lpart) cudaFreeAsync(lpart, s);
    return rc;
}
