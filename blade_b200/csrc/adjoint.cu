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
// is one read of the voltages.  Other shapes take the one-CTA-per-(f, p) kernel.
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

extern "C" int blade_beamform_detect_adjoint(const void* in, const void* phasors, void* grad, double* loss, uint64_t B,
                                             uint64_t A, uint64_t F, uint64_t T, uint64_t P, blade_stream_t stream) {
    using namespace bb;
    if (P != 1 && P != 2) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: P must be 1 or 2");
    if (B == 0 || A == 0 || F == 0) return BLADE_SUCCESS;
    if (!in || !phasors || !grad) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: null buffer");
    if (F * P > 0x7fffffffull || T >= (1ull << 32) || T == 0)
        return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: dimensions out of range");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t Q = B * A;
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
