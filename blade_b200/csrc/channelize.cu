// Channelizer: hand-written FP32 Stockham FFT replacing the reference's
// pre_channelizer kernel + cuFFT.
//
// Reference: src/modules/channelizer/base.cc:9-146 multiplies by (-1)^t
// (channelizer.cu:5-19, an fftshift for even rates) and runs one cuFFT C2C plan
// per polarisation, in place; it only accepts rate == T or rate == 1
// (base.cc:30-35) because the in-place output is [A][F][T/C][C][P], which is
// [A][F*C][T/C][P] only when T/C = 1.  The general-rate layout is the test oracle
// tests/modules/channelizer/advanced.py:49-65:
//   out[a, f*C + k, s, p] = fftshift(FFT_C(x[a, f, s*C:(s+1)*C, p]))[k].
//
// Here, rate <= 4096: one CTA loads whole spectra of one (a, f) (all
// polarisations) with coalesced loads into shared memory, runs mixed-radix
// Stockham passes (radix 8/4/2 and direct odd-prime DFTs, twiddles from a
// shared-memory table computed with sincospif) and writes the spectra transposed
// into the [A, F*C, T/C, P] layout with the fftshift folded into the store index.
// rate > 4096: a four-step FFT (C = N1 * N2): column FFTs of length N1 with the
// inter-step twiddle, written to a workspace, then row FFTs of length N2 written
// to the output.
#include "common.cuh"

namespace bb {
namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSmallMax = 4096;

struct Plan {
    int n;       // number of passes
    int r[20];   // radix of each pass
};

bool make_plan(uint64_t N, Plan& p) {
    p.n = 0;
    uint64_t n = N;
    while (n % 8 == 0) { p.r[p.n++] = 8; n /= 8; }
    while (n % 4 == 0) { p.r[p.n++] = 4; n /= 4; }
    while (n % 2 == 0) { p.r[p.n++] = 2; n /= 2; }
    for (uint64_t q = 3; n > 1; q += 2) {
        while (n % q == 0) {
            if (q > 61 || p.n >= 20) return false;
            p.r[p.n++] = (int)q;
            n /= q;
        }
    }
    return true;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }  // -i * a

// exp(-2 pi i m / N)
__device__ __forceinline__ float2 twiddle(uint32_t m, uint32_t N) {
    float s, c;
    sincospif(-2.0f * (float)m / (float)N, &s, &c);
    return make_float2(c, s);
}

__device__ __forceinline__ void dft4(float2& a, float2& b, float2& c, float2& d) {
    const float2 e0 = cadd(a, c), e1 = csub(a, c), o0 = cadd(b, d), o1 = mul_mi(csub(b, d));
    a = cadd(e0, o0);
    b = cadd(e1, o1);
    c = csub(e0, o0);
    d = csub(e1, o1);
}

// Stockham passes over G transforms of length N stored back to back in b0.
// W holds exp(-2 pi i m / N), m < N.  Returns the buffer holding the result.
__device__ float2* stockham(float2* b0, float2* b1, const float2* W, uint32_t N, uint32_t G, const Plan& plan) {
    uint32_t Ns = 1;
    for (int ps = 0; ps < plan.n; ps++) {
        const uint32_t R = plan.r[ps];
        const uint32_t NR = N / R;
        const uint32_t total = G * NR;
        const uint32_t tws = N / (Ns * R);  // twiddle index stride
        for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
            const uint32_t g = e / NR, j = e - g * NR;
            const float2* src = b0 + g * N;
            float2* dst = b1 + g * N;
            const uint32_t jm = j % Ns;
            const uint32_t idxD = (j - jm) * R + jm;
            const uint32_t tw = jm * tws;
            if (R == 8) {
                float2 v[8];
#pragma unroll
                for (int r = 0; r < 8; r++) v[r] = src[j + r * NR];
#pragma unroll
                for (int r = 1; r < 8; r++) v[r] = cmul(v[r], W[tw * r]);
                dft4(v[0], v[2], v[4], v[6]);
                dft4(v[1], v[3], v[5], v[7]);
                const float c = 0.70710678118654752f;
                const float2 t0 = v[1];
                const float2 t1 = make_float2(c * (v[3].x + v[3].y), c * (v[3].y - v[3].x));
                const float2 t2 = mul_mi(v[5]);
                const float2 t3 = make_float2(c * (v[7].y - v[7].x), -c * (v[7].x + v[7].y));
                dst[idxD + 0 * Ns] = cadd(v[0], t0);
                dst[idxD + 4 * Ns] = csub(v[0], t0);
                dst[idxD + 1 * Ns] = cadd(v[2], t1);
                dst[idxD + 5 * Ns] = csub(v[2], t1);
                dst[idxD + 2 * Ns] = cadd(v[4], t2);
                dst[idxD + 6 * Ns] = csub(v[4], t2);
                dst[idxD + 3 * Ns] = cadd(v[6], t3);
                dst[idxD + 7 * Ns] = csub(v[6], t3);
            } else if (R == 4) {
                float2 v0 = src[j], v1 = src[j + NR], v2 = src[j + 2 * NR], v3 = src[j + 3 * NR];
                v1 = cmul(v1, W[tw]);
                v2 = cmul(v2, W[2 * tw]);
                v3 = cmul(v3, W[3 * tw]);
                dft4(v0, v1, v2, v3);
                dst[idxD] = v0;
                dst[idxD + Ns] = v1;
                dst[idxD + 2 * Ns] = v2;
                dst[idxD + 3 * Ns] = v3;
            } else if (R == 2) {
                const float2 v0 = src[j], v1 = cmul(src[j + NR], W[tw]);
                dst[idxD] = cadd(v0, v1);
                dst[idxD + Ns] = csub(v0, v1);
            } else {
                float2 v[61];
                for (uint32_t r = 0; r < R; r++) v[r] = cmul(src[j + r * NR], W[tw * r]);
                for (uint32_t k = 0; k < R; k++) {
                    float2 acc = v[0];
                    for (uint32_t m = 1; m < R; m++) acc = cadd(acc, cmul(v[m], W[((m * k) % R) * NR]));
                    dst[idxD + k * Ns] = acc;
                }
            }
        }
        __syncthreads();
        float2* t = b0;
        b0 = b1;
        b1 = t;
        Ns *= R;
    }
    return b0;
}

// ---- rate <= 4096 --------------------------------------------------------

template <int P>
__global__ void __launch_bounds__(kThreads) fft_small_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                             uint32_t A, uint32_t F, uint32_t T, uint32_t N,
                                                             uint32_t SB, Plan plan) {
    extern __shared__ __align__(16) float2 smem[];
    const uint32_t S = T / N;
    const uint32_t G = SB * P;
    float2* W = smem;
    float2* b0 = smem + N;
    float2* b1 = b0 + (size_t)G * N;
    for (uint32_t m = threadIdx.x; m < N; m += blockDim.x) W[m] = twiddle(m, N);
    const uint32_t nsb = (S + SB - 1) / SB;
    const uint64_t groups = (uint64_t)A * F * nsb;
    for (uint64_t grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const uint64_t af = grp / nsb;
        const uint32_t s0 = (uint32_t)(grp - af * nsb) * SB;
        const uint32_t sb = min(SB, S - s0);
        const uint32_t g = sb * P;
        // Load sb spectra x P polarisations (contiguous in the input).
        const float2* src = in + (af * T + (uint64_t)s0 * N) * P;
        const uint32_t nsamp = sb * N;
        for (uint32_t e = threadIdx.x; e < nsamp; e += blockDim.x) {
            const uint32_t sl = e / N, j = e - sl * N;
            if (P == 2) {
                const float4 v = ldg_nc_f4(src + 2 * (uint64_t)e);
                b0[(sl * 2 + 0) * N + j] = make_float2(v.x, v.y);
                b0[(sl * 2 + 1) * N + j] = make_float2(v.z, v.w);
            } else {
                b0[sl * N + j] = src[e];
            }
        }
        __syncthreads();
        const float2* res = stockham(b0, b1, W, N, g, plan);
        // Store: out[a, f*N + k, s, p] = X[(k + N/2) % N]; (s, p) fastest.
        const uint64_t obase = af * N;  // row (a, f*N) in units of output rows
        const uint32_t half = N / 2;
        for (uint32_t e = threadIdx.x; e < nsamp; e += blockDim.x) {
            const uint32_t k = e / sb, sl = e - k * sb;
            uint32_t kk = k + half;
            if (kk >= N) kk -= N;
            float2* dst = out + ((obase + k) * S + s0 + sl) * P;
            if (P == 2) {
                const float2 x0 = res[(sl * 2 + 0) * N + kk], x1 = res[(sl * 2 + 1) * N + kk];
                stg_f4(dst, make_float4(x0.x, x0.y, x1.x, x1.y));
            } else {
                dst[0] = res[sl * N + kk];
            }
        }
        __syncthreads();
    }
}

// ---- rate > 4096: four-step ------------------------------------------------
// N = N1 * N2, j = N2 j1 + j2, k = k1 + N1 k2:
//   X[k1 + N1 k2] = sum_j2 w_N2^(j2 k2) [ w_N^(j2 k1) sum_j1 x[N2 j1 + j2] w_N1^(j1 k1) ]

constexpr uint32_t kJB = 16;  // columns per CTA in the first step

template <int P>
__global__ void __launch_bounds__(kThreads) fft_cols_kernel(const float2* __restrict__ in, float2* __restrict__ ws,
                                                            uint32_t A, uint32_t F, uint32_t T, uint32_t N1,
                                                            uint32_t N2, Plan plan) {
    extern __shared__ __align__(16) float2 smem[];
    const uint32_t N = N1 * N2;
    const uint32_t S = T / N;
    const uint32_t G = kJB * P;
    float2* W = smem;
    float2* b0 = smem + N1;
    float2* b1 = b0 + (size_t)G * N1;
    for (uint32_t m = threadIdx.x; m < N1; m += blockDim.x) W[m] = twiddle(m, N1);
    const uint32_t ncb = N2 / kJB;
    const uint64_t groups = (uint64_t)A * F * S * ncb;
    for (uint64_t grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const uint64_t batch = grp / ncb;  // (a, f, s)
        const uint32_t c0 = (uint32_t)(grp - batch * ncb) * kJB;
        const float2* src = in + batch * (uint64_t)N * P;
        for (uint32_t e = threadIdx.x; e < N1 * kJB; e += blockDim.x) {
            const uint32_t j1 = e / kJB, jl = e - j1 * kJB;
            const uint64_t idx = (uint64_t)j1 * N2 + c0 + jl;
            if (P == 2) {
                const float4 v = ldg_nc_f4(src + 2 * idx);
                b0[(0 * kJB + jl) * N1 + j1] = make_float2(v.x, v.y);
                b0[(1 * kJB + jl) * N1 + j1] = make_float2(v.z, v.w);
            } else {
                b0[jl * N1 + j1] = src[idx];
            }
        }
        __syncthreads();
        const float2* res = stockham(b0, b1, W, N1, G, plan);
        // Twiddle and store ws[((batch*P + p)*N1 + k1)*N2 + j2].
        for (uint32_t e = threadIdx.x; e < G * N1; e += blockDim.x) {
            const uint32_t jl = e % kJB, k1 = (e / kJB) % N1, p = e / (kJB * N1);
            const uint32_t j2 = c0 + jl;
            const uint32_t m = (uint32_t)(((uint64_t)j2 * k1) % N);
            const float2 v = cmul(res[(p * kJB + jl) * N1 + k1], twiddle(m, N));
            ws[((batch * P + p) * N1 + k1) * (uint64_t)N2 + j2] = v;
        }
        __syncthreads();
    }
}

template <int P>
__global__ void __launch_bounds__(kThreads) fft_rows_kernel(const float2* __restrict__ ws, float2* __restrict__ out,
                                                            uint32_t A, uint32_t F, uint32_t T, uint32_t N1,
                                                            uint32_t N2, uint32_t SB, Plan plan) {
    extern __shared__ __align__(16) float2 smem[];
    const uint32_t N = N1 * N2;
    const uint32_t S = T / N;
    const uint32_t G = SB * P;
    float2* W = smem;
    float2* b0 = smem + N2;
    float2* b1 = b0 + (size_t)G * N2;
    for (uint32_t m = threadIdx.x; m < N2; m += blockDim.x) W[m] = twiddle(m, N2);
    const uint32_t nsb = (S + SB - 1) / SB;
    const uint64_t groups = (uint64_t)A * F * N1 * nsb;
    for (uint64_t grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const uint32_t sbi = (uint32_t)(grp % nsb);
        const uint64_t r = grp / nsb;
        const uint32_t k1 = (uint32_t)(r % N1);
        const uint64_t af = r / N1;
        const uint32_t s0 = sbi * SB, sb = min(SB, S - s0);
        // Rows (af, s, p, k1) for s in [s0, s0+sb).
        for (uint32_t e = threadIdx.x; e < sb * P * N2; e += blockDim.x) {
            const uint32_t j2 = e % N2, q = e / N2;  // q = sl*P + p
            const uint32_t sl = q / P, p = q - sl * P;
            const uint64_t batch = af * S + s0 + sl;
            b0[q * N2 + j2] = ws[((batch * P + p) * N1 + k1) * (uint64_t)N2 + j2];
        }
        __syncthreads();
        const float2* res = stockham(b0, b1, W, N2, sb * P, plan);
        const uint32_t half = N / 2;
        for (uint32_t e = threadIdx.x; e < N2 * sb; e += blockDim.x) {
            const uint32_t k2 = e / sb, sl = e - k2 * sb;
            uint32_t kout = k1 + N1 * k2 + half;  // fftshift destination of X[k1 + N1 k2]
            if (kout >= N) kout -= N;
            float2* dst = out + ((af * N + kout) * S + s0 + sl) * P;
            if (P == 2) {
                const float2 x0 = res[(sl * 2 + 0) * N2 + k2], x1 = res[(sl * 2 + 1) * N2 + k2];
                stg_f4(dst, make_float4(x0.x, x0.y, x1.x, x1.y));
            } else {
                dst[0] = res[sl * N2 + k2];
            }
        }
        __syncthreads();
    }
}

template <typename K>
int prepare_smem(K kernel, size_t bytes) {
    return ensure_smem(reinterpret_cast<const void*>(kernel), bytes);
}

bool split_large(uint64_t N, uint64_t& N1, uint64_t& N2) {
    // Most balanced N1 * N2 = N with both <= kSmallMax and N2 % kJB == 0.
    uint64_t best = 0;
    for (uint64_t d = 2; d <= kSmallMax; d++) {
        if (N % d) continue;
        uint64_t e = N / d;
        if (e > kSmallMax || e % kJB) continue;
        if (best == 0 || (d > e ? d - e : e - d) < (best > N / best ? best - N / best : N / best - best)) best = d;
    }
    if (!best) return false;
    N1 = best;
    N2 = N / best;
    return true;
}

}  // namespace
}  // namespace bb

extern "C" uint64_t blade_channelize_workspace_size(uint64_t A, uint64_t F, uint64_t T, uint64_t P, uint64_t rate) {
    if (rate <= bb::kSmallMax) return 0;
    return A * F * T * P * sizeof(float2);
}

extern "C" int blade_channelize(const void* in, void* out, void* workspace, uint64_t A, uint64_t F, uint64_t T,
                                uint64_t P, uint64_t rate, blade_stream_t stream) {
    using namespace bb;
    if (rate == 0) return set_error(BLADE_ERROR, "blade_channelize: rate must be positive");
    if (T % rate != 0)
        return set_error(BLADE_ERROR, "blade_channelize: the number of time samples (%llu) should be divisible by "
                         "the channelizer rate (%llu)", (unsigned long long)T, (unsigned long long)rate);
    if ((rate % 2) != 0 && rate != 1)
        return set_error(BLADE_ERROR, "blade_channelize: the channelizer rate (%llu) should be divisible by 2",
                         (unsigned long long)rate);
    if (P != 1 && P != 2)
        return set_error(BLADE_ERROR, "blade_channelize: number of polarizations (%llu) should be one or two",
                         (unsigned long long)P);
    const uint64_t total = A * F * T;
    if (total == 0) return BLADE_SUCCESS;
    if (!in || !out) return set_error(BLADE_ERROR, "blade_channelize: null buffer");
    if (rate == 1) return in == out ? BLADE_SUCCESS : blade_duplicate(in, out, total * P * sizeof(float2), stream);
    if (in == out && rate != T)
        return set_error(BLADE_ERROR, "blade_channelize: in-place operation needs rate == T");
    if (!aligned16(in) || !aligned16(out)) return set_error(BLADE_ERROR, "blade_channelize: buffers must be 16-byte aligned");
    if (A * F > (1ull << 40) || T >= (1ull << 32)) return set_error(BLADE_ERROR, "blade_channelize: dimensions out of range");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const float2* src = static_cast<const float2*>(in);
    float2* dst = static_cast<float2*>(out);
    const uint64_t S = T / rate;
    const int blocks_per_sm = 2;
    if (rate <= kSmallMax) {
        Plan plan;
        if (!make_plan(rate, plan))
            return set_error(BLADE_ERROR, "blade_channelize: rate %llu has a prime factor above 61",
                             (unsigned long long)rate);
        uint64_t SB = 4096 / (rate * P);
        if (SB < 1) SB = 1;
        if (SB > S) SB = S;
        const size_t smem = (rate + 2 * SB * P * rate) * sizeof(float2);
        const uint64_t groups = A * F * ceil_div(S, SB);
        const unsigned grid = (unsigned)(groups < (uint64_t)sm_count() * blocks_per_sm ? groups
                                                                                      : (uint64_t)sm_count() * blocks_per_sm);
        int rc;
        if (P == 2) {
            if ((rc = prepare_smem(fft_small_kernel<2>, smem))) return rc;
            fft_small_kernel<2><<<grid, kThreads, smem, s>>>(src, dst, (uint32_t)A, (uint32_t)F, (uint32_t)T,
                                                            (uint32_t)rate, (uint32_t)SB, plan);
        } else {
            if ((rc = prepare_smem(fft_small_kernel<1>, smem))) return rc;
            fft_small_kernel<1><<<grid, kThreads, smem, s>>>(src, dst, (uint32_t)A, (uint32_t)F, (uint32_t)T,
                                                            (uint32_t)rate, (uint32_t)SB, plan);
        }
        return check_launch("blade_channelize");
    }
    if (!workspace) return set_error(BLADE_ERROR, "blade_channelize: rate %llu needs a workspace of %llu bytes",
                                     (unsigned long long)rate,
                                     (unsigned long long)blade_channelize_workspace_size(A, F, T, P, rate));
    uint64_t N1, N2;
    if (!split_large(rate, N1, N2))
        return set_error(BLADE_ERROR, "blade_channelize: rate %llu cannot be split into two factors <= %u",
                         (unsigned long long)rate, kSmallMax);
    Plan p1, p2;
    if (!make_plan(N1, p1) || !make_plan(N2, p2))
        return set_error(BLADE_ERROR, "blade_channelize: rate %llu has a prime factor above 61", (unsigned long long)rate);
    float2* ws = static_cast<float2*>(workspace);
    const size_t smem1 = (N1 + 2 * kJB * P * N1) * sizeof(float2);
    uint64_t SB2 = 4096 / (N2 * P);
    if (SB2 < 1) SB2 = 1;
    if (SB2 > S) SB2 = S;
    const size_t smem2 = (N2 + 2 * SB2 * P * N2) * sizeof(float2);
    const uint64_t g1 = A * F * S * (N2 / kJB);
    const uint64_t g2 = A * F * N1 * ceil_div(S, SB2);
    const uint64_t cap = (uint64_t)sm_count() * blocks_per_sm;
    int rc;
    if (P == 2) {
        if ((rc = prepare_smem(fft_cols_kernel<2>, smem1))) return rc;
        if ((rc = prepare_smem(fft_rows_kernel<2>, smem2))) return rc;
        fft_cols_kernel<2><<<(unsigned)(g1 < cap ? g1 : cap), kThreads, smem1, s>>>(
            src, ws, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, p1);
        fft_rows_kernel<2><<<(unsigned)(g2 < cap ? g2 : cap), kThreads, smem2, s>>>(
            ws, dst, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, (uint32_t)SB2, p2);
    } else {
        if ((rc = prepare_smem(fft_cols_kernel<1>, smem1))) return rc;
        if ((rc = prepare_smem(fft_rows_kernel<1>, smem2))) return rc;
        fft_cols_kernel<1><<<(unsigned)(g1 < cap ? g1 : cap), kThreads, smem1, s>>>(
            src, ws, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, p1);
        fft_rows_kernel<1><<<(unsigned)(g2 < cap ? g2 : cap), kThreads, smem2, s>>>(
            ws, dst, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, (uint32_t)SB2, p2);
    }
    return check_launch("blade_channelize");
}
