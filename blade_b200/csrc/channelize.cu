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
#include "autotune.cuh"
#include "common.cuh"
#include "tc_ptx.cuh"

namespace bb {

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kSmallMax = 4096;

struct Plan {
    int n;       // number of passes
    int r[20];   // radix of each pass
    int log2n;   // log2 N when N is a power of two, else -1 (shift/mask indexing)
};

bool make_plan(uint64_t N, Plan& p) {
    p.n = 0;
    p.log2n = -1;
    if ((N & (N - 1)) == 0) {
        p.log2n = 0;
        while ((1ull << p.log2n) < N) p.log2n++;
    }
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

// Complex product with its two fused multiply-adds spelled out, so that every
// kernel rounds it the same way whatever the compiler would contract.
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -(a.y * b.y)), fmaf(a.x, b.y, a.y * b.x));
}
// Complex add and subtract as one packed FP32x2 instruction each (both lanes round
// as the scalar add would; a - b is fma(b, -1, a), whose product is exact).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
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
    const bool pow2 = plan.log2n >= 0;
    for (int ps = 0; ps < plan.n; ps++) {
        const uint32_t R = plan.r[ps];
        const uint32_t NR = N / R;
        const uint32_t total = G * NR;
        const uint32_t tws = N / (Ns * R);  // twiddle index stride
        const uint32_t lnr = pow2 ? (uint32_t)plan.log2n - (R == 8 ? 3u : R == 4 ? 2u : 1u) : 0u;
        for (uint32_t e = threadIdx.x; e < total; e += blockDim.x) {
            const uint32_t g = pow2 ? e >> lnr : e / NR, j = e - g * NR;
            const float2* src = b0 + g * N;
            float2* dst = b1 + g * N;
            const uint32_t jm = pow2 ? (j & (Ns - 1u)) : j % Ns;
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
constexpr int kThreads4 = 512;  // threads of the four-step kernels (one CTA per SM for the column step)

template <int P>
__global__ void __launch_bounds__(kThreads4) fft_cols_kernel(const float2* __restrict__ in, float2* __restrict__ ws,
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
            const uint32_t jk = j2 * k1;  // < N1 N2 <= 2^24
            const uint32_t m = (N & (N - 1u)) == 0 ? (jk & (N - 1u)) : jk % N;
            const float2 v = cmul(res[(p * kJB + jl) * N1 + k1], twiddle(m, N));
            ws[((batch * P + p) * N1 + k1) * (uint64_t)N2 + j2] = v;
        }
        __syncthreads();
    }
}

template <int P>
__global__ void __launch_bounds__(kThreads4) fft_rows_kernel(const float2* __restrict__ ws, float2* __restrict__ out,
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

// ---- rate 65536 = 256 x 256: register-blocked four-step --------------------
// A 256-point FFT runs on 16 threads: n = 16 n1 + n2, k = k1 + 16 k2,
//   X[k1 + 16 k2] = sum_n2 w16^(n2 k2) [ w256^(n2 k1) sum_n1 x[16 n1 + n2] w16^(n1 k1) ],
// thread n2 does the inner 16-point DFT in registers, the products go through
// shared memory once, thread k1 does the outer one.  A 16-point DFT is 4 x 4:
// four DFT-4s over n1 (stride 4), the w16 twiddles, four DFT-4s over n2.
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
    // v[n], n = 4 a + b -> in place, result index k = c + 4 d at position c + 4 d
#pragma unroll
    for (int b = 0; b < 4; b++) dft4(v[b], v[4 + b], v[8 + b], v[12 + b]);  // over a: U[b][c] at v[4 c + b]
    const float c1 = 0.92387953251128676f, s1 = 0.38268343236508977f, h = 0.70710678118654752f;
    // w16^(b c) for b, c in 1..3: exponents 1, 2, 3, 2, 4, 6, 3, 6, 9
    v[4 + 1] = cmul(v[4 + 1], make_float2(c1, -s1));   // b 1, c 1: w^1
    v[8 + 1] = cmul(v[8 + 1], make_float2(h, -h));     // b 1, c 2: w^2
    v[12 + 1] = cmul(v[12 + 1], make_float2(s1, -c1)); // b 1, c 3: w^3
    v[4 + 2] = cmul(v[4 + 2], make_float2(h, -h));     // b 2, c 1: w^2
    v[8 + 2] = mul_mi(v[8 + 2]);                       // b 2, c 2: w^4 = -i
    v[12 + 2] = cmul(v[12 + 2], make_float2(-h, -h));  // b 2, c 3: w^6
    v[4 + 3] = cmul(v[4 + 3], make_float2(s1, -c1));   // b 3, c 1: w^3
    v[8 + 3] = cmul(v[8 + 3], make_float2(-h, -h));    // b 3, c 2: w^6
    v[12 + 3] = cmul(v[12 + 3], make_float2(-c1, s1)); // b 3, c 3: w^9
#pragma unroll
    for (int c = 0; c < 4; c++) dft4(v[4 * c + 0], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);  // over b: X[c + 4 d] at v[4 c + d]
    // reorder: position 4 c + d holds X[c + 4 d]; transpose the 4 x 4 in registers
    float2 t[16];
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
        for (int d = 0; d < 4; d++) t[c + 4 * d] = v[4 * c + d];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = t[k];
}

// ---- rates 2, 4, 8, 16: one spectrum per thread in registers ----------------
// The shared-memory Stockham above pays a load / sync / pass / sync / store round per
// group; a transform this short fits a thread's registers instead.  Thread = one
// spectrum s of one (a, f): R consecutive samples (P = 2: both polarisations in one
// 16-byte word) in, the R fftshifted bins out, bin k of every spectrum of the row
// block written side by side (consecutive threads, consecutive 16-byte stores).
template <int R>
__device__ __forceinline__ void dft_small(float2 (&v)[R]) {
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        dft4(v[0], v[1], v[2], v[3]);  // outputs in natural order
    } else if constexpr (R == 8) {
        // radix 2 x 4: X[k] = E[k mod 4] + w8^k O[k mod 4], E / O = DFT-4 of the even / odd samples
        float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4(e0, e1, e2, e3);
        dft4(o0, o1, o2, o3);
        const float h = 0.70710678118654752f;
        const float2 t0 = o0, t1 = make_float2(h * (o1.x + o1.y), h * (o1.y - o1.x)), t2 = mul_mi(o2),
                     t3 = make_float2(h * (o3.y - o3.x), -h * (o3.x + o3.y));
        v[0] = cadd(e0, t0);
        v[4] = csub(e0, t0);
        v[1] = cadd(e1, t1);
        v[5] = csub(e1, t1);
        v[2] = cadd(e2, t2);
        v[6] = csub(e2, t2);
        v[3] = cadd(e3, t3);
        v[7] = csub(e3, t3);
    } else {
        static_assert(R == 16, "rates 2, 4, 8, 16");
        dft16(v);
    }
}

template <int R, int P>
__global__ void __launch_bounds__(256) fft_reg_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                      uint64_t rows, uint32_t S) {
    const uint64_t n = rows * S;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t af = i / S;
        const uint32_t sp = (uint32_t)(i - af * S);
        const float2* src = in + i * R * P;  // spectrum sp of row af starts at sample (af S + sp) R
        float2 x[P][R];
#pragma unroll
        for (int r = 0; r < R; r++) {
            if constexpr (P == 2) {
                const float4 v = __ldg(reinterpret_cast<const float4*>(src) + r);
                x[0][r] = make_float2(v.x, v.y);
                x[1][r] = make_float2(v.z, v.w);
            } else {
                x[0][r] = __ldg(src + r);
            }
        }
#pragma unroll
        for (int p = 0; p < P; p++) dft_small<R>(x[p]);
        // out[a, f R + k, s, p] = X[(k + R / 2) mod R]
        float2* dst = out + ((af * R) * S + sp) * P;
#pragma unroll
        for (int k = 0; k < R; k++) {
            const int kk = (k + R / 2) % R;
            if constexpr (P == 2) {
                stg_f4(dst + (uint64_t)k * S * 2, make_float4(x[0][kk].x, x[0][kk].y, x[1][kk].x, x[1][kk].y));
            } else {
                dst[(uint64_t)k * S] = x[0][kk];
            }
        }
    }
}

// ---- rate 8192: one transform per CTA unit, no workspace ---------------------
// N = 8192 = 16 x 16 x 32, n = t + 512 m, t = 32 u + v, k = k1 + 16 k2a + 256 k2b:
//   Y[k1][t]      = w8192^(t k1)  DFT16_m(x[t + 512 m])[k1]
//   Z[k1][k2a][v] = w512^(v k2a)  DFT16_u(Y[k1][32 u + v])[k2a]
//   X[k]          = DFT32_v(Z[k1][k2a][v])[k2b]
// A unit is one polarisation of one spectrum (a, f, s); 256 threads, the 8192
// values in shared memory between the three register stages (Y and Z share one
// buffer, rows padded to 529 and 33 so that every access of a half-warp is one
// wavefront).  Twiddle powers come from one sincospif and a recurrence of 15
// complex products (a few FP32 ulps).  The output bins of a unit are its own
// (written after all of its inputs are read), so rate == T runs in place.
constexpr uint32_t kN8 = 8192, kZ1 = 529, kZ2 = 33;

// w32^k = exp(-2 pi i k / 32), k < 16
__device__ __constant__ float2 c_w32[16] = {
    {1.000000000e+00f, -0.000000000e+00f}, {9.807852804e-01f, -1.950903220e-01f},
    {9.238795325e-01f, -3.826834324e-01f}, {8.314696123e-01f, -5.555702330e-01f},
    {7.071067812e-01f, -7.071067812e-01f}, {5.555702330e-01f, -8.314696123e-01f},
    {3.826834324e-01f, -9.238795325e-01f}, {1.950903220e-01f, -9.807852804e-01f},
    {0.000000000e+00f, -1.000000000e+00f}, {-1.950903220e-01f, -9.807852804e-01f},
    {-3.826834324e-01f, -9.238795325e-01f}, {-5.555702330e-01f, -8.314696123e-01f},
    {-7.071067812e-01f, -7.071067812e-01f}, {-8.314696123e-01f, -5.555702330e-01f},
    {-9.238795325e-01f, -3.826834324e-01f}, {-9.807852804e-01f, -1.950903220e-01f}};

template <int P>
__global__ void __launch_bounds__(256, 2) fft8192_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                                                          uint64_t units, uint32_t S) {
    extern __shared__ __align__(16) float2 sm[];  // 16 rows of kZ1
    const uint32_t tid = threadIdx.x;
    for (uint64_t unit = blockIdx.x; unit < units; unit += gridDim.x) {
        const uint32_t p = (uint32_t)(unit % P);
        const uint64_t as = unit / P;  // (a, f) row x S + s
        const uint64_t af = as / S;
        const uint32_t s = (uint32_t)(as - af * S);
        const float2* src = in + as * (uint64_t)kN8 * P + p;  // sample n at src[n P]
        if (tid < 16 && unit + gridDim.x < units)  // the next unit's spectrum into L2 while this one runs
            tc::prefetch_l2_bulk(in + ((unit + gridDim.x) / P) * (uint64_t)kN8 * P + 512 * P * tid, 4096u * P);
        // stage A: columns t = tid, tid + 256
#pragma unroll 1
        for (uint32_t c = 0; c < 2; c++) {
            const uint32_t t = tid + 256 * c;
            float2 v[16];
#pragma unroll
            for (int m = 0; m < 16; m++) v[m] = src[(uint64_t)(t + 512 * m) * P];
            dft16(v);
            float2 w1, wk = make_float2(1.f, 0.f);
            sincospif(-2.f * (float)t / 8192.f, &w1.y, &w1.x);
#pragma unroll
            for (int k1 = 0; k1 < 16; k1++) {
                if (k1) {
                    wk = cmul(wk, w1);
                    v[k1] = cmul(v[k1], wk);
                }
                sm[k1 * kZ1 + t] = v[k1];
            }
        }
        __syncthreads();
        // stage B: pairs q = tid, tid + 256 -> (k1, v) = (q / 32, q % 32); all reads first
        float2 y[2][16];
#pragma unroll
        for (uint32_t c = 0; c < 2; c++) {
            const uint32_t q = tid + 256 * c, k1 = q >> 5, vv = q & 31;
#pragma unroll
            for (int u = 0; u < 16; u++) y[c][u] = sm[k1 * kZ1 + 32 * u + vv];
        }
        __syncthreads();
#pragma unroll
        for (uint32_t c = 0; c < 2; c++) {
            const uint32_t q = tid + 256 * c, k1 = q >> 5, vv = q & 31;
            dft16(y[c]);
            float2 w1, wk = make_float2(1.f, 0.f);
            sincospif(-2.f * (float)vv / 512.f, &w1.y, &w1.x);
#pragma unroll
            for (int k2a = 0; k2a < 16; k2a++) {
                if (k2a) {
                    wk = cmul(wk, w1);
                    y[c][k2a] = cmul(y[c][k2a], wk);
                }
                sm[k1 * kZ1 + k2a * kZ2 + vv] = y[c][k2a];
            }
        }
        __syncthreads();
        // stage C: thread (k1, k2a) = (tid % 16, tid / 16), a 32-point DFT over v as
        // two 16-point DFTs of the even and odd samples
        {
            const uint32_t k1 = tid & 15, k2a = tid >> 4;
            float2 e[16], o[16];
#pragma unroll
            for (int i = 0; i < 16; i++) {
                e[i] = sm[k1 * kZ1 + k2a * kZ2 + 2 * i];
                o[i] = sm[k1 * kZ1 + k2a * kZ2 + 2 * i + 1];
            }
            dft16(e);
            dft16(o);
            // out[a, f N + kout, s, p], kout = (k + N / 2) mod N (fftshift)
            float2* dst = out + ((af * kN8) * S + s) * P + p;
#pragma unroll
            for (int k = 0; k < 16; k++) {
                const float2 t = cmul(o[k], c_w32[k]);
                const uint32_t k0 = k1 + 16 * k2a + 256 * k, k16 = k0 + 4096;  // X[k0] and X[k0 + 4096]
                dst[(uint64_t)((k0 + 4096) & 8191) * S * P] = cadd(e[k], t);
                dst[(uint64_t)((k16 + 4096) & 8191) * S * P] = csub(e[k], t);
            }
        }
        __syncthreads();
    }
}

// Column step for N = 65536 (N1 = N2 = 256): one CTA = one (a, f, s) spectrum, 16
// consecutive columns j2, both polarisations (32 FFTs x 16 threads = 512 threads).
// Output ws[((batch P + p) 256 + k1) 256 + j2] = w65536^(j2 k1) FFT256_j1(x[256 j1 + j2])[k1].
// Padded stride of a 256-point column / row in shared memory: odd, so columns
// read or written side by side fall in different banks, and >= 16 * 17 so the
// 16 x 16 exchange can use row stride 17 (conflict-free in both directions).
constexpr uint32_t kLd = 273;
constexpr uint32_t kZ = 17;

// v[k] *= w^k for k = 0..15 by recurrence from w (15 complex products, relative
// error a few FP32 ulps): replaces 16 strided, bank-conflicting table lookups.
__device__ __forceinline__ void twiddle_run(float2 (&v)[16], float2 base, float2 w) {
    float2 acc = base;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        v[k] = cmul(v[k], acc);
        acc = cmul(acc, w);
    }
}

// CI8 = true: the input is CI8 [.., T, 2] (one 4-byte word per dual-polarisation
// sample), cast exactly to FP32 on load (the fused spectrometer).
template <int P, bool CI8 = false>
__global__ void __launch_bounds__(512, 2) fft256_cols_kernel(const void* __restrict__ vin, float2* __restrict__ ws,
                                                          uint64_t batches) {
    extern __shared__ __align__(16) float2 sm[];
    float2* tile = sm;                   // [p][jc][kLd]   (16 P columns)
    float2* w256 = tile + 16 * P * kLd;  // w256^m, m < 256
    float2* wlo = w256 + 256;            // w65536^m, m < 256
    for (uint32_t m = threadIdx.x; m < 256; m += blockDim.x) {
        w256[m] = twiddle(m, 256);
        wlo[m] = twiddle(m, 65536);
    }
    const uint32_t t = threadIdx.x & 15u, jc = (threadIdx.x >> 4) & 15u, p = threadIdx.x >> 8;
    const bool active = p < (uint32_t)P;
    float2* col = tile + (p * 16 + jc) * kLd;
    constexpr uint32_t kPer = 256u * 16u / 512u;  // words loaded per thread per group
    // CI8: the next group's words are loaded into registers while this group's FFTs
    // run (8 registers), so the loads of consecutive groups overlap the arithmetic.
    uint32_t nxt[kPer];
    auto load_ci8 = [&](uint64_t g, uint32_t (&w)[kPer]) {
        const uint32_t* src = static_cast<const uint32_t*>(vin) + (g >> 4) * 65536ull + (uint32_t)(g & 15u) * 16u;
#pragma unroll
        for (uint32_t u = 0; u < kPer; u++) {
            const uint32_t e = threadIdx.x + u * 512u;
            w[u] = __ldg(src + (uint64_t)(e >> 4) * 256u + (e & 15u));
        }
    };
    if constexpr (CI8)
        if (blockIdx.x < batches * 16) load_ci8(blockIdx.x, nxt);
    for (uint64_t grp = blockIdx.x; grp < batches * 16; grp += gridDim.x) {
        const uint64_t batch = grp >> 4;
        const uint32_t c0 = (uint32_t)(grp & 15u) * 16u;
        __syncthreads();
        // coalesced load: rows j1 of 16 columns x P (256 B per row for P = 2); all of a
        // thread's loads are issued before any shared-memory store
        if constexpr (CI8) {
            uint32_t ld[kPer];
#pragma unroll
            for (uint32_t u = 0; u < kPer; u++) ld[u] = nxt[u];
            if (grp + gridDim.x < batches * 16) load_ci8(grp + gridDim.x, nxt);
#pragma unroll
            for (uint32_t u = 0; u < kPer; u++) {
                const uint32_t e = threadIdx.x + u * 512u, j1 = e >> 4, jl = e & 15u;
                const uint32_t w = ld[u];
                tile[(0 * 16 + jl) * kLd + j1] = make_float2((float)(int8_t)(w & 0xFFu), (float)(int8_t)((w >> 8) & 0xFFu));
                tile[(1 * 16 + jl) * kLd + j1] = make_float2((float)(int8_t)((w >> 16) & 0xFFu), (float)(int8_t)(w >> 24));
            }
        } else if (P == 2) {
            const float2* src = static_cast<const float2*>(vin) + batch * 65536ull * P;
#pragma unroll
            for (uint32_t h = 0; h < 2; h++) {  // two batches of four 16-byte loads in flight
                float4 ld[kPer / 2];
#pragma unroll
                for (uint32_t u = 0; u < kPer / 2; u++) {
                    const uint32_t e = threadIdx.x + (h * kPer / 2 + u) * 512u, j1 = e >> 4, jl = e & 15u;
                    ld[u] = ldg_nc_f4(src + 2 * ((uint64_t)j1 * 256u + c0 + jl));
                }
#pragma unroll
                for (uint32_t u = 0; u < kPer / 2; u++) {
                    const uint32_t e = threadIdx.x + (h * kPer / 2 + u) * 512u, j1 = e >> 4, jl = e & 15u;
                    tile[(0 * 16 + jl) * kLd + j1] = make_float2(ld[u].x, ld[u].y);
                    tile[(1 * 16 + jl) * kLd + j1] = make_float2(ld[u].z, ld[u].w);
                }
            }
        } else {
            const float2* src = static_cast<const float2*>(vin) + batch * 65536ull * P;
            float2 ld[kPer];
#pragma unroll
            for (uint32_t u = 0; u < kPer; u++) {
                const uint32_t e = threadIdx.x + u * 512u, j1 = e >> 4, jl = e & 15u;
                ld[u] = src[(uint64_t)j1 * 256u + c0 + jl];
            }
#pragma unroll
            for (uint32_t u = 0; u < kPer; u++) {
                const uint32_t e = threadIdx.x + u * 512u, j1 = e >> 4, jl = e & 15u;
                tile[jl * kLd + j1] = ld[u];
            }
        }
        __syncthreads();
        float2 v[16];
        if (active) {
#pragma unroll
            for (int n1 = 0; n1 < 16; n1++) v[n1] = col[16 * n1 + t];  // thread n2 = t
            dft16(v);
            twiddle_run(v, make_float2(1.f, 0.f), w256[t]);  // w256^(t k1)
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int k1 = 0; k1 < 16; k1++) col[kZ * t + k1] = v[k1];  // Z[n2 = t][k1]
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) v[n2] = col[kZ * n2 + t];  // thread k1 = t
            dft16(v);  // X[t + 16 k2]
            // inter-step twiddle w65536^(j2 (t + 16 k2)): base w^(j2 t), step w^(16 j2),
            // each from the two-level table w256^(m >> 8) w65536^(m & 255)
            const uint32_t j2 = c0 + jc;
            const uint32_t m0 = j2 * t, m1 = (16u * j2) & 65535u;
            twiddle_run(v, cmul(w256[m0 >> 8], wlo[m0 & 255u]), cmul(w256[m1 >> 8], wlo[m1 & 255u]));
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int k2 = 0; k2 < 16; k2++) col[t + 16 * k2] = v[k2];  // col[k1] = result, k1 = t + 16 k2
        }
        __syncthreads();
        // coalesced store: for each (p, k1), 16 consecutive j2
        for (uint32_t e = threadIdx.x; e < (uint32_t)P * 256u * 16u; e += blockDim.x) {
            const uint32_t jl = e & 15u, k1 = (e >> 4) & 255u, pp = e >> 12;
            ws[((batch * P + pp) * 256u + k1) * 256ull + c0 + jl] = tile[(pp * 16 + jl) * kLd + k1];
        }
    }
}

// Loads the rows (s, p, k1) of one (a, f) for all S spectra x P polarisations
// (q = s * P + p < nq) from the workspace into shared memory: 256 contiguous values
// per row.
__device__ __forceinline__ void load_rows(const float2* __restrict__ ws, float2* rows, uint64_t af, uint32_t S,
                                          uint32_t P, uint32_t k1, uint32_t nq) {
    // Asynchronous 8-byte copies straight into shared memory: all of a group's loads
    // are in flight at once without holding registers (rows are 273 float2 apart, so
    // 8 bytes is the widest aligned copy); consecutive threads take consecutive j2.
    const uint32_t n = nq * 256u;
    for (uint32_t e = threadIdx.x; e < n; e += blockDim.x) {
        const uint32_t qq = e >> 8, j2 = e & 255u;
        const float2* src = ws + (((af * S) * P + qq) * 256u + k1) * 256ull + j2;
        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(rows + qq * kLd + j2));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src) : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// Row step for N = 65536: one CTA = one (a, f) and one k1, all S spectra x P
// polarisations (S P <= 32 FFTs, 16 threads each).  X[k1 + 256 k2] goes to the
// fftshifted channel k1 + 256 k2 + N/2 (mod N) of [A, F*N, S, P].
template <int P>
__global__ void __launch_bounds__(512, 2) fft256_rows_kernel(const float2* __restrict__ ws, float2* __restrict__ out,
                                                          uint64_t AF, uint32_t S) {
    extern __shared__ __align__(16) float2 sm[];
    float2* rows = sm;                     // [q = s P + p][kLd], q < S P <= 32
    float2* w256 = rows + 32 * kLd;
    for (uint32_t m = threadIdx.x; m < 256; m += blockDim.x) w256[m] = twiddle(m, 256);
    const uint32_t t = threadIdx.x & 15u, q = threadIdx.x >> 4;
    const uint32_t nq = S * P;
    const bool active = q < nq;
    float2* row = rows + q * kLd;
    for (uint64_t grp = blockIdx.x; grp < AF * 256u; grp += gridDim.x) {
        const uint64_t af = grp >> 8;
        const uint32_t k1 = (uint32_t)(grp & 255u);
        __syncthreads();
        load_rows(ws, rows, af, S, P, k1, nq);
        __syncthreads();
        float2 v[16];
        if (active) {
#pragma unroll
            for (int n1 = 0; n1 < 16; n1++) v[n1] = row[16 * n1 + t];
            dft16(v);
            twiddle_run(v, make_float2(1.f, 0.f), w256[t]);
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int k = 0; k < 16; k++) row[kZ * t + k] = v[k];
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) v[n2] = row[kZ * n2 + t];
            dft16(v);  // X2[t + 16 c] = final X[k1 + 256 (t + 16 c)]
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int c = 0; c < 16; c++) row[t + 16 * c] = v[c];
        }
        __syncthreads();
        // out[(af N + kout) S + s][p], kout = (k1 + 256 k2 + 32768) mod 65536; (s, p) fastest
        for (uint32_t e = threadIdx.x; e < 256u * nq; e += blockDim.x) {
            const uint32_t qq = e % nq, k2 = e / nq;
            const uint32_t kout = (k1 + 256u * k2 + 32768u) & 65535u;
            out[((af * 65536ull + kout) * S) * P + qq] = rows[qq * kLd + k2];
        }
    }
}

// Row step of the fused spectrometer: the row FFTs of fft256_rows_kernel, then
// per output channel the optional circular conversion (L, R) = (X + iY, X - iY)
// (Polarizer), the detector over windows of I spectra (Stokes-I |X|^2 + |Y|^2, or
// (|X|^2, |Y|^2, Re X conj Y, Im X conj Y)) and the output cast, straight to
// out[A, F*N, S/I, OP]: only the products reach HBM.
template <int OP, typename OT>
__global__ void __launch_bounds__(512, 2) fft256_rows_detect_kernel(const float2* __restrict__ ws, OT* __restrict__ out,
                                                                 uint64_t AF, uint32_t S, uint32_t I, int circular) {
    extern __shared__ __align__(16) float2 sm[];
    constexpr uint32_t P = 2;
    float2* rows = sm;  // [q = s P + p][kLd], q < S P <= 32
    float2* w256 = rows + 32 * kLd;
    for (uint32_t m = threadIdx.x; m < 256; m += blockDim.x) w256[m] = twiddle(m, 256);
    const uint32_t t = threadIdx.x & 15u, q = threadIdx.x >> 4;
    const uint32_t nq = S * P, U = S / I;
    const bool active = q < nq;
    float2* row = rows + q * kLd;
    for (uint64_t grp = blockIdx.x; grp < AF * 256u; grp += gridDim.x) {
        const uint64_t af = grp >> 8;
        const uint32_t k1 = (uint32_t)(grp & 255u);
        __syncthreads();
        load_rows(ws, rows, af, S, P, k1, nq);
        __syncthreads();
        float2 v[16];
        if (active) {
#pragma unroll
            for (int n1 = 0; n1 < 16; n1++) v[n1] = row[16 * n1 + t];
            dft16(v);
            twiddle_run(v, make_float2(1.f, 0.f), w256[t]);
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int k = 0; k < 16; k++) row[kZ * t + k] = v[k];
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int n2 = 0; n2 < 16; n2++) v[n2] = row[kZ * n2 + t];
            dft16(v);
        }
        __syncthreads();
        if (active) {
#pragma unroll
            for (int c = 0; c < 16; c++) row[t + 16 * c] = v[c];
        }
        __syncthreads();
        // one thread per (k2, u): window sum over I spectra, OP products
        for (uint32_t e = threadIdx.x; e < 256u * U; e += blockDim.x) {
            const uint32_t u = e % U, k2 = e / U;
            float acc[OP];
#pragma unroll
            for (int o = 0; o < OP; o++) acc[o] = 0.f;
            for (uint32_t s = u * I; s < (u + 1) * I; s++) {
                float2 x = rows[(s * 2 + 0) * kLd + k2], y = rows[(s * 2 + 1) * kLd + k2];
                if (circular) {
                    const float2 l = make_float2(x.x - y.y, x.y + y.x), r = make_float2(x.x + y.y, x.y - y.x);
                    x = l;
                    y = r;
                }
                if constexpr (OP == 1) {
                    acc[0] += x.x * x.x + x.y * x.y + y.x * y.x + y.y * y.y;
                } else {
                    acc[0] += x.x * x.x + x.y * x.y;
                    acc[1] += y.x * y.x + y.y * y.y;
                    acc[2] += x.x * y.x + x.y * y.y;  // Re x conj(y)
                    acc[3] += x.y * y.x - x.x * y.y;  // Im x conj(y)
                }
            }
            const uint32_t kout = (k1 + 256u * k2 + 32768u) & 65535u;
            OT* dst = out + ((af * 65536ull + kout) * U + u) * OP;
#pragma unroll
            for (int o = 0; o < OP; o++) dst[o] = (OT)acc[o];
        }
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
    if (rate <= bb::kSmallMax || rate == bb::kN8) return 0;
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
    if ((rate == 2 || rate == 4 || rate == 8 || rate == 16) && S < (1ull << 32)) {
        const uint64_t rows = A * F;
        const unsigned grid = grid_for(rows * S, 256);
#define BB_FFT_REG(RR)                                                                               \
    do {                                                                                             \
        if (P == 2) fft_reg_kernel<RR, 2><<<grid, 256, 0, s>>>(src, dst, rows, (uint32_t)S);         \
        else fft_reg_kernel<RR, 1><<<grid, 256, 0, s>>>(src, dst, rows, (uint32_t)S);                \
    } while (0)
        if (rate == 2) BB_FFT_REG(2);
        else if (rate == 4) BB_FFT_REG(4);
        else if (rate == 8) BB_FFT_REG(8);
        else BB_FFT_REG(16);
#undef BB_FFT_REG
        return check_launch("blade_channelize");
    }
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
    if (rate == kN8) {
        const uint64_t units = A * F * S * P;
        const size_t smem = 16 * kZ1 * sizeof(float2);
        const uint64_t cap = (uint64_t)sm_count() * 2;
        const unsigned grid = (unsigned)(units < cap ? units : cap);
        int rc;
        if (P == 2) {
            if ((rc = prepare_smem(fft8192_kernel<2>, smem))) return rc;
            fft8192_kernel<2><<<grid, 256, smem, s>>>(src, dst, units, (uint32_t)S);
        } else {
            if ((rc = prepare_smem(fft8192_kernel<1>, smem))) return rc;
            fft8192_kernel<1><<<grid, 256, smem, s>>>(src, dst, units, (uint32_t)S);
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
    if (N1 == 256 && N2 == 256 && S * P <= 32) {
        const uint64_t batches = A * F * S;
        const size_t sm1 = (16 * P * kLd + 512) * sizeof(float2), sm2 = (32 * kLd + 256) * sizeof(float2);
        const uint64_t cap = (uint64_t)sm_count() * 2;
        const uint64_t g1 = batches * 16, g2 = A * F * 256;
        int rc;
        if (P == 2) {
            if ((rc = prepare_smem(fft256_cols_kernel<2>, sm1))) return rc;
            if ((rc = prepare_smem(fft256_rows_kernel<2>, sm2))) return rc;
            fft256_cols_kernel<2><<<(unsigned)(g1 < cap ? g1 : cap), 512, sm1, s>>>(in, ws, batches);
            fft256_rows_kernel<2><<<(unsigned)(g2 < cap ? g2 : cap), 512, sm2, s>>>(ws, dst, A * F, (uint32_t)S);
        } else {
            if ((rc = prepare_smem(fft256_cols_kernel<1>, sm1))) return rc;
            if ((rc = prepare_smem(fft256_rows_kernel<1>, sm2))) return rc;
            fft256_cols_kernel<1><<<(unsigned)(g1 < cap ? g1 : cap), 512, sm1, s>>>(in, ws, batches);
            fft256_rows_kernel<1><<<(unsigned)(g2 < cap ? g2 : cap), 512, sm2, s>>>(ws, dst, A * F, (uint32_t)S);
        }
        return check_launch("blade_channelize");
    }
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
        fft_cols_kernel<2><<<(unsigned)(g1 < cap ? g1 : cap), kThreads4, smem1, s>>>(
            src, ws, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, p1);
        fft_rows_kernel<2><<<(unsigned)(g2 < cap ? g2 : cap), kThreads4, smem2, s>>>(
            ws, dst, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, (uint32_t)SB2, p2);
    } else {
        if ((rc = prepare_smem(fft_cols_kernel<1>, smem1))) return rc;
        if ((rc = prepare_smem(fft_rows_kernel<1>, smem2))) return rc;
        fft_cols_kernel<1><<<(unsigned)(g1 < cap ? g1 : cap), kThreads4, smem1, s>>>(
            src, ws, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, p1);
        fft_rows_kernel<1><<<(unsigned)(g2 < cap ? g2 : cap), kThreads4, smem2, s>>>(
            ws, dst, (uint32_t)A, (uint32_t)F, (uint32_t)T, (uint32_t)N1, (uint32_t)N2, (uint32_t)SB2, p2);
    }
    return check_launch("blade_channelize");
}

// ---- fused spectrometer (Cast -> Channelizer -> Polarizer -> Detector -> Cast) ----

extern "C" uint64_t blade_spectrometer_workspace_size(uint64_t A, uint64_t F, uint64_t T, uint64_t P, uint64_t rate) {
    if (P != 2 || rate != 65536 || T % rate) return 0;
    return A * F * T * P * sizeof(float2);
}

namespace bb {
void spec_per_sm(const uint64_t (&key)[8], uint32_t (&per_sm)[2], bool* tuned = nullptr, TuneEntry* entry = nullptr);
int spectrometer_launch(int in_type, const void* in, int out_type, void* out, void* workspace, uint64_t A, uint64_t F,
                        uint64_t T, uint64_t integration, uint64_t out_pols, int circular,
                        const uint32_t (&per_sm)[2], cudaStream_t s);
}  // namespace bb

extern "C" int blade_spectrometer(int in_type, const void* in, int out_type, void* out, void* workspace, uint64_t A,
                                  uint64_t F, uint64_t T, uint64_t P, uint64_t rate, uint64_t integration,
                                  uint64_t out_pols, int circular, blade_stream_t stream) {
    using namespace bb;
    if (in_type != BLADE_CI8 && in_type != BLADE_CF32)
        return set_error(BLADE_ERROR, "blade_spectrometer: input must be CI8 or CF32");
    if (out_type != BLADE_F32 && out_type != BLADE_F16)
        return set_error(BLADE_ERROR, "blade_spectrometer: output must be F32 or F16");
    if (P != 2) return set_error(BLADE_ERROR, "blade_spectrometer: the polarizer needs two polarizations (P = %llu)",
                                 (unsigned long long)P);
    if (rate != 65536)
        return set_error(BLADE_ERROR, "blade_spectrometer: the fused path runs rate 65536 (256 x 256); use the "
                         "module chain for rate %llu", (unsigned long long)rate);
    if (T % rate != 0)
        return set_error(BLADE_ERROR, "blade_spectrometer: the number of time samples (%llu) should be divisible by "
                         "the channelizer rate (%llu)", (unsigned long long)T, (unsigned long long)rate);
    const uint64_t S = T / rate;
    if (S > 16) return set_error(BLADE_ERROR, "blade_spectrometer: at most 16 spectra per block (T <= 2^20)");
    if (integration == 0)
        return set_error(BLADE_ERROR, "blade_spectrometer: integration size (%llu) should be more than zero",
                         (unsigned long long)integration);
    if (S % integration != 0)
        return set_error(BLADE_ERROR, "blade_spectrometer: the number of spectra (%llu) should be divisible by the "
                         "integration size (%llu)", (unsigned long long)S, (unsigned long long)integration);
    if (out_pols != 1 && out_pols != 4)
        return set_error(BLADE_ERROR, "blade_spectrometer: number of output polarizations (%llu) not supported",
                         (unsigned long long)out_pols);
    if (A * F == 0) return BLADE_SUCCESS;
    if (!in || !out || !workspace) return set_error(BLADE_ERROR, "blade_spectrometer: null buffer");
    if (!aligned16(in) || !aligned16(workspace) || (reinterpret_cast<uintptr_t>(out) & 3))
        return set_error(BLADE_ERROR, "blade_spectrometer: input and workspace must be 16-byte aligned");
    uint32_t per_sm[2];
    const uint64_t key[8] = {A, F, T, P, rate, integration, out_pols, (uint64_t)in_type};
    spec_per_sm(key, per_sm);
    return spectrometer_launch(in_type, in, out_type, out, workspace, A, F, T, integration, out_pols, circular,
                               per_sm, reinterpret_cast<cudaStream_t>(stream));
}

namespace bb {

// CTAs per SM of the column and row steps (both grid-stride loops): the tuned pair
// for this shape on this device when blade_spectrometer_autotune stored one, else 2, 2.
void spec_per_sm(const uint64_t (&key)[8], uint32_t (&per_sm)[2], bool* tuned, TuneEntry* entry) {
    per_sm[0] = per_sm[1] = 2;
    if (tuned) *tuned = false;
    TuneEntry e;
    if (tune_lookup(BLADE_TUNE_SPECTROMETER, key, &e) && e.params[0] >= 1 && e.params[0] <= 4 && e.params[1] >= 1 &&
        e.params[1] <= 4) {
        per_sm[0] = e.params[0];
        per_sm[1] = e.params[1];
        if (tuned) *tuned = true;
        if (entry) *entry = e;
    }
}

int spec_query(const uint64_t (&shape)[8], uint32_t* params, float* us, int* tuned) {
    bool t = false;
    TuneEntry e;
    uint32_t per_sm[2];
    spec_per_sm(shape, per_sm, &t, &e);
    for (int i = 0; i < kTuneParams; i++) params[i] = t ? e.params[i] : 0u;
    params[0] = per_sm[0];
    params[1] = per_sm[1];
    *us = t ? e.us : 0.f;
    *tuned = t ? 1 : 0;
    return BLADE_SUCCESS;
}

int spectrometer_launch(int in_type, const void* in, int out_type, void* out, void* workspace, uint64_t A, uint64_t F,
                        uint64_t T, uint64_t integration, uint64_t out_pols, int circular,
                        const uint32_t (&per_sm)[2], cudaStream_t s) {
    const uint64_t S = T / 65536;
    float2* ws = static_cast<float2*>(workspace);
    const uint64_t batches = A * F * S;
    const size_t sm1 = (16 * 2 * kLd + 512) * sizeof(float2), sm2 = (32 * kLd + 256) * sizeof(float2);
    const uint64_t cap1 = (uint64_t)sm_count() * per_sm[0], cap2 = (uint64_t)sm_count() * per_sm[1];
    const uint64_t g1 = batches * 16, g2 = A * F * 256;
    const unsigned grid1 = (unsigned)(g1 < cap1 ? g1 : cap1), grid2 = (unsigned)(g2 < cap2 ? g2 : cap2);
    int rc;
    if (in_type == BLADE_CI8) {
        if ((rc = prepare_smem(fft256_cols_kernel<2, true>, sm1))) return rc;
        fft256_cols_kernel<2, true><<<grid1, 512, sm1, s>>>(in, ws, batches);
    } else {
        if ((rc = prepare_smem(fft256_cols_kernel<2, false>, sm1))) return rc;
        fft256_cols_kernel<2, false><<<grid1, 512, sm1, s>>>(in, ws, batches);
    }
    if ((rc = check_launch("blade_spectrometer"))) return rc;
    const uint32_t S32 = (uint32_t)S, I32 = (uint32_t)integration;
#define BB_SPEC_ROWS(OPN, OTY)                                                                              \
    do {                                                                                                    \
        if ((rc = prepare_smem(fft256_rows_detect_kernel<OPN, OTY>, sm2))) return rc;                       \
        fft256_rows_detect_kernel<OPN, OTY><<<grid2, 512, sm2, s>>>(ws, static_cast<OTY*>(out), A * F, S32, \
                                                                    I32, circular ? 1 : 0);                 \
    } while (0)
    if (out_type == BLADE_F32) {
        if (out_pols == 1) BB_SPEC_ROWS(1, float);
        else BB_SPEC_ROWS(4, float);
    } else {
        if (out_pols == 1) BB_SPEC_ROWS(1, __half);
        else BB_SPEC_ROWS(4, __half);
    }
#undef BB_SPEC_ROWS
    return check_launch("blade_spectrometer");
}

}  // namespace bb

extern "C" int blade_spectrometer_autotune(int in_type, int out_type, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                           uint64_t rate, uint64_t integration, uint64_t out_pols,
                                           blade_stream_t stream) {
    using namespace bb;
    const char* who = "blade_spectrometer_autotune";
    if (A * F == 0 || P != 2 || rate != 65536 || T % rate != 0)
        return set_error(BLADE_ERROR, "%s: unsupported configuration", who);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const size_t n = (size_t)A * F * T * P;
    const size_t in_bytes = n * (in_type == BLADE_CI8 ? 2 : 8);
    const size_t ws_bytes = blade_spectrometer_workspace_size(A, F, T, P, rate);
    const size_t out_bytes = (size_t)A * F * T / integration * out_pols * (out_type == BLADE_F16 ? 2 : 4);
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
    void* ws = get(ws_bytes);
    void* ref = get(out_bytes);
    void* out = get(out_bytes);
    if (!in || !ws || !ref || !out) return set_error(BLADE_CUDA_ERROR, "%s: allocation failed", who);
    if (in_type == BLADE_CI8) {
        if (int rc = tune_fill_ci8(in, in_bytes, st)) return rc;
    } else {
        if (int rc = tune_fill_phasors(in, n, st)) return rc;
    }
    // the public entry validates the configuration
    if (int rc = blade_spectrometer(in_type, in, out_type, ref, ws, A, F, T, P, rate, integration, out_pols, 1, stream))
        return rc;
    std::vector<std::pair<uint32_t, uint32_t>> cands{{2u, 2u}};
    for (uint32_t a = 1; a <= 3; a++)
        for (uint32_t b = 1; b <= 3; b++)
            if (!(a == 2 && b == 2)) cands.push_back({a, b});
    int best = -1;
    float best_us = 0.f;
    uint32_t ndiff = 0, ntimed = 0;
    for (size_t i = 0; i < cands.size(); i++) {
        const uint32_t per_sm[2] = {cands[i].first, cands[i].second};
        void* dst = i == 0 ? ref : out;
        const float us = tune_time(
            [&]() {
                return spectrometer_launch(in_type, in, out_type, dst, ws, A, F, T, integration, out_pols, 1, per_sm,
                                           st);
            },
            st);
        if (us < 0.f) return set_error(BLADE_CUDA_ERROR, "%s: candidate %zu failed: %s", who, i, blade_last_error());
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
    e.params[0] = cands[best].first;
    e.params[1] = cands[best].second;
    e.params[4] = ntimed;
    e.params[5] = ndiff;
    e.us = best_us;
    const uint64_t key[8] = {A, F, T, P, rate, integration, out_pols, (uint64_t)in_type};
    tune_store(BLADE_TUNE_SPECTROMETER, key, e);
    return BLADE_SUCCESS;
}
