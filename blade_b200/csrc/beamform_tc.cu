// Tensor-core (tcgen05 / TMEM) beamform + channelize + detect chain for sm_100a.
//
// Computes, for CI8 voltages x[A, F, T, 2] and phasors w[B, A, F, 1, 2],
//   y[b, f, t, p]            = sum_a x[a, f, t, p] w[b, a, f, 0, p]
//   Y[b, f*R + k, s, p]      = fftshift(FFT_R(y[b, f, sR:(s+1)R, p]))[k],  R in {1, 2, 4}
//   out[b, f*R + k, u, 0]    = sum_{s in window u of I spectra} sum_p |Y[b, f*R + k, s, p]|^2
// i.e. the reference chain Cast -> Beamformer::ATA -> Channelizer -> Detector
// (src/modules/cast/cast.cu, src/modules/beamformer/beamformer.cu:13-62,
// src/modules/channelizer/base.cc + channelizer.cu, src/modules/detector/detector.cu:34-51),
// fused so that only the Stokes-I output reaches HBM.
//
// Numerics.  CI8 values are exact in FP16.  The rate-R DFT with the (-1)^t
// fftshift pre-multiply has coefficients in {+-1, +-i}, so it is applied to the
// integer voltages while the MMA operand is built (values <= 4 * 128, still
// exact in FP16): Y = X_R . w with X_R exact.  Each phasor component is split into
// FP16 hi = rn(w) and lo = rn(w - hi) (about 22 significant bits); both products
// accumulate in FP32 in tensor memory.
//
// GEMM mapping per (channel f, polarisation p): D[m, n] = sum_k A[m, k] B[n, k]
// with m = one of 128 rows of a tile (R consecutive samples per spectrum,
// row = k * (128/R) + spectrum), k = antenna (K = A padded to 16), and the complex
// product embedded in reals with N = 2 NB (NB = beams padded to 16):
//   D[:, 0:NB]   = Xr Wr - Xi Wi  (Re y),   D[:, NB:2NB] = Xr Wi + Xi Wr  (Im y)
//   D = Xr . [Wr | Wi]^T + Xi . [-Wi | Wr]^T
// The phasor image stores the three blocks [-Wi | Wr | Wi] per (p, hi/lo), so both
// B operands are contiguous windows of it.  Operands use the K-major no-swizzle
// core-matrix layout (8 rows x 16 bytes per 128-byte core matrix).
//
// CTA organisation (persistent, one CTA per SM, 14 warps):
//   warp 0      TMEM allocation; lane 0 issues tcgen05.mma and commits
//   warp 1      lane 0 loads the per-channel phasor image with one bulk copy
//   warps 2-5   epilogue: tcgen05.ld of the accumulators, |.|^2 over both
//               polarisations, window sums with lane shuffles, Stokes-I stores
//   warps 6-13  operand build: CI8 loads, DFT, exact int8 -> FP16 conversion,
//               stores in the UMMA core-matrix layout
// Pipelines: operand stages (full/empty mbarriers), two TMEM accumulator buffers
// (full/empty), phasor image (full/empty).  Every wait is bounded (clock budget
// plus a shared abort flag); on expiry the kernel records a status word, drains
// its own MMAs and bulk copies, frees TMEM and returns.
#include <mutex>

#include "common.cuh"
#include "tc_ptx.cuh"

namespace bb {

// Non-zero after a bounded wait expired in the tensor-core kernel (read and
// cleared by blade_device_status()).
__device__ unsigned int g_tc_status = 0;

namespace {

using namespace tc;

constexpr int kM = 128;  // tile rows
constexpr int kConvWarps = 8;
constexpr int kEpiWarps = 4;
constexpr int kThreads = (2 + kEpiWarps + kConvWarps) * 32;  // 448
constexpr int kMaxNB = 64;
constexpr int kMaxKA = 64;
constexpr long long kWaitBudget = 4000000000ll;  // cycles (~2 s) before a wait gives up

struct TcArgs {
    const uint8_t* in;    // CI8 [A, F, T, 2]
    const uint8_t* plan;  // phasor images, one per channel, img_bytes each
    float* out;           // [beams, F*R, U]
    uint32_t A, F, T, beams, U, integ;
    uint32_t NB, KA, stages;
    uint32_t img_bytes, tiles_per_ch;
    uint64_t total_tiles;
};

__device__ __forceinline__ uint32_t cvt_pair(uint32_t v) {
    // bytes 0 and 2 of v hold two int8 values; returns them as an exact half2.
    uint32_t x = (v & 0x00FF00FFu) ^ 0x64806480u;  // 1024 + (b + 128) in each half
    half2 h = *reinterpret_cast<half2*>(&x);
    const half2 bias = __halves2half2(__ushort_as_half(0x6480), __ushort_as_half(0x6480));  // 1152
    h = __hsub2(h, bias);
    return *reinterpret_cast<uint32_t*>(&h);
}

// One sample word [p0 re, p0 im, p1 re, p1 im] -> half2 (re, im) of polarisation p.
__device__ __forceinline__ half2 sample_h2(uint32_t w, int p) {
    uint32_t v = __byte_perm(w, 0, p == 0 ? 0x0100 : 0x0302);
    uint32_t r = cvt_pair(v);
    return *reinterpret_cast<half2*>(&r);
}

__device__ __forceinline__ uint32_t h2u(half2 h) { return *reinterpret_cast<uint32_t*>(&h); }

// Byte offset of element (row, k) inside an operand block with K extent KA.
__device__ __forceinline__ uint32_t cm_off(uint32_t row, uint32_t kchunk, uint32_t KA) {
    return (row >> 3) * (16u * KA) + kchunk * 128u + (row & 7u) * 16u;
}

__device__ __forceinline__ void record_abort(volatile int* abort, unsigned code) {
    *abort = 1;
    atomicCAS(&g_tc_status, 0u, code);
}

template <int R>
__global__ void __launch_bounds__(kThreads, 1) bf_tc_kernel(const TcArgs g) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const uint32_t NB = g.NB, KA = g.KA, S = g.stages;
    const uint32_t blkW = NB * KA * 2;      // one [NB x KA] fp16 block
    const uint32_t blkA = kM * KA * 2;      // one [128 x KA] fp16 block
    uint8_t* w_smem = smem;                 // 12 blocks: [p][h][-Wi | Wr | Wi]
    uint8_t* a_smem = smem + 12 * blkW;     // S stages x 4 blocks: [p][Xr | Xi]
    uint64_t* bars = reinterpret_cast<uint64_t*>(a_smem + (size_t)S * 4 * blkA);
    uint64_t* a_full = bars;
    uint64_t* a_empty = bars + S;
    uint64_t* d_full = bars + 2 * S;
    uint64_t* d_empty = d_full + 2;
    uint64_t* w_full = d_empty + 2;
    uint64_t* w_empty = w_full + 1;
    uint64_t* fin = w_empty + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(fin + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int never = 0;  // abort flag that is never raised (drain waits)
    const uint32_t tmem_cols = (8 * NB <= 32) ? 32 : (8 * NB <= 64) ? 64 : (8 * NB <= 128) ? 128 : (8 * NB <= 256) ? 256 : 512;

    if (threadIdx.x == 0) {
        for (uint32_t i = 0; i < S; i++) {
            mbar_init(&a_full[i], kConvWarps);
            mbar_init(&a_empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            mbar_init(&d_full[i], 1);
            mbar_init(&d_empty[i], kEpiWarps);
        }
        mbar_init(w_full, 1);
        mbar_init(w_empty, 1);
        mbar_init(fin, 1);
        *abort = 0;
        fence_mbar_init();
    }
    if (warp == 0) {
        tmem_alloc(tmem_slot, tmem_cols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // This CTA's contiguous range of (channel, time-tile) tiles.
    const uint64_t per = (g.total_tiles + gridDim.x - 1) / gridDim.x;
    const uint64_t L0 = (uint64_t)blockIdx.x * per;
    const uint64_t L1 = min(g.total_tiles, L0 + per);
    const uint32_t tpc = g.tiles_per_ch;

    if (warp == 0) {
        // ---------------- MMA issuer ----------------
        if (lane == 0 && L0 < L1) {
            const uint32_t idesc = idesc_f16(kM, 2 * NB);
            const uint32_t sbo = 16 * KA;
            const uint32_t w_base = smem_u32(w_smem), a_base = smem_u32(a_smem);
            uint32_t st = 0, aph = 0, db = 0, dph = 0, wph = 0;
            bool ok = true;
            for (uint64_t L = L0; L < L1 && ok; L++) {
                const uint32_t tt = (uint32_t)(L % tpc);
                if (L == L0 || tt == 0) {
                    if (!mbar_wait(w_full, wph, abort, kWaitBudget)) { record_abort(abort, 1); ok = false; break; }
                }
                if (!mbar_wait(&a_full[st], aph, abort, kWaitBudget)) { record_abort(abort, 2); ok = false; break; }
                if (!mbar_wait(&d_empty[db], dph ^ 1, abort, kWaitBudget)) { record_abort(abort, 3); ok = false; break; }
                tc_fence_after();
                const uint32_t a_stage = a_base + st * 4 * blkA;
                for (uint32_t p = 0; p < 2; p++) {
                    const uint32_t d = tmem + db * (4 * NB) + p * (2 * NB);
                    uint32_t acc = 0;
                    for (uint32_t h = 0; h < 2; h++) {
                        const uint32_t wblk = w_base + (p * 2 + h) * 3 * blkW;
                        for (uint32_t ri = 0; ri < 2; ri++) {
                            const uint32_t abase = a_stage + (p * 2 + ri) * blkA;
                            const uint32_t bbase = wblk + (ri == 0 ? 1 : 0) * blkW;
                            for (uint32_t ks = 0; ks < KA / 16; ks++) {
                                const uint64_t ad = smem_desc(abase + ks * 256, 128, sbo);
                                const uint64_t bd = smem_desc(bbase + ks * 256, 128, sbo);
                                mma_f16(d, ad, bd, idesc, acc);
                                acc = 1;
                            }
                        }
                    }
                }
                mma_commit(&a_empty[st]);
                mma_commit(&d_full[db]);
                if (tt == tpc - 1 || L + 1 == L1) {
                    mma_commit(w_empty);
                    wph ^= 1;
                }
                if (++st == S) { st = 0; aph ^= 1; }
                if (++db == 2) { db = 0; dph ^= 1; }
            }
            // Drain every MMA issued by this thread before TMEM is released
            // (bounded, but not cut short by the abort flag).
            mma_commit(fin);
            if (!mbar_wait(fin, 0, &never, kWaitBudget)) record_abort(abort, 4);
        }
    } else if (warp == 1) {
        // ---------------- phasor image loader ----------------
        if (lane == 0 && L0 < L1) {
            uint32_t wph = 0;
            bool issued = false;
            for (uint64_t L = L0; L < L1; L++) {
                const uint32_t tt = (uint32_t)(L % tpc);
                if (!(L == L0 || tt == 0)) continue;
                if (!mbar_wait(w_empty, wph ^ 1, abort, kWaitBudget)) { record_abort(abort, 5); break; }
                const uint32_t f = (uint32_t)(L / tpc);
                mbar_arrive_expect_tx(w_full, g.img_bytes);
                bulk_g2s(w_smem, g.plan + (uint64_t)f * g.img_bytes, g.img_bytes, w_full);
                issued = true;
                wph ^= 1;
            }
            // The last copy must land before the CTA exits.
            if (issued && !mbar_wait(w_full, wph ^ 1, &never, kWaitBudget)) record_abort(abort, 6);
        }
    } else if (warp < 2 + kEpiWarps) {
        // ---------------- epilogue ----------------
        const uint32_t q = warp & 3;  // TMEM lane quarter this warp may access
        const uint32_t rows_per_k = kM / R;
        const uint32_t row = 32 * q + lane;
        const uint32_t k = row / rows_per_k;
        const uint32_t s_local = row - k * rows_per_k;
        const uint32_t I = g.integ;
        const bool leader = (lane % I) == 0;
        uint32_t db = 0, dph = 0;
        for (uint64_t L = L0; L < L1; L++) {
            if (!mbar_wait(&d_full[db], dph, abort, kWaitBudget)) { record_abort(abort, 7); break; }
            tc_fence_after();
            const uint32_t f = (uint32_t)(L / tpc), tt = (uint32_t)(L % tpc);
            const uint32_t u = (tt * rows_per_k + s_local) / I;
            const uint32_t lane_addr = tmem + ((32 * q) << 16) + db * (4 * NB);
            for (uint32_t bc = 0; bc < NB; bc += 16) {
                float pw[16];
#pragma unroll
                for (int j = 0; j < 16; j++) pw[j] = 0.f;
#pragma unroll
                for (uint32_t p = 0; p < 2; p++) {
                    uint32_t re[16], im[16];
                    tmem_ld16(lane_addr + p * (2 * NB) + bc, re);
                    tmem_ld16(lane_addr + p * (2 * NB) + NB + bc, im);
                    tmem_ld_wait();
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        const float a = __uint_as_float(re[j]), b = __uint_as_float(im[j]);
                        pw[j] = fmaf(a, a, fmaf(b, b, pw[j]));
                    }
                }
                for (uint32_t o = 1; o < I; o <<= 1) {
#pragma unroll
                    for (int j = 0; j < 16; j++) pw[j] += __shfl_xor_sync(0xffffffffu, pw[j], o);
                }
                if (leader) {
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        const uint32_t b = bc + j;
                        if (b < g.beams) g.out[((uint64_t)(b * (uint64_t)g.F + f) * R + k) * g.U + u] = pw[j];
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&d_empty[db]);
            if (++db == 2) { db = 0; dph ^= 1; }
        }
    } else {
        // ---------------- operand build ----------------
        const uint32_t ct = threadIdx.x - (2 + kEpiWarps) * 32;  // 0..255
        const uint32_t spectra = kM / R;
        const uint32_t groups = KA / 8;
        const uint32_t ntasks = spectra * groups;
        const uint64_t ch_stride = (uint64_t)g.T * 4;  // bytes between (a, f) rows... per channel
        uint32_t st = 0, aph = 0;
        for (uint64_t L = L0; L < L1; L++) {
            if (!mbar_wait(&a_empty[st], aph ^ 1, abort, kWaitBudget)) { record_abort(abort, 8); break; }
            const uint32_t f = (uint32_t)(L / tpc), tt = (uint32_t)(L % tpc);
            uint8_t* stage = a_smem + (size_t)st * 4 * blkA;
            for (uint32_t task = ct; task < ntasks; task += kConvWarps * 32) {
                const uint32_t s = task % spectra, grp = task / spectra;
                const uint32_t t = tt * kM + s * R;
                // Raw samples: [antenna][R samples], one 32-bit word per sample.
                uint32_t raw[8][R];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const uint32_t a = grp * 8 + i;
                    if (a < g.A) {
                        const uint8_t* src = g.in + ((uint64_t)a * g.F + f) * ch_stride + (uint64_t)t * 4;
                        if (R == 4) {
                            uint4 v = ldg_nc_u4(src);
                            raw[i][0] = v.x;
                            raw[i][R > 1 ? 1 : 0] = v.y;
                            raw[i][R > 2 ? 2 : 0] = v.z;
                            raw[i][R > 3 ? 3 : 0] = v.w;
                        } else if (R == 2) {
                            uint2 v = __ldg(reinterpret_cast<const uint2*>(src));
                            raw[i][0] = v.x;
                            raw[i][R > 1 ? 1 : 0] = v.y;
                        } else {
                            raw[i][0] = __ldg(reinterpret_cast<const uint32_t*>(src));
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < R; j++) raw[i][j] = 0u;
                    }
                }
#pragma unroll
                for (int p = 0; p < 2; p++) {
                    // Z[i][k] = (re, im) half2 of fine channel k for antenna 8 grp + i.
                    half2 Z[8][R];
#pragma unroll
                    for (int i = 0; i < 8; i++) {
                        if (R == 1) {
                            Z[i][0] = sample_h2(raw[i][0], p);
                        } else if (R == 2) {
                            const half2 x0 = sample_h2(raw[i][0], p), x1 = sample_h2(raw[i][R - 1], p);
                            Z[i][0] = __hsub2(x0, x1);       // k = 0: x0 - x1
                            Z[i][R - 1] = __hadd2(x0, x1);   // k = 1: x0 + x1
                        } else {
                            const half2 x0 = sample_h2(raw[i][0], p), x1 = sample_h2(raw[i][R > 1 ? 1 : 0], p);
                            const half2 x2 = sample_h2(raw[i][R > 2 ? 2 : 0], p), x3 = sample_h2(raw[i][R > 3 ? 3 : 0], p);
                            const half2 e02 = __hadd2(x0, x2), d02 = __hsub2(x0, x2);
                            const half2 e13 = __hadd2(x1, x3), d13 = __hsub2(x1, x3);
                            // i * d13 = (-d13.im, d13.re)
                            const half2 id13 = __hmul2(__lowhigh2highlow(d13),
                                                       __halves2half2(__float2half(-1.f), __float2half(1.f)));
                            Z[i][0] = __hsub2(e02, e13);                  // x0 - x1 + x2 - x3
                            Z[i][R > 1 ? 1 : 0] = __hadd2(d02, id13);     // x0 + i x1 - x2 - i x3
                            Z[i][R > 2 ? 2 : 0] = __hadd2(e02, e13);      // x0 + x1 + x2 + x3
                            Z[i][R > 3 ? 3 : 0] = __hsub2(d02, id13);     // x0 - i x1 - x2 + i x3
                        }
                    }
#pragma unroll
                    for (int kk = 0; kk < R; kk++) {
                        uint4 vr, vi;
                        uint32_t* pr = &vr.x;
                        uint32_t* pi = &vi.x;
#pragma unroll
                        for (int i = 0; i < 4; i++) {
                            const uint32_t lo = h2u(Z[2 * i][kk]), hi = h2u(Z[2 * i + 1][kk]);
                            pr[i] = __byte_perm(lo, hi, 0x5410);  // (re_a, re_a+1)
                            pi[i] = __byte_perm(lo, hi, 0x7632);  // (im_a, im_a+1)
                        }
                        const uint32_t r = kk * spectra + s;
                        const uint32_t off = cm_off(r, grp, KA);
                        *reinterpret_cast<uint4*>(stage + (p * 2 + 0) * blkA + off) = vr;
                        *reinterpret_cast<uint4*>(stage + (p * 2 + 1) * blkA + off) = vi;
                    }
                }
            }
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(&a_full[st]);
            if (++st == S) { st = 0; aph ^= 1; }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, tmem_cols);
    }
}

// ---- phasor image ------------------------------------------------------------
// plan[chunk][f][p][h][blk][core-matrix layout of NB x KA fp16],
// blk 0 = -Wi, 1 = Wr, 2 = Wi; h 0 = hi = rn(w), h 1 = lo = rn(w - hi).
__global__ void __launch_bounds__(256) tc_prepare_kernel(const float2* __restrict__ ph, uint8_t* __restrict__ plan,
                                                         uint32_t B, uint32_t A, uint32_t F, uint32_t NB,
                                                         uint32_t KA, uint32_t nchunks) {
    const uint64_t n = (uint64_t)nchunks * F * 2 * NB * KA;
    const uint32_t blk = NB * KA * 2;
    const uint64_t img = 12ull * blk;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t a = (uint32_t)(i % KA);
        uint64_t r = i / KA;
        const uint32_t nb = (uint32_t)(r % NB);
        r /= NB;
        const uint32_t p = (uint32_t)(r % 2);
        r /= 2;
        const uint32_t f = (uint32_t)(r % F);
        const uint32_t c = (uint32_t)(r / F);
        const uint32_t b = c * kMaxNB + nb;
        float wr = 0.f, wi = 0.f;
        if (a < A && b < B && nb < NB) {
            const float2 w = ph[((uint64_t)(b * (uint64_t)A + a) * F + f) * 2 + p];
            wr = w.x;
            wi = w.y;
        }
        const __half rh = __float2half_rn(wr), ih = __float2half_rn(wi);
        const __half rl = __float2half_rn(wr - __half2float(rh)), il = __float2half_rn(wi - __half2float(ih));
        uint8_t* base = plan + ((uint64_t)c * F + f) * img;
        const uint32_t off = (nb >> 3) * (16u * KA) + (a >> 3) * 128u + (nb & 7u) * 16u + (a & 7u) * 2u;
        __half* hb = reinterpret_cast<__half*>(base + (p * 2 + 0) * 3 * blk + off);
        __half* lb = reinterpret_cast<__half*>(base + (p * 2 + 1) * 3 * blk + off);
        hb[0] = __hneg(ih);
        hb[blk / 2] = rh;
        hb[blk] = ih;
        lb[0] = __hneg(il);
        lb[blk / 2] = rl;
        lb[blk] = il;
    }
}

struct TcShape {
    uint32_t NB, KA, nchunks, img_bytes, stages;
    size_t smem;
};

bool tc_shape(uint64_t B, uint64_t A, TcShape& s) {
    if (A == 0 || A > kMaxKA || B == 0) return false;
    const uint64_t bc = B < (uint64_t)kMaxNB ? B : (uint64_t)kMaxNB;
    s.NB = (uint32_t)((bc + 15) / 16 * 16);
    s.KA = (uint32_t)((A + 15) / 16 * 16);
    s.nchunks = (uint32_t)((B + kMaxNB - 1) / kMaxNB);
    s.img_bytes = 12u * s.NB * s.KA * 2u;
    const size_t stage = 4ull * kM * s.KA * 2;
    const size_t fixed = s.img_bytes + 256;  // barriers, TMEM slot, abort flag
    const size_t limit = 227 * 1024;
    size_t st = (limit - fixed) / stage;
    if (st > 4) st = 4;
    if (st < 2) return false;
    s.stages = (uint32_t)st;
    s.smem = fixed + st * stage;
    return true;
}

int g_tc_sms = 0;

}  // namespace
}  // namespace bb

using namespace bb;

extern "C" uint64_t blade_beamform_tc_plan_size(uint64_t B, uint64_t A, uint64_t F, uint64_t P) {
    TcShape s;
    if (P != 2 || !tc_shape(B, A, s)) return 0;
    return (uint64_t)s.nchunks * F * s.img_bytes;
}

extern "C" int blade_beamform_tc_prepare(const void* phasors, void* plan, uint64_t B, uint64_t A, uint64_t F,
                                         uint64_t P, blade_stream_t stream) {
    TcShape s;
    if (P != 2) return set_error(BLADE_ERROR, "blade_beamform_tc_prepare: P must be 2");
    if (!tc_shape(B, A, s))
        return set_error(BLADE_ERROR, "blade_beamform_tc_prepare: unsupported shape (A=%llu must be 1..64)",
                         (unsigned long long)A);
    if (F == 0) return BLADE_SUCCESS;
    if (!phasors || !plan) return set_error(BLADE_ERROR, "blade_beamform_tc_prepare: null buffer");
    if (!aligned16(plan)) return set_error(BLADE_ERROR, "blade_beamform_tc_prepare: plan must be 16-byte aligned");
    const uint64_t n = (uint64_t)s.nchunks * F * 2 * s.NB * s.KA;
    tc_prepare_kernel<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        static_cast<const float2*>(phasors), static_cast<uint8_t*>(plan), (uint32_t)B, (uint32_t)A, (uint32_t)F,
        s.NB, s.KA, s.nchunks);
    return check_launch("blade_beamform_tc_prepare");
}

extern "C" int blade_beamform_detect_tc_supported(uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                                  uint64_t rate, uint64_t integration) {
    TcShape s;
    if (P != 2 || !tc_shape(B, A, s)) return 0;
    if (rate != 1 && rate != 2 && rate != 4) return 0;
    if (integration == 0 || integration > 32 || (integration & (integration - 1)) != 0) return 0;
    if (T == 0 || T % kM != 0 || F == 0) return 0;
    if (F > 0xffffffffull / (T / kM) || T >= (1ull << 31)) return 0;
    return 1;
}

extern "C" int blade_beamform_detect_tc(const void* in, const void* plan, void* out, uint64_t B, uint64_t A,
                                        uint64_t F, uint64_t T, uint64_t P, uint64_t rate, uint64_t integration,
                                        blade_stream_t stream) {
    if (!blade_beamform_detect_tc_supported(B, A, F, T, P, rate, integration))
        return set_error(BLADE_ERROR,
                         "blade_beamform_detect_tc: unsupported configuration (B=%llu A=%llu T=%llu P=%llu rate=%llu "
                         "I=%llu): needs P=2, 1<=A<=64, T%%128==0, rate in {1,2,4}, I a power of two <= 32",
                         (unsigned long long)B, (unsigned long long)A, (unsigned long long)T, (unsigned long long)P,
                         (unsigned long long)rate, (unsigned long long)integration);
    if (!in || !plan || !out) return set_error(BLADE_ERROR, "blade_beamform_detect_tc: null buffer");
    if (!aligned16(in) || !aligned16(plan) || (reinterpret_cast<uintptr_t>(out) & 3))
        return set_error(BLADE_ERROR, "blade_beamform_detect_tc: input and plan must be 16-byte aligned");
    TcShape s;
    tc_shape(B, A, s);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const void* fn = rate == 1 ? reinterpret_cast<const void*>(bf_tc_kernel<1>)
                     : rate == 2 ? reinterpret_cast<const void*>(bf_tc_kernel<2>)
                                 : reinterpret_cast<const void*>(bf_tc_kernel<4>);
    if (int rc = ensure_smem(fn, s.smem)) return rc;
    const uint32_t U = (uint32_t)(T / (rate * integration));
    for (uint32_t c = 0; c < s.nchunks; c++) {
        TcArgs g;
        g.in = static_cast<const uint8_t*>(in);
        g.plan = static_cast<const uint8_t*>(plan) + (uint64_t)c * F * s.img_bytes;
        g.out = static_cast<float*>(out) + (uint64_t)c * kMaxNB * F * rate * U;
        g.A = (uint32_t)A;
        g.F = (uint32_t)F;
        g.T = (uint32_t)T;
        const uint64_t rem = B - (uint64_t)c * kMaxNB;
        g.beams = (uint32_t)(rem < (uint64_t)kMaxNB ? rem : kMaxNB);
        g.U = U;
        g.integ = (uint32_t)integration;
        g.NB = s.NB;
        g.KA = s.KA;
        g.stages = s.stages;
        g.img_bytes = s.img_bytes;
        g.tiles_per_ch = (uint32_t)(T / kM);
        g.total_tiles = (uint64_t)F * (T / kM);
        uint64_t grid = (uint64_t)sm_count();
        if (grid > g.total_tiles) grid = g.total_tiles;
        if (rate == 1) bf_tc_kernel<1><<<(unsigned)grid, kThreads, s.smem, st>>>(g);
        else if (rate == 2) bf_tc_kernel<2><<<(unsigned)grid, kThreads, s.smem, st>>>(g);
        else bf_tc_kernel<4><<<(unsigned)grid, kThreads, s.smem, st>>>(g);
        if (int rc = check_launch("blade_beamform_detect_tc")) return rc;
    }
    (void)g_tc_sms;
    return BLADE_SUCCESS;
}

extern "C" int blade_device_status(uint32_t* status) {
    unsigned int v = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(v));
    if (e != cudaSuccess) return check_cuda(e, "blade_device_status");
    e = cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(zero));
    if (e != cudaSuccess) return check_cuda(e, "blade_device_status");
    if (status) *status = v;
    return BLADE_SUCCESS;
}

// ---- allocation-free variant ---------------------------------------------------
// For callers that must not allocate device memory while they stream: an online
// beamformer that sizes its whole GPU budget once at start-up and then runs a
// fixed-cadence loop cannot call cudaMalloc / cudaFree per block, because those
// calls synchronise the device and take unbounded time, which the loop's
// real-time deadline cannot absorb.  This entry point keeps the phasor image in a
// fixed device array that every GPU loading the library holds until exit.

// Scratch for the phasor image: 8 MiB per device.
static __device__ __align__(256) uint8_t g_tc_noalloc_plan[8u << 20];

namespace {

constexpr uint64_t kNoAllocPlanBytes = 8ull << 20;

// Device address of g_tc_noalloc_plan, looked up once per device with that device
// current (the host-side name is only a stand-in for the device array).
int noalloc_plan_address(void** out) {
    static std::mutex mu;
    static void* addr[64] = {nullptr};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return check_cuda(e, "blade_beamform_detect_tc_noalloc");
    if (dev < 0 || dev >= 64) return set_error(BLADE_ERROR, "blade_beamform_detect_tc_noalloc: device %d", dev);
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_tc_noalloc_plan);
        if (e != cudaSuccess) return check_cuda(e, "blade_beamform_detect_tc_noalloc: cudaGetSymbolAddress");
        addr[dev] = p;
    }
    *out = addr[dev];
    return BLADE_SUCCESS;
}

}  // namespace

extern "C" int blade_beamform_detect_tc_noalloc(const void* in, const void* phasors, void* out, uint64_t B,
                                                uint64_t A, uint64_t F, uint64_t T, uint64_t P, uint64_t rate,
                                                uint64_t integration, blade_stream_t stream) {
    if (!blade_beamform_detect_tc_supported(B, A, F, T, P, rate, integration))
        return set_error(BLADE_ERROR,
                         "blade_beamform_detect_tc_noalloc: unsupported configuration (needs P=2, 1<=A<=64, "
                         "T%%128==0, rate in {1,2,4}, I a power of two <= 32)");
    const uint64_t need = blade_beamform_tc_plan_size(B, A, F, P);
    if (need > kNoAllocPlanBytes)
        return set_error(BLADE_ERROR,
                         "blade_beamform_detect_tc_noalloc: the phasor image for B=%llu A=%llu F=%llu needs %llu "
                         "bytes, above the %llu-byte static workspace; use blade_beamform_tc_prepare + "
                         "blade_beamform_detect_tc with a caller-allocated image",
                         (unsigned long long)B, (unsigned long long)A, (unsigned long long)F,
                         (unsigned long long)need, (unsigned long long)kNoAllocPlanBytes);
    void* plan = nullptr;
    if (int rc = noalloc_plan_address(&plan)) return rc;
    if (int rc = blade_beamform_tc_prepare(phasors, plan, B, A, F, P, stream)) return rc;
    return blade_beamform_detect_tc(in, plan, out, B, A, F, T, P, rate, integration, stream);
}
