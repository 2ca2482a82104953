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
// row = k * (128/R) + spectrum), k = [Xr of KA antennas | Xi of KA antennas]
// (KA = 32 or 64, antennas zero-padded), and the complex product embedded in reals
// (NB = beams of a 64-beam chunk padded to 16):
//   Re y = Xr Wr - Xi Wi,   Im y = Xr Wi + Xi Wr
// Three phasor-image layouts, all K-major with the 128-byte swizzle:
//   NB <= 32 ("stacked"): rows [hi Re | hi Im | lo Re | lo Im] x NB, K = 2 KA, so
//            one MMA per k-step with N = 4 NB gives both hi and lo products;
//   KA = 64: blocks [-Wi | Wr | Wi] per (p, hi/lo); the Xr k-steps read the window
//            [Wr | Wi], the Xi k-steps [-Wi | Wr] (N = 2 NB);
//   KA = 32: one embedded block of 2 NB rows per (p, hi/lo), K = 2 KA.
// Each 64-element K block of an operand is 128 rows x 128 bytes (16 KB).
//
// CTA organisation (persistent, one CTA per SM, 15 warps):
//   warp 0      TMEM allocation; lane 0 issues tcgen05.mma and commits (MMA
//               issuer 0; warp 14 is issuer 1 when two issuers apply)
//   warp 1      loader: the per-channel phasor image (one bulk copy) and the raw
//               CI8 tiles (one 3-D TMA tensor load per tile: 128 samples x 1
//               channel x A antennas) into a ring of raw stages
//   warps 2-5   epilogue: tcgen05.ld of the accumulators, |.|^2 over both
//               polarisations, window sums with lane shuffles, Stokes-I stores
//   warps 6-13  operand build from the raw ring: DFT, exact int8 -> FP16
//               conversion, swizzled stores; both polarisations of a tile in one
//               pass when the operand ring holds at least two tiles
// Pipelines (full/empty mbarrier pairs): raw stages, operand stages (one per tile
// and polarisation), up to four TMEM accumulator buffers, the phasor image.  Every
// wait is bounded (clock budget plus a shared abort flag) and sleeps on the
// mbarrier rather than spinning; on expiry the kernel records a status word,
// drains its own MMAs and copies, frees TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <string.h>

#include <mutex>

#include "autotune.cuh"
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
constexpr int kEpiWarps = 4;  // one or two per TMEM lane quarter
constexpr int kEpiGroups = kEpiWarps / 4;  // warps per lane quarter, each a share of the beams
constexpr int kWarps = 3 + kEpiWarps + kConvWarps;  // + MMA issuer 0, loader, MMA issuer 1
constexpr int kThreads = kWarps * 32;               // 480
constexpr int kMaxNB = 64;
constexpr int kMaxKA = 64;
constexpr int kMaxAcc = 4;   // TMEM accumulator buffers
constexpr int kMaxStages = 8;  // operand stages and raw stages, each
constexpr long long kWaitBudget = 4000000000ll;  // cycles (~2 s) before a wait gives up

struct TcArgs {
    const uint8_t* in;    // CI8 [A, F, T, 2]
    const uint8_t* plan;  // phasor images, one per channel, img_bytes each
    float* out;           // [beams, F*R, U]
    uint32_t A, F, T, beams, U;
    uint32_t NB, KA, a_stages, r_stages, stacked;
    uint32_t img_bytes, raw_bytes, tiles_per_ch;
    uint32_t raw_tiles, raw_row;  // tiles per raw stage (1, 2 or 4) and its antenna row stride (raw_tiles * 512)
    uint64_t total_tiles;
    uint32_t pdl;  // launched as a programmatic dependent of the phasor split: wait for it before the image
    uint32_t direct;  // R = 1 CI8 without a raw ring: converter threads load the voltages themselves
    uint32_t transposed;  // outputs along TMEM lanes, samples along columns (64-beam chunks, rate 1, I = 8 or 16)
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
__device__ __forceinline__ half2 u2h(uint32_t u) { return *reinterpret_cast<half2*>(&u); }

// Address of K element k_total (a multiple of 4) of row `row` in one
// polarisation's operand: Xr occupies k_total in [0, KA), Xi [KA, 2 KA); every
// 64 K elements form one 128-row x 128-byte swizzled block of 16 KB.
__device__ __forceinline__ uint32_t op_off(uint32_t row, uint32_t k_total) {
    return (k_total >> 6) * 16384u + sw128_off(row, (k_total >> 3) & 7u) + ((k_total & 4u) << 1);
}

__device__ __forceinline__ void record_abort(volatile int* abort, unsigned code) {
    *abort = 1;
    atomicCAS(&g_tc_status, 0u, code);
}

// rate-4 spectrum of one antenna and polarisation from its 4 sample words:
// Z[k] = sum_j (-1)^j x_j e^{-2 pi i j k / 4}, exact in FP16 (|Z| <= 512).
__device__ __forceinline__ void dft4_h2(uint4 v, int p, half2 (&Z)[4]) {
    const half2 x0 = sample_h2(v.x, p), x1 = sample_h2(v.y, p), x2 = sample_h2(v.z, p), x3 = sample_h2(v.w, p);
    const half2 e02 = __hadd2(x0, x2), d02 = __hsub2(x0, x2);
    const half2 e13 = __hadd2(x1, x3), d13 = __hsub2(x1, x3);
    const half2 id13 = __hmul2(__lowhigh2highlow(d13), __halves2half2(__float2half(-1.f), __float2half(1.f)));
    Z[0] = __hsub2(e02, e13);  // x0 - x1 + x2 - x3
    Z[1] = __hadd2(d02, id13); // x0 + i x1 - x2 - i x3
    Z[2] = __hadd2(e02, e13);  // x0 + x1 + x2 + x3
    Z[3] = __hsub2(d02, id13); // x0 - i x1 - x2 + i x3
}

// R = 1 operand chunk: 8 antennas of one sample -> (re, im) chunks of polarisation p.
__device__ __forceinline__ void r1_chunks(const uint32_t (&w)[8], int p, uint4& vr, uint4& vi) {
    const uint32_t sre = p ? 0x0602u : 0x0400u, sim = p ? 0x0703u : 0x0501u;
    vr.x = cvt_pair(__byte_perm(w[0], w[1], sre));
    vr.y = cvt_pair(__byte_perm(w[2], w[3], sre));
    vr.z = cvt_pair(__byte_perm(w[4], w[5], sre));
    vr.w = cvt_pair(__byte_perm(w[6], w[7], sre));
    vi.x = cvt_pair(__byte_perm(w[0], w[1], sim));
    vi.y = cvt_pair(__byte_perm(w[2], w[3], sim));
    vi.z = cvt_pair(__byte_perm(w[4], w[5], sim));
    vi.w = cvt_pair(__byte_perm(w[6], w[7], sim));
}

// Builds the operand rows of polarisation p for one tile from the raw stage in
// shared memory (antenna-major rows of rrow bytes; `raw` points at this tile's
// 128 samples x 4 bytes in the first row).
// Row = k * (128 / R) + spectrum.  Consecutive lanes take consecutive rows, so
// every 16-byte store of a warp lands in a distinct bank group of the swizzle.
template <int R>
__device__ __forceinline__ void build_operand(const uint8_t* raw, uint32_t rrow, uint8_t* op, uint32_t A, uint32_t KA,
                                              int p, uint32_t ct) {
    constexpr uint32_t kStride = kConvWarps * 32;
    if constexpr (R == 1) {
        const uint32_t ntasks = kM * (KA / 8);
        // Two tasks per pass: both tasks' shared-memory loads are in flight together.
        for (uint32_t t0 = ct; t0 < ntasks; t0 += 2 * kStride) {
            const uint32_t t1 = t0 + kStride;
            const bool has1 = t1 < ntasks;
            const uint32_t s0 = t0 % kM, g0 = t0 / kM, s1 = t1 % kM, g1 = t1 / kM;
            uint32_t w0[8], w1[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const uint32_t a0 = g0 * 8 + i, a1 = g1 * 8 + i;
                w0[i] = a0 < A ? *reinterpret_cast<const uint32_t*>(raw + a0 * rrow + s0 * 4) : 0u;
                w1[i] = (has1 && a1 < A) ? *reinterpret_cast<const uint32_t*>(raw + a1 * rrow + s1 * 4) : 0u;
            }
            uint4 vr, vi;
            r1_chunks(w0, p, vr, vi);
            *reinterpret_cast<uint4*>(op + op_off(s0, g0 * 8)) = vr;
            *reinterpret_cast<uint4*>(op + op_off(s0, KA + g0 * 8)) = vi;
            if (has1) {
                r1_chunks(w1, p, vr, vi);
                *reinterpret_cast<uint4*>(op + op_off(s1, g1 * 8)) = vr;
                *reinterpret_cast<uint4*>(op + op_off(s1, KA + g1 * 8)) = vi;
            }
        }
    } else if constexpr (R == 2) {
        const uint32_t ntasks = (kM / 2) * (KA / 8);
        for (uint32_t task = ct; task < ntasks; task += kStride) {
            const uint32_t s = task % (kM / 2), grp = task / (kM / 2);
            uint2 v[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const uint32_t a = grp * 8 + i;
                v[i] = a < A ? *reinterpret_cast<const uint2*>(raw + a * rrow + s * 8) : make_uint2(0u, 0u);
            }
            half2 Z0[8], Z1[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const half2 x0 = sample_h2(v[i].x, p), x1 = sample_h2(v[i].y, p);
                Z0[i] = __hsub2(x0, x1);  // k = 0: x0 - x1
                Z1[i] = __hadd2(x0, x1);  // k = 1: x0 + x1
            }
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const half2* Z = k ? Z1 : Z0;
                uint4 vr, vi;
                vr.x = __byte_perm(h2u(Z[0]), h2u(Z[1]), 0x5410);
                vr.y = __byte_perm(h2u(Z[2]), h2u(Z[3]), 0x5410);
                vr.z = __byte_perm(h2u(Z[4]), h2u(Z[5]), 0x5410);
                vr.w = __byte_perm(h2u(Z[6]), h2u(Z[7]), 0x5410);
                vi.x = __byte_perm(h2u(Z[0]), h2u(Z[1]), 0x7632);
                vi.y = __byte_perm(h2u(Z[2]), h2u(Z[3]), 0x7632);
                vi.z = __byte_perm(h2u(Z[4]), h2u(Z[5]), 0x7632);
                vi.w = __byte_perm(h2u(Z[6]), h2u(Z[7]), 0x7632);
                const uint32_t row = k * (kM / 2) + s;
                *reinterpret_cast<uint4*>(op + op_off(row, grp * 8)) = vr;
                *reinterpret_cast<uint4*>(op + op_off(row, KA + grp * 8)) = vi;
            }
        }
    } else {
        // R == 4: a task is one spectrum of 4 antennas (half a K chunk, 8-byte stores).
        const uint32_t ntasks = (kM / 4) * (KA / 4);
        for (uint32_t task = ct; task < ntasks; task += kStride) {
            const uint32_t s = task % (kM / 4), g4 = task / (kM / 4);
            uint4 v[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t a = g4 * 4 + i;
                v[i] = a < A ? *reinterpret_cast<const uint4*>(raw + a * rrow + s * 16) : make_uint4(0u, 0u, 0u, 0u);
            }
            half2 Z[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++) dft4_h2(v[i], p, Z[i]);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                uint2 vr, vi;
                vr.x = __byte_perm(h2u(Z[0][k]), h2u(Z[1][k]), 0x5410);
                vr.y = __byte_perm(h2u(Z[2][k]), h2u(Z[3][k]), 0x5410);
                vi.x = __byte_perm(h2u(Z[0][k]), h2u(Z[1][k]), 0x7632);
                vi.y = __byte_perm(h2u(Z[2][k]), h2u(Z[3][k]), 0x7632);
                const uint32_t row = k * (kM / 4) + s;
                *reinterpret_cast<uint2*>(op + op_off(row, g4 * 4)) = vr;
                *reinterpret_cast<uint2*>(op + op_off(row, KA + g4 * 4)) = vi;
            }
        }
    }
}

// R = 4, both polarisations in one pass.  Each sample word is split into two
// half2 words with the polarisations in the two halves, RE = (p0 re, p1 re) and
// IM = (p0 im, p1 im), read exactly as 1024 + (x + 128) = 1152 + x through the
// 0x64 exponent byte (one XOR of the sign bits, two byte permutes).  The DFT then
// runs in FP16 on the FMA pipe (the integer pipe issues at half rate): every
// intermediate is an integer of magnitude < 2048, so all of it is exact, and the
// 1152 biases cancel in differences or are removed together (x0 + x2 =
// ((1024 + u0) - 2304) + (1024 + u2) with both steps exact).  A warp covers 16
// spectra x 8 antennas (two 4-antenna groups): lanes 0-7 and 8-15 write the two
// 8-byte halves of one 16-byte chunk for 8 rows with distinct swizzle slots, lanes
// 16-31 the next 8 rows, so each 8-byte store is two conflict-free wavefronts.
// Row k * 32 + s of an operand sits 4096 * k bytes after row s (the swizzle phase
// depends on s only), so a task's addresses are fixed offsets computed once.
struct R4Task {
    uint32_t raw_off;  // a0 * rrow + s * 16 in the raw stage
    uint32_t o_r, o_i; // operand offsets of (row s, K = a0) and (row s, K = KA + a0)
    uint32_t nvalid;   // antennas a0 .. a0 + nvalid - 1 exist (0..4)
};

__device__ __forceinline__ R4Task r4_task(uint32_t wt, uint32_t lane, uint32_t A, uint32_t KA, uint32_t rrow) {
    const uint32_t c = wt >> 1;
    const uint32_t s = (wt & 1u) * 16u + (lane & 7u) + ((lane >> 4) << 3);
    const uint32_t a0 = (2u * c + ((lane >> 3) & 1u)) * 4u;
    R4Task t;
    t.raw_off = a0 * rrow + s * 16u;
    t.o_r = op_off(s, a0);
    t.o_i = op_off(s, KA + a0);
    t.nvalid = a0 < A ? min(4u, A - a0) : 0u;
    return t;
}

__device__ __forceinline__ void r4_pair_task(const uint8_t* raw, uint32_t rrow, uint8_t* op0, uint8_t* op1,
                                             const R4Task& t) {
    const half2 h2304 = __halves2half2(__ushort_as_half(0x6880), __ushort_as_half(0x6880));  // 2304
    uint2 out_r[2][4], out_i[2][4];  // [pol][k]
    if (t.nvalid) {
        half2 zr[4][4], zi[4][4];  // [antenna][k], halves = (pol 0, pol 1)
        const uint8_t* src = raw + t.raw_off;
#pragma unroll
        for (uint32_t i = 0; i < 4; i++) {
            const uint4 v = i < t.nvalid ? *reinterpret_cast<const uint4*>(src + i * rrow) : make_uint4(0u, 0u, 0u, 0u);
            const uint32_t w[4] = {v.x ^ 0x80808080u, v.y ^ 0x80808080u, v.z ^ 0x80808080u, v.w ^ 0x80808080u};
            half2 re[4], im[4];  // 1152 + x
#pragma unroll
            for (int j = 0; j < 4; j++) {
                re[j] = u2h(__byte_perm(w[j], 0x64646464u, 0x4240));
                im[j] = u2h(__byte_perm(w[j], 0x64646464u, 0x4341));
            }
            const half2 aR = __hadd2(__hsub2(re[0], h2304), re[2]);  // x0 + x2
            const half2 bR = __hadd2(__hsub2(re[1], h2304), re[3]);  // x1 + x3
            const half2 cR = __hsub2(re[0], re[2]), dR = __hsub2(re[1], re[3]);
            const half2 aI = __hadd2(__hsub2(im[0], h2304), im[2]);
            const half2 bI = __hadd2(__hsub2(im[1], h2304), im[3]);
            const half2 cI = __hsub2(im[0], im[2]), dI = __hsub2(im[1], im[3]);
            zr[i][0] = __hsub2(aR, bR);  // x0 - x1 + x2 - x3
            zi[i][0] = __hsub2(aI, bI);
            zr[i][1] = __hsub2(cR, dI);  // x0 + i x1 - x2 - i x3
            zi[i][1] = __hadd2(cI, dR);
            zr[i][2] = __hadd2(aR, bR);  // x0 + x1 + x2 + x3
            zi[i][2] = __hadd2(aI, bI);
            zr[i][3] = __hadd2(cR, dI);  // x0 - i x1 - x2 + i x3
            zi[i][3] = __hsub2(cI, dR);
        }
#pragma unroll
        for (int p = 0; p < 2; p++) {
            const uint32_t sel = p ? 0x7632u : 0x5410u;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                out_r[p][k].x = __byte_perm(h2u(zr[0][k]), h2u(zr[1][k]), sel);
                out_r[p][k].y = __byte_perm(h2u(zr[2][k]), h2u(zr[3][k]), sel);
                out_i[p][k].x = __byte_perm(h2u(zi[0][k]), h2u(zi[1][k]), sel);
                out_i[p][k].y = __byte_perm(h2u(zi[2][k]), h2u(zi[3][k]), sel);
            }
        }
    } else {
#pragma unroll
        for (int p = 0; p < 2; p++)
#pragma unroll
            for (int k = 0; k < 4; k++) out_r[p][k] = out_i[p][k] = make_uint2(0u, 0u);
    }
#pragma unroll
    for (uint32_t k = 0; k < 4; k++) {
        *reinterpret_cast<uint2*>(op0 + t.o_r + k * 4096u) = out_r[0][k];
        *reinterpret_cast<uint2*>(op0 + t.o_i + k * 4096u) = out_i[0][k];
        *reinterpret_cast<uint2*>(op1 + t.o_r + k * 4096u) = out_r[1][k];
        *reinterpret_cast<uint2*>(op1 + t.o_i + k * 4096u) = out_i[1][k];
    }
}

// Rate 1 from CF16 voltages (the ModeB path: channelized and polarized on the
// way in, exact in FP16): raw rows of 128 samples x 8 bytes [p0 (re, im) | p1 (re,
// im)] per antenna.  A task is one sample of 8 antennas -> the (re, im) chunks of
// polarisation p; consecutive lanes take consecutive samples (rows).
__device__ __forceinline__ void build_operand_h16(const uint8_t* raw, uint32_t rrow, uint8_t* op, uint32_t A,
                                                  uint32_t KA, int p, uint32_t ct) {
    constexpr uint32_t kStride = kConvWarps * 32;
    const uint32_t ntasks = kM * (KA / 8);
    for (uint32_t t = ct; t < ntasks; t += kStride) {
        const uint32_t s = t % kM, g = t / kM;
        uint32_t h[8];  // half2 (re, im) of polarisation p, antennas g*8 .. g*8+7
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint32_t a = g * 8 + i;
            h[i] = a < A ? *reinterpret_cast<const uint32_t*>(raw + a * rrow + s * 8 + p * 4) : 0u;
        }
        uint4 vr, vi;
        vr.x = __byte_perm(h[0], h[1], 0x5410);
        vr.y = __byte_perm(h[2], h[3], 0x5410);
        vr.z = __byte_perm(h[4], h[5], 0x5410);
        vr.w = __byte_perm(h[6], h[7], 0x5410);
        vi.x = __byte_perm(h[0], h[1], 0x7632);
        vi.y = __byte_perm(h[2], h[3], 0x7632);
        vi.z = __byte_perm(h[4], h[5], 0x7632);
        vi.w = __byte_perm(h[6], h[7], 0x7632);
        *reinterpret_cast<uint4*>(op + op_off(s, g * 8)) = vr;
        *reinterpret_cast<uint4*>(op + op_off(s, KA + g * 8)) = vi;
    }
}

// Both polarisations of one CF16 tile in one pass: one 8-byte load per (antenna,
// sample) feeds both operands (consecutive lanes read consecutive 8-byte samples,
// so a warp's loads are conflict-free).
__device__ __forceinline__ void build_operand_h16_pair(const uint8_t* raw, uint32_t rrow, uint8_t* op0, uint8_t* op1,
                                                       uint32_t A, uint32_t KA, uint32_t ct) {
    constexpr uint32_t kStride = kConvWarps * 32;
    const uint32_t ntasks = kM * (KA / 8);
    for (uint32_t t = ct; t < ntasks; t += kStride) {
        const uint32_t s = t % kM, g = t / kM;
        uint2 v[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const uint32_t a = g * 8 + i;
            v[i] = a < A ? *reinterpret_cast<const uint2*>(raw + a * rrow + s * 8) : make_uint2(0u, 0u);
        }
#pragma unroll
        for (int p = 0; p < 2; p++) {
            uint32_t h[8];
#pragma unroll
            for (int i = 0; i < 8; i++) h[i] = p ? v[i].y : v[i].x;
            uint4 vr, vi;
            vr.x = __byte_perm(h[0], h[1], 0x5410);
            vr.y = __byte_perm(h[2], h[3], 0x5410);
            vr.z = __byte_perm(h[4], h[5], 0x5410);
            vr.w = __byte_perm(h[6], h[7], 0x5410);
            vi.x = __byte_perm(h[0], h[1], 0x7632);
            vi.y = __byte_perm(h[2], h[3], 0x7632);
            vi.z = __byte_perm(h[4], h[5], 0x7632);
            vi.w = __byte_perm(h[6], h[7], 0x7632);
            uint8_t* op = p ? op1 : op0;
            *reinterpret_cast<uint4*>(op + op_off(s, g * 8)) = vr;
            *reinterpret_cast<uint4*>(op + op_off(s, KA + g * 8)) = vi;
        }
    }
}

// R = 1 CI8, both polarisations of a tile in one pass.  Thread (converter warp w,
// lane l) owns samples 4l .. 4l + 3 (rows of the operand) and one group g of 8
// antennas, fixed for the whole kernel:
//   KA = 64: g = (l + w) & 7,         warps 0-7;
//   KA = 32: g = ((l >> 1) + w) & 3,  warps 0-3 (warps 4-7 only keep the handshakes).
// Loads: one 16-byte load per antenna (4 samples x [p0 re, p0 im, p1 re, p1 im]);
// the 8 lanes of a quarter-warp read 8 consecutive 16-byte slots of a row, so each
// is one wavefront.  Stores: a 16-byte chunk of row 4l + j holds 8 antennas of one
// component; its bank group is g ^ (row & 7) = g ^ 4 (l & 1) ^ j, which the
// mappings above make distinct over every quarter-warp.  Conversion: byte permutes
// gather one component of two antennas ([a p0, b p0, a p1, b p1]), the XOR with
// 0x80 per byte and a second permute with the 0x64 exponent byte give the half2
// (1024 + x + 128) per polarisation, and one subtraction of 1152 makes it exact x.
struct R1Task {
    uint32_t raw_off;        // 8 g * rrow + 16 l in the raw tile
    uint32_t o_r[4], o_i[4];  // operand offsets of (row 4l + j, K = 8 g) and (row 4l + j, K = KA + 8 g)
    uint32_t nvalid;         // antennas 8 g .. 8 g + nvalid - 1 exist (0..8)
    uint32_t active;
};

__device__ __forceinline__ R1Task r1_task(uint32_t w, uint32_t l, uint32_t A, uint32_t KA, uint32_t rrow) {
    R1Task t;
    const uint32_t ng = KA / 8;
    const uint32_t g = ng == 8 ? ((l + w) & 7u) : (((l >> 1) + w) & 3u);
    t.active = w < ng;
    t.raw_off = 8u * g * rrow + 16u * l;
    const uint32_t a0 = 8u * g;
    t.nvalid = (t.active && a0 < A) ? min(8u, A - a0) : 0u;
#pragma unroll
    for (uint32_t j = 0; j < 4; j++) {
        t.o_r[j] = op_off(4u * l + j, a0);
        t.o_i[j] = op_off(4u * l + j, KA + a0);
    }
    return t;
}

// One sample of 8 antennas -> the (re, im) chunks of both polarisations (exact
// int8 -> FP16; see the R1Task comment).
__device__ __forceinline__ void r1_convert_store(const uint32_t (&wv)[8], uint8_t* op0, uint8_t* op1, uint32_t o_r,
                                                 uint32_t o_i) {
    const half2 h1152 = __halves2half2(__ushort_as_half(0x6480), __ushort_as_half(0x6480));
    uint32_t r0[4], i0[4], r1[4], i1[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const uint32_t tr = __byte_perm(wv[2 * q], wv[2 * q + 1], 0x6240) ^ 0x80808080u;
        const uint32_t ti = __byte_perm(wv[2 * q], wv[2 * q + 1], 0x7351) ^ 0x80808080u;
        r0[q] = h2u(__hsub2(u2h(__byte_perm(tr, 0x64646464u, 0x4140)), h1152));
        r1[q] = h2u(__hsub2(u2h(__byte_perm(tr, 0x64646464u, 0x4342)), h1152));
        i0[q] = h2u(__hsub2(u2h(__byte_perm(ti, 0x64646464u, 0x4140)), h1152));
        i1[q] = h2u(__hsub2(u2h(__byte_perm(ti, 0x64646464u, 0x4342)), h1152));
    }
    *reinterpret_cast<uint4*>(op0 + o_r) = make_uint4(r0[0], r0[1], r0[2], r0[3]);
    *reinterpret_cast<uint4*>(op0 + o_i) = make_uint4(i0[0], i0[1], i0[2], i0[3]);
    *reinterpret_cast<uint4*>(op1 + o_r) = make_uint4(r1[0], r1[1], r1[2], r1[3]);
    *reinterpret_cast<uint4*>(op1 + o_i) = make_uint4(i1[0], i1[1], i1[2], i1[3]);
}

__device__ __forceinline__ void r1_pair_task(const uint8_t* raw, uint32_t rrow, uint8_t* op0, uint8_t* op1,
                                             const R1Task& t) {
    if (!t.active) return;
    const uint8_t* src = raw + t.raw_off;
    uint4 v[8];
#pragma unroll
    for (uint32_t i = 0; i < 8; i++)
        v[i] = i < t.nvalid ? *reinterpret_cast<const uint4*>(src + i * rrow) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        uint32_t wv[8];
#pragma unroll
        for (int i = 0; i < 8; i++) wv[i] = j == 0 ? v[i].x : j == 1 ? v[i].y : j == 2 ? v[i].z : v[i].w;
        r1_convert_store(wv, op0, op1, t.o_r[j], t.o_i[j]);
    }
}

// R = 1 CI8 "direct" mode (no raw ring in shared memory, which leaves room for
// four operand stages beside a large phasor image): each converter thread loads
// its voltage words from global memory itself, one tile ahead of the one it
// builds.  Thread (converter warp w, lane l) owns antenna group g of 8 and the
// rows l + 32 j (j in its set of sample quarters), fixed for the kernel:
//   KA = 64: g = w, j = 0..3;   KA = 32: g = w & 3, j = 2 (w >> 2) and 2 (w >> 2) + 1.
// Loads: 4-byte words, consecutive lanes at consecutive samples of one antenna
// (128 contiguous bytes per warp load).  Stores: the 16-byte chunk (row l + 32 j,
// group g) has bank group g ^ (l & 7), distinct over a quarter-warp.
constexpr uint32_t kDirectMaxJ = 4;

struct DirectTask {
    uint32_t a0, nvalid, j0, nj;
    uint32_t o_r[kDirectMaxJ], o_i[kDirectMaxJ];  // offsets of (row l + 32 (j0 + j), K = a0) and (..., K = KA + a0)
};

__device__ __forceinline__ DirectTask direct_task(uint32_t w, uint32_t l, uint32_t A, uint32_t KA) {
    DirectTask t;
    const bool wide = KA == 64;
    const uint32_t g = wide ? w : (w & 3u);
    t.j0 = wide ? 0u : 2u * (w >> 2);
    t.nj = wide ? 4u : 2u;
    t.a0 = 8u * g;
    t.nvalid = t.a0 < A ? min(8u, A - t.a0) : 0u;
#pragma unroll
    for (uint32_t j = 0; j < kDirectMaxJ; j++) {
        const uint32_t row = l + 32u * (t.j0 + (j < t.nj ? j : 0u));
        t.o_r[j] = op_off(row, t.a0);
        t.o_i[j] = op_off(row, KA + t.a0);
    }
    return t;
}

// The words [j][i] = sample (t0 + l + 32 (j0 + j)) of antenna a0 + i in channel f.
__device__ __forceinline__ void direct_load(const uint32_t* in, uint32_t F, uint32_t T, uint32_t f, uint32_t t0,
                                            uint32_t l, const DirectTask& t, uint32_t (&v)[kDirectMaxJ][8]) {
#pragma unroll
    for (uint32_t i = 0; i < 8; i++) {
        const uint32_t* row = in + ((uint64_t)(t.a0 + i) * F + f) * T + t0 + l + 32u * t.j0;
#pragma unroll
        for (uint32_t j = 0; j < kDirectMaxJ; j++)
            v[j][i] = (i < t.nvalid && j < t.nj) ? __ldg(row + 32u * j) : 0u;
    }
}

__device__ __forceinline__ void direct_build(const uint32_t (&v)[kDirectMaxJ][8], uint8_t* op0, uint8_t* op1,
                                             const DirectTask& t) {
#pragma unroll
    for (uint32_t j = 0; j < kDirectMaxJ; j++)
        if (j < t.nj) r1_convert_store(v[j], op0, op1, t.o_r[j], t.o_i[j]);
}

// Both polarisations of one tile for R = 1 and 2: two single-polarisation passes.
template <int R>
__device__ __forceinline__ void build_operand_pair(const uint8_t* raw, uint32_t rrow, uint8_t* op0, uint8_t* op1, uint32_t A,
                                                   uint32_t KA, uint32_t ct) {
    build_operand<R>(raw, rrow, op0, A, KA, 0, ct);
    build_operand<R>(raw, rrow, op1, A, KA, 1, ct);
}

// Window sum of NV per-beam values over I = 2^LOGI adjacent lanes by a butterfly
// reduce-scatter: after min(LOGI, log2 NV) halving rounds each lane holds the
// window sums of NV >> min(LOGI, log2 NV) consecutive beams starting at *first; the
// remaining rounds (I > NV) are a plain exchange.  Returns the number of values
// this lane stores (0 for the lanes that hold duplicates when I > NV).
template <int NV, int LOGI>
__device__ __forceinline__ int window_reduce(float (&v)[NV], uint32_t lane, uint32_t* first) {
    constexpr int LOGNV = NV == 16 ? 4 : NV == 8 ? 3 : NV == 4 ? 2 : NV == 2 ? 1 : 0;
    constexpr int RS = LOGI < LOGNV ? LOGI : LOGNV;
    uint32_t off = 0;
#pragma unroll
    for (int s = 0; s < RS; s++) {
        const int half = NV >> (s + 1);
        const bool upper = (lane >> s) & 1u;
#pragma unroll
        for (int j = 0; j < half; j++) {
            const float send = upper ? v[j] : v[half + j];
            const float recv = __shfl_xor_sync(0xffffffffu, send, 1 << s);
            v[j] = (upper ? v[half + j] : v[j]) + recv;
        }
        if (upper) off += half;
    }
#pragma unroll
    for (int s = RS; s < LOGI; s++) v[0] += __shfl_xor_sync(0xffffffffu, v[0], 1 << s);
    *first = off;
    if (LOGI > LOGNV && ((lane >> LOGNV) & ((1u << (LOGI > LOGNV ? LOGI - LOGNV : 0)) - 1u))) return 0;
    return NV >> RS;
}

// ---- MMA issue ----------------------------------------------------------------
// Descriptors are built once per stage and stepped by adding 16-byte units to the
// start-address field, so each tcgen05.mma costs a handful of integer adds.
// A operand k-step j: column block j / 4 (16 KB each), 32 bytes per step in a row.
__device__ __forceinline__ uint64_t a_step(uint64_t ad, int j) {
    return ad + (uint64_t)((((j >> 2) * 16384) + (j & 3) * 32) >> 4);
}

// hi and lo stacked along N (4 NB rows per column block of the image): one MMA per k-step.
template <int KSTEPS>
__device__ __forceinline__ void issue_stacked(uint32_t d, uint64_t ad, uint64_t wd, uint32_t wblk16, uint32_t idesc) {
#pragma unroll
    for (int j = 0; j < KSTEPS; j++)
        mma_f16(d, a_step(ad, j), wd + (uint64_t)((j >> 2) * wblk16 + (j & 3) * 2), idesc, j > 0 ? 1u : 0u);
}

// KA = 64, hi and lo as separate MMAs: the Xr steps read blocks [Wr | Wi], the Xi
// steps [-Wi | Wr] of the [-Wi | Wr | Wi] image (nb16 = one block, 16-byte units).
__device__ __forceinline__ void issue_ka64(uint32_t d, uint64_t ad, uint64_t wd, uint32_t nb16, uint32_t idesc) {
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int j = 0; j < 8; j++)
            mma_f16(d, a_step(ad, j), wd + (uint64_t)(h * 3 * nb16 + (j < 4 ? nb16 : 0) + (j & 3) * 2), idesc,
                    (h | j) ? 1u : 0u);
}

// KA = 32, hi and lo as separate MMAs over one block of 2 NB rows per (p, h).
__device__ __forceinline__ void issue_ka32(uint32_t d, uint64_t ad, uint64_t wd, uint32_t nb16, uint32_t idesc) {
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int j = 0; j < 4; j++)
            mma_f16(d, a_step(ad, j), wd + (uint64_t)(h * 2 * nb16 + j * 2), idesc, (h | j) ? 1u : 0u);
}

// The same products with the roles of the operands swapped: the image blocks are
// the A operand (M = 128 rows: Re outputs of the 64 beams, then Im outputs) and the
// tile's samples the B operand (N = 128), so the accumulator holds one output row
// per TMEM lane and the tile's samples along its columns.
__device__ __forceinline__ void issue_ka64_t(uint32_t d, uint64_t ad, uint64_t wd, uint32_t nb16, uint32_t idesc) {
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int j = 0; j < 8; j++)
            mma_f16(d, wd + (uint64_t)(h * 3 * nb16 + (j < 4 ? nb16 : 0) + (j & 3) * 2), a_step(ad, j), idesc,
                    (h | j) ? 1u : 0u);
}

__device__ __forceinline__ void issue_ka32_t(uint32_t d, uint64_t ad, uint64_t wd, uint32_t nb16, uint32_t idesc) {
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int j = 0; j < 4; j++)
            mma_f16(d, wd + (uint64_t)(h * 2 * nb16 + j * 2), a_step(ad, j), idesc, (h | j) ? 1u : 0u);
}

// Epilogue of the transposed accumulator (rate 1 CI8, windows of I = 8 or 16
// samples, one 64-beam chunk): TMEM lane m holds output row m (Re of beam m for
// m < 64, Im of beam m - 64 after) and column c sample c of the tile, so a thread
// adds the squares of its row over each window of I consecutive columns (two
// columns per packed FP32x2 FMA) without any lane exchange.  Warps 0 and 1 of the
// lane quarters (the Re rows) store their window sums of both polarisations to
// the output; warps 2 and 3 (the Im rows) keep theirs in registers and add them to
// the stored partial sums one tile later, once pr_full says those are there.  The
// Re half signals a tile's partial sums after reading the next tile from TMEM, so
// neither half waits on the round trip through memory.
//
// Phases of pr_full: an mbarrier wait tests only the parity of its phase, so the Re
// half must never complete a barrier's next phase before the Im half has waited
// for the current one.  Inside the range, the Re half's signal for tile m needs the
// accumulator of tile m + 1, which needs the Im half's release of tile m + 1 - nacc,
// which it gives only after its wait for tile m - nacc, the previous phase of the
// same barrier.  The signal for the range's last tile comes after the loop with no
// accumulator to gate it, so the Re half first waits for the release of tile
// n - nacc (that wait of the Im half precedes it).
//
// At rate 1 a channel holds tpc tiles of NW outputs and U = tpc NW, so tile L of
// the chunk's F tpc tiles writes outputs L NW .. L NW + NW - 1 of each beam row.
template <int LOGI>
__device__ __forceinline__ void epilogue_transposed(const TcArgs& g, uint32_t tmem, uint32_t d_cols, uint32_t nacc,
                                                    uint64_t* d_full, uint64_t* d_empty, uint64_t* pr_full,
                                                    volatile int* abort, uint64_t L0, uint64_t L1, uint32_t q,
                                                    uint32_t lane) {
    constexpr uint32_t I = 1u << LOGI;
    constexpr int NW = kM / I;                      // windows per tile: 16 or 8
    constexpr int kCols = LOGI == 3 ? 32 : 16;      // TMEM columns read per wait
    const bool re_half = q < 2;
    const uint32_t b = 32u * (q & 1u) + lane;
    const bool valid = b < g.beams;
    float* row = g.out + (uint64_t)b * g.F * g.U + L0 * NW;  // this beam's outputs of tile L0
    const uint32_t n = (uint32_t)(L1 - L0);
    uint32_t db = 0, dph = 0;
    float pend[NW];  // Im half: the previous tile's own window sums
    uint32_t i = 0;
    for (; i < n; i++) {
        if (!mbar_wait(&d_full[db], dph, abort, kWaitBudget)) { record_abort(abort, 7); break; }
        tc_fence_after();
        const uint32_t lane_addr = tmem + ((32 * q) << 16) + db * (2 * d_cols);
        float2 acc[NW];
#pragma unroll
        for (int w = 0; w < NW; w++) acc[w] = make_float2(0.f, 0.f);
#pragma unroll
        for (uint32_t p = 0; p < 2; p++) {
#pragma unroll
            for (int c0 = 0; c0 < kM; c0 += kCols) {
                uint32_t r[kCols / 16][16];
#pragma unroll
                for (int k = 0; k < kCols / 16; k++) tmem_ld16(lane_addr + p * d_cols + c0 + 16 * k, r[k]);
                tmem_ld_wait();
#pragma unroll
                for (int k = 0; k < kCols / 16; k++)
#pragma unroll
                    for (int j = 0; j < 8; j++) {
                        const int w = (c0 + 16 * k + 2 * j) / I;
                        const float2 v = make_float2(__uint_as_float(r[k][2 * j]), __uint_as_float(r[k][2 * j + 1]));
                        acc[w] = __ffma2_rn(v, v, acc[w]);
                    }
            }
        }
        tc_fence_before();
        __syncwarp();
        // the previous tile's accumulator slot and phase
        const uint32_t pdb = db ? db - 1 : nacc - 1, pph = db ? dph : dph ^ 1u;
        float* o = row + (uint64_t)i * NW;
        if (re_half) {
            if (lane == 0) {
                mbar_arrive(&d_empty[db]);
                if (i) mbar_arrive(&pr_full[pdb]);  // stored a tile ago
            }
            if (valid) {
#pragma unroll
                for (int w = 0; w < NW; w += 4)
                    *reinterpret_cast<float4*>(o + w) = make_float4(acc[w].x + acc[w].y, acc[w + 1].x + acc[w + 1].y,
                                                                    acc[w + 2].x + acc[w + 2].y, acc[w + 3].x + acc[w + 3].y);
            }
            __threadfence_block();  // ordered before lane 0's next arrive on pr_full
            __syncwarp();
        } else {
            if (i && !mbar_wait(&pr_full[pdb], pph, abort, kWaitBudget)) { record_abort(abort, 12); break; }
            __syncwarp();
            if (lane == 0) mbar_arrive(&d_empty[db]);
            if (i && valid) {
#pragma unroll
                for (int w = 0; w < NW; w += 4) {
                    const float4 r = *reinterpret_cast<const float4*>(o - NW + w);
                    *reinterpret_cast<float4*>(o - NW + w) =
                        make_float4(r.x + pend[w], r.y + pend[w + 1], r.z + pend[w + 2], r.w + pend[w + 3]);
                }
            }
#pragma unroll
            for (int w = 0; w < NW; w++) pend[w] = acc[w].x + acc[w].y;
        }
        if (++db == nacc) { db = 0; dph ^= 1; }
    }
    if (i == n && n) {
        // the last tile's exchange (db, dph now name tile n's slot and phase)
        const uint32_t pdb = db ? db - 1 : nacc - 1, pph = db ? dph : dph ^ 1u;
        float* o = row + (uint64_t)(n - 1) * NW;
        if (re_half) {
            // tile n - nacc used this slot in the phase before: wait for its release
            if (n >= nacc && !mbar_wait(&d_empty[db], dph ^ 1u, abort, kWaitBudget)) record_abort(abort, 13);
            else if (lane == 0) mbar_arrive(&pr_full[pdb]);
        } else if (mbar_wait(&pr_full[pdb], pph, abort, kWaitBudget)) {
            __syncwarp();
            if (valid) {
#pragma unroll
                for (int w = 0; w < NW; w += 4) {
                    const float4 r = *reinterpret_cast<const float4*>(o + w);
                    *reinterpret_cast<float4*>(o + w) =
                        make_float4(r.x + pend[w], r.y + pend[w + 1], r.z + pend[w + 2], r.w + pend[w + 3]);
                }
            }
        } else {
            record_abort(abort, 12);
        }
    }
}

// ES = bytes per dual-polarisation input sample: 4 (CI8) or 8 (CF16, rate 1 only).
template <int R, int LOGI, int ES = 4>
__global__ void __launch_bounds__(kThreads, 1) bf_tc_kernel(const TcArgs g, const __grid_constant__ CUtensorMap tmap) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // Swizzled operands need 1024-byte aligned atoms: align the working base.
    uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    const uint32_t NB = g.NB, KA = g.KA, AS = g.a_stages, RS = g.r_stages;
    const uint32_t op_bytes = (2 * KA / 64) * 16384u;  // one polarisation's operand
    uint8_t* w_smem = smem;                              // phasor image
    uint8_t* a_smem = w_smem + g.img_bytes;              // AS operand stages
    uint8_t* r_smem = a_smem + (size_t)AS * op_bytes;    // RS raw tiles
    uint64_t* bars = reinterpret_cast<uint64_t*>(r_smem + (size_t)RS * g.raw_bytes);
    uint64_t* a_full = bars;
    uint64_t* a_empty = a_full + AS;
    uint64_t* r_full = a_empty + AS;
    uint64_t* r_empty = r_full + RS;
    uint64_t* d_full = r_empty + RS;
    uint64_t* d_empty = d_full + kMaxAcc;
    uint64_t* w_full = d_empty + kMaxAcc;
    uint64_t* w_empty = w_full + 1;
    uint64_t* fin = w_empty + 1;  // one per MMA issuer
    uint64_t* pr_full = fin + 2;  // transposed epilogue: the Re half's partial sums are stored
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(pr_full + kMaxAcc);
    volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int never = 0;  // abort flag that is never raised (drain waits)
    // Accumulator columns per polarisation: [re | im] (2 NB), or with hi/lo stacked
    // along N [hi re | hi im | lo re | lo im] (4 NB).
    const uint32_t d_cols = (g.stacked ? 4u : 2u) * NB;
    // Accumulator buffers (tiles in flight between MMA and epilogue): as many as
    // fit the 512 TMEM columns, at most kMaxAcc.
    const uint32_t nacc = min((uint32_t)kMaxAcc, 512u / (2u * d_cols));
    const uint32_t need_cols = nacc * 2u * d_cols;
    const uint32_t tmem_cols = need_cols <= 32 ? 32 : need_cols <= 64 ? 64 : need_cols <= 128 ? 128 : need_cols <= 256 ? 256 : 512;
    // Pair mode: the converter builds both polarisations of a tile in one pass and
    // signals them together on the second stage of the pair.
    const bool pair = AS >= 4 && (AS & 1u) == 0;

    // Two MMA issuers (warp 0 and the last warp, lane 0 each) take alternate tiles
    // when the operand ring holds an even number of tile pairs and the accumulator
    // count is even, so that every barrier is only ever used by one issuer.  An
    // issue of tcgen05.mma holds its thread for about the MMA's duration, so one
    // issuer's waits and commits overlap the other's MMAs.
    const uint32_t nis = (pair && ((AS / 2) & 1u) == 0 && (nacc & 1u) == 0) ? 2u : 1u;
    // Split operand build (R = 4, two issuers, two-tile raw stages): converter warps
    // 0-3 build the even tiles of the CTA's range (the first tile of each raw stage,
    // issuer 0's) and warps 4-7 the odd ones, so the two halves run independently
    // and each operand pair has four producers.
    const bool split = R == 4 && nis == 2 && g.raw_tiles == 2;

    if (threadIdx.x == 0) {
        for (uint32_t i = 0; i < AS; i++) {
            mbar_init(&a_full[i], split ? kConvWarps / 2 : kConvWarps);
            mbar_init(&a_empty[i], 1);
        }
        for (uint32_t i = 0; i < RS; i++) {
            mbar_init(&r_full[i], 1);
            mbar_init(&r_empty[i], kConvWarps);
        }
        for (uint32_t i = 0; i < nacc; i++) {
            mbar_init(&d_full[i], 1);
            mbar_init(&d_empty[i], kEpiWarps);
            mbar_init(&pr_full[i], kEpiWarps / 2);
        }
        mbar_init(w_full, 1);
        mbar_init(w_empty, nis);
        mbar_init(&fin[0], 1);
        mbar_init(&fin[1], 1);
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

    // This CTA's contiguous range of (channel, time-tile) tiles, a whole number of
    // raw stages (tiles per channel is a multiple of raw_tiles).
    const uint64_t per = ((g.total_tiles + gridDim.x - 1) / gridDim.x + g.raw_tiles - 1) / g.raw_tiles * g.raw_tiles;
    const uint64_t L0 = (uint64_t)blockIdx.x * per;
    const uint64_t L1 = min(g.total_tiles, L0 + per);
    const uint32_t tpc = g.tiles_per_ch;
    const int issuer = warp == 0 ? 0 : (warp == kWarps - 1 ? 1 : -1);

    if (issuer >= 0) {
        // ---------------- MMA issuers ----------------
        const uint32_t j = (uint32_t)issuer;
        // The whole warp runs the loop and the waits (a lone active lane beside lanes
        // parked at the final barrier progressed slowly); lane 0 issues the MMAs and
        // the commits, which track that thread's MMAs.
        auto wait_all = [&](uint64_t* bar, uint32_t parity, unsigned code) -> bool {
            const bool w = __all_sync(0xffffffffu, mbar_wait(bar, parity, abort, kWaitBudget));
            if (!w && lane == 0) record_abort(abort, code);
            return w;
        };
        if (L0 < L1 && j < nis) {
            const uint32_t idesc = idesc_f16(kM, d_cols);
            const uint64_t w_desc = smem_desc_sw128(smem_u32(w_smem));
            const uint64_t a_desc = smem_desc_sw128(smem_u32(a_smem));
            const uint32_t op16 = op_bytes >> 4;   // operand stage stride, 16-byte units
            const uint32_t nb16 = NB * 8;          // NB rows x 128 bytes, 16-byte units
            // Phasor image stride per polarisation, 16-byte units:
            //   stacked: (2 KA / 64) column blocks of 4 NB rows;
            //   KA = 64: two (hi, lo) x three NB-row blocks; KA = 32: two x one 2 NB-row block.
            const uint32_t wpol16 = g.stacked ? (2 * KA / 64) * 4 * nb16 : (KA == 64 ? 6 * nb16 : 4 * nb16);
            // This issuer's first tile is local tile j: operand stage 2 j (pair mode)
            // or 0, accumulator j; both advance by nis tiles per own tile.
            uint32_t as = pair ? 2 * j : 0, aph = 0, db = j, dph = 0, wph = 0;
            uint32_t tt = (uint32_t)(L0 % tpc);  // time tile within the channel, stepped below
            bool ok = true;
            uint32_t i = 0;
            for (uint64_t L = L0; L < L1 && ok; L++, i++) {
                if (L == L0 || tt == 0) {
                    if (!wait_all(w_full, wph, 1)) { ok = false; break; }
                }
                if ((i % nis) == j) {
                    if (!wait_all(&d_empty[db], dph ^ 1, 3)) { ok = false; break; }
                    const uint32_t np = pair ? 1u : 2u;  // operand handshakes per tile
                    for (uint32_t h = 0; h < np; h++) {
                        // pair mode: the converter signals both polarisation stages on as + 1
                        const uint32_t sig = pair ? as + 1 : as;
                        if (!wait_all(&a_full[sig], aph, 2)) { ok = false; break; }
                        tc_fence_after();
                        if (lane == 0) {
                            for (uint32_t p = pair ? 0u : h; p < (pair ? 2u : h + 1); p++) {
                                const uint64_t ad = a_desc + (uint64_t)((as + (pair ? p : 0u)) * op16);
                                const uint64_t wd = w_desc + (uint64_t)(p * wpol16);
                                const uint32_t d = tmem + db * (2 * d_cols) + p * d_cols;
                                if (g.stacked) {
                                    if (KA == 64) issue_stacked<8>(d, ad, wd, 4 * nb16, idesc);
                                    else issue_stacked<4>(d, ad, wd, 4 * nb16, idesc);
                                } else if (g.transposed) {
                                    if (KA == 64) issue_ka64_t(d, ad, wd, nb16, idesc);
                                    else issue_ka32_t(d, ad, wd, nb16, idesc);
                                } else if (KA == 64) {
                                    issue_ka64(d, ad, wd, nb16, idesc);
                                } else {
                                    issue_ka32(d, ad, wd, nb16, idesc);
                                }
                            }
                            mma_commit(&a_empty[sig]);
                        }
                        __syncwarp();
                        as += pair ? 2u * nis : 1u;
                        if (as >= AS) { as -= AS; aph ^= 1; }
                    }
                    if (!ok) break;
                    if (lane == 0) mma_commit(&d_full[db]);
                    __syncwarp();
                    db += nis;
                    if (db >= nacc) { db -= nacc; dph ^= 1; }
                }
                // Every issuer releases the phasor image at the end of each channel
                // segment (the barrier counts one arrival per issuer).
                if (tt == tpc - 1 || L + 1 == L1) {
                    if (lane == 0) mma_commit(w_empty);
                    __syncwarp();
                    wph ^= 1;
                }
                if (++tt == tpc) tt = 0;
            }
            // Drain every MMA issued by this thread before TMEM is released
            // (bounded, but not cut short by the abort flag).
            if (lane == 0) {
                mma_commit(&fin[j]);
                if (!mbar_wait(&fin[j], 0, &never, kWaitBudget)) record_abort(abort, 4);
            }
            __syncwarp();
        }
    } else if (warp == 1) {
        // ---------------- loader: phasor image + raw CI8 tiles (bulk copies) ----------------
        if (L0 < L1 && g.direct) {
            // direct mode: the converter threads load the voltages; only the images here
            uint32_t wph = 0;
            bool w_issued = false;
            uint32_t f = (uint32_t)(L0 / tpc);
            for (uint64_t L = L0; L < L1; L = (uint64_t)(++f) * tpc) {
                int ok = 1;
                if (lane == 0) {
                    if (g.pdl && L == L0) asm volatile("griddepcontrol.wait;" ::: "memory");
                    ok = mbar_wait(w_empty, wph ^ 1, abort, kWaitBudget);
                    if (ok) {
                        mbar_arrive_expect_tx(w_full, g.img_bytes);
                        bulk_g2s(w_smem, g.plan + (uint64_t)f * g.img_bytes, g.img_bytes, w_full);
                    } else {
                        record_abort(abort, 5);
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) break;
                w_issued = true;
                wph ^= 1;
            }
            if (lane == 0 && w_issued && !mbar_wait(w_full, wph ^ 1, &never, kWaitBudget)) record_abort(abort, 6);
            __syncwarp();
        } else if (L0 < L1) {
            uint32_t rs = 0, rph = 0, wph = 0;
            bool w_issued = false;
            uint32_t issued_mask = 0, issued_par = 0;  // per raw stage: issued?, parity of last issue
            // One raw stage = raw_tiles consecutive tiles of one channel, loaded as one or
            // two TMA boxes of up to 256 samples x 1 channel x A antennas (rows of
            // raw_row bytes per antenna: 512-byte rows per tile leave DRAM bandwidth
            // unused, 1-2 KB rows do not).
            const uint32_t RT = g.raw_tiles, box = g.raw_row / ES, nbox = RT * kM / box;
            uint32_t f = (uint32_t)(L0 / tpc), tt = (uint32_t)(L0 % tpc);  // stepped below
            for (uint64_t L = L0; L < L1; L += RT) {
                int ok = 1;
                if (L == L0 || tt == 0) {
                    if (lane == 0) {
                        // the phasor image is the preceding grid's output: with a programmatic
                        // launch, everything above overlapped that grid, and here it must be done
                        if (g.pdl && L == L0) asm volatile("griddepcontrol.wait;" ::: "memory");
                        ok = mbar_wait(w_empty, wph ^ 1, abort, kWaitBudget);
                        if (ok) {
                            mbar_arrive_expect_tx(w_full, g.img_bytes);
                            bulk_g2s(w_smem, g.plan + (uint64_t)f * g.img_bytes, g.img_bytes, w_full);
                        } else {
                            record_abort(abort, 5);
                        }
                    }
                    ok = __shfl_sync(0xffffffffu, ok, 0);
                    if (!ok) break;
                    w_issued = true;
                    wph ^= 1;
                }
                if (lane == 0) {
                    ok = mbar_wait(&r_empty[rs], rph ^ 1, abort, kWaitBudget);
                    if (ok) {
                        mbar_arrive_expect_tx(&r_full[rs], g.A * (uint32_t)(kM * ES) * RT);
                        uint8_t* dst = r_smem + (size_t)rs * g.raw_bytes;
                        for (uint32_t b = 0; b < nbox; b++)
                            tma_load_3d(dst + (size_t)b * g.A * g.raw_row, &tmap, (int)(tt * kM + b * box), (int)f, 0,
                                        &r_full[rs]);
                    } else {
                        record_abort(abort, 9);
                    }
                }
                ok = __shfl_sync(0xffffffffu, ok, 0);
                if (!ok) break;
                issued_mask |= 1u << rs;
                issued_par = (issued_par & ~(1u << rs)) | (rph << rs);
                if (++rs == RS) { rs = 0; rph ^= 1; }
                tt += RT;
                if (tt == tpc) { tt = 0; f++; }
            }
            // Every bulk copy this warp issued must land before the CTA exits.
            if (lane == 0) {
                if (w_issued && !mbar_wait(w_full, wph ^ 1, &never, kWaitBudget)) record_abort(abort, 6);
                for (uint32_t s = 0; s < RS; s++)
                    if ((issued_mask >> s) & 1u)
                        if (!mbar_wait(&r_full[s], (issued_par >> s) & 1u, &never, kWaitBudget)) record_abort(abort, 10);
            }
            __syncwarp();
        }
    } else if (warp < 2 + kEpiWarps) {
        bool done = false;
        if constexpr (R == 1 && (LOGI == 3 || LOGI == 4) && ES == 4 && kEpiWarps == 4) {
            if (g.transposed) {
                epilogue_transposed<LOGI>(g, tmem, d_cols, nacc, d_full, d_empty, pr_full, abort, L0, L1,
                                          (uint32_t)(warp & 3), (uint32_t)lane);
                done = true;
            }
        }
        if (!done) {
            // ---------------- epilogue ----------------
            constexpr uint32_t I = 1u << LOGI;
            const uint32_t q = warp & 3;               // TMEM lane quarter this warp may access
            const uint32_t hw = (warp - 2) >> 2;       // which share of the beams
            const uint32_t nbh = NB / kEpiGroups;      // beams per warp, a multiple of 8
            constexpr uint32_t rows_per_k = kM / R;
            const uint32_t row = 32 * q + lane;
            const uint32_t k = row / rows_per_k;
            const uint32_t s_local = row - k * rows_per_k;
            const uint64_t bstride = (uint64_t)g.F * R * g.U;
            uint32_t db = 0, dph = 0;
            uint32_t f = (uint32_t)(L0 / tpc), tt = (uint32_t)(L0 % tpc);  // stepped below
            for (uint64_t L = L0; L < L1; L++) {
                if (!mbar_wait(&d_full[db], dph, abort, kWaitBudget)) { record_abort(abort, 7); break; }
                tc_fence_after();
                const uint32_t u = (tt * rows_per_k + s_local) / I;
                const uint32_t lane_addr = tmem + ((32 * q) << 16) + db * (2 * d_cols);
                float* obase = g.out + ((uint64_t)f * R + k) * g.U + u;
                constexpr int CH = 16 / kEpiGroups;  // beams per TMEM load (16 or 8)
                for (uint32_t bc = hw * nbh; bc < (hw + 1) * nbh; bc += CH) {
                    // Two beams per packed FP32x2 instruction (each lane of the pair rounds
                    // exactly as the scalar add / multiply / FMA would).
                    float2 pw2[CH / 2];
                    float(&pw)[CH] = *reinterpret_cast<float(*)[CH]>(pw2);
                    if (g.stacked) {
                        // per polarisation: (hi + lo) re, (hi + lo) im
    #pragma unroll
                        for (int j = 0; j < CH; j++) pw[j] = 0.f;
    #pragma unroll
                        for (uint32_t p = 0; p < 2; p++) {
                            uint32_t hr[CH], hi[CH], lr[CH], li[CH];
                            const uint32_t pa = lane_addr + p * d_cols + bc;
                            tmem_ld(pa, hr);
                            tmem_ld(pa + NB, hi);
                            tmem_ld(pa + 2 * NB, lr);
                            tmem_ld(pa + 3 * NB, li);
                            tmem_ld_wait();
    #pragma unroll
                            for (int j = 0; j < CH / 2; j++) {
                                const float2 a = __fadd2_rn(make_float2(__uint_as_float(hr[2 * j]), __uint_as_float(hr[2 * j + 1])),
                                                            make_float2(__uint_as_float(lr[2 * j]), __uint_as_float(lr[2 * j + 1])));
                                const float2 b = __fadd2_rn(make_float2(__uint_as_float(hi[2 * j]), __uint_as_float(hi[2 * j + 1])),
                                                            make_float2(__uint_as_float(li[2 * j]), __uint_as_float(li[2 * j + 1])));
                                pw2[j] = __ffma2_rn(a, a, __ffma2_rn(b, b, pw2[j]));
                            }
                        }
                    } else {
                        uint32_t r0[CH], i0[CH], r1[CH], i1[CH];
                        tmem_ld(lane_addr + bc, r0);
                        tmem_ld(lane_addr + NB + bc, i0);
                        tmem_ld(lane_addr + 2 * NB + bc, r1);
                        tmem_ld(lane_addr + 3 * NB + bc, i1);
                        tmem_ld_wait();
    #pragma unroll
                        for (int j = 0; j < CH / 2; j++) {
                            const float2 a0 = make_float2(__uint_as_float(r0[2 * j]), __uint_as_float(r0[2 * j + 1]));
                            const float2 b0 = make_float2(__uint_as_float(i0[2 * j]), __uint_as_float(i0[2 * j + 1]));
                            const float2 a1 = make_float2(__uint_as_float(r1[2 * j]), __uint_as_float(r1[2 * j + 1]));
                            const float2 b1 = make_float2(__uint_as_float(i1[2 * j]), __uint_as_float(i1[2 * j + 1]));
                            pw2[j] = __ffma2_rn(a0, a0, __ffma2_rn(b0, b0, __ffma2_rn(a1, a1, __fmul2_rn(b1, b1))));
                        }
                    }
                    uint32_t first;
                    const int cnt = window_reduce<CH, LOGI>(pw, lane, &first);
    #pragma unroll
                    for (int j = 0; j < CH; j++) {
                        if (j < cnt) {
                            const uint32_t b = bc + first + j;
                            if (b < g.beams) obase[b * bstride] = pw[j];
                        }
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&d_empty[db]);
                if (++db == nacc) { db = 0; dph ^= 1; }
                if (++tt == tpc) { tt = 0; f++; }
            }
        }
    } else if (warp < 2 + kEpiWarps + kConvWarps) {
        // ---------------- operand build ----------------
        const uint32_t ct = threadIdx.x - (2 + kEpiWarps) * 32;  // 0 .. 32 kConvWarps - 1
        if constexpr (R == 4) {
            if (split) {
                // Group grp takes local tiles grp, grp + 2, ...: tile `grp` of every raw
                // stage (512 bytes into each 1 KB antenna row) and operand pair 2 grp,
                // 2 grp + 4, ... (the pairs issuer grp consumes).  The CTA's range is a
                // whole number of two-tile stages, so both groups see every stage once.
                constexpr uint32_t kGroup = kConvWarps / 2;
                constexpr uint32_t kMaxTk = kMaxKA / 4 / kGroup;
                const uint32_t cw = ct >> 5, grp = cw / kGroup, gw = cw % kGroup;
                const uint32_t ntk = KA / 4 / kGroup;
                R4Task tk[kMaxTk];
#pragma unroll
                for (uint32_t i = 0; i < kMaxTk; i++) tk[i] = r4_task(gw + i * kGroup, lane, g.A, KA, g.raw_row);
                uint32_t rs = 0, rph = 0, as = 2 * grp, aph = 0;
                for (uint64_t L = L0 + grp; L < L1; L += 2) {
                    if (!mbar_wait(&r_full[rs], rph, abort, kWaitBudget)) { record_abort(abort, 11); break; }
                    if (!mbar_wait(&a_empty[as + 1], aph ^ 1, abort, kWaitBudget)) { record_abort(abort, 8); break; }
                    const uint8_t* raw = r_smem + (size_t)rs * g.raw_bytes + grp * (kM * 4u);
                    uint8_t* op0 = a_smem + (size_t)as * op_bytes;
                    uint8_t* op1 = op0 + op_bytes;
#pragma unroll
                    for (uint32_t i = 0; i < kMaxTk; i++)
                        if (i < ntk) r4_pair_task(raw, g.raw_row, op0, op1, tk[i]);
                    fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0) {
                        mbar_arrive(&a_full[as + 1]);
                        mbar_arrive(&r_empty[rs]);
                    }
                    as += 4;
                    if (as >= AS) { as -= AS; aph ^= 1; }
                    if (++rs == RS) { rs = 0; rph ^= 1; }
                }
            }
        }
        if constexpr (R == 1 && ES == 4) {
            if (g.direct) {
                // Pair mode without a raw ring: registers hold this tile's words, loaded
                // while the previous tile was built; the next tile's loads go out first.
                const DirectTask dt = direct_task(ct >> 5, lane, g.A, KA);
                const uint32_t* in32 = reinterpret_cast<const uint32_t*>(g.in);
                uint32_t va[kDirectMaxJ][8], vb[kDirectMaxJ][8];
                uint32_t f = (uint32_t)(L0 / tpc), tt = (uint32_t)(L0 % tpc);
                if (L0 < L1) direct_load(in32, g.F, g.T, f, tt * kM, lane, dt, va);
                uint32_t as = 0, aph = 0;
                for (uint64_t L = L0; L < L1; L += 2) {
                    // tile L from va (tile L + 1 into vb first), then tile L + 1 from vb
                    // (tile L + 2 into va first)
#pragma unroll
                    for (int half = 0; half < 2; half++) {
                        if (half == 1 && L + 1 >= L1) break;
                        uint32_t nf = f, ntt = tt + 1;
                        if (ntt == tpc) { ntt = 0; nf++; }
                        if (L + half + 1 < L1) direct_load(in32, g.F, g.T, nf, ntt * kM, lane, dt, half ? va : vb);
                        if (lane < dt.nvalid && L + half + 2 < L1) {
                            // the tile after next into L2: lanes 0-7 prefetch this thread group's rows
                            uint32_t pf = nf, pt = ntt + 1;
                            if (pt == tpc) { pt = 0; pf++; }
                            prefetch_l2_bulk(in32 + ((uint64_t)(dt.a0 + lane) * g.F + pf) * g.T + pt * kM + 32u * dt.j0,
                                             dt.nj * 128u);
                        }
                        if (!mbar_wait(&a_empty[as + 1], aph ^ 1, abort, kWaitBudget)) {
                            record_abort(abort, 8);
                            L = L1;
                            break;
                        }
                        uint8_t* op0 = a_smem + (size_t)as * op_bytes;
                        direct_build(half ? vb : va, op0, op0 + op_bytes, dt);
                        fence_proxy_async_smem();
                        __syncwarp();
                        if (lane == 0) mbar_arrive(&a_full[as + 1]);
                        as += 2;
                        if (as == AS) { as = 0; aph ^= 1; }
                        f = nf;
                        tt = ntt;
                    }
                }
            }
        }
        if (!(R == 4 && split) && !g.direct) {
        // R = 4 pair mode: this warp's warp-tasks (KA / 4 of them over kConvWarps warps),
        // addresses fixed for the kernel
        constexpr uint32_t kMaxT4 = kMaxKA / 4 / kConvWarps;
        const uint32_t nt4 = KA / 4 / kConvWarps;
        R4Task t4[kMaxT4];
        if constexpr (R == 4) {
#pragma unroll
            for (uint32_t i = 0; i < kMaxT4; i++) t4[i] = r4_task((ct >> 5) + i * kConvWarps, lane, g.A, KA, g.raw_row);
        }
        R1Task t1;
        if constexpr (R == 1 && ES == 4) t1 = r1_task(ct >> 5, lane, g.A, KA, g.raw_row);
        uint32_t rs = 0, rph = 0, as = 0, aph = 0;
        uint32_t sub = 0;  // tile within the raw stage (CTA ranges are stage-aligned)
        bool ok = true;
        for (uint64_t L = L0; L < L1 && ok; L++) {
            if (sub == 0) {
                if (!mbar_wait(&r_full[rs], rph, abort, kWaitBudget)) { record_abort(abort, 11); break; }
            }
            // this tile inside the stage: box (sub * 128 / box), column (sub * 128 % box)
            const uint32_t sb = sub * kM, box = g.raw_row / ES;
            const uint8_t* raw = r_smem + (size_t)rs * g.raw_bytes + (sb / box) * g.A * g.raw_row + (sb % box) * ES;
            if (pair) {
                // Both polarisations in one pass into stages as, as + 1 (AS is even).
                if (!mbar_wait(&a_empty[as + 1], aph ^ 1, abort, kWaitBudget)) {
                    record_abort(abort, 8);
                    break;
                }
                uint8_t* op0 = a_smem + (size_t)as * op_bytes;
                uint8_t* op1 = op0 + op_bytes;
                if constexpr (R == 4) {
#pragma unroll
                    for (uint32_t i = 0; i < kMaxT4; i++)
                        if (i < nt4) r4_pair_task(raw, g.raw_row, op0, op1, t4[i]);
                } else if constexpr (ES == 8) {
                    build_operand_h16_pair(raw, g.raw_row, op0, op1, g.A, KA, ct);
                } else if constexpr (R == 1) {
                    r1_pair_task(raw, g.raw_row, op0, op1, t1);
                } else {
                    build_operand_pair<R>(raw, g.raw_row, op0, op1, g.A, KA, ct);
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) mbar_arrive(&a_full[as + 1]);
                as += 2;
                if (as == AS) { as = 0; aph ^= 1; }
            } else {
                for (int p = 0; p < 2; p++) {
                    if (!mbar_wait(&a_empty[as], aph ^ 1, abort, kWaitBudget)) { record_abort(abort, 8); ok = false; break; }
                    if constexpr (ES == 8) build_operand_h16(raw, g.raw_row, a_smem + (size_t)as * op_bytes, g.A, KA, p, ct);
                    else build_operand<R>(raw, g.raw_row, a_smem + (size_t)as * op_bytes, g.A, KA, p, ct);
                    fence_proxy_async_smem();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&a_full[as]);
                    if (++as == AS) { as = 0; aph ^= 1; }
                }
                if (!ok) break;
            }
            if (++sub == g.raw_tiles) {
                sub = 0;
                __syncwarp();
                if (lane == 0) mbar_arrive(&r_empty[rs]);
                if (++rs == RS) { rs = 0; rph ^= 1; }
            }
        }
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
// plan[chunk][f][p] in the 128-byte-swizzled K-major layout (K = 2 KA: Xr part
// then Xi part), h 0 = hi = rn(w), h 1 = lo = rn(w - hi):
//   stacked (NB <= 32): per p, (2 KA / 64) column blocks of 4 NB rows
//            [hi: b -> (Wr | -Wi), NB + b -> (Wi | Wr) ; lo: the same],
//   KA = 64, NB > 32: per (p, h) three blocks of NB rows x 64 K: [-Wi | Wr | Wi],
//   KA = 32, NB > 32: per (p, h) one block of 2 NB rows: b -> [Wr | -Wi], NB + b -> [Wi | Wr].
// One thread writes the 16-byte chunks of one (chunk c, channel f, polarisation p,
// beam row nb, 8-antenna group j) for hi and lo: 8 phasors in, 8 or 12 chunk
// stores out.  Consecutive threads take consecutive channels, so the phasor loads
// of a warp are 16 bytes apart.
__device__ __forceinline__ uint4 pack8(const __half (&v)[8]) {
    uint4 u;
    u.x = (uint32_t)__half_as_ushort(v[0]) | ((uint32_t)__half_as_ushort(v[1]) << 16);
    u.y = (uint32_t)__half_as_ushort(v[2]) | ((uint32_t)__half_as_ushort(v[3]) << 16);
    u.z = (uint32_t)__half_as_ushort(v[4]) | ((uint32_t)__half_as_ushort(v[5]) << 16);
    u.w = (uint32_t)__half_as_ushort(v[6]) | ((uint32_t)__half_as_ushort(v[7]) << 16);
    return u;
}

// 16-byte chunk holding K elements [k_total, k_total + 8) of `row` in a stack of
// 64-wide column blocks of `rows` rows each.
__device__ __forceinline__ void put_chunk(uint8_t* base, uint32_t rows, uint32_t row, uint32_t k_total, uint4 v) {
    *reinterpret_cast<uint4*>(base + (k_total >> 6) * rows * 128u + sw128_off(row, (k_total >> 3) & 7u)) = v;
}

__global__ void __launch_bounds__(256) tc_prepare_kernel(const float2* __restrict__ ph, uint8_t* __restrict__ plan,
                                                         uint32_t B, uint32_t A, uint32_t F, uint32_t NB,
                                                         uint32_t KA, uint32_t nchunks, uint32_t img_bytes,
                                                         uint32_t stacked) {
    // a chain kernel launched as this grid's programmatic dependent may start its
    // prologue now; it waits for this grid to finish before it reads the image
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const uint32_t groups = KA / 8;
    const uint32_t n = nchunks * F * 2u * NB * groups;
    const uint32_t ph_bytes = (KA == 64 ? 3u : 2u) * NB * 128u;
    const uint32_t pol_stacked = (2 * KA / 64) * 4 * NB * 128u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t r = i;
        const uint32_t f = r % F;
        r /= F;
        const uint32_t p = r & 1u;
        r >>= 1;
        const uint32_t nb = r % NB;
        r /= NB;
        const uint32_t j = r % groups;
        const uint32_t c = r / groups;
        const uint32_t b = c * kMaxNB + nb;
        // hi = rn(w), lo = rn(w - hi) per component; padded antennas and beams are 0
        __half rh[8], ih[8], rl[8], il[8], nih[8], nil[8];
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const uint32_t a = j * 8 + e;
            float wr = 0.f, wi = 0.f;
            if (a < A && b < B) {
                const float2 w = ph[((uint64_t)(b * (uint64_t)A + a) * F + f) * 2 + p];
                wr = w.x;
                wi = w.y;
            }
            rh[e] = __float2half_rn(wr);
            ih[e] = __float2half_rn(wi);
            rl[e] = __float2half_rn(wr - __half2float(rh[e]));
            il[e] = __float2half_rn(wi - __half2float(ih[e]));
            nih[e] = __hneg(ih[e]);
            nil[e] = __hneg(il[e]);
        }
        const uint32_t k0 = j * 8;
        if (stacked) {
            // per p, (2 KA / 64) column blocks of 4 NB rows:
            //   hi: row nb -> [Wr | -Wi], row NB + nb -> [Wi | Wr]; lo: the same at rows + 2 NB
            uint8_t* base = plan + ((uint64_t)c * F + f) * img_bytes + (uint64_t)p * pol_stacked;
            const uint32_t rows = 4 * NB;
            put_chunk(base, rows, nb, k0, pack8(rh));
            put_chunk(base, rows, nb, KA + k0, pack8(nih));
            put_chunk(base, rows, NB + nb, k0, pack8(ih));
            put_chunk(base, rows, NB + nb, KA + k0, pack8(rh));
            put_chunk(base, rows, 2 * NB + nb, k0, pack8(rl));
            put_chunk(base, rows, 2 * NB + nb, KA + k0, pack8(nil));
            put_chunk(base, rows, 3 * NB + nb, k0, pack8(il));
            put_chunk(base, rows, 3 * NB + nb, KA + k0, pack8(rl));
            continue;
        }
        uint8_t* base = plan + ((uint64_t)c * F + f) * img_bytes + (uint64_t)p * 2 * ph_bytes;
        for (int h = 0; h < 2; h++) {
            uint8_t* blk = base + h * ph_bytes;
            const uint4 re = pack8(h ? rl : rh), im = pack8(h ? il : ih), nim = pack8(h ? nil : nih);
            if (KA == 64) {
                // three blocks of NB rows x 64 K: [-Wi | Wr | Wi]
                put_chunk(blk, NB, nb, k0, nim);
                put_chunk(blk + NB * 128u, NB, nb, k0, re);
                put_chunk(blk + 2u * NB * 128u, NB, nb, k0, im);
            } else {
                // one block of 2 NB rows x 64 K: row nb -> [Wr | -Wi], row NB + nb -> [Wi | Wr]
                put_chunk(blk, 2 * NB, nb, k0, re);
                put_chunk(blk, 2 * NB, nb, 32u + k0, nim);
                put_chunk(blk, 2 * NB, NB + nb, k0, im);
                put_chunk(blk, 2 * NB, NB + nb, 32u + k0, re);
            }
        }
    }
}

// The same split for KA = 64 images without stacking (more than 32 beams per
// chunk), through shared memory: a CTA takes 8 beams x 2 channels x both
// polarisations of one chunk (20 KB of shared memory; the dense block's 1024
// CTAs are resident at once).  It reads each (beam, antenna) row's 2 x 2 phasors
// as one 32-byte run, and each warp then writes 4 whole 128-byte image rows per
// block (lanes: 8 antenna groups x 4 beams), where the one-thread-per-chunk form
// writes 32 chunks into 32 different channels' images.  Same arithmetic per
// element, so the image is bit-identical.
constexpr uint32_t kPrepBeams = 8, kPrepChans = 2, kPrepPad = 10;  // float2 per 8-antenna group (8 + 2 pad)
__global__ void __launch_bounds__(256) tc_prepare_wide_kernel(const float2* __restrict__ ph, uint8_t* __restrict__ plan,
                                                              uint32_t B, uint32_t A, uint32_t F, uint32_t NB,
                                                              uint32_t img_bytes) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    // [beam][channel][pol][antenna group][8 antennas + pad]: a task's 8 phasors are
    // contiguous, and the 80-byte group pitch keeps a quarter-warp's 16-byte reads
    // (8 groups) on distinct banks
    __shared__ __align__(16) float2 sp[kPrepBeams][kPrepChans][2][8][kPrepPad];
    const uint32_t f0 = blockIdx.x * kPrepChans, nb0 = blockIdx.y * kPrepBeams, c = blockIdx.z;
    // load: element q = (bl, a, col), col = 2 fl + p fastest (the phasors' own order)
    constexpr uint32_t kCol = 2 * kPrepChans;
#pragma unroll 4
    for (uint32_t q = threadIdx.x; q < kPrepBeams * 64 * kCol; q += blockDim.x) {
        const uint32_t col = q % kCol, a = (q / kCol) % 64u, bl = q / (64u * kCol);
        const uint32_t fl = col >> 1, pp = col & 1u;
        const uint32_t b = c * kMaxNB + nb0 + bl;
        float2 w = make_float2(0.f, 0.f);
        if (b < B && a < A && f0 + fl < F) w = ph[((uint64_t)(b * (uint64_t)A + a) * F + f0 + fl) * 2 + pp];
        sp[bl][fl][pp][a >> 3][a & 7u] = w;
    }
    __syncthreads();
    const uint32_t ph_bytes = 3u * NB * 128u;
    // tasks t = (j, bl, p, fl), j fastest: a warp covers 8 groups x 4 beams
    for (uint32_t t = threadIdx.x; t < kPrepBeams * 8 * 2 * kPrepChans; t += blockDim.x) {
        const uint32_t j = t & 7u, bl = (t / 8u) % kPrepBeams, pp = (t / (8u * kPrepBeams)) & 1u,
                       fl = t / (16u * kPrepBeams);
        const uint32_t f = f0 + fl;
        if (f >= F) continue;
        __half rh[8], ih[8], rl[8], il[8], nih[8], nil[8];
        const float4* src = reinterpret_cast<const float4*>(&sp[bl][fl][pp][j][0]);
#pragma unroll
        for (int e2 = 0; e2 < 4; e2++) {
            const float4 v = src[e2];
            const float wr[2] = {v.x, v.z}, wi[2] = {v.y, v.w};
#pragma unroll
            for (int u = 0; u < 2; u++) {
                const int e = 2 * e2 + u;
                rh[e] = __float2half_rn(wr[u]);
                ih[e] = __float2half_rn(wi[u]);
                rl[e] = __float2half_rn(wr[u] - __half2float(rh[e]));
                il[e] = __float2half_rn(wi[u] - __half2float(ih[e]));
                nih[e] = __hneg(ih[e]);
                nil[e] = __hneg(il[e]);
            }
        }
        const uint32_t nb = nb0 + bl, k0 = j * 8;
        uint8_t* base = plan + ((uint64_t)c * F + f) * img_bytes + (uint64_t)pp * 2 * ph_bytes;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            uint8_t* blk = base + h * ph_bytes;
            // three blocks of NB rows x 64 K: [-Wi | Wr | Wi]
            put_chunk(blk, NB, nb, k0, pack8(h ? nil : nih));
            put_chunk(blk + NB * 128u, NB, nb, k0, pack8(h ? rl : rh));
            put_chunk(blk + 2u * NB * 128u, NB, nb, k0, pack8(h ? il : ih));
        }
    }
}

struct TcShape {
    uint32_t NB, KA, nchunks, img_bytes, raw_bytes, a_stages, r_stages, stacked;
    uint32_t raw_tiles, raw_row, direct;
    size_t smem;
};

// T = 0 sizes only the phasor image (the ring layout needs the tiles per channel).
bool tc_shape(uint64_t B, uint64_t A, TcShape& s, uint64_t T = 0, uint32_t es = 4, uint64_t rate = 0) {
    s.direct = 0;
    if (A == 0 || A > kMaxKA || B == 0) return false;
    const uint64_t bc = B < (uint64_t)kMaxNB ? B : (uint64_t)kMaxNB;
    s.NB = (uint32_t)((bc + 15) / 16 * 16);
    s.KA = A <= 32 ? 32u : 64u;
    s.nchunks = (uint32_t)((B + kMaxNB - 1) / kMaxNB);
    // hi/lo stacked along N (one MMA per k-step, N = 4 NB <= 128) whenever the
    // doubled accumulators still fit twice in tensor memory.
    s.stacked = s.NB <= 32 ? 1u : 0u;
    s.img_bytes = s.stacked ? (2 * s.KA / 64) * 1024u * s.NB : (s.KA == 64 ? 1536u : 1024u) * s.NB;
    s.raw_bytes = (uint32_t)A * kM * es;
    const size_t op = (2ull * s.KA / 64) * 16384;   // one polarisation's operand
    // barriers (2 x 8 operand + 2 x 8 raw + 3 x 4 accumulator + 4, 8 bytes each),
    // TMEM slot and abort flag, alignment slack
    const size_t fixed = s.img_bytes + 512 + 1024;
    const size_t limit = 227 * 1024;
    // Two-tile raw stages (1 KB per antenna row) when the channel's tile count is even
    // and one of these rings fits: four operand tile pairs and two raw stages (the
    // operand build runs up to four tiles ahead of the MMAs), else two pairs and
    // four or three raw stages.
    const uint64_t tpc = T / kM;
    if (T && es == 8) {
        // CF16 input: single-tile raw stages of 1 KB rows; four operand pairs and two
        // raw stages (two issuers), else two pairs and four or three raw stages.
        const uint32_t cand[][2] = {{8, 2}, {4, 4}, {4, 3}};
        for (const auto& c : cand) {
            if (fixed + c[0] * op + c[1] * (size_t)s.raw_bytes <= limit) {
                s.raw_tiles = 1;
                s.raw_row = kM * es;
                s.a_stages = c[0];
                s.r_stages = c[1];
                s.smem = fixed + c[0] * op + c[1] * (size_t)s.raw_bytes;
                return true;
            }
        }
    }
    if (T && es == 4 && tpc % 2 == 0) {
        const size_t raw2 = (size_t)A * 1024u;
        const uint32_t cand[][2] = {{8, 2}, {4, 4}, {4, 3}};
        for (const auto& c : cand) {
            if (fixed + c[0] * op + c[1] * raw2 <= limit) {
                s.raw_tiles = 2;
                s.raw_row = 1024;
                s.raw_bytes = (uint32_t)raw2;
                s.a_stages = c[0];
                s.r_stages = c[1];
                s.smem = fixed + c[0] * op + c[1] * raw2;
                return true;
            }
        }
    }
    s.raw_tiles = 1;
    s.raw_row = kM * es;
    // Deepest rings that fit: operand stages in pairs (one per polarisation) down to
    // four, raw stages down to three, then both down to the minimum.
    uint32_t as = kMaxStages, rs = 6;
    while (fixed + as * op + rs * (size_t)s.raw_bytes > limit) {
        if (rs > 3 && (rs > as / 2 || as <= 4)) rs--;
        else if (as > 4) as -= 2;
        else if (rs > 2) rs--;
        else if (as > 2) as--;
        else if (rs > 1) rs--;
        else return false;
    }
    s.a_stages = as;
    s.r_stages = rs;
    s.smem = fixed + as * op + rs * (size_t)s.raw_bytes;
    if (T && es == 4 && rate == 1 && as < 4) {
        // A phasor image this large leaves no room for a raw ring and a build-ahead
        // operand ring together: at rate 1 the converter threads load the voltages
        // themselves and the shared memory holds operand tile pairs only (two pairs
        // at least, so that the build runs a tile ahead and two issuers alternate).
        for (uint32_t c : {8u, 4u}) {
            if (fixed + c * op <= limit) {
                s.direct = 1;
                s.a_stages = c;
                s.r_stages = 0;
                s.raw_bytes = 0;
                s.smem = fixed + c * op;
                return true;
            }
        }
    }
    return true;
}

// A launch choice of the chain: mode 0 = raw ring of TMA tiles, 1 = converter
// threads load the voltages (rate 1 CI8), with the operand ring depth, the raw
// ring depth and the tiles per raw stage.
struct TcChoice {
    uint32_t mode, a_stages, r_stages, raw_tiles;
};

TcChoice tc_choice_of(const TcShape& s) {
    return TcChoice{s.direct ? 1u : 0u, s.a_stages, s.r_stages, s.raw_tiles};
}

// Lays out shape s (image part from tc_shape) for choice c; false when c does not
// apply to the shape or does not fit in shared memory.  Every choice computes the
// same arithmetic in the same order within a kernel (the ring depths only change
// scheduling), so modes 0 and 1 give bit-identical outputs.
bool tc_apply(TcShape& s, uint64_t A, uint64_t T, uint32_t es, uint64_t rate, const TcChoice& c) {
    const size_t op = (2ull * s.KA / 64) * 16384;
    const size_t limit = 227 * 1024;
    if (c.a_stages < 1 || c.a_stages > (uint32_t)kMaxStages) return false;
    s.direct = 0;
    s.a_stages = c.a_stages;
    if (c.mode == 1) {
        // direct loads run in pair mode: an even operand ring of at least four stages
        if (es != 4 || rate != 1 || (c.a_stages & 1u) || c.a_stages < 4u) return false;
        s.direct = 1;
        s.raw_tiles = 1;
        s.raw_row = kM * es;
        s.raw_bytes = 0;
        s.r_stages = 0;
        s.smem = s.img_bytes + 1536 + c.a_stages * op;
        return s.smem <= limit;
    }
    if (c.mode != 0 || c.r_stages < 1 || c.r_stages > (uint32_t)kMaxStages) return false;
    if (c.raw_tiles == 2) {
        if (es != 4 || (T / kM) % 2) return false;
        s.raw_row = 1024;
        s.raw_bytes = (uint32_t)A * 1024u;
    } else if (c.raw_tiles == 1) {
        s.raw_row = kM * es;
        s.raw_bytes = (uint32_t)A * kM * es;
    } else {
        return false;
    }
    s.raw_tiles = c.raw_tiles;
    s.r_stages = c.r_stages;
    s.smem = s.img_bytes + 1536 + c.a_stages * op + c.r_stages * (size_t)s.raw_bytes;
    return s.smem <= limit;
}

// The launch layout of a chain call: the tuned choice for this shape on this device
// when blade_beamform_detect_tc_autotune stored one, else the heuristic default.
bool tc_layout(uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t rate, uint64_t integration, uint32_t es,
               TcShape& s, bool* tuned = nullptr, TuneEntry* entry = nullptr) {
    if (!tc_shape(B, A, s, T, es, rate)) return false;
    if (tuned) *tuned = false;
    const uint64_t key[8] = {B, A, F, T, 2, rate, integration, es};
    TuneEntry e;
    if (tune_lookup(BLADE_TUNE_TC, key, &e)) {
        TcShape t = s;
        if (tc_apply(t, A, T, es, rate, TcChoice{e.params[0], e.params[1], e.params[2], e.params[3]})) {
            s = t;
            if (tuned) *tuned = true;
            if (entry) *entry = e;
        }
    }
    return true;
}

using TcKernel = void (*)(const TcArgs, const CUtensorMap);

// Tensor map of the voltages seen as samples [A][F][T] of es bytes (CI8: one
// 4-byte word, CF16: one 8-byte word = both polarisations of one sample);
// box = `box` samples x 1 channel x A.
int encode_voltage_map(CUtensorMap* tm, const void* in, uint64_t A, uint64_t F, uint64_t T, uint32_t box_t,
                       uint32_t es = 4) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!encode) {
            cudaDriverEntryPointQueryResult q;
            void* fn = nullptr;
            if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &fn, 12000, cudaEnableDefault, &q) !=
                    cudaSuccess ||
                q != cudaDriverEntryPointSuccess || !fn)
                return set_error(BLADE_CUDA_ERROR, "blade_beamform_detect_tc: cuTensorMapEncodeTiled unavailable");
            encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        }
    }
    const cuuint64_t dims[3] = {T, F, A};
    const cuuint64_t strides[2] = {T * es, F * T * es};
    const cuuint32_t box[3] = {box_t, 1, (cuuint32_t)A};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(tm, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, const_cast<void*>(in), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(BLADE_CUDA_ERROR, "blade_beamform_detect_tc: tensor map encode (%d)", (int)r);
    return BLADE_SUCCESS;
}

template <int R>
TcKernel pick_logi(uint32_t logi) {
    switch (logi) {
        case 0: return bf_tc_kernel<R, 0>;
        case 1: return bf_tc_kernel<R, 1>;
        case 2: return bf_tc_kernel<R, 2>;
        case 3: return bf_tc_kernel<R, 3>;
        case 4: return bf_tc_kernel<R, 4>;
        default: return bf_tc_kernel<R, 5>;
    }
}

TcKernel pick_kernel(uint64_t rate, uint64_t integration) {
    uint32_t logi = 0;
    while ((1ull << logi) < integration) logi++;
    if (rate == 1) return pick_logi<1>(logi);
    if (rate == 2) return pick_logi<2>(logi);
    return pick_logi<4>(logi);
}

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
    const uint64_t n = (uint64_t)s.nchunks * F * 2 * s.NB * (s.KA / 8);
    if (n > 0xFFFFFFFFull) return set_error(BLADE_ERROR, "blade_beamform_tc_prepare: too many channels");
    if (!s.stacked && s.KA == 64) {
        const dim3 grid((unsigned)((F + kPrepChans - 1) / kPrepChans), s.NB / kPrepBeams, s.nchunks);
        tc_prepare_wide_kernel<<<grid, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            static_cast<const float2*>(phasors), static_cast<uint8_t*>(plan), (uint32_t)B, (uint32_t)A, (uint32_t)F,
            s.NB, s.img_bytes);
    } else {
        tc_prepare_kernel<<<grid_for(n, 256), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
            static_cast<const float2*>(phasors), static_cast<uint8_t*>(plan), (uint32_t)B, (uint32_t)A, (uint32_t)F,
            s.NB, s.KA, s.nchunks, s.img_bytes, s.stacked);
    }
    return check_launch("blade_beamform_tc_prepare");
}

extern "C" int blade_beamform_detect_tc_supported(uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                                  uint64_t rate, uint64_t integration) {
    TcShape s;
    if (P != 2 || !tc_shape(B, A, s)) return 0;
    if (rate != 1 && rate != 2 && rate != 4) return 0;
    if (integration == 0 || integration > 32 || (integration & (integration - 1)) != 0) return 0;
    if (T == 0 || T % kM != 0 || F == 0) return 0;
    if (F > 0xffffffffull / (T / kM) || T >= (1ull << 31) || (uint64_t)A * F * T >= (1ull << 40)) return 0;
    return 1;
}

namespace bb {
namespace {

// Launches the chain over the 64-beam chunks once the arguments are checked.
int tc_run(const char* who, const void* in, const void* plan, void* out, uint64_t B, uint64_t A, uint64_t F,
           uint64_t T, uint64_t rate, uint64_t integration, uint32_t es, TcKernel fn, blade_stream_t stream,
           bool pdl = false, const TcShape* force = nullptr) {
    TcShape s;
    if (force) {
        s = *force;
    } else {
        tc_layout(B, A, F, T, rate, integration, es, s);
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int rc = ensure_smem(reinterpret_cast<const void*>(fn), s.smem)) return rc;
    const uint32_t U = (uint32_t)(T / (rate * integration));
    CUtensorMap tmap;
    if (int rc = encode_voltage_map(&tmap, in, A, F, T, s.raw_row / es, es)) return rc;
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
        g.NB = s.NB;
        g.KA = s.KA;
        g.a_stages = s.a_stages;
        g.r_stages = s.r_stages;
        g.img_bytes = s.img_bytes;
        g.raw_bytes = s.raw_bytes;
        g.raw_tiles = s.raw_tiles;
        g.raw_row = s.raw_row;
        g.stacked = s.stacked;
        g.tiles_per_ch = (uint32_t)(T / kM);
        g.total_tiles = (uint64_t)F * (T / kM);
        g.pdl = (pdl && c == 0) ? 1u : 0u;
        g.direct = s.direct;
        // outputs along TMEM lanes: full 64-beam chunks (separate hi/lo products),
        // rate 1 CI8, windows of 8 or 16 samples, 16-byte aligned output rows
        g.transposed = (!s.stacked && s.NB == 64 && rate == 1 && es == 4 && (integration == 8 || integration == 16) &&
                        U % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15u) == 0) ? 1u : 0u;
        // Whole raw stages per CTA (the kernel rounds its share up to raw_tiles); no
        // CTA is left without tiles.
        const uint64_t sms = (uint64_t)sm_count();
        const uint64_t per = ((g.total_tiles + sms - 1) / sms + s.raw_tiles - 1) / s.raw_tiles * s.raw_tiles;
        const uint64_t grid = (g.total_tiles + per - 1) / per;
        if (g.pdl) {
            // programmatic dependent of the phasor split launched just before on this
            // stream: prologue and raw loads overlap it (the kernel waits before the image)
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)grid, 1, 1);
            cfg.blockDim = dim3(kThreads, 1, 1);
            cfg.dynamicSmemBytes = s.smem;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            const cudaError_t e = cudaLaunchKernelEx(&cfg, fn, g, tmap);
            if (e != cudaSuccess) return check_cuda(e, who);
        } else {
            fn<<<(unsigned)grid, kThreads, s.smem, st>>>(g, tmap);
        }
        if (int rc = check_launch(who)) return rc;
    }
    return BLADE_SUCCESS;
}

TcKernel pick_cf16(uint64_t integration) {
    uint32_t logi = 0;
    while ((1ull << logi) < integration) logi++;
    switch (logi) {
        case 0: return bf_tc_kernel<1, 0, 8>;
        case 1: return bf_tc_kernel<1, 1, 8>;
        case 2: return bf_tc_kernel<1, 2, 8>;
        case 3: return bf_tc_kernel<1, 3, 8>;
        case 4: return bf_tc_kernel<1, 4, 8>;
        default: return bf_tc_kernel<1, 5, 8>;
    }
}

}  // namespace
}  // namespace bb

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
    return tc_run("blade_beamform_detect_tc", in, plan, out, B, A, F, T, rate, integration, 4,
                  pick_kernel(rate, integration), stream);
}

extern "C" int blade_beamform_prepare_detect_tc(const void* phasors, void* plan, const void* in, void* out,
                                                uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                                uint64_t rate, uint64_t integration, blade_stream_t stream) {
    if (!blade_beamform_detect_tc_supported(B, A, F, T, P, rate, integration))
        return set_error(BLADE_ERROR,
                         "blade_beamform_prepare_detect_tc: unsupported configuration (B=%llu A=%llu T=%llu P=%llu "
                         "rate=%llu I=%llu): needs P=2, 1<=A<=64, T%%128==0, rate in {1,2,4}, I a power of two <= 32",
                         (unsigned long long)B, (unsigned long long)A, (unsigned long long)T, (unsigned long long)P,
                         (unsigned long long)rate, (unsigned long long)integration);
    if (!in || !plan || !out || !phasors) return set_error(BLADE_ERROR, "blade_beamform_prepare_detect_tc: null buffer");
    if (!aligned16(in) || !aligned16(plan) || (reinterpret_cast<uintptr_t>(out) & 3))
        return set_error(BLADE_ERROR, "blade_beamform_prepare_detect_tc: input and plan must be 16-byte aligned");
    if (F == 0) return BLADE_SUCCESS;  // no split launched: nothing may follow it programmatically
    if (int rc = blade_beamform_tc_prepare(phasors, plan, B, A, F, P, stream)) return rc;
    return tc_run("blade_beamform_prepare_detect_tc", in, plan, out, B, A, F, T, rate, integration, 4,
                  pick_kernel(rate, integration), stream, true);
}

extern "C" int blade_beamform_detect_tc_cf16(const void* in, const void* plan, void* out, uint64_t B, uint64_t A,
                                             uint64_t F, uint64_t T, uint64_t P, uint64_t integration,
                                             blade_stream_t stream) {
    if (!blade_beamform_detect_tc_supported(B, A, F, T, P, 1, integration))
        return set_error(BLADE_ERROR,
                         "blade_beamform_detect_tc_cf16: unsupported configuration (B=%llu A=%llu T=%llu P=%llu "
                         "I=%llu): needs P=2, 1<=A<=64, T%%128==0, I a power of two <= 32",
                         (unsigned long long)B, (unsigned long long)A, (unsigned long long)T, (unsigned long long)P,
                         (unsigned long long)integration);
    if (!in || !plan || !out) return set_error(BLADE_ERROR, "blade_beamform_detect_tc_cf16: null buffer");
    if (!aligned16(in) || !aligned16(plan) || (reinterpret_cast<uintptr_t>(out) & 3))
        return set_error(BLADE_ERROR, "blade_beamform_detect_tc_cf16: input and plan must be 16-byte aligned");
    return tc_run("blade_beamform_detect_tc_cf16", in, plan, out, B, A, F, T, 1, integration, 8,
                  pick_cf16(integration), stream);
}

extern "C" int blade_beamform_prepare_detect_tc_cf16(const void* phasors, void* plan, const void* in, void* out,
                                                     uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                                     uint64_t integration, blade_stream_t stream) {
    if (!blade_beamform_detect_tc_supported(B, A, F, T, P, 1, integration))
        return set_error(BLADE_ERROR,
                         "blade_beamform_prepare_detect_tc_cf16: unsupported configuration (B=%llu A=%llu T=%llu "
                         "P=%llu I=%llu): needs P=2, 1<=A<=64, T%%128==0, I a power of two <= 32",
                         (unsigned long long)B, (unsigned long long)A, (unsigned long long)T, (unsigned long long)P,
                         (unsigned long long)integration);
    if (!in || !plan || !out || !phasors)
        return set_error(BLADE_ERROR, "blade_beamform_prepare_detect_tc_cf16: null buffer");
    if (!aligned16(in) || !aligned16(plan) || (reinterpret_cast<uintptr_t>(out) & 3))
        return set_error(BLADE_ERROR, "blade_beamform_prepare_detect_tc_cf16: input and plan must be 16-byte aligned");
    if (F == 0) return BLADE_SUCCESS;
    if (int rc = blade_beamform_tc_prepare(phasors, plan, B, A, F, P, stream)) return rc;
    return tc_run("blade_beamform_prepare_detect_tc_cf16", in, plan, out, B, A, F, T, 1, integration, 8,
                  pick_cf16(integration), stream, true);
}

namespace bb {
int adjoint_status_take(uint32_t* v);
}

extern "C" int blade_device_status(uint32_t* status) {
    unsigned int v = 0, zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_status, sizeof(v));
    if (e != cudaSuccess) return check_cuda(e, "blade_device_status");
    e = cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(zero));
    if (e != cudaSuccess) return check_cuda(e, "blade_device_status");
    // the tensor-core adjoint's word: codes 0x100 | 1 (a phase wait expired), 0x100 | 2 (the drain did)
    uint32_t adj = 0;
    if (int rc = bb::adjoint_status_take(&adj)) return rc;
    if (!v && adj) v = 0x100u | adj;
    if (status) *status = v;
    return BLADE_SUCCESS;
}

// ---- bounded-wait self-test ---------------------------------------------------
// One thread waits on an mbarrier that nothing ever completes, through the same
// bounded wait as the pipelined kernels; when the budget runs out it records
// kSelftestCode in the status word and the kernel returns normally, so the
// expiry path is exercised without a fault and the context stays usable.
namespace bb {
namespace {
constexpr unsigned kSelftestCode = 0x20u;

__global__ void wait_selftest_kernel(long long budget) {
    __shared__ __align__(8) uint64_t bar;
    volatile int never = 0;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);  // one arrival completes phase 0; none is ever made
        tc::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !tc::mbar_wait(&bar, 0, &never, budget)) atomicCAS(&g_tc_status, 0u, kSelftestCode);
}
}  // namespace
}  // namespace bb

extern "C" int blade_wait_selftest(uint64_t budget_cycles, blade_stream_t stream) {
    using namespace bb;
    if (budget_cycles == 0 || budget_cycles > 10000000000ull)
        return set_error(BLADE_ERROR, "blade_wait_selftest: budget must be 1 .. 1e10 cycles (got %llu)",
                         (unsigned long long)budget_cycles);
    wait_selftest_kernel<<<1, 32, 0, reinterpret_cast<cudaStream_t>(stream)>>>((long long)budget_cycles);
    return check_launch("blade_wait_selftest");
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

template <typename Fn>
int driver_entry(const char* name, unsigned version, Fn* fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPointByVersion(name, &p, version, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
        return set_error(BLADE_CUDA_ERROR, "blade_beamform_detect_tc_noalloc: %s unavailable", name);
    *fn = reinterpret_cast<Fn>(p);
    return BLADE_SUCCESS;
}

// Device address of g_tc_noalloc_plan, looked up with the device current (the
// host-side name is only a stand-in for the device array) once per device and
// context: the cache is keyed on the current context's unique id as well, so
// after a cudaDeviceReset, which destroys the primary context and this module's
// copy of the array with it, the next call looks the address up again.
int noalloc_plan_address(void** out) {
    static std::mutex mu;
    static void* addr[64] = {nullptr};
    static unsigned long long ctx_of[64] = {0};
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return check_cuda(e, "blade_beamform_detect_tc_noalloc");
    if (dev < 0 || dev >= 64) return set_error(BLADE_ERROR, "blade_beamform_detect_tc_noalloc: device %d", dev);
    // makes the device's primary context current, creating it if a reset destroyed it
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) return check_cuda(e, "blade_beamform_detect_tc_noalloc: cudaSetDevice");
    std::lock_guard<std::mutex> lock(mu);
    if (!get_current) {
        if (int rc = driver_entry("cuCtxGetCurrent", 4000, &get_current)) return rc;
        if (int rc = driver_entry("cuCtxGetId", 12000, &get_id)) return rc;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return set_error(BLADE_CUDA_ERROR, "blade_beamform_detect_tc_noalloc: no current CUDA context");
    if (!addr[dev] || ctx_of[dev] != id) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_tc_noalloc_plan);
        if (e != cudaSuccess) return check_cuda(e, "blade_beamform_detect_tc_noalloc: cudaGetSymbolAddress");
        addr[dev] = p;
        ctx_of[dev] = id;
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
    return blade_beamform_prepare_detect_tc(phasors, plan, in, out, B, A, F, T, P, rate, integration, stream);
}

// ---- autotuner ------------------------------------------------------------------

namespace bb {
namespace {

// Device buffers of one tuning run, freed on every return path.
struct DevBufs {
    std::vector<void*> p;
    ~DevBufs() {
        for (void* q : p) cudaFree(q);
    }
    void* get(size_t bytes) {
        void* q = nullptr;
        if (cudaMalloc(&q, bytes < 16 ? 16 : bytes) != cudaSuccess) return nullptr;
        p.push_back(q);
        return q;
    }
};

}  // namespace

// Output bytes a and b (device) are identical; false on a copy failure too.
bool tune_same(const void* a, const void* b, size_t bytes) {
    std::vector<uint8_t> ha(bytes), hb(bytes);
    if (cudaMemcpy(ha.data(), a, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    if (cudaMemcpy(hb.data(), b, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    return memcmp(ha.data(), hb.data(), bytes) == 0;
}

int tc_query(const uint64_t (&shape)[8], uint32_t* params, float* us, int* tuned) {
    TcShape s;
    bool t = false;
    TuneEntry e;
    const uint32_t es = shape[7] ? (uint32_t)shape[7] : 4u;
    if (shape[4] != 2 || !tc_layout(shape[0], shape[1], shape[2], shape[3], shape[5], shape[6], es, s, &t, &e))
        return set_error(BLADE_ERROR, "blade_autotune_query: unsupported tensor-core shape");
    const TcChoice c = tc_choice_of(s);
    for (int i = 0; i < kTuneParams; i++) params[i] = t ? e.params[i] : 0u;
    params[0] = c.mode;
    params[1] = c.a_stages;
    params[2] = c.r_stages;
    params[3] = c.raw_tiles;
    *us = t ? e.us : 0.f;
    *tuned = t ? 1 : 0;
    return BLADE_SUCCESS;
}

}  // namespace bb

extern "C" int blade_beamform_detect_tc_autotune(uint64_t B, uint64_t A, uint64_t F, uint64_t T, uint64_t P,
                                                 uint64_t rate, uint64_t integration, blade_stream_t stream) {
    using namespace bb;
    const char* who = "blade_beamform_detect_tc_autotune";
    if (!blade_beamform_detect_tc_supported(B, A, F, T, P, rate, integration))
        return set_error(BLADE_ERROR, "%s: unsupported configuration", who);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t U = T / (rate * integration);
    const size_t in_bytes = (size_t)A * F * T * 4, ph_count = (size_t)B * A * F * 2;
    const size_t plan_bytes = blade_beamform_tc_plan_size(B, A, F, P);
    const size_t out_bytes = (size_t)B * F * rate * U * sizeof(float);
    DevBufs bufs;
    void* in = bufs.get(in_bytes);
    void* ph = bufs.get(ph_count * sizeof(float2));
    void* plan = bufs.get(plan_bytes);
    void* ref = bufs.get(out_bytes);
    void* out = bufs.get(out_bytes);
    if (!in || !ph || !plan || !ref || !out) return set_error(BLADE_CUDA_ERROR, "%s: allocation failed", who);
    if (int rc = tune_fill_ci8(in, in_bytes, st)) return rc;
    if (int rc = tune_fill_phasors(ph, ph_count, st)) return rc;
    if (int rc = blade_beamform_tc_prepare(ph, plan, B, A, F, P, stream)) return rc;
    TcShape base;
    tc_shape(B, A, base, T, 4, rate);
    const TcKernel fn = pick_kernel(rate, integration);
    // candidates: the default first, then every ring layout that fits
    std::vector<TcChoice> cands{tc_choice_of(base)};
    auto add = [&](TcChoice c) {
        for (const auto& d : cands)
            if (d.mode == c.mode && d.a_stages == c.a_stages && d.r_stages == c.r_stages && d.raw_tiles == c.raw_tiles)
                return;
        TcShape t = base;
        if (tc_apply(t, A, T, 4, rate, c)) cands.push_back(c);
    };
    const uint32_t rings[][2] = {{8, 2}, {8, 3}, {6, 2}, {4, 4}, {4, 3}, {4, 2}, {2, 4}, {2, 2}};
    for (uint32_t rt : {2u, 1u})
        for (const auto& r : rings) add(TcChoice{0, r[0], r[1], rt});
    for (uint32_t a : {8u, 6u, 4u}) add(TcChoice{1, a, 0, 1});
    int best = -1;
    float best_us = 0.f;
    uint32_t ndiff = 0, ntimed = 0;
    for (size_t i = 0; i < cands.size(); i++) {
        TcShape t = base;
        tc_apply(t, A, T, 4, rate, cands[i]);
        void* dst = i == 0 ? ref : out;
        const float us = tune_time(
            [&]() { return tc_run(who, in, plan, dst, B, A, F, T, rate, integration, 4, fn, stream, false, &t); }, st);
        if (us < 0.f) return set_error(BLADE_CUDA_ERROR, "%s: candidate %zu failed: %s", who, i, blade_last_error());
        uint32_t status = 0;
        if (int rc = blade_device_status(&status)) return rc;
        if (status != 0) return set_error(BLADE_CUDA_ERROR, "%s: candidate %zu: device status %u", who, i, status);
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
    e.params[0] = cands[best].mode;
    e.params[1] = cands[best].a_stages;
    e.params[2] = cands[best].r_stages;
    e.params[3] = cands[best].raw_tiles;
    e.params[4] = ntimed;
    e.params[5] = ndiff;
    e.us = best_us;
    const uint64_t key[8] = {B, A, F, T, P, rate, integration, 4};
    tune_store(BLADE_TUNE_TC, key, e);
    return BLADE_SUCCESS;
}
