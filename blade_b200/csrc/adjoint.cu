// Adjoint of beamform + Stokes-I detect with respect to the complex weights.
// No reference counterpart (the reference has no differentiation).
//
// L = -sum_{b,f,t,p} |y[b,f,t,p]|^2,  y[b,f,t,p] = sum_a x[a,f,t,p] w[b,a,f,0,p]
// dL/d conj(w[b,a,f,0,p]) = -sum_t y[b,f,t,p] conj(x[a,f,t,p])
// (detector integration windows do not change the sum, so they drop out).
//
// One CTA owns one (f, p) and walks the time axis in tiles of 256 samples: the
// tile's voltages are staged in shared memory, the beam voltages y are recomputed
// for the tile (never stored to HBM), and the products y conj(x) are reduced over
// the tile by (beam, antenna) pair with the tile's samples split across threads;
// the per-pair partial sums are added in a fixed order, so results are
// deterministic.  HBM traffic is one read of the voltages.  The loss is returned
// per (f, p) (the caller adds the F*P partials), which keeps every sum ordered.
#include "common.cuh"

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
        if (tid == 0) loss[fp] = -lred[0];
    }
}

}  // namespace
}  // namespace bb

extern "C" int blade_beamform_detect_adjoint(const void* in, const void* phasors, void* grad, double* loss, uint64_t B,
                                             uint64_t A, uint64_t F, uint64_t T, uint64_t P, blade_stream_t stream) {
    using namespace bb;
    if (P != 1 && P != 2) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: P must be 1 or 2");
    if (B == 0 || A == 0 || F == 0) return BLADE_SUCCESS;
    if (!in || !phasors || !grad) return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: null buffer");
    const size_t smem = ((size_t)B * A * 2 + (size_t)A * kT + (size_t)B * kT + kT) * sizeof(float2) +
                        kT * sizeof(double);
    if (smem > 227 * 1024)
        return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: B=%llu x A=%llu exceeds shared memory",
                         (unsigned long long)B, (unsigned long long)A);
    if (F * P > 0x7fffffffull || T >= (1ull << 32))
        return set_error(BLADE_ERROR, "blade_beamform_detect_adjoint: dimensions out of range");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (int rc = ensure_smem(reinterpret_cast<const void*>(adjoint_kernel), smem)) return rc;
    adjoint_kernel<<<(unsigned)(F * P), kT, smem, s>>>(static_cast<const float2*>(in),
                                                       static_cast<const float2*>(phasors),
                                                       static_cast<float2*>(grad), loss, (uint32_t)B, (uint32_t)A,
                                                       (uint32_t)F, (uint32_t)T, (uint32_t)P);
    return check_launch("blade_beamform_detect_adjoint");
}
