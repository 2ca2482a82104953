// Byte-movement modules: Duplicate, Gather, Permutation.  All bit-exact.
//
// Reference: Duplicate = cudaMemcpyAsync D2D (src/modules/duplicate/base.cc:34-37);
// Gather = one scalar scatter per thread or Copy2D (src/modules/gather/base.cc:70-111,
// gather.cu:6-18); Permutation = one scalar scatter per thread through
// offset -> coordinates -> permuted offset (src/modules/permutation/permutation.cu:6-20).
// Here: 128-bit copies where alignment allows, row copies for gather and for
// permutations that keep the innermost axis, and a shared-memory tiled transpose
// (coalesced reads and writes) for permutations that move it.
#include "common.cuh"

namespace bb {
namespace {

template <int N> struct Bytes;
template <> struct Bytes<1> { using T = uint8_t; };
template <> struct Bytes<2> { using T = uint16_t; };
template <> struct Bytes<4> { using T = uint32_t; };
template <> struct Bytes<8> { using T = uint2; };
template <> struct Bytes<16> { using T = uint4; };

// 2-D strided copy: rows of `vpr` vectors; src row r at src + r*src_pitch,
// dst row r at dst + r*dst_pitch (pitches in vectors).
template <typename V>
__global__ void __launch_bounds__(256) copy2d_kernel(const V* __restrict__ src, V* __restrict__ dst,
                                                     uint64_t rows, uint64_t vpr, uint64_t src_pitch,
                                                     uint64_t dst_pitch) {
    const uint64_t total = rows * vpr;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        uint64_t r = i / vpr, c = i - r * vpr;
        dst[r * dst_pitch + c] = src[r * src_pitch + c];
    }
}

template <typename V>
int launch_copy2d(const void* src, void* dst, uint64_t rows, uint64_t vpr, uint64_t sp, uint64_t dp,
                  cudaStream_t s) {
    uint64_t total = rows * vpr;
    if (total == 0) return BLADE_SUCCESS;
    copy2d_kernel<V><<<grid_for(total, 256), 256, 0, s>>>(static_cast<const V*>(src), static_cast<V*>(dst), rows,
                                                          vpr, sp, dp);
    return BLADE_SUCCESS;
}

// Copies `rows` rows of `row_bytes` bytes with byte pitches, picking the widest
// vector that every address and size allows.
int copy_rows(const void* src, void* dst, uint64_t rows, uint64_t row_bytes, uint64_t src_pitch_b,
              uint64_t dst_pitch_b, cudaStream_t s) {
    uintptr_t a = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst) | row_bytes |
                  src_pitch_b | dst_pitch_b;
    int rc;
    if ((a & 15) == 0)
        rc = launch_copy2d<uint4>(src, dst, rows, row_bytes / 16, src_pitch_b / 16, dst_pitch_b / 16, s);
    else if ((a & 7) == 0)
        rc = launch_copy2d<uint2>(src, dst, rows, row_bytes / 8, src_pitch_b / 8, dst_pitch_b / 8, s);
    else if ((a & 3) == 0)
        rc = launch_copy2d<uint32_t>(src, dst, rows, row_bytes / 4, src_pitch_b / 4, dst_pitch_b / 4, s);
    else if ((a & 1) == 0)
        rc = launch_copy2d<uint16_t>(src, dst, rows, row_bytes / 2, src_pitch_b / 2, dst_pitch_b / 2, s);
    else
        rc = launch_copy2d<uint8_t>(src, dst, rows, row_bytes, src_pitch_b, dst_pitch_b, s);
    if (rc) return rc;
    return check_launch("copy");
}

// Tiled transpose for a 4-D permutation that moves the innermost input axis.
// X = input axis 3 (contiguous in the input), Y = input axis that becomes the
// output's innermost (contiguous in the output).  U, V = the other two axes.
struct PermGeom {
    uint64_t nX, nY, nU, nV;         // extents
    uint64_t isY, isU, isV;          // input strides (elements); isX = 1
    uint64_t osX, osU, osV;          // output strides (elements); osY = 1
};

template <typename T>
__global__ void __launch_bounds__(256) transpose_kernel(const T* __restrict__ in, T* __restrict__ out, PermGeom g,
                                                        uint64_t tiles_x, uint64_t tiles_y, uint64_t batches) {
    __shared__ T tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    const uint64_t ntiles = tiles_x * tiles_y * batches;
    for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        uint64_t b = t / (tiles_x * tiles_y);
        uint64_t r = t - b * tiles_x * tiles_y;
        uint64_t yt = r / tiles_x, xt = r - yt * tiles_x;
        uint64_t u = b / g.nV, v = b - u * g.nV;
        uint64_t x0 = xt * 32, y0 = yt * 32;
        const T* ib = in + u * g.isU + v * g.isV;
        T* ob = out + u * g.osU + v * g.osV;
#pragma unroll
        for (int k = 0; k < 32; k += 8) {
            uint64_t x = x0 + tx, y = y0 + ty + k;
            if (x < g.nX && y < g.nY) tile[ty + k][tx] = ib[y * g.isY + x];
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 32; k += 8) {
            uint64_t y = y0 + tx, x = x0 + ty + k;
            if (x < g.nX && y < g.nY) ob[x * g.osX + y] = tile[tx][ty + k];
        }
        __syncthreads();
    }
}

template <int ES>
int launch_transpose(const void* in, void* out, const PermGeom& g, cudaStream_t s) {
    using T = typename Bytes<ES>::T;
    uint64_t tx = ceil_div(g.nX, 32), ty = ceil_div(g.nY, 32), nb = g.nU * g.nV;
    uint64_t ntiles = tx * ty * nb;
    if (ntiles == 0) return BLADE_SUCCESS;
    uint64_t grid = ntiles < (uint64_t)sm_count() * 16 ? ntiles : (uint64_t)sm_count() * 16;
    transpose_kernel<T><<<(unsigned)grid, 256, 0, s>>>(static_cast<const T*>(in), static_cast<T*>(out), g, tx, ty,
                                                       nb);
    return check_launch("blade_permute");
}


// Permutation that keeps the innermost axis: output row r = (o0, o1, o2)
// copies vpr vectors from input offset o0*s0 + o1*s1 + o2*s2 (vector units).
struct PermRows {
    uint64_t rows, n1, n2, vpr, s0, s1, s2;
};

template <typename V>
__global__ void __launch_bounds__(256) perm_rows_kernel(const V* __restrict__ in, V* __restrict__ out, PermRows r) {
    const uint64_t total = r.rows * r.vpr;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += stride) {
        uint64_t row = i / r.vpr, c = i - row * r.vpr;
        uint64_t o2 = row % r.n2, t = row / r.n2;
        uint64_t o1 = t % r.n1, o0 = t / r.n1;
        out[i] = in[o0 * r.s0 + o1 * r.s1 + o2 * r.s2 + c];
    }
}

template <typename V>
int launch_perm_rows(const void* in, void* out, const PermRows& r, cudaStream_t s) {
    uint64_t total = r.rows * r.vpr;
    perm_rows_kernel<V><<<grid_for(total, 256), 256, 0, s>>>(static_cast<const V*>(in), static_cast<V*>(out), r);
    return check_launch("blade_permute");
}

}  // namespace
}  // namespace bb

extern "C" int blade_duplicate(const void* in, void* out, uint64_t bytes, blade_stream_t stream) {
    using namespace bb;
    if (bytes == 0 || in == out) return BLADE_SUCCESS;
    if (!in || !out) return set_error(BLADE_ERROR, "blade_duplicate: null buffer");
    return copy_rows(in, out, 1, bytes, bytes, bytes, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int blade_gather(uint64_t elem_bytes, const void* in, void* out, const uint64_t shape[4], uint64_t axis,
                            uint64_t multiplier, uint64_t step, blade_stream_t stream) {
    using namespace bb;
    if (!shape) return set_error(BLADE_ERROR, "blade_gather: null shape");
    if (axis >= 4) return set_error(BLADE_ERROR, "blade_gather: axis (%llu) is larger than the rank (4)",
                                    (unsigned long long)axis);
    if (multiplier == 0) return set_error(BLADE_ERROR, "blade_gather: multiplier should be more than zero");
    if (step >= multiplier)
        return set_error(BLADE_ERROR, "blade_gather: step (%llu) must be below the multiplier (%llu)",
                         (unsigned long long)step, (unsigned long long)multiplier);
    if (elem_bytes == 0) return set_error(BLADE_ERROR, "blade_gather: element size is zero");
    uint64_t height = 1, width = 1;
    for (uint64_t i = 0; i < axis; i++) height *= shape[i];
    for (uint64_t i = axis; i < 4; i++) width *= shape[i];
    if (height * width == 0) return BLADE_SUCCESS;
    if (!in || !out) return set_error(BLADE_ERROR, "blade_gather: null buffer");
    const uint64_t wb = width * elem_bytes;
    return copy_rows(in, static_cast<char*>(out) + step * wb, height, wb, wb, wb * multiplier,
                     reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int blade_permute(uint64_t elem_bytes, const void* in, void* out, const uint64_t shape[4],
                             const uint64_t indexes[4], blade_stream_t stream) {
    using namespace bb;
    if (!shape || !indexes) return set_error(BLADE_ERROR, "blade_permute: null shape or indexes");
    int seen = 0;
    for (int i = 0; i < 4; i++) {
        if (indexes[i] >= 4) return set_error(BLADE_ERROR, "blade_permute: index %llu out of range",
                                              (unsigned long long)indexes[i]);
        if (seen & (1 << indexes[i]))
            return set_error(BLADE_ERROR, "blade_permute: repeated index %llu in permutation",
                             (unsigned long long)indexes[i]);
        seen |= 1 << indexes[i];
    }
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16)
        return set_error(BLADE_ERROR, "blade_permute: unsupported element size %llu", (unsigned long long)elem_bytes);
    uint64_t n = shape[0] * shape[1] * shape[2] * shape[3];
    if (n == 0) return BLADE_SUCCESS;
    if (!in || !out) return set_error(BLADE_ERROR, "blade_permute: null buffer");
    if (in == out) return set_error(BLADE_ERROR, "blade_permute: in-place permutation is not supported");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

    // Input axes that stay adjacent and in order in the output move as one axis:
    // merge them first (e.g. AFTP -> ATPF is [A][F][T P] -> [A][T P][F], a batched
    // transpose of full-width tiles instead of tiles two elements wide), then pad
    // the merged rank back to four with leading axes of extent 1.
    uint64_t mshape[4] = {1, 1, 1, 1}, midx[4] = {0, 1, 2, 3};
    {
        int first[4], last[4], ng = 0;  // groups of input axes in output order
        for (int i = 0; i < 4; i++) {
            if (ng > 0 && indexes[i] == (uint64_t)last[ng - 1] + 1) {
                last[ng - 1] = (int)indexes[i];
            } else {
                first[ng] = last[ng] = (int)indexes[i];
                ng++;
            }
        }
        int rank[4];  // each group's position among the groups in input order
        for (int g = 0; g < ng; g++) {
            rank[g] = 0;
            for (int h = 0; h < ng; h++)
                if (first[h] < first[g]) rank[g]++;
        }
        const int pad = 4 - ng;
        for (int g = 0; g < ng; g++) {
            uint64_t ext = 1;
            for (int d = first[g]; d <= last[g]; d++) ext *= shape[d];
            mshape[pad + rank[g]] = ext;
            midx[pad + g] = (uint64_t)(pad + rank[g]);
        }
        for (int i = 0; i < pad; i++) midx[i] = (uint64_t)i;
        shape = mshape;
        indexes = midx;
    }

    // Input strides and output strides expressed per input axis.
    uint64_t is[4], os_out[4], os_in[4], oshape[4];
    is[3] = 1;
    for (int d = 2; d >= 0; d--) is[d] = is[d + 1] * shape[d + 1];
    for (int i = 0; i < 4; i++) oshape[i] = shape[indexes[i]];
    os_out[3] = 1;
    for (int i = 2; i >= 0; i--) os_out[i] = os_out[i + 1] * oshape[i + 1];
    for (int i = 0; i < 4; i++) os_in[indexes[i]] = os_out[i];

    if (indexes[3] == 3) {
        // Innermost axis stays: rows of shape[3] contiguous elements, one row
        // per output (o0, o1, o2); vectors as wide as alignment allows.
        PermRows r;
        r.n1 = oshape[1];
        r.n2 = oshape[2];
        r.rows = oshape[0] * oshape[1] * oshape[2];
        const uint64_t rb = shape[3] * elem_bytes;
        uintptr_t a = reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out) | rb;
        uint64_t vb = (a & 15) == 0 ? 16 : (a & 7) == 0 ? 8 : (a & 3) == 0 ? 4 : (a & 1) == 0 ? 2 : 1;
        r.vpr = rb / vb;
        r.s0 = is[indexes[0]] * elem_bytes / vb;
        r.s1 = is[indexes[1]] * elem_bytes / vb;
        r.s2 = is[indexes[2]] * elem_bytes / vb;
        switch (vb) {
            case 16: return launch_perm_rows<uint4>(in, out, r, s);
            case 8: return launch_perm_rows<uint2>(in, out, r, s);
            case 4: return launch_perm_rows<uint32_t>(in, out, r, s);
            case 2: return launch_perm_rows<uint16_t>(in, out, r, s);
            default: return launch_perm_rows<uint8_t>(in, out, r, s);
        }
    }

    PermGeom g;
    const int X = 3;
    const int Y = (int)indexes[3];
    int others[2], k = 0;
    for (int d = 0; d < 4; d++)
        if (d != X && d != Y) others[k++] = d;
    g.nX = shape[X];
    g.nY = shape[Y];
    g.nU = shape[others[0]];
    g.nV = shape[others[1]];
    g.isY = is[Y];
    g.isU = is[others[0]];
    g.isV = is[others[1]];
    g.osX = os_in[X];
    g.osU = os_in[others[0]];
    g.osV = os_in[others[1]];
    if (os_in[Y] != 1) return set_error(BLADE_ASSERTION_ERROR, "blade_permute: internal stride error");
    switch (elem_bytes) {
        case 1: return launch_transpose<1>(in, out, g, s);
        case 2: return launch_transpose<2>(in, out, g, s);
        case 4: return launch_transpose<4>(in, out, g, s);
        case 8: return launch_transpose<8>(in, out, g, s);
        default: return launch_transpose<16>(in, out, g, s);
    }
}
