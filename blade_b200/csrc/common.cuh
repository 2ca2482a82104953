// Shared helpers for the sm_100a kernels behind the blade_b200 C ABI.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>
#include <stdio.h>

#include "blade_b200.h"

namespace bb {

// Records a message for blade_last_error() and returns the status code.
int set_error(int code, const char* fmt, ...);

// Status of the last launch on this thread (cudaPeekAtLastError semantics,
// as include/blade/module.hh:77-80 does after each reference launch).
int check_launch(const char* what);

inline int check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        return set_error(BLADE_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
    }
    return BLADE_SUCCESS;
}

__host__ __device__ inline uint64_t ceil_div(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Number of SMs of the current device (cached per device).
int sm_count();

// Raises a kernel's dynamic shared-memory limit to `bytes` once per device (the
// attribute call is skipped afterwards, so launches stay capturable in graphs).
int ensure_smem(const void* func, size_t bytes);

// Grid size for a grid-stride loop: enough CTAs to fill every SM `per_sm` times,
// never more than the work needs.
inline unsigned grid_for(uint64_t work_items, unsigned block, unsigned per_sm = 8) {
    uint64_t need = ceil_div(work_items, block);
    uint64_t cap = (uint64_t)sm_count() * per_sm;
    if (need > cap) need = cap;
    if (need == 0) need = 1;
    return (unsigned)need;
}

// Bytes per element of a BLADE_* dtype (complex types count both parts).
inline uint64_t dtype_bytes(int t) {
    switch (t) {
        case BLADE_I8: return 1;
        case BLADE_I32: return 4;
        case BLADE_F16: return 2;
        case BLADE_F32: return 4;
        case BLADE_F64: return 8;
        case BLADE_CI8: return 2;
        case BLADE_CF16: return 4;
        case BLADE_CF32: return 8;
        case BLADE_CF64: return 16;
        default: return 0;
    }
}

inline bool dtype_is_complex(int t) {
    return t == BLADE_CI8 || t == BLADE_CF16 || t == BLADE_CF32 || t == BLADE_CF64;
}

// ---- device helpers -------------------------------------------------------

// Streaming 16-byte loads of data that is read-only for the whole kernel.  Not
// volatile, so the compiler may batch several of them ahead of their uses.
__device__ __forceinline__ float4 ldg_nc_f4(const void* p) {
    float4 v;
    asm("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
    return v;
}

__device__ __forceinline__ uint4 ldg_nc_u4(const void* p) {
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
    return v;
}

__device__ __forceinline__ void stg_f4(void* p, float4 v) {
    *reinterpret_cast<float4*>(p) = v;
}

}  // namespace bb
