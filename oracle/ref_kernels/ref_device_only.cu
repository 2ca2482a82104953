// Test-only checker, device code only: the reference's own polarizer, gather
// (accumulate) and permutation kernels, compiled from the reference sources where
// they lie by build.sh with `nvcc -cubin`, one kernel per cubin (REF_PICK).
//
// These kernels take ArrayTensor arguments by value whose element type
// (Blade::ops::complex) the reference defines for device code only, so nvcc
// cannot generate their host launch stubs (the reference itself compiles them
// with NVRTC at run time).  A device-only cubin needs no stub: the tests load it
// and launch its single kernel through the CUDA driver API with the argument
// bytes laid out as the reference's Vector<Device::CUDA, T, ArrayShape>
// (oracle/ref_kernels/cubin.py).  Nothing in blade_b200 links or loads these.
//
//   REF_PICK 1  src/modules/polarizer/polarizer.cu:5-25      polarizer<CF32, CF32>
//   REF_PICK 2  src/modules/polarizer/polarizer.cu:5-25      polarizer<CF16, CF16>
//   REF_PICK 3  src/modules/gather/gather.cu:6-18            accumulate<CF32>
//   REF_PICK 4  src/modules/permutation/permutation.cu:6-20  permutation<CF32>
#include <cassert>

#if REF_PICK == 1 || REF_PICK == 2
#include "src/modules/polarizer/polarizer.cu"
#if REF_PICK == 1
template __global__ void polarizer<CF32, CF32>(const ArrayTensor<Device::CUDA, CF32>,
                                               ArrayTensor<Device::CUDA, CF32>);
#else
template __global__ void polarizer<CF16, CF16>(const ArrayTensor<Device::CUDA, CF16>,
                                               ArrayTensor<Device::CUDA, CF16>);
#endif
#elif REF_PICK == 3
#include "src/modules/gather/gather.cu"
template __global__ void accumulate<CF32>(const ArrayTensor<Device::CUDA, CF32>, ArrayTensor<Device::CUDA, CF32>,
                                          const U64, const U64);
#elif REF_PICK == 4
#include "src/modules/permutation/permutation.cu"
template __global__ void permutation<CF32>(const ArrayTensor<Device::CUDA, CF32>, ArrayTensor<Device::CUDA, CF32>,
                                           ArrayShape);
#else
#error "REF_PICK must be 1..4"
#endif
