// Core types of the C++ host layer: element types, Result, Taint, POL, Device.
//
// Mirrors include/blade/macros.hh:11-48 (Taint, Result with the soft-error bit 4),
// include/blade/types.hh:14-49 (POL) and include/blade/memory/types.hh (element
// types) of the reference, so module code written against Blade:: compiles
// unchanged against this layer.
#ifndef BLADE_B200_TYPES_HH
#define BLADE_B200_TYPES_HH

#include <cuda_runtime.h>
#include <stdint.h>

#include <complex>
#include <stdexcept>
#include <string>

#include "blade_b200.h"

namespace Blade {

using U64 = uint64_t;
using I64 = int64_t;
using I32 = int32_t;
using I8 = int8_t;
using F32 = float;
using F64 = double;
using BOOL = bool;

struct F16 {
    uint16_t bits;
};
struct CI8 {
    int8_t re, im;
};
struct CF16 {
    uint16_t re, im;
};
using CF32 = std::complex<float>;
using CF64 = std::complex<double>;

// A CUDA stream handle (the reference wraps cudaStream_t the same way).
using Stream = cudaStream_t;

enum class Device : uint8_t { CPU, CUDA };

enum class Taint : uint8_t {
    NONE = 0 << 0,
    CONSUMER = 1 << 0,
    PRODUCER = 1 << 1,
    MODIFIER = 1 << 2,
    CHRONOUS = 1 << 3,
};

inline constexpr Taint operator|(Taint a, Taint b) { return static_cast<Taint>(uint8_t(a) | uint8_t(b)); }
inline constexpr Taint operator&(Taint a, Taint b) { return static_cast<Taint>(uint8_t(a) & uint8_t(b)); }

enum class Result : uint8_t {
    SUCCESS = 0,
    ERROR = 1,
    CUDA_ERROR,
    ASSERTION_ERROR,
    RUNNER_QUEUE_FULL = 0 | (1 << 4),
    RUNNER_QUEUE_EMPTY = 1 | (1 << 4),
    RUNNER_QUEUE_NONE_AVAILABLE = 2 | (1 << 4),
    PIPELINE_EXHAUSTED = 3 | (1 << 4),
};

inline constexpr bool IsSoft(Result r) { return (uint8_t(r) & (1 << 4)) != 0; }

enum class POL : uint8_t { X, Y, L, R, XY, LR };

// C-ABI status -> Result (the codes are the same numbers).
inline Result FromABI(int rc) { return static_cast<Result>(rc); }

// Constructor checks throw like BL_CHECK_THROW (include/blade/macros.hh:125-135).
struct Error : std::runtime_error {
    Result result;
    Error(Result r, const std::string& what) : std::runtime_error(what), result(r) {}
};

inline void Check(int rc, const char* what) {
    if (rc != BLADE_SUCCESS) throw Error(FromABI(rc), std::string(what) + ": " + blade_last_error());
}

template <typename T> struct TypeInfo;
template <> struct TypeInfo<I8> { static constexpr int code = BLADE_I8; static constexpr bool complex = false; static constexpr const char* name = "I8"; };
template <> struct TypeInfo<I32> { static constexpr int code = BLADE_I32; static constexpr bool complex = false; static constexpr const char* name = "I32"; };
template <> struct TypeInfo<F16> { static constexpr int code = BLADE_F16; static constexpr bool complex = false; static constexpr const char* name = "F16"; };
template <> struct TypeInfo<F32> { static constexpr int code = BLADE_F32; static constexpr bool complex = false; static constexpr const char* name = "F32"; };
template <> struct TypeInfo<F64> { static constexpr int code = BLADE_F64; static constexpr bool complex = false; static constexpr const char* name = "F64"; };
template <> struct TypeInfo<CI8> { static constexpr int code = BLADE_CI8; static constexpr bool complex = true; static constexpr const char* name = "CI8"; };
template <> struct TypeInfo<CF16> { static constexpr int code = BLADE_CF16; static constexpr bool complex = true; static constexpr const char* name = "CF16"; };
template <> struct TypeInfo<CF32> { static constexpr int code = BLADE_CF32; static constexpr bool complex = true; static constexpr const char* name = "CF32"; };
template <> struct TypeInfo<CF64> { static constexpr int code = BLADE_CF64; static constexpr bool complex = true; static constexpr const char* name = "CF64"; };

}  // namespace Blade

#endif
