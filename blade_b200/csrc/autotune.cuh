// Launch-shape autotuner: a per-device cache of measured launch choices, keyed by
// kernel family and problem shape, which the launch paths consult.  The tuning
// entry points (blade_*_autotune) time every candidate on the caller's shape with
// CUDA events and store the fastest whose output is bit-identical to the default
// candidate's; blade_autotune_query reports what a launch of a shape will use.
#pragma once

#include <stdint.h>

#include <vector>

#include "common.cuh"

namespace bb {

constexpr int kTuneParams = 8;

// params[0..3]: the family's launch choice (see include/blade_b200.h);
// params[4]: candidates timed; params[5]: candidates whose output differed from
// the default candidate's (never chosen).
struct TuneEntry {
    uint32_t params[kTuneParams];
    float us;
};

// Looks up the tuned choice of (family, shape) on the current device.
bool tune_lookup(int family, const uint64_t (&shape)[8], TuneEntry* out);
void tune_store(int family, const uint64_t (&shape)[8], const TuneEntry& e);

// Per-family resolution of what a launch of `shape` uses now (tuned or default).
int tc_query(const uint64_t (&shape)[8], uint32_t* params, float* us, int* tuned);
int f32_query(const uint64_t (&shape)[8], uint32_t* params, float* us, int* tuned);
int spec_query(const uint64_t (&shape)[8], uint32_t* params, float* us, int* tuned);

// Output bytes a and b (device memory) are identical.
bool tune_same(const void* a, const void* b, size_t bytes);

// Fills n bytes with int8 values in [-127, 127] (deterministic hash of the index).
int tune_fill_ci8(void* p, uint64_t n, cudaStream_t s);
// Fills n complex64 values with unit-modulus phasors (deterministic).
int tune_fill_phasors(void* p, uint64_t n, cudaStream_t s);

// Times `launch` (warm-up, then `reps` launches between CUDA events on `s`) and
// returns the median launch time in microseconds (< 0 on a failed launch).
template <typename Fn>
float tune_time(Fn&& launch, cudaStream_t s, int reps = 5) {
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return -1.f;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return -1.f;
    }
    float result = -1.f;
    std::vector<float> t;
    if (launch() == BLADE_SUCCESS && launch() == BLADE_SUCCESS) {
        bool ok = true;
        for (int i = 0; i < reps && ok; i++) {
            cudaEventRecord(a, s);
            ok = launch() == BLADE_SUCCESS;
            cudaEventRecord(b, s);
            float ms = 0.f;
            ok = ok && cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess;
            t.push_back(ms * 1000.f);
        }
        if (ok) {
            for (size_t i = 1; i < t.size(); i++)
                for (size_t j = i; j > 0 && t[j] < t[j - 1]; j--) std::swap(t[j], t[j - 1]);
            result = t[t.size() / 2];
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return result;
}

}  // namespace bb
