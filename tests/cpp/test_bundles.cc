// C++ bundles: Bundles::ATA::ModeB and Bundles::Generic::ModeH (and the
// Beamformer::MeerKAT module) connected to a Pipeline like the reference's C++
// examples (examples/pipeline-cpp), one block each.  Writes every case's inputs and outputs as raw little-endian arrays into
// the directory given as argv[1] (<case>_in.bin, <case>_ph.bin, <case>_out.bin)
// and prints one JSON line per case; tests/test_cpp.py compares the outputs with
// the FP64 oracle.
// Usage: test_bundles <out-dir>   (exit code 0 = every case ran)
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "blade/base.hh"

using namespace Blade;

static uint32_t lcg(uint32_t& x) { return x = 1664525u * x + 1013904223u; }

template <typename T, typename S>
static bool dump(const std::string& path, const Vector<Device::CUDA, T, S>& dev) {
    std::vector<T> h(dev.size());
    if (cudaMemcpy(h.data(), dev.data(), dev.size_bytes(), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(h.data(), sizeof(T), h.size(), f) == h.size();
    std::fclose(f);
    return ok;
}

template <typename T>
static void fill(Vector<Device::CUDA, T, ArrayShape>& dev, uint32_t seed) {
    std::vector<T> h(dev.size());
    for (auto& v : h) {
        const float re = (float)(int8_t)((lcg(seed) >> 24) & 0x7F) - 64.f, im = (float)(int8_t)((lcg(seed) >> 24) & 0x7F) - 64.f;
        if constexpr (std::is_same<T, CI8>::value) {
            v.re = (int8_t)re;
            v.im = (int8_t)im;
        } else {
            v = T(re / 16.f, im / 16.f);
        }
    }
    cudaMemcpy(dev.data(), h.data(), dev.size_bytes(), cudaMemcpyHostToDevice);
}

static void phasors(PhasorTensor<Device::CUDA, CF32>& dev, uint32_t seed) {
    std::vector<CF32> h(dev.size());
    for (U64 i = 0; i < h.size(); i += 2) {  // both polarisations share a phase
        const double ph = 2.0 * M_PI * (lcg(seed) / 4294967296.0);
        h[i] = h[i + 1] = CF32((float)std::cos(ph), (float)std::sin(ph));
    }
    cudaMemcpy(dev.data(), h.data(), dev.size_bytes(), cudaMemcpyHostToDevice);
}

template <typename Block, typename Out>
static bool run(Pipeline& p, const std::string& dir, const std::string& name, const Out& out, bool fused,
                bool tc = false) {
    if (p.compute(0) != Result::SUCCESS || p.synchronize(0) != Result::SUCCESS) {
        std::fprintf(stderr, "%s: compute failed: %s\n", name.c_str(), blade_last_error());
        return false;
    }
    if (!dump(dir + "/" + name + "_out.bin", out)) return false;
    std::printf("{\"case\": \"%s\", \"fused\": %s, \"tc\": %s}\n", name.c_str(), fused ? "true" : "false",
                tc ? "true" : "false");
    return true;
}

template <typename IT, typename OT>
static bool mode_b(const std::string& dir, const std::string& name, U64 A, U64 F, U64 T, U64 B, U64 R, bool circ,
                   bool inc, bool det, U64 I, U64 OP, uint32_t seed) {
    using Bundle = Bundles::ATA::ModeB<IT, OT>;
    ArrayTensor<Device::CUDA, IT> in(ArrayShape({A, F, T, 2}));
    PhasorTensor<Device::CUDA, CF32> ph(PhasorShape({B, A, F * R, 1, 2}));
    fill(in, seed);
    phasors(ph, seed + 1);
    const U64 nb = B + (inc ? 1 : 0);
    const ArrayShape out = det ? ArrayShape({nb, F * R, T / (R * I), OP}) : ArrayShape({nb, F * R, T / R, 2});
    Pipeline p;
    std::shared_ptr<Bundle> b;
    try {
        p.connect(b,
                  {.inputShape = ArrayShape({A, F, T, 2}), .outputShape = out, .preBeamformerChannelizerRate = R,
                   .preBeamformerPolarizerConvertToCircular = circ, .beamformerIncoherentBeam = inc,
                   .detectorEnable = det, .detectorIntegrationSize = I, .detectorNumberOfOutputPolarizations = OP},
                  {in, ph});
    } catch (const Error& e) {
        std::fprintf(stderr, "%s: construction failed: %s\n", name.c_str(), e.what());
        return false;
    }
    if (!dump(dir + "/" + name + "_in.bin", in) || !dump(dir + "/" + name + "_ph.bin", ph)) return false;
    return run<Bundle>(p, dir, name, b->getOutputBuffer(), b->isFused(), b->usesTensorCores());
}

template <typename IT, typename OT>
static bool mode_h(const std::string& dir, const std::string& name, U64 A, U64 F, U64 T, bool circ, U64 I, U64 OP,
                   uint32_t seed) {
    using Bundle = Bundles::Generic::ModeH<IT, OT>;
    ArrayTensor<Device::CUDA, IT> in(ArrayShape({A, F, T, 2}));
    fill(in, seed);
    Pipeline p;
    std::shared_ptr<Bundle> b;
    try {
        p.connect(b,
                  {.inputShape = ArrayShape({A, F, T, 2}), .outputShape = ArrayShape({A, F * T, 1 / I, OP}),
                   .polarizerConvertToCircular = circ, .detectorIntegrationSize = I,
                   .detectorNumberOfOutputPolarizations = OP},
                  {in});
    } catch (const Error& e) {
        std::fprintf(stderr, "%s: construction failed: %s\n", name.c_str(), e.what());
        return false;
    }
    if (!dump(dir + "/" + name + "_in.bin", in)) return false;
    return run<Bundle>(p, dir, name, b->getOutputBuffer(), b->isFused());
}

static bool meerkat(const std::string& dir, uint32_t seed) {
    const U64 A = 6, F = 3, T = 128, B = 4;
    ArrayTensor<Device::CUDA, CF32> in(ArrayShape({A, F, T, 2}));
    PhasorTensor<Device::CUDA, CF32> ph(PhasorShape({B, A, F, 1, 2}));
    fill(in, seed);
    phasors(ph, seed + 1);
    Pipeline p;
    std::shared_ptr<Modules::Beamformer::MeerKAT<CF32, CF32>> bf;
    try {
        p.connect(bf, {.enableIncoherentBeam = true}, {in, ph});
    } catch (const Error& e) {
        std::fprintf(stderr, "meerkat: construction failed: %s\n", e.what());
        return false;
    }
    if (!dump(dir + "/meerkat_in.bin", in) || !dump(dir + "/meerkat_ph.bin", ph)) return false;
    return run<void>(p, dir, "meerkat", bf->getOutputBuffer(), false);
}

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: test_bundles <out-dir>\n");
        return 2;
    }
    const std::string dir = argv[1];
    bool ok = true;
    ok &= mode_b<CI8, F32>(dir, "modeb_ci8_r4", 12, 4, 512, 3, 4, true, true, true, 2, 1, 11);
    ok &= mode_b<CF32, F32>(dir, "modeb_cf32_r1", 20, 8, 512, 2, 1, false, false, true, 4, 1, 12);
    ok &= mode_b<CI8, CF32>(dir, "modeb_ci8_beams", 8, 4, 256, 2, 2, false, true, false, 1, 1, 13);
    ok &= mode_b<CI8, F32>(dir, "modeb_ci8_r4_tc", 12, 4, 1024, 3, 4, true, false, true, 2, 1, 17);
    ok &= mode_h<CI8, F32>(dir, "modeh_ci8_65536", 1, 2, 65536, true, 1, 4, 14);
    ok &= mode_h<CF32, F32>(dir, "modeh_cf32_1024", 2, 3, 1024, false, 1, 1, 15);
    ok &= meerkat(dir, 16);
    return ok ? 0 : 1;
}
