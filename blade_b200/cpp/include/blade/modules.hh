// Modules of the beamform -> channelize -> detect path for C++ callers, with the
// reference's class names, Config / Input structs, constructor checks and
// process() signature (include/blade/modules/*.hh of the reference).  Each
// process() is one C-ABI call into libblade_b200.so on the given stream.
#ifndef BLADE_B200_MODULES_HH
#define BLADE_B200_MODULES_HH

#include <string>
#include <type_traits>
#include <vector>

#include "blade/module.hh"

namespace Blade::Modules {

// ---------------------------------------------------------------- Cast
// include/blade/modules/cast.hh:9-70, src/modules/cast/base.cc:12-66
template <typename IT, typename OT>
class Cast : public Module {
   public:
    struct Config {
        U64 blockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Cast(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(input.buf.shape()) {
        if (TypeInfo<IT>::complex != TypeInfo<OT>::complex)
            throw Error(Result::ERROR, "Cannot cast between complex and non-complex types.");
    }
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "Cast"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        return FromABI(blade_cast(TypeInfo<IT>::code, TypeInfo<OT>::code, input.buf.data(), out.get().data(),
                                  input.buf.size(), stream));
    }

   private:
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
};

// ---------------------------------------------------------------- Beamformer::ATA
namespace Beamformer {
// include/blade/modules/beamformer/{generic,ata}.hh, src/modules/beamformer/ata.cc:7-74
template <typename IT, typename OT>
class ATA : public Module {
   public:
    struct Config {
        BOOL enableIncoherentBeam = false;
        BOOL enableIncoherentBeamSqrt = false;
        U64 blockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
        const PhasorTensor<Device::CUDA, IT>& phasors;
    };

    ATA(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {}

    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "Beamformer"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        const auto& s = input.buf.shape();
        return FromABI(blade_beamform_f32(input.buf.data(), input.phasors.data(), out.get().data(),
                                          input.phasors.shape().numberOfBeams(), s.numberOfAspects(),
                                          s.numberOfFrequencyChannels(), s.numberOfTimeSamples(),
                                          s.numberOfPolarizations(), config.enableIncoherentBeam,
                                          config.enableIncoherentBeamSqrt, stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        const auto& s = in.buf.shape();
        const auto& p = in.phasors.shape();
        if (p.numberOfFrequencyChannels() != s.numberOfFrequencyChannels())
            throw Error(Result::ERROR, "Number of frequency channels mismatch between phasors and buffer.");
        if (p.numberOfPolarizations() != s.numberOfPolarizations())
            throw Error(Result::ERROR, "Number of polarizations mismatch between phasors and buffer.");
        if (p.numberOfAntennas() != s.numberOfAspects())
            throw Error(Result::ERROR, "Number of antennas mismatch between phasors and buffer.");
        return ArrayShape({p.numberOfBeams() + (c.enableIncoherentBeam ? 1 : 0), s.numberOfFrequencyChannels(),
                           s.numberOfTimeSamples(), s.numberOfPolarizations()});
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
};

// include/blade/modules/beamformer/meerkat.hh, src/modules/beamformer/meerkat.cc:8-39:
// one weight per (beam, antenna), the first B*A values of the phasor tensor, for
// every channel and polarisation; the incoherent beam is sized but zero (the
// reference kernel never writes it).
template <typename IT, typename OT>
class MeerKAT : public Module {
   public:
    using Config = typename ATA<IT, OT>::Config;
    using Input = typename ATA<IT, OT>::Input;

    MeerKAT(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {}

    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "Beamformer"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        const auto& s = input.buf.shape();
        return FromABI(blade_beamform_meerkat_f32(input.buf.data(), input.phasors.data(), out.get().data(),
                                                  input.phasors.shape().numberOfBeams(), s.numberOfAspects(),
                                                  s.numberOfFrequencyChannels(), s.numberOfTimeSamples(),
                                                  s.numberOfPolarizations(), config.enableIncoherentBeam, stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        const auto& s = in.buf.shape();
        return ArrayShape({in.phasors.shape().numberOfBeams() + (c.enableIncoherentBeam ? 1 : 0),
                           s.numberOfFrequencyChannels(), s.numberOfTimeSamples(), s.numberOfPolarizations()});
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
};
}  // namespace Beamformer

// ---------------------------------------------------------------- Channelizer
// include/blade/modules/channelizer/base.hh:12-87, src/modules/channelizer/base.cc:9-146;
// any even rate dividing T (the reference accepts only rate == T or 1).
template <typename IT, typename OT>
class Channelizer : public Module {
   public:
    struct Config {
        U64 rate = 4;
        U64 blockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Channelizer(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {
        const auto& s = input.buf.shape();
        const U64 ws = blade_channelize_workspace_size(s[0], s[1], s[2], s[3], config.rate);
        if (ws) workspace = Vector<Device::CUDA, uint8_t, VectorShape>(VectorShape({ws}));
    }
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::MODIFIER; }
    std::string name() const override { return "Channelizer"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        const auto& s = input.buf.shape();
        return FromABI(blade_channelize(input.buf.data(), out.get().data(),
                                        workspace.empty() ? nullptr : workspace.data(), s[0], s[1], s[2], s[3],
                                        config.rate, stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        const auto& s = in.buf.shape();
        if (c.rate == 0 || s[2] % c.rate != 0)
            throw Error(Result::ERROR, "The number of time samples should be divisable by the channelizer rate.");
        if (c.rate % 2 != 0 && c.rate != 1) throw Error(Result::ERROR, "The channelizer rate should be divisable by 2.");
        if (s[3] != 1 && s[3] != 2) throw Error(Result::ERROR, "Number of polarizations should be one or two.");
        return ArrayShape({s[0], s[1] * c.rate, s[2] / c.rate, s[3]});
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
    Vector<Device::CUDA, uint8_t, VectorShape> workspace;
};

// ---------------------------------------------------------------- Polarizer (in place)
// include/blade/modules/polarizer.hh:9-71, src/modules/polarizer/base.cc:12-68
template <typename IT, typename OT>
class Polarizer : public Module {
    static_assert(std::is_same<IT, OT>::value, "Polarizer requires the same input and output type");

   public:
    struct Config {
        POL inputPolarization = POL::XY;
        POL outputPolarization = POL::LR;
        U64 blockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Polarizer(const Config& config, const Input& input, const Stream& = nullptr) : config(config), input(input) {
        if (input.buf.shape()[3] != 2) throw Error(Result::ERROR, "Polarizer needs two polarizations.");
    }
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return input.buf; }
    Taint getTaint() const override { return Taint::MODIFIER; }
    std::string name() const override { return "Polarizer"; }
    Result process(const U64&, const Stream& stream = nullptr) override {
        if (config.inputPolarization == config.outputPolarization) return Result::SUCCESS;
        const auto& s = input.buf.shape();
        return FromABI(blade_polarize(TypeInfo<IT>::code, input.buf.data(), input.buf.data(), s[0] * s[1] * s[2],
                                      stream));
    }

   private:
    const Config config;
    const Input input;
};

// ---------------------------------------------------------------- Detector
// include/blade/modules/detector.hh:12-81, src/modules/detector/base.cc:9-85
template <typename IT, typename OT>
class Detector : public Module {
   public:
    struct Config {
        U64 integrationSize;
        U64 numberOfOutputPolarizations = 4;
        U64 blockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Detector(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {}
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "Detector"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        const auto& s = input.buf.shape();
        return FromABI(blade_detect(input.buf.data(), out.get().data(), s[0], s[1], s[2], s[3], config.integrationSize,
                                    config.numberOfOutputPolarizations, stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        const auto& s = in.buf.shape();
        if (c.integrationSize == 0) throw Error(Result::ERROR, "Integration size should be more than zero.");
        if (s[2] % c.integrationSize != 0)
            throw Error(Result::ERROR, "The number of time samples should be divisable by the integration size.");
        if (s[3] != 2) throw Error(Result::ERROR, "Number of polarizations should be two (2).");
        if (c.numberOfOutputPolarizations != 1 && c.numberOfOutputPolarizations != 4)
            throw Error(Result::ERROR, "Number of output polarizations not supported.");
        return ArrayShape({s[0], s[1], s[2] / c.integrationSize, c.numberOfOutputPolarizations});
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
};

// ---------------------------------------------------------------- Gather (CHRONOUS)
// include/blade/modules/gather.hh:12-95, src/modules/gather/base.cc:12-111
template <typename IT, typename OT>
class Gather : public Module {
    static_assert(std::is_same<IT, OT>::value, "Casting isn't supported by Gather");

   public:
    struct Config {
        U64 axis = 0;
        U64 multiplier = 1;
        U64 copySizeThreshold = 512;
        U64 blockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Gather(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {}
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER | Taint::CHRONOUS; }
    U64 getComputeRatio() const override { return config.multiplier; }
    std::string name() const override { return "Gather"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64& step, const Stream& stream = nullptr) override {
        return FromABI(blade_gather(sizeof(IT), input.buf.data(), out.get().data(), input.buf.shape().data(),
                                    config.axis, config.multiplier, step, stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        if (c.axis >= 4) throw Error(Result::ERROR, "Selected input axis is larger than input shape dimensions.");
        if (c.multiplier == 0) throw Error(Result::ERROR, "Multiplier should be more than zero.");
        ArrayShape s = in.buf.shape();
        s[c.axis] *= c.multiplier;
        return s;
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
};

// ---------------------------------------------------------------- Permutation
// include/blade/modules/permutation.hh:11-78, src/modules/permutation/base.cc:12-73
template <typename IT, typename OT>
class Permutation : public Module {
    static_assert(std::is_same<IT, OT>::value, "Casting isn't supported by Permutation");

   public:
    struct Config {
        ArrayShape indexes;
        U64 blockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Permutation(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {}
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "Permutation"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        return FromABI(blade_permute(sizeof(IT), input.buf.data(), out.get().data(), input.buf.shape().data(),
                                     config.indexes.data(), stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        bool seen[4] = {false, false, false, false};
        ArrayShape s;
        for (U64 i = 0; i < 4; i++) {
            if (c.indexes[i] >= 4 || seen[c.indexes[i]]) throw Error(Result::ERROR, "Repeated index in permutation.");
            seen[c.indexes[i]] = true;
            s[i] = in.buf.shape()[c.indexes[i]];
        }
        return s;
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
};

// ---------------------------------------------------------------- Duplicate
// include/blade/modules/duplicate.hh:11-64, src/modules/duplicate/base.cc:12-37
template <typename IT, typename OT>
class Duplicate : public Module {
    static_assert(std::is_same<IT, OT>::value, "Casting isn't supported by Duplicate");

   public:
    struct Config {};
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Duplicate(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(input.buf.shape()) {}
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "Duplicate"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        return FromABI(blade_duplicate(input.buf.data(), out.get().data(), input.buf.size_bytes(), stream));
    }

   private:
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
};

// ---------------------------------------------------------------- BeamformDetect (fused chain)
// Beamformer -> Channelizer -> Detector of include/blade/bundles/ata/mode_b.hh:99-199
// in one launch: tensor cores (CI8 input) when the shape allows, else FP32 cores.
template <typename IT, typename OT>
class BeamformDetect : public Module {
   public:
    struct Config {
        U64 rate = 1;
        U64 integrationSize = 1;
        bool tensorCores = true;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
        const PhasorTensor<Device::CUDA, CF32>& phasors;
    };

    BeamformDetect(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {
        const auto& s = input.buf.shape();
        const U64 B = input.phasors.shape()[0];
        tc = config.tensorCores && TypeInfo<IT>::code == BLADE_CI8 &&
             blade_beamform_detect_tc_supported(B, s[0], s[1], s[2], s[3], config.rate, config.integrationSize);
        if (tc) plan = Vector<Device::CUDA, uint8_t, VectorShape>(
                    VectorShape({blade_beamform_tc_plan_size(B, s[0], s[1], s[3])}));
    }
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    bool usesTensorCores() const { return tc; }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "BeamformDetect"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        const auto& s = input.buf.shape();
        const U64 B = input.phasors.shape()[0];
        if (tc) {
            return FromABI(blade_beamform_prepare_detect_tc(input.phasors.data(), plan.data(), input.buf.data(),
                                                            out.get().data(), B, s[0], s[1], s[2], s[3], config.rate,
                                                            config.integrationSize, stream));
        }
        return FromABI(blade_beamform_detect_f32(TypeInfo<IT>::code, input.buf.data(), input.phasors.data(),
                                                 out.get().data(), B, s[0], s[1], s[2], s[3], config.rate,
                                                 config.integrationSize, stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        const auto& s = in.buf.shape();
        if (c.rate == 0 || c.integrationSize == 0 || s[2] % (c.rate * c.integrationSize) != 0)
            throw Error(Result::ERROR, "T must be a multiple of rate x integration.");
        return ArrayShape({in.phasors.shape()[0], s[1] * c.rate, s[2] / (c.rate * c.integrationSize), 1});
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
    Vector<Device::CUDA, uint8_t, VectorShape> plan;
    bool tc = false;
};

}  // namespace Blade::Modules

#endif
