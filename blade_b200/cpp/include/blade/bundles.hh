// Bundles of the C++ host layer: Bundle (include/blade/bundle.hh:12-45 of the
// reference), Bundles::ATA::ModeB (include/blade/bundles/ata/mode_b.hh:17-225) and
// Bundles::Generic::ModeH (include/blade/bundles/generic/mode_h.hh:13-130) with the
// reference's Config / Input / getOutputBuffer shapes.  A Pipeline that connects a
// bundle registers the bundle's modules in order (pipeline.hh:44-62), so a bundle
// steps and captures into CUDA graphs like hand-connected modules.
//
// Differences from the reference, each deliberate:
//  * ModeB takes the phasors [B, A, F*rate, 1, P] as input: the geometric delay
//    engine of Phasor::ATA (ERFA astrometry, src/modules/phasor/ata.cc:9-173) is
//    not part of this library (blade_phasor_from_delays turns delays into phasors).
//  * ModeB with the detector, rate 1, no circular conversion, no incoherent beam and
//    Stokes-I is one fused launch (Modules::BeamformDetect: tensor cores for CI8);
//    with CI8 at rate 2 or 4 (Stokes-I) it runs the
//    pre-beamformer stages into exact FP16 and the tensor-core chain on the fine
//    channels (Modules::ModeBTensorCore).
//  * ModeH at rate 65536 is one fused module (blade_spectrometer); other rates run
//    the module chain Cast -> Channelizer -> Polarizer -> Detector -> Cast.
#ifndef BLADE_B200_BUNDLES_HH
#define BLADE_B200_BUNDLES_HH

#include <memory>
#include <type_traits>
#include <vector>

#include "blade/modules.hh"

namespace Blade {

class Bundle {
   public:
    explicit Bundle(const Stream& stream) : stream(stream) {}
    virtual ~Bundle() = default;
    std::vector<std::shared_ptr<Module>>& getModules() { return modules; }

   protected:
    template <typename Block>
    void connect(std::shared_ptr<Block>& module, const typename Block::Config& config,
                 const typename Block::Input& input) {
        module = std::make_shared<Block>(config, input, stream);
        modules.push_back(module);
    }

   private:
    const Stream stream;
    std::vector<std::shared_ptr<Module>> modules;
};

namespace Modules {

// Fused ModeH chain (Cast -> Channelizer(65536) -> Polarizer -> Detector -> Cast) in
// blade_spectrometer, with its FP32 workspace.
template <typename IT, typename OT>
class Spectrometer : public Module {
   public:
    struct Config {
        BOOL convertToCircular = false;
        U64 integrationSize = 1;
        U64 numberOfOutputPolarizations = 1;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buf;
    };

    Spectrometer(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input), out(outShape(config, input)) {
        const auto& s = input.buf.shape();
        workspace = Vector<Device::CUDA, uint8_t, VectorShape>(
            VectorShape({blade_spectrometer_workspace_size(s[0], s[1], s[2], s[3], 65536)}));
    }
    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "Spectrometer"; }
    void setSlot(U64 i) override { out.set(i); }
    Result process(const U64&, const Stream& stream = nullptr) override {
        const auto& s = input.buf.shape();
        return FromABI(blade_spectrometer(TypeInfo<IT>::code, input.buf.data(), TypeInfo<OT>::code, out.get().data(),
                                          workspace.data(), s[0], s[1], s[2], s[3], 65536, config.integrationSize,
                                          config.numberOfOutputPolarizations, config.convertToCircular ? 1 : 0,
                                          stream));
    }

   private:
    static ArrayShape outShape(const Config& c, const Input& in) {
        const auto& s = in.buf.shape();
        if (s[3] != 2) throw Error(Result::ERROR, "The polarizer needs two polarizations.");
        if (s[2] % 65536 != 0) throw Error(Result::ERROR, "The number of time samples must be a multiple of 65536.");
        const U64 S = s[2] / 65536;
        if (c.integrationSize == 0 || S % c.integrationSize != 0)
            throw Error(Result::ERROR, "The number of spectra should be divisible by the integration size.");
        if (c.numberOfOutputPolarizations != 1 && c.numberOfOutputPolarizations != 4)
            throw Error(Result::ERROR, "Number of output polarizations not supported.");
        return ArrayShape({s[0], s[1] * 65536, S / c.integrationSize, c.numberOfOutputPolarizations});
    }
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, OT>> out;
    Vector<Device::CUDA, uint8_t, VectorShape> workspace;
};

// ModeB's pre-beamformer stages and beamformer + detector on tensor cores for CI8
// voltages at rate 2 or 4 (Stokes-I): blade_prechannelize_cf16 into an exact CF16
// buffer, then the per-fine-channel phasor split and the chain
// (blade_beamform_prepare_detect_tc_cf16), and with the incoherent beam its detected row
// (blade_incoherent_detect_cf16).
class ModeBTensorCore : public Module {
   public:
    struct Config {
        U64 rate = 4;
        BOOL convertToCircular = false;
        U64 integrationSize = 1;
        BOOL incoherentBeam = false;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, CI8>& buf;
        const PhasorTensor<Device::CUDA, CF32>& phasors;
    };

    static bool applies(const ArrayShape& s, U64 B, U64 rate, U64 integration) {
        return (rate == 2 || rate == 4) && s[3] == 2 && s[2] % rate == 0 &&
               blade_beamform_detect_tc_supported(B, s[0], s[1] * rate, s[2] / rate, 2, 1, integration) == 1;
    }

    ModeBTensorCore(const Config& config, const Input& input, const Stream& = nullptr)
        : config(config), input(input),
          pre(ArrayShape({input.buf.shape()[0], input.buf.shape()[1] * config.rate,
                          input.buf.shape()[2] / config.rate, 2})),
          plan(VectorShape({blade_beamform_tc_plan_size(input.phasors.shape()[0], input.buf.shape()[0],
                                                        input.buf.shape()[1] * config.rate, 2)})),
          out(ArrayShape({input.phasors.shape()[0] + (config.incoherentBeam ? 1 : 0), input.buf.shape()[1] * config.rate,
                          input.buf.shape()[2] / (config.rate * config.integrationSize), 1})) {}
    const ArrayTensor<Device::CUDA, F32>& getOutputBuffer() const { return out.get(); }
    Taint getTaint() const override { return Taint::CONSUMER | Taint::PRODUCER; }
    std::string name() const override { return "ModeBTensorCore"; }
    void setSlot(U64 i) override {
        pre.set(i);
        plan.set(i);
        out.set(i);
    }
    Result process(const U64&, const Stream& stream = nullptr) override {
        const auto& s = input.buf.shape();
        const U64 B = input.phasors.shape()[0], R = config.rate;
        int rc = blade_prechannelize_cf16(input.buf.data(), pre.get().data(), s[0], s[1], s[2], 2, R,
                                          config.convertToCircular ? 1 : 0, stream);
        if (!rc)
            rc = blade_beamform_prepare_detect_tc_cf16(input.phasors.data(), plan.get().data(), pre.get().data(),
                                                       out.get().data(), B, s[0], s[1] * R, s[2] / R, 2,
                                                       config.integrationSize, stream);
        if (!rc && config.incoherentBeam)  // beam row B
            rc = blade_incoherent_detect_cf16(pre.get().data(), input.phasors.data(),
                                              out.get().data() + B * s[1] * R * (s[2] / (R * config.integrationSize)),
                                              s[0], s[1] * R, s[2] / R, 2, config.integrationSize, stream);
        return FromABI(rc);
    }

   private:
    const Config config;
    const Input input;
    SlotOutput<ArrayTensor<Device::CUDA, CF16>> pre;
    SlotOutput<Vector<Device::CUDA, uint8_t, VectorShape>> plan;
    SlotOutput<ArrayTensor<Device::CUDA, F32>> out;
};

}  // namespace Modules

namespace Bundles {
namespace ATA {

template <typename IT, typename OT>
class ModeB : public Bundle {
    static_assert(std::is_same<OT, F32>::value || std::is_same<OT, CF32>::value,
                  "ModeB produces F32 (detector enabled) or CF32 beams");

   public:
    struct Config {
        ArrayShape inputShape;
        ArrayShape outputShape;
        U64 preBeamformerChannelizerRate = 1;
        BOOL preBeamformerPolarizerConvertToCircular = false;
        BOOL beamformerIncoherentBeam = false;
        BOOL detectorEnable = false;
        U64 detectorIntegrationSize = 1;
        U64 detectorNumberOfOutputPolarizations = 1;
        U64 castBlockSize = 512;
        U64 channelizerBlockSize = 512;
        U64 beamformerBlockSize = 512;
        U64 polarizerBlockSize = 512;
        U64 detectorBlockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buffer;
        const PhasorTensor<Device::CUDA, CF32>& phasors;
    };

    ModeB(const Config& config, const Input& input, const Stream& stream)
        : Bundle(stream), config(config), input(input) {
        if (input.buffer.shape() != config.inputShape)
            throw Error(Result::ERROR, "Expected input buffer size mismatch with actual size.");
        if ((std::is_same<OT, F32>::value) != config.detectorEnable)
            throw Error(Result::ERROR, "ModeB produces F32 with the detector enabled and CF32 without it.");
        const U64 R = config.preBeamformerChannelizerRate;
        const auto& s = input.buffer.shape();
        const auto& p = input.phasors.shape();
        if (p[1] != s[0] || p[2] != s[1] * R || p[4] != s[3])
            throw Error(Result::ERROR, "Phasor shape does not match the channelized voltages.");
        fused = config.detectorEnable && R == 1 && !config.preBeamformerPolarizerConvertToCircular &&
                !config.beamformerIncoherentBeam && config.detectorNumberOfOutputPolarizations == 1 && s[3] == 2;
        if constexpr (std::is_same<OT, F32>::value) {
            if (fused) {
                this->connect(beamformDetect, {.rate = 1, .integrationSize = config.detectorIntegrationSize},
                              {input.buffer, input.phasors});
                checkOutput(beamformDetect->getOutputBuffer().shape());
                return;
            }
            if constexpr (std::is_same<IT, CI8>::value) {
                if (config.detectorEnable && config.detectorNumberOfOutputPolarizations == 1 &&
                    Modules::ModeBTensorCore::applies(s, p[0], R, config.detectorIntegrationSize)) {
                    this->connect(tensorCore, {.rate = R,
                                               .convertToCircular = config.preBeamformerPolarizerConvertToCircular,
                                               .integrationSize = config.detectorIntegrationSize,
                                               .incoherentBeam = config.beamformerIncoherentBeam},
                                  {input.buffer, input.phasors});
                    checkOutput(tensorCore->getOutputBuffer().shape());
                    return;
                }
            }
        }
        const ArrayTensor<Device::CUDA, CF32>* x = nullptr;
        if constexpr (std::is_same<IT, CF32>::value) {
            x = &input.buffer;
        } else {
            this->connect(inputCast, {.blockSize = config.castBlockSize}, {input.buffer});
            x = &inputCast->getOutputBuffer();
        }
        if (R != 1) {
            this->connect(channelizer, {.rate = R, .blockSize = config.channelizerBlockSize}, {*x});
            x = &channelizer->getOutputBuffer();
        }
        if (config.preBeamformerPolarizerConvertToCircular) {
            this->connect(polarizer, {.inputPolarization = POL::XY, .outputPolarization = POL::LR,
                                      .blockSize = config.polarizerBlockSize},
                          {*x});
            x = &polarizer->getOutputBuffer();
        }
        this->connect(beamformer, {.enableIncoherentBeam = config.beamformerIncoherentBeam,
                                   .enableIncoherentBeamSqrt = config.detectorEnable,
                                   .blockSize = config.beamformerBlockSize},
                      {*x, input.phasors});
        if constexpr (std::is_same<OT, F32>::value) {
            this->connect(detector, {.integrationSize = config.detectorIntegrationSize,
                                     .numberOfOutputPolarizations = config.detectorNumberOfOutputPolarizations,
                                     .blockSize = config.detectorBlockSize},
                          {beamformer->getOutputBuffer()});
        }
        checkOutput(getOutputBuffer().shape());
    }

    const Config& getConfig() const { return config; }
    const ArrayTensor<Device::CUDA, IT>& getInputBuffer() const { return input.buffer; }
    bool isFused() const { return fused; }
    bool usesTensorCores() const { return tensorCore != nullptr; }

    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const {
        if constexpr (std::is_same<OT, F32>::value) {
            if (tensorCore) return tensorCore->getOutputBuffer();
            return fused ? beamformDetect->getOutputBuffer() : detector->getOutputBuffer();
        } else {
            return beamformer->getOutputBuffer();
        }
    }

   private:
    void checkOutput(const ArrayShape& shape) const {
        if (shape != config.outputShape)
            throw Error(Result::ERROR, "Expected output buffer size mismatch with actual size.");
    }

    const Config config;
    const Input input;
    bool fused = false;
    std::shared_ptr<Modules::Cast<IT, CF32>> inputCast;
    std::shared_ptr<Modules::Channelizer<CF32, CF32>> channelizer;
    std::shared_ptr<Modules::Polarizer<CF32, CF32>> polarizer;
    std::shared_ptr<Modules::Beamformer::ATA<CF32, CF32>> beamformer;
    std::shared_ptr<Modules::Detector<CF32, F32>> detector;
    std::shared_ptr<Modules::BeamformDetect<IT, F32>> beamformDetect;
    std::shared_ptr<Modules::ModeBTensorCore> tensorCore;
};

}  // namespace ATA

namespace Generic {

template <typename IT, typename OT>
class ModeH : public Bundle {
   public:
    struct Config {
        ArrayShape inputShape;
        ArrayShape outputShape;
        BOOL polarizerConvertToCircular = false;
        U64 detectorIntegrationSize = 1;
        U64 detectorNumberOfOutputPolarizations = 1;
        U64 castBlockSize = 512;
        U64 polarizerBlockSize = 512;
        U64 channelizerBlockSize = 512;
        U64 detectorBlockSize = 512;
    };
    struct Input {
        const ArrayTensor<Device::CUDA, IT>& buffer;
    };

    ModeH(const Config& config, const Input& input, const Stream& stream)
        : Bundle(stream), config(config), input(input) {
        if (input.buffer.shape() != config.inputShape)
            throw Error(Result::ERROR, "Expected input buffer size mismatch with actual size.");
        const auto& s = input.buffer.shape();
        // the reference's ModeH channelizes at rate = the number of time samples
        if (s[2] == 65536) {
            this->connect(spectrometer, {.convertToCircular = config.polarizerConvertToCircular,
                                         .integrationSize = config.detectorIntegrationSize,
                                         .numberOfOutputPolarizations = config.detectorNumberOfOutputPolarizations},
                          {input.buffer});
        } else {
            const ArrayTensor<Device::CUDA, CF32>* x = nullptr;
            if constexpr (std::is_same<IT, CF32>::value) {
                x = &input.buffer;
            } else {
                this->connect(inputCast, {.blockSize = config.castBlockSize}, {input.buffer});
                x = &inputCast->getOutputBuffer();
            }
            this->connect(channelizer, {.rate = s[2], .blockSize = config.channelizerBlockSize}, {*x});
            this->connect(polarizer, {.inputPolarization = POL::XY,
                                      .outputPolarization = config.polarizerConvertToCircular ? POL::LR : POL::XY,
                                      .blockSize = config.polarizerBlockSize},
                          {channelizer->getOutputBuffer()});
            this->connect(detector, {.integrationSize = config.detectorIntegrationSize,
                                     .numberOfOutputPolarizations = config.detectorNumberOfOutputPolarizations,
                                     .blockSize = config.detectorBlockSize},
                          {polarizer->getOutputBuffer()});
            if constexpr (!std::is_same<OT, F32>::value)
                this->connect(outputCast, {.blockSize = config.castBlockSize}, {detector->getOutputBuffer()});
        }
        if (getOutputBuffer().shape() != config.outputShape)
            throw Error(Result::ERROR, "Expected output buffer size mismatch with actual size.");
    }

    const Config& getConfig() const { return config; }
    const ArrayTensor<Device::CUDA, IT>& getInputBuffer() const { return input.buffer; }
    bool isFused() const { return spectrometer != nullptr; }

    const ArrayTensor<Device::CUDA, OT>& getOutputBuffer() const {
        if (spectrometer) return spectrometer->getOutputBuffer();
        if constexpr (std::is_same<OT, F32>::value) {
            return detector->getOutputBuffer();
        } else {
            return outputCast->getOutputBuffer();
        }
    }

   private:
    const Config config;
    const Input input;
    std::shared_ptr<Modules::Spectrometer<IT, OT>> spectrometer;
    std::shared_ptr<Modules::Cast<IT, CF32>> inputCast;
    std::shared_ptr<Modules::Channelizer<CF32, CF32>> channelizer;
    std::shared_ptr<Modules::Polarizer<CF32, CF32>> polarizer;
    std::shared_ptr<Modules::Detector<CF32, F32>> detector;
    std::shared_ptr<Modules::Cast<F32, OT>> outputCast;
};

}  // namespace Generic
}  // namespace Bundles
}  // namespace Blade

#endif
