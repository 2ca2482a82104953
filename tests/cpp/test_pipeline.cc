// C++ drop-in check: BLADE-style Runner + Modules (blade/base.hh over the C ABI).
//
// Builds the reference's ModeB-order chain module by module
//   Cast<CI8,CF32> -> Beamformer::ATA<CF32,CF32> -> Channelizer(rate 4) -> Detector(I=4, Stokes-I)
// and the fused BeamformDetect<CI8,F32> on the same input, streams several blocks
// through both Runners with enqueue/dequeue (CUDA graphs on), and checks that the
// two Stokes-I outputs agree to 1e-5 relative L2 for every block.
// Usage: test_pipeline [--no-graphs]   (exit code 0 = pass)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "blade/base.hh"

using namespace Blade;

static uint32_t lcg(uint32_t& x) { return x = 1664525u * x + 1013904223u; }

int main(int argc, char** argv) {
    const bool graphs = !(argc > 1 && std::strcmp(argv[1], "--no-graphs") == 0);
    const U64 A = 28, F = 8, T = 2048, P = 2, B = 16, R = 4, I = 4, NBLK = 5;

    Runner chain, fused;
    chain.enableGraphs(graphs);
    fused.enableGraphs(graphs);

    Duet<ArrayTensor<Device::CUDA, CI8>> in(ArrayShape({A, F, T, P}));
    Duet<PhasorTensor<Device::CUDA, CF32>> ph(PhasorShape({B, A, F, 1, P}));

    std::shared_ptr<Modules::Cast<CI8, CF32>> cast;
    std::shared_ptr<Modules::Beamformer::ATA<CF32, CF32>> bf;
    std::shared_ptr<Modules::Channelizer<CF32, CF32>> ch;
    std::shared_ptr<Modules::Detector<CF32, F32>> det;
    std::shared_ptr<Modules::BeamformDetect<CI8, F32>> bd;
    try {
        chain.connect(cast, {}, {in.fixed()});
        chain.connect(bf, {}, {cast->getOutputBuffer(), ph.fixed()});
        chain.connect(ch, {.rate = R}, {bf->getOutputBuffer()});
        chain.connect(det, {.integrationSize = I, .numberOfOutputPolarizations = 1}, {ch->getOutputBuffer()});
        fused.connect(bd, {.rate = R, .integrationSize = I, .tensorCores = true}, {in.fixed(), ph.fixed()});
    } catch (const Error& e) {
        std::fprintf(stderr, "construction failed: %s\n", e.what());
        return 2;
    }
    if (!bd->usesTensorCores()) {
        std::fprintf(stderr, "expected the tensor-core path\n");
        return 3;
    }

    // Pinned host blocks.
    std::vector<ArrayTensor<Device::CPU, CI8>> hin;
    std::vector<PhasorTensor<Device::CPU, CF32>> hph;
    std::vector<ArrayTensor<Device::CPU, F32>> hout1, hout2;
    uint32_t seed = 12345;
    for (U64 k = 0; k < NBLK; k++) {
        hin.emplace_back(ArrayShape({A, F, T, P}));
        hph.emplace_back(PhasorShape({B, A, F, 1, P}));
        hout1.emplace_back(ArrayShape({B, F * R, T / (R * I), 1}));
        hout2.emplace_back(ArrayShape({B, F * R, T / (R * I), 1}));
        for (U64 i = 0; i < hin[k].size(); i++) {
            hin[k][i].re = (int8_t)((lcg(seed) >> 24) - 128);
            hin[k][i].im = (int8_t)((lcg(seed) >> 24) - 128);
        }
        for (U64 i = 0; i < hph[k].size(); i++) {
            const double phase = 2.0 * M_PI * (lcg(seed) / 4294967296.0);
            hph[k][i] = CF32((float)std::cos(phase), (float)std::sin(phase));
        }
    }

    // Both runners, several blocks each, two slots in flight.
    Duet<ArrayTensor<Device::CUDA, F32>> out1(ArrayShape({B, F * R, T / (R * I), 1}));
    Duet<ArrayTensor<Device::CUDA, F32>> out2(ArrayShape({B, F * R, T / (R * I), 1}));
    auto drive = [&](Runner& r, Duet<ArrayTensor<Device::CUDA, F32>>& out, const ArrayTensor<Device::CUDA, F32>& src,
                     std::vector<ArrayTensor<Device::CPU, F32>>& host) -> bool {
        U64 k = 0, done = 0;
        while (done < NBLK) {
            if (k < NBLK) {
                const U64 j = k;
                const Result e = r.enqueue(
                    [&] {
                        if (r.copy(in, hin[j]) != Result::SUCCESS) return Result::ERROR;
                        return r.copy(ph, hph[j]);
                    },
                    [&] {
                        if (r.copy(out, src) != Result::SUCCESS) return Result::ERROR;
                        return Copy(host[j], out[r.headIndex()], r.stream(r.headIndex()));
                    },
                    j, j);
                if (e == Result::SUCCESS) {
                    k++;
                    continue;
                }
                if (!IsSoft(e)) return false;
            }
            const Result d = r.dequeue([&](const U64&, const U64&, const bool&) {
                done++;
                return Result::SUCCESS;
            });
            if (d != Result::SUCCESS && !IsSoft(d)) return false;
        }
        return true;
    };
    if (!drive(chain, out1, det->getOutputBuffer(), hout1) || !drive(fused, out2, bd->getOutputBuffer(), hout2)) {
        std::fprintf(stderr, "runner failed: %s\n", blade_last_error());
        return 4;
    }
    cudaDeviceSynchronize();

    double worst = 0;
    for (U64 k = 0; k < NBLK; k++) {
        double num = 0, den = 0;
        for (U64 i = 0; i < hout1[k].size(); i++) {
            const double a = hout1[k][i], b = hout2[k][i];
            num += (a - b) * (a - b);
            den += a * a;
        }
        const double rel = std::sqrt(num / (den > 0 ? den : 1));
        if (rel > worst) worst = rel;
    }
    std::printf("{\"blocks\": %llu, \"graphs\": %s, \"max_rel_l2_chain_vs_fused\": %.3e}\n",
                (unsigned long long)NBLK, graphs ? "true" : "false", worst);
    return worst < 1e-5 ? 0 : 1;
}
