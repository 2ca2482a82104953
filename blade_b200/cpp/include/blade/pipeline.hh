// Pipeline and Runner of the C++ host layer.
//
// Pipeline mirrors include/blade/pipeline.hh:15-89 and src/pipeline.cc:7-141:
// two non-blocking streams, connect()/addModule() with CHRONOUS compute-ratio
// stepping, compute(index), synchronize(), isSynchronized(), willOutput().
// Runner mirrors include/blade/runner.hh:14-52 and src/runner.cc:7-68: the
// two-slot enqueue/dequeue queue and copy() into the head slot.
// Differences: every module output is per slot (setSlot), and with
// enableGraphs() the steady-state compute(index) of each slot is captured once
// into a CUDA graph and replayed.
#ifndef BLADE_B200_PIPELINE_HH
#define BLADE_B200_PIPELINE_HH

#include <functional>
#include <memory>
#include <queue>
#include <thread>
#include <tuple>
#include <vector>

#include "blade/bundles.hh"
#include "blade/modules.hh"

namespace Blade {

class Pipeline {
   public:
    Pipeline() {
        for (auto& s : _streams)
            Check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess ? BLADE_SUCCESS
                                                                                        : BLADE_CUDA_ERROR,
                  "Pipeline: cudaStreamCreate");
    }
    virtual ~Pipeline() {
        for (U64 i = 0; i < 2; i++) {
            cudaStreamSynchronize(_streams[i]);
            if (_execs[i]) cudaGraphExecDestroy(_execs[i]);
            cudaStreamDestroy(_streams[i]);
        }
    }
    Pipeline(const Pipeline&) = delete;
    Pipeline& operator=(const Pipeline&) = delete;

    bool computeComplete() const { return _step + 1 == _stepsPerCycle; }
    const U64& computeCurrentStepCount() const { return _step; }
    const U64& computeStepsPerCycle() const { return _stepsPerCycle; }
    const U64& computeLifetimeCycles() const { return _cycles; }
    const bool& commited() const { return _commited; }
    bool willOutput() const { return _stepsPerCycle == _step + 1; }
    const Stream& stream(U64 index = 0) const { return _streams[index]; }
    U64 numberOfStreams() const { return 2; }
    void enableGraphs(bool on = true) { _graphs = on; }

    template <typename Block>
    void connect(std::shared_ptr<Block>& module, const typename Block::Config& config,
                 const typename Block::Input& input) {
        if (_commited) throw Error(Result::ERROR, "Can't connect new module after Pipeline is commited.");
        module = std::make_shared<Block>(config, input, _streams[0]);
        if constexpr (std::is_base_of<Bundle, Block>::value) {
            for (auto& m : module->getModules()) addModule(m);  // a bundle runs as its modules, in order
        } else {
            addModule(module);
        }
    }

    void addModule(const std::shared_ptr<Module>& module) {
        if ((module->getTaint() & Taint::CHRONOUS) == Taint::CHRONOUS && module->getComputeRatio() > 1) {
            _stepsPerCycle *= module->getComputeRatio();
            _ratios.push_back(module->getComputeRatio());
        }
        _modules.push_back(module);
    }

    Result compute(const U64& index) {
        if (!_commited) {
            _ratios.push_back(1);
            _commited = true;
        }
        for (auto& m : _modules) m->setSlot(index);
        Result r;
        if (_graphs && _stepsPerCycle == 1 && _warm[index]) {
            if (!_execs[index]) {
                cudaGraph_t g = nullptr;
                if (cudaStreamBeginCapture(_streams[index], cudaStreamCaptureModeThreadLocal) != cudaSuccess)
                    return Result::CUDA_ERROR;
                r = runModules(index);
                if (cudaStreamEndCapture(_streams[index], &g) != cudaSuccess || r != Result::SUCCESS) {
                    if (g) cudaGraphDestroy(g);
                    return r != Result::SUCCESS ? r : Result::CUDA_ERROR;
                }
                const cudaError_t e = cudaGraphInstantiate(&_execs[index], g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return Result::CUDA_ERROR;
            }
            r = cudaGraphLaunch(_execs[index], _streams[index]) == cudaSuccess ? Result::SUCCESS : Result::CUDA_ERROR;
        } else {
            r = runModules(index);
            _warm[index] = true;
        }
        if (r != Result::SUCCESS) return r;
        if (cudaPeekAtLastError() != cudaSuccess) return Result::CUDA_ERROR;
        if (++_step == _stepsPerCycle) {
            _step = 0;
            _cycles += 1;
        }
        return Result::SUCCESS;
    }

    Result synchronize(const U64& index) {
        return cudaStreamSynchronize(_streams[index]) == cudaSuccess ? Result::SUCCESS : Result::CUDA_ERROR;
    }
    bool isSynchronized(const U64& index) { return cudaStreamQuery(_streams[index]) == cudaSuccess; }

   private:
    // src/pipeline.cc:89-141: modules after a ratio-R module run on its last sub-step.
    Result runModules(const U64& index) {
        U64 offset = 1, ratioIndex = 0;
        for (auto& m : _modules) {
            const U64 local = _step / offset % _ratios[ratioIndex];
            const Result r = m->process(local, _streams[index]);
            if (r != Result::SUCCESS) return r;
            if (m->getComputeRatio() > 1) {
                if (local == _ratios[ratioIndex] - 1) {
                    offset += local;
                    ratioIndex += 1;
                } else {
                    break;
                }
            }
        }
        return Result::SUCCESS;
    }

    Stream _streams[2] = {nullptr, nullptr};
    cudaGraphExec_t _execs[2] = {nullptr, nullptr};
    bool _warm[2] = {false, false};
    bool _graphs = false;
    bool _commited = false;
    std::vector<std::shared_ptr<Module>> _modules;
    U64 _step = 0, _stepsPerCycle = 1, _cycles = 0;
    std::vector<U64> _ratios;
};

class Runner : public Pipeline {
   public:
    using DequeueCallback = std::function<Result(const U64& inputId, const U64& outputId, const bool& didOutput)>;

    Result enqueue(const std::function<Result()>& inputCallback, const std::function<Result()>& outputCallback,
                   U64 inputId, U64 outputId) {
        if (_queue.size() == numberOfStreams()) {
            std::this_thread::yield();
            return Result::RUNNER_QUEUE_FULL;
        }
        const bool will = willOutput();
        Result r = inputCallback();
        if (r != Result::SUCCESS && !IsSoft(r)) return r;
        r = compute(_head);
        if (r != Result::SUCCESS && !IsSoft(r)) return r;
        if (will) {
            r = outputCallback();
            if (r != Result::SUCCESS && !IsSoft(r)) return r;
        }
        _queue.push({_head, inputId, outputId, will});
        _head = (_head + 1) % numberOfStreams();
        return Result::SUCCESS;
    }

    Result dequeue(const DequeueCallback& callback) {
        if (_queue.empty()) {
            std::this_thread::yield();
            return Result::RUNNER_QUEUE_EMPTY;
        }
        const auto [front, inId, outId, did] = _queue.front();
        if (_queue.size() < numberOfStreams()) {
            if (!isSynchronized(front)) return Result::RUNNER_QUEUE_NONE_AVAILABLE;
        } else if (synchronize(front) != Result::SUCCESS) {
            return Result::CUDA_ERROR;
        }
        _queue.pop();
        return callback(inId, outId, did);
    }

    template <typename DT, typename ST>
    Result copy(DT& dst, const ST& src) {
        return Copy(dst, src, stream(_head));
    }
    template <typename V, typename ST>
    Result copy(Duet<V>& dst, const ST& src) {
        return Copy(dst[_head], src, stream(_head));
    }
    U64 headIndex() const { return _head; }

   private:
    U64 _head = 0;
    std::queue<std::tuple<U64, U64, U64, bool>> _queue;
};

}  // namespace Blade

#endif
