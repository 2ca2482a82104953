// Module base of the C++ host layer (include/blade/module.hh:20-115 of the
// reference): taint, compute ratio, name and process(step, stream).  There is no
// run-time kernel compilation: every module calls an ahead-of-time sm_100a kernel
// through the C ABI of libblade_b200.so.
#ifndef BLADE_B200_MODULE_HH
#define BLADE_B200_MODULE_HH

#include <string>

#include "blade/memory.hh"

namespace Blade {

class Module {
   public:
    virtual ~Module() = default;
    virtual Taint getTaint() const { return Taint::NONE; }
    virtual U64 getComputeRatio() const { return 1; }
    virtual std::string name() const = 0;
    virtual Result process(const U64& currentStepCount, const Stream& stream = nullptr) = 0;
    // Selects the Runner slot whose output buffers the next process() writes.
    virtual void setSlot(U64) {}

   protected:
    template <Device D, typename T, typename S>
    static Result Link(Vector<D, T, S>& dst, const Vector<D, T, S>& src) {
        dst = src;
        return Result::SUCCESS;
    }
};

// A module output owned per Runner slot: the two slots of the Runner never share
// an intermediate buffer (the reference shares one, src/runner.cc:17-68).
template <typename V>
class SlotOutput {
   public:
    SlotOutput() = default;
    template <typename S>
    explicit SlotOutput(const S& shape) : _duet(shape) {}
    V& get() { return _duet.fixed(); }
    const V& get() const { return const_cast<Duet<V>&>(_duet).fixed(); }
    void set(U64 i) { _duet.set(i); }

   private:
    Duet<V> _duet;
};

}  // namespace Blade

#endif
