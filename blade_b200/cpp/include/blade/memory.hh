// Memory of the C++ host layer: named shapes, ref-counted device/host vectors,
// the two-slot Duet and Copy.
//
// Mirrors include/blade/memory/shape.hh:10-108 (row-major Shape<N>),
// custom.hh:10-163 (ArrayShape [A,F,T,P], PhasorShape [B,A,F,T,P], DelayShape
// [B,A], VectorShape), vector.hh:15-278 (ref-counted Vector<Device, T, Shape>),
// helper.hh:13-49 (Duet: operator[] re-points the fixed slot) and copy.hh:11-33
// (Copy with shape checks) of the reference.
#ifndef BLADE_B200_MEMORY_HH
#define BLADE_B200_MEMORY_HH

#include <array>
#include <memory>

#include "blade/types.hh"

namespace Blade {

template <U64 N>
struct Shape {
    using Type = std::array<U64, N>;

    Shape() { _shape.fill(0); }
    Shape(const Type& s) : _shape(s) {}

    U64 size() const {
        U64 n = 1;
        for (auto d : _shape) n *= d;
        return n;
    }
    static constexpr U64 dimensions() { return N; }
    const U64& operator[](U64 i) const { return _shape[i]; }
    U64& operator[](U64 i) { return _shape[i]; }
    const U64* data() const { return _shape.data(); }
    bool operator==(const Shape& o) const { return _shape == o._shape; }
    bool operator!=(const Shape& o) const { return !(*this == o); }
    operator Type() const { return _shape; }

   protected:
    Type _shape;
};

struct ArrayShape : Shape<4> {
    using Shape<4>::Shape;
    const U64& numberOfAspects() const { return (*this)[0]; }
    const U64& numberOfFrequencyChannels() const { return (*this)[1]; }
    const U64& numberOfTimeSamples() const { return (*this)[2]; }
    const U64& numberOfPolarizations() const { return (*this)[3]; }
};

struct PhasorShape : Shape<5> {
    using Shape<5>::Shape;
    const U64& numberOfBeams() const { return (*this)[0]; }
    const U64& numberOfAntennas() const { return (*this)[1]; }
    const U64& numberOfFrequencyChannels() const { return (*this)[2]; }
    const U64& numberOfTimeSamples() const { return (*this)[3]; }
    const U64& numberOfPolarizations() const { return (*this)[4]; }
};

struct DelayShape : Shape<2> {
    using Shape<2>::Shape;
    const U64& numberOfBeams() const { return (*this)[0]; }
    const U64& numberOfAntennas() const { return (*this)[1]; }
};

struct VectorShape : Shape<1> {
    using Shape<1>::Shape;
};

// Ref-counted buffer.  Copies share the allocation (like the reference's Vector).
template <Device D, typename T, typename S>
class Vector {
   public:
    Vector() = default;
    explicit Vector(const S& shape) : _shape(shape) {
        const U64 bytes = shape.size() * sizeof(T);
        if (bytes == 0) return;
        void* p = nullptr;
        if (D == Device::CUDA) {
            Check(cudaMalloc(&p, bytes) == cudaSuccess ? BLADE_SUCCESS : BLADE_CUDA_ERROR, "Vector: cudaMalloc");
            _data = std::shared_ptr<void>(p, [](void* q) { cudaFree(q); });
        } else {
            Check(cudaMallocHost(&p, bytes) == cudaSuccess ? BLADE_SUCCESS : BLADE_CUDA_ERROR,
                  "Vector: cudaMallocHost");
            _data = std::shared_ptr<void>(p, [](void* q) { cudaFreeHost(q); });
        }
    }

    T* data() const { return static_cast<T*>(_data.get()); }
    const S& shape() const { return _shape; }
    U64 size() const { return _shape.size(); }
    U64 size_bytes() const { return _shape.size() * sizeof(T); }
    static constexpr Device device() { return D; }
    bool empty() const { return !_data; }

    // Reinterpret with another shape of the same size (Module::Link with a shape).
    Result reshape(const S& s) {
        if (s.size() != _shape.size()) return Result::ERROR;
        _shape = s;
        return Result::SUCCESS;
    }

    T& operator[](U64 i) const { return data()[i]; }

   private:
    std::shared_ptr<void> _data;
    S _shape;
};

template <Device D, typename T> using ArrayTensor = Vector<D, T, ArrayShape>;
template <Device D, typename T> using PhasorTensor = Vector<D, T, PhasorShape>;
template <Device D, typename T> using DelayTensor = Vector<D, T, DelayShape>;
template <Device D, typename T> using Tensor = Vector<D, T, VectorShape>;

// Two slots and a fixed Vector that operator[] re-points at slot i, so a module
// holding the fixed Vector by reference sees the current slot's data.
template <typename V>
class Duet {
   public:
    Duet() = default;
    template <typename Sh>
    explicit Duet(const Sh& shape) : _slots{V(shape), V(shape)}, _fixed(_slots[0]) {}

    void set(U64 i) { _fixed = _slots[i]; }
    V& operator[](U64 i) {
        set(i);
        return _fixed;
    }
    const V& at(U64 i) const { return _slots[i]; }
    V& fixed() { return _fixed; }
    operator V&() { return _fixed; }

   private:
    std::array<V, 2> _slots;
    V _fixed;
};

// Asynchronous copy with shape and type checks (copy.hh:11-33).
template <Device DD, Device SD, typename T, typename S>
Result Copy(Vector<DD, T, S>& dst, const Vector<SD, T, S>& src, Stream stream = nullptr) {
    if (dst.shape() != src.shape()) return Result::ERROR;
    const cudaError_t e = cudaMemcpyAsync(dst.data(), src.data(), src.size_bytes(), cudaMemcpyDefault, stream);
    return e == cudaSuccess ? Result::SUCCESS : Result::CUDA_ERROR;
}

}  // namespace Blade

#endif
