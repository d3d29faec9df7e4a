// Bohrium constants (the immediate operand of an instruction).
//
// Layout and API follow include/bohrium/bh_constant.hpp:25-199 of the reference: a union of every
// element type plus the type tag. The value union crosses the kernel-argument boundary by value,
// so its size (16 bytes) and member order are kept.
#pragma once

#include <complex>
#include <iostream>
#include <bohrium/bh_type.hpp>

union bh_constant_value {
    bh_bool bool8;
    bh_int8 int8;
    bh_int16 int16;
    bh_int32 int32;
    bh_int64 int64;
    bh_uint8 uint8;
    bh_uint16 uint16;
    bh_uint32 uint32;
    bh_uint64 uint64;
    bh_float32 float32;
    bh_float64 float64;
    bh_complex64 complex64;
    bh_complex128 complex128;
    bh_r123 r123;

    bh_constant_value() = default;
    bh_constant_value(bool val) : bool8(val) {}
    bh_constant_value(int8_t val) : int8(val) {}
    bh_constant_value(int16_t val) : int16(val) {}
    bh_constant_value(int32_t val) : int32(val) {}
    bh_constant_value(int64_t val) : int64(val) {}
    bh_constant_value(uint8_t val) : uint8(val) {}
    bh_constant_value(uint16_t val) : uint16(val) {}
    bh_constant_value(uint32_t val) : uint32(val) {}
    bh_constant_value(uint64_t val) : uint64(val) {}
    bh_constant_value(float val) : float32(val) {}
    bh_constant_value(double val) : float64(val) {}
    bh_constant_value(std::complex<float> val) : complex64{val.real(), val.imag()} {}
    bh_constant_value(std::complex<double> val) : complex128{val.real(), val.imag()} {}
    bh_constant_value(bh_r123 val) : r123(val) {}
};
static_assert(sizeof(bh_constant_value) == 16, "bh_constant_value must be 16 bytes");

class bh_constant {
public:
    bh_constant_value value;
    bh_type type;

    // Store `v` converted (static_cast) to this constant's type.
    template <typename T>
    void set_value(T v) {
        switch (type) {
            case bh_type::BOOL: value = bh_constant_value{static_cast<bool>(v)}; return;
            case bh_type::INT8: value = bh_constant_value{static_cast<int8_t>(v)}; return;
            case bh_type::INT16: value = bh_constant_value{static_cast<int16_t>(v)}; return;
            case bh_type::INT32: value = bh_constant_value{static_cast<int32_t>(v)}; return;
            case bh_type::INT64: value = bh_constant_value{static_cast<int64_t>(v)}; return;
            case bh_type::UINT8: value = bh_constant_value{static_cast<uint8_t>(v)}; return;
            case bh_type::UINT16: value = bh_constant_value{static_cast<uint16_t>(v)}; return;
            case bh_type::UINT32: value = bh_constant_value{static_cast<uint32_t>(v)}; return;
            case bh_type::UINT64: value = bh_constant_value{static_cast<uint64_t>(v)}; return;
            case bh_type::FLOAT32: value = bh_constant_value{static_cast<float>(v)}; return;
            case bh_type::FLOAT64: value = bh_constant_value{static_cast<double>(v)}; return;
            case bh_type::COMPLEX64: value = bh_constant_value{std::complex<float>(static_cast<float>(v))}; return;
            case bh_type::COMPLEX128: value = bh_constant_value{std::complex<double>(static_cast<double>(v))}; return;
            case bh_type::R123: value = bh_constant_value{static_cast<uint64_t>(v)}; return;
        }
        throw std::runtime_error("set_value(): unknown constant type");
    }
    void set_value(bh_r123 v) {
        if (type != bh_type::R123)
            throw std::runtime_error("set_value(): can only set BH_R123 constants with type `bh_r123`");
        value = bh_constant_value{v};
    }

    bh_constant() = default;
    template <typename T>
    bh_constant(T val) : value(val), type(bh_type_from_template<T>()) {}
    template <typename T>
    bh_constant(T val, bh_type t) : type(t) { set_value(val); }

    static bh_constant get_min(bh_type type);
    static bh_constant get_max(bh_type type);
    int64_t get_int64() const;
    uint64_t get_uint64() const;
    double get_double() const;
    void set_double(double value);
    bool operator==(const bh_constant &other) const;
    bool operator!=(const bh_constant &other) const { return !(other == *this); }
    void pprint(std::ostream &out, bool opencl = false) const;
};

std::ostream &operator<<(std::ostream &out, const bh_constant &constant);
