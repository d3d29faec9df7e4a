// Element types, constants and opcode properties.
// Semantics follow core/bh_type.cpp, core/bh_constant.cpp and the opcode flags of
// core/codegen/opcodes.json in the reference.
#include <cmath>
#include <complex>
#include <limits>
#include <sstream>
#include <bohrium/bh_type.hpp>
#include <bohrium/bh_constant.hpp>
#include <bohrium/bh_opcode.h>

using namespace std;

int bh_type_size(bh_type type) {
    switch (type) {
        case bh_type::BOOL: case bh_type::INT8: case bh_type::UINT8: return 1;
        case bh_type::INT16: case bh_type::UINT16: return 2;
        case bh_type::INT32: case bh_type::UINT32: case bh_type::FLOAT32: return 4;
        case bh_type::INT64: case bh_type::UINT64: case bh_type::FLOAT64: case bh_type::COMPLEX64: return 8;
        case bh_type::COMPLEX128: case bh_type::R123: return 16;
    }
    throw runtime_error("bh_type_size(): unknown type");
}

const char *bh_type_text(bh_type type) {
    switch (type) {
        case bh_type::BOOL: return "BH_BOOL";
        case bh_type::INT8: return "BH_INT8";
        case bh_type::INT16: return "BH_INT16";
        case bh_type::INT32: return "BH_INT32";
        case bh_type::INT64: return "BH_INT64";
        case bh_type::UINT8: return "BH_UINT8";
        case bh_type::UINT16: return "BH_UINT16";
        case bh_type::UINT32: return "BH_UINT32";
        case bh_type::UINT64: return "BH_UINT64";
        case bh_type::FLOAT32: return "BH_FLOAT32";
        case bh_type::FLOAT64: return "BH_FLOAT64";
        case bh_type::COMPLEX64: return "BH_COMPLEX64";
        case bh_type::COMPLEX128: return "BH_COMPLEX128";
        case bh_type::R123: return "BH_R123";
    }
    return "Unknown type";
}

int bh_type_is_signed_integer(bh_type t) {
    return t == bh_type::INT8 || t == bh_type::INT16 || t == bh_type::INT32 || t == bh_type::INT64;
}
int bh_type_is_unsigned_integer(bh_type t) {
    return t == bh_type::UINT8 || t == bh_type::UINT16 || t == bh_type::UINT32 || t == bh_type::UINT64;
}
int bh_type_is_integer(bh_type t) { return bh_type_is_signed_integer(t) || bh_type_is_unsigned_integer(t); }
int bh_type_is_float(bh_type t) { return t == bh_type::FLOAT32 || t == bh_type::FLOAT64; }
int bh_type_is_complex(bh_type t) { return t == bh_type::COMPLEX64 || t == bh_type::COMPLEX128; }

uint64_t bh_type_limit_max_integer(bh_type t) {
    switch (t) {
        case bh_type::BOOL: return 1;
        case bh_type::INT8: return numeric_limits<int8_t>::max();
        case bh_type::INT16: return numeric_limits<int16_t>::max();
        case bh_type::INT32: return numeric_limits<int32_t>::max();
        case bh_type::INT64: return numeric_limits<int64_t>::max();
        case bh_type::UINT8: return numeric_limits<uint8_t>::max();
        case bh_type::UINT16: return numeric_limits<uint16_t>::max();
        case bh_type::UINT32: return numeric_limits<uint32_t>::max();
        case bh_type::UINT64: return numeric_limits<uint64_t>::max();
        default: throw runtime_error("bh_type_limit_max_integer(): not an integer type");
    }
}
int64_t bh_type_limit_min_integer(bh_type t) {
    switch (t) {
        case bh_type::BOOL: return 0;
        case bh_type::INT8: return numeric_limits<int8_t>::min();
        case bh_type::INT16: return numeric_limits<int16_t>::min();
        case bh_type::INT32: return numeric_limits<int32_t>::min();
        case bh_type::INT64: return numeric_limits<int64_t>::min();
        case bh_type::UINT8: case bh_type::UINT16: case bh_type::UINT32: case bh_type::UINT64: return 0;
        default: throw runtime_error("bh_type_limit_min_integer(): not an integer type");
    }
}
double bh_type_limit_max_float(bh_type t) {
    if (t == bh_type::FLOAT32) return numeric_limits<float>::max();
    if (t == bh_type::FLOAT64) return numeric_limits<double>::max();
    throw runtime_error("bh_type_limit_max_float(): not a float type");
}
double bh_type_limit_min_float(bh_type t) {
    if (t == bh_type::FLOAT32) return numeric_limits<float>::min();
    if (t == bh_type::FLOAT64) return numeric_limits<double>::min();
    throw runtime_error("bh_type_limit_min_float(): not a float type");
}

// The "minimum" constant used as the identity of BH_MAXIMUM_REDUCE. As in the reference
// (core/bh_constant.cpp get_min), signed integers use min()+1 and floating point uses the
// smallest positive normal number (numeric_limits<T>::min()), not the lowest value.
bh_constant bh_constant::get_min(bh_type type) {
    switch (type) {
        case bh_type::BOOL: return bh_constant(bh_bool{0});
        case bh_type::INT8: return bh_constant(static_cast<int8_t>(numeric_limits<int8_t>::min() + 1));
        case bh_type::INT16: return bh_constant(static_cast<int16_t>(numeric_limits<int16_t>::min() + 1));
        case bh_type::INT32: return bh_constant(static_cast<int32_t>(numeric_limits<int32_t>::min() + 1));
        case bh_type::INT64: return bh_constant(static_cast<int64_t>(numeric_limits<int64_t>::min() + 1));
        case bh_type::UINT8: return bh_constant(uint8_t{0});
        case bh_type::UINT16: return bh_constant(uint16_t{0});
        case bh_type::UINT32: return bh_constant(uint32_t{0});
        case bh_type::UINT64: return bh_constant(uint64_t{0});
        case bh_type::FLOAT32: return bh_constant(numeric_limits<float>::min());
        case bh_type::FLOAT64: return bh_constant(numeric_limits<double>::min());
        case bh_type::COMPLEX64:
            return bh_constant(complex<float>(numeric_limits<float>::min(), numeric_limits<float>::min()));
        case bh_type::COMPLEX128:
            return bh_constant(complex<double>(numeric_limits<double>::min(), numeric_limits<double>::min()));
        case bh_type::R123: return bh_constant(bh_r123{0, 0});
    }
    throw runtime_error("bh_constant::get_min(): unknown type");
}

bh_constant bh_constant::get_max(bh_type type) {
    switch (type) {
        case bh_type::BOOL: return bh_constant(bh_bool{1});
        case bh_type::INT8: return bh_constant(numeric_limits<int8_t>::max());
        case bh_type::INT16: return bh_constant(numeric_limits<int16_t>::max());
        case bh_type::INT32: return bh_constant(numeric_limits<int32_t>::max());
        case bh_type::INT64: return bh_constant(numeric_limits<int64_t>::max());
        case bh_type::UINT8: return bh_constant(numeric_limits<uint8_t>::max());
        case bh_type::UINT16: return bh_constant(numeric_limits<uint16_t>::max());
        case bh_type::UINT32: return bh_constant(numeric_limits<uint32_t>::max());
        case bh_type::UINT64: return bh_constant(numeric_limits<uint64_t>::max());
        case bh_type::FLOAT32: return bh_constant(numeric_limits<float>::max());
        case bh_type::FLOAT64: return bh_constant(numeric_limits<double>::max());
        case bh_type::COMPLEX64:
            return bh_constant(complex<float>(numeric_limits<float>::max(), numeric_limits<float>::max()));
        case bh_type::COMPLEX128:
            return bh_constant(complex<double>(numeric_limits<double>::max(), numeric_limits<double>::max()));
        case bh_type::R123:
            return bh_constant(bh_r123{numeric_limits<uint64_t>::max(), numeric_limits<uint64_t>::max()});
    }
    throw runtime_error("bh_constant::get_max(): unknown type");
}

int64_t bh_constant::get_int64() const {
    switch (type) {
        case bh_type::BOOL: return value.bool8;
        case bh_type::INT8: return value.int8;
        case bh_type::INT16: return value.int16;
        case bh_type::INT32: return value.int32;
        case bh_type::INT64: return value.int64;
        case bh_type::UINT8: return value.uint8;
        case bh_type::UINT16: return value.uint16;
        case bh_type::UINT32: return value.uint32;
        case bh_type::UINT64:
            if (value.uint64 < static_cast<uint64_t>(numeric_limits<int64_t>::max()))
                return static_cast<int64_t>(value.uint64);
            break;
        default: break;
    }
    throw overflow_error("Constant cannot be converted to int64_t");
}

uint64_t bh_constant::get_uint64() const {
    switch (type) {
        case bh_type::UINT8: return value.uint8;
        case bh_type::UINT16: return value.uint16;
        case bh_type::UINT32: return value.uint32;
        case bh_type::UINT64: return value.uint64;
        default: throw overflow_error("Constant cannot be converted to uint64_t");
    }
}

double bh_constant::get_double() const {
    switch (type) {
        case bh_type::BOOL: return value.bool8;
        case bh_type::INT8: return value.int8;
        case bh_type::INT16: return value.int16;
        case bh_type::INT32: return value.int32;
        case bh_type::INT64: return static_cast<double>(value.int64);
        case bh_type::UINT8: return value.uint8;
        case bh_type::UINT16: return value.uint16;
        case bh_type::UINT32: return value.uint32;
        case bh_type::UINT64: return static_cast<double>(value.uint64);
        case bh_type::FLOAT32: return value.float32;
        case bh_type::FLOAT64: return value.float64;
        case bh_type::COMPLEX64:
            if (value.complex64.imag != 0) throw overflow_error("Complex64 with imag != 0 cannot become a double");
            return value.complex64.real;
        case bh_type::COMPLEX128:
            if (value.complex128.imag != 0) throw overflow_error("Complex128 with imag != 0 cannot become a double");
            return value.complex128.real;
        case bh_type::R123: throw overflow_error("R123 cannot be converted to double");
    }
    throw runtime_error("Unknown constant type in get_double");
}

void bh_constant::set_double(double v) {
    switch (type) {
        case bh_type::BOOL: value.bool8 = static_cast<bool>(v); return;
        case bh_type::INT8: value.int8 = static_cast<int8_t>(v); return;
        case bh_type::INT16: value.int16 = static_cast<int16_t>(v); return;
        case bh_type::INT32: value.int32 = static_cast<int32_t>(v); return;
        case bh_type::INT64: value.int64 = static_cast<int64_t>(v); return;
        case bh_type::UINT8: value.uint8 = static_cast<uint8_t>(v); return;
        case bh_type::UINT16: value.uint16 = static_cast<uint16_t>(v); return;
        case bh_type::UINT32: value.uint32 = static_cast<uint32_t>(v); return;
        case bh_type::UINT64: value.uint64 = static_cast<uint64_t>(v); return;
        case bh_type::FLOAT32: value.float32 = static_cast<float>(v); return;
        case bh_type::FLOAT64: value.float64 = v; return;
        case bh_type::COMPLEX64: value.complex64.real = static_cast<float>(v); value.complex64.imag = 0; return;
        case bh_type::COMPLEX128: value.complex128.real = v; value.complex128.imag = 0; return;
        case bh_type::R123: throw overflow_error("double to R123 isn't possible");
    }
    throw runtime_error("Unknown constant type in set_double");
}

bool bh_constant::operator==(const bh_constant &o) const {
    if (o.type != type) return false;
    switch (type) {
        case bh_type::BOOL: return o.value.bool8 == value.bool8;
        case bh_type::INT8: return o.value.int8 == value.int8;
        case bh_type::INT16: return o.value.int16 == value.int16;
        case bh_type::INT32: return o.value.int32 == value.int32;
        case bh_type::INT64: return o.value.int64 == value.int64;
        case bh_type::UINT8: return o.value.uint8 == value.uint8;
        case bh_type::UINT16: return o.value.uint16 == value.uint16;
        case bh_type::UINT32: return o.value.uint32 == value.uint32;
        case bh_type::UINT64: return o.value.uint64 == value.uint64;
        case bh_type::FLOAT32: return o.value.float32 == value.float32;
        case bh_type::FLOAT64: return o.value.float64 == value.float64;
        case bh_type::COMPLEX64:
            return o.value.complex64.real == value.complex64.real && o.value.complex64.imag == value.complex64.imag;
        case bh_type::COMPLEX128:
            return o.value.complex128.real == value.complex128.real &&
                   o.value.complex128.imag == value.complex128.imag;
        case bh_type::R123: return o.value.r123.start == value.r123.start && o.value.r123.key == value.r123.key;
    }
    return false;
}

void bh_constant::pprint(ostream &out, bool) const {
    out.precision(17);
    switch (type) {
        case bh_type::BOOL: out << (value.bool8 ? "true" : "false"); break;
        case bh_type::INT8: out << static_cast<int>(value.int8); break;
        case bh_type::INT16: out << value.int16; break;
        case bh_type::INT32: out << value.int32; break;
        case bh_type::INT64: out << value.int64; break;
        case bh_type::UINT8: out << static_cast<unsigned>(value.uint8); break;
        case bh_type::UINT16: out << value.uint16; break;
        case bh_type::UINT32: out << value.uint32; break;
        case bh_type::UINT64: out << value.uint64; break;
        case bh_type::FLOAT32: out << value.float32; break;
        case bh_type::FLOAT64: out << value.float64; break;
        case bh_type::COMPLEX64: out << "(" << value.complex64.real << "+" << value.complex64.imag << "i)"; break;
        case bh_type::COMPLEX128: out << "(" << value.complex128.real << "+" << value.complex128.imag << "i)"; break;
        case bh_type::R123: out << "{start: " << value.r123.start << ", key: " << value.r123.key << "}"; break;
    }
}

ostream &operator<<(ostream &out, const bh_constant &c) {
    c.pprint(out);
    return out;
}

// ---------------------------------------------------------------------------------------------
// Opcode table: name, number of operands and the flags (elementwise, system, reduction,
// accumulate) of each opcode id.
namespace {
struct OpInfo {
    int id;
    const char *name;
    int nop;
    bool elementwise, system, reduction, accumulate;
};
constexpr OpInfo kOps[] = {
    {BH_ADD, "BH_ADD", 3, true, false, false, false},
    {BH_SUBTRACT, "BH_SUBTRACT", 3, true, false, false, false},
    {BH_MULTIPLY, "BH_MULTIPLY", 3, true, false, false, false},
    {BH_DIVIDE, "BH_DIVIDE", 3, true, false, false, false},
    {BH_POWER, "BH_POWER", 3, true, false, false, false},
    {BH_ABSOLUTE, "BH_ABSOLUTE", 2, true, false, false, false},
    {BH_GREATER, "BH_GREATER", 3, true, false, false, false},
    {BH_GREATER_EQUAL, "BH_GREATER_EQUAL", 3, true, false, false, false},
    {BH_LESS, "BH_LESS", 3, true, false, false, false},
    {BH_LESS_EQUAL, "BH_LESS_EQUAL", 3, true, false, false, false},
    {BH_EQUAL, "BH_EQUAL", 3, true, false, false, false},
    {BH_NOT_EQUAL, "BH_NOT_EQUAL", 3, true, false, false, false},
    {BH_LOGICAL_AND, "BH_LOGICAL_AND", 3, true, false, false, false},
    {BH_LOGICAL_OR, "BH_LOGICAL_OR", 3, true, false, false, false},
    {BH_LOGICAL_XOR, "BH_LOGICAL_XOR", 3, true, false, false, false},
    {BH_LOGICAL_NOT, "BH_LOGICAL_NOT", 2, true, false, false, false},
    {BH_MAXIMUM, "BH_MAXIMUM", 3, true, false, false, false},
    {BH_MINIMUM, "BH_MINIMUM", 3, true, false, false, false},
    {BH_BITWISE_AND, "BH_BITWISE_AND", 3, true, false, false, false},
    {BH_BITWISE_OR, "BH_BITWISE_OR", 3, true, false, false, false},
    {BH_BITWISE_XOR, "BH_BITWISE_XOR", 3, true, false, false, false},
    {BH_INVERT, "BH_INVERT", 2, true, false, false, false},
    {BH_LEFT_SHIFT, "BH_LEFT_SHIFT", 3, true, false, false, false},
    {BH_RIGHT_SHIFT, "BH_RIGHT_SHIFT", 3, true, false, false, false},
    {BH_COS, "BH_COS", 2, true, false, false, false},
    {BH_SIN, "BH_SIN", 2, true, false, false, false},
    {BH_TAN, "BH_TAN", 2, true, false, false, false},
    {BH_COSH, "BH_COSH", 2, true, false, false, false},
    {BH_SINH, "BH_SINH", 2, true, false, false, false},
    {BH_TANH, "BH_TANH", 2, true, false, false, false},
    {BH_ARCSIN, "BH_ARCSIN", 2, true, false, false, false},
    {BH_ARCCOS, "BH_ARCCOS", 2, true, false, false, false},
    {BH_ARCTAN, "BH_ARCTAN", 2, true, false, false, false},
    {BH_ARCSINH, "BH_ARCSINH", 2, true, false, false, false},
    {BH_ARCCOSH, "BH_ARCCOSH", 2, true, false, false, false},
    {BH_ARCTANH, "BH_ARCTANH", 2, true, false, false, false},
    {BH_ARCTAN2, "BH_ARCTAN2", 3, true, false, false, false},
    {BH_EXP, "BH_EXP", 2, true, false, false, false},
    {BH_EXP2, "BH_EXP2", 2, true, false, false, false},
    {BH_EXPM1, "BH_EXPM1", 2, true, false, false, false},
    {BH_LOG, "BH_LOG", 2, true, false, false, false},
    {BH_LOG2, "BH_LOG2", 2, true, false, false, false},
    {BH_LOG10, "BH_LOG10", 2, true, false, false, false},
    {BH_LOG1P, "BH_LOG1P", 2, true, false, false, false},
    {BH_SQRT, "BH_SQRT", 2, true, false, false, false},
    {BH_CEIL, "BH_CEIL", 2, true, false, false, false},
    {BH_TRUNC, "BH_TRUNC", 2, true, false, false, false},
    {BH_FLOOR, "BH_FLOOR", 2, true, false, false, false},
    {BH_RINT, "BH_RINT", 2, true, false, false, false},
    {BH_MOD, "BH_MOD", 3, true, false, false, false},
    {BH_ISNAN, "BH_ISNAN", 2, true, false, false, false},
    {BH_ISINF, "BH_ISINF", 2, true, false, false, false},
    {BH_IDENTITY, "BH_IDENTITY", 2, true, false, false, false},
    {BH_FREE, "BH_FREE", 1, false, true, false, false},
    {BH_NONE, "BH_NONE", 0, true, true, false, false},
    {BH_TALLY, "BH_TALLY", 0, false, true, false, false},
    {BH_ADD_REDUCE, "BH_ADD_REDUCE", 3, false, false, true, false},
    {BH_MULTIPLY_REDUCE, "BH_MULTIPLY_REDUCE", 3, false, false, true, false},
    {BH_MINIMUM_REDUCE, "BH_MINIMUM_REDUCE", 3, false, false, true, false},
    {BH_MAXIMUM_REDUCE, "BH_MAXIMUM_REDUCE", 3, false, false, true, false},
    {BH_LOGICAL_AND_REDUCE, "BH_LOGICAL_AND_REDUCE", 3, false, false, true, false},
    {BH_BITWISE_AND_REDUCE, "BH_BITWISE_AND_REDUCE", 3, false, false, true, false},
    {BH_LOGICAL_OR_REDUCE, "BH_LOGICAL_OR_REDUCE", 3, false, false, true, false},
    {BH_BITWISE_OR_REDUCE, "BH_BITWISE_OR_REDUCE", 3, false, false, true, false},
    {BH_LOGICAL_XOR_REDUCE, "BH_LOGICAL_XOR_REDUCE", 3, false, false, true, false},
    {BH_BITWISE_XOR_REDUCE, "BH_BITWISE_XOR_REDUCE", 3, false, false, true, false},
    {BH_RANDOM, "BH_RANDOM", 2, false, false, false, false},
    {BH_RANGE, "BH_RANGE", 1, false, false, false, false},
    {BH_REAL, "BH_REAL", 2, true, false, false, false},
    {BH_IMAG, "BH_IMAG", 2, true, false, false, false},
    {BH_ADD_ACCUMULATE, "BH_ADD_ACCUMULATE", 3, false, false, false, true},
    {BH_MULTIPLY_ACCUMULATE, "BH_MULTIPLY_ACCUMULATE", 3, false, false, false, true},
    {BH_SIGN, "BH_SIGN", 2, true, false, false, false},
    {BH_GATHER, "BH_GATHER", 3, false, false, false, false},
    {BH_SCATTER, "BH_SCATTER", 3, false, false, false, false},
    {BH_REMAINDER, "BH_REMAINDER", 3, true, false, false, false},
    {BH_COND_SCATTER, "BH_COND_SCATTER", 4, false, false, false, false},
    {BH_ISFINITE, "BH_ISFINITE", 2, true, false, false, false},
    {BH_CONJ, "BH_CONJ", 2, true, false, false, false},
};
static_assert(sizeof(kOps) / sizeof(kOps[0]) == BH_NO_OPCODES, "opcode table size");

const OpInfo *find_op(bh_opcode op) {
    static const OpInfo *table[BH_MAX_OPCODE_ID + 1] = {nullptr};
    static bool init = false;
    if (!init) {
        for (const OpInfo &o : kOps) table[o.id] = &o;
        init = true;
    }
    if (op < 0 || op > BH_MAX_OPCODE_ID) return nullptr;
    return table[op];
}
} // namespace

extern "C" {
const char *bh_opcode_text(bh_opcode opcode) {
    const OpInfo *o = find_op(opcode);
    return o ? o->name : "Unknown opcode";
}
int bh_opcode_nop(bh_opcode opcode) {
    const OpInfo *o = find_op(opcode);
    return o ? o->nop : -1;
}
bool bh_opcode_is_system(bh_opcode opcode) {
    const OpInfo *o = find_op(opcode);
    return o && o->system;
}
bool bh_opcode_is_reduction(bh_opcode opcode) {
    const OpInfo *o = find_op(opcode);
    return o && o->reduction;
}
bool bh_opcode_is_accumulate(bh_opcode opcode) {
    const OpInfo *o = find_op(opcode);
    return o && o->accumulate;
}
bool bh_opcode_is_elementwise(bh_opcode opcode) {
    const OpInfo *o = find_op(opcode);
    return o && o->elementwise;
}
bool bh_opcode_is_sweep(bh_opcode opcode) {
    return bh_opcode_is_reduction(opcode) || bh_opcode_is_accumulate(opcode);
}
}
