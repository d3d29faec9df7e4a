// Bohrium opcodes.
//
// The numeric ids are the bytecode's wire values shared with every bridge and component, so they
// match the ids of the reference's opcode specification (core/codegen/opcodes.json; the generated
// enum lives at include/bohrium/bh_opcode.h in a reference build). Ids 54, 56, 69, 70 and 78 are
// unused there and here. Extension methods are assigned ids above BH_MAX_OPCODE_ID.
#pragma once

#include <bohrium/bh_type.hpp>

#ifdef __cplusplus
extern "C" {
#endif

enum { /* bh_opcode */
    BH_ADD = 1,
    BH_SUBTRACT = 2,
    BH_MULTIPLY = 3,
    BH_DIVIDE = 4,
    BH_POWER = 5,
    BH_ABSOLUTE = 6,
    BH_GREATER = 7,
    BH_GREATER_EQUAL = 8,
    BH_LESS = 9,
    BH_LESS_EQUAL = 10,
    BH_EQUAL = 11,
    BH_NOT_EQUAL = 12,
    BH_LOGICAL_AND = 13,
    BH_LOGICAL_OR = 14,
    BH_LOGICAL_XOR = 15,
    BH_LOGICAL_NOT = 16,
    BH_MAXIMUM = 17,
    BH_MINIMUM = 18,
    BH_BITWISE_AND = 19,
    BH_BITWISE_OR = 20,
    BH_BITWISE_XOR = 21,
    BH_INVERT = 22,
    BH_LEFT_SHIFT = 23,
    BH_RIGHT_SHIFT = 24,
    BH_COS = 25,
    BH_SIN = 26,
    BH_TAN = 27,
    BH_COSH = 28,
    BH_SINH = 29,
    BH_TANH = 30,
    BH_ARCSIN = 31,
    BH_ARCCOS = 32,
    BH_ARCTAN = 33,
    BH_ARCSINH = 34,
    BH_ARCCOSH = 35,
    BH_ARCTANH = 36,
    BH_ARCTAN2 = 37,
    BH_EXP = 38,
    BH_EXP2 = 39,
    BH_EXPM1 = 40,
    BH_LOG = 41,
    BH_LOG2 = 42,
    BH_LOG10 = 43,
    BH_LOG1P = 44,
    BH_SQRT = 45,
    BH_CEIL = 46,
    BH_TRUNC = 47,
    BH_FLOOR = 48,
    BH_RINT = 49,
    BH_MOD = 50,
    BH_ISNAN = 51,
    BH_ISINF = 52,
    BH_IDENTITY = 53,
    BH_FREE = 55,
    BH_NONE = 57,
    BH_TALLY = 58,
    BH_ADD_REDUCE = 59,
    BH_MULTIPLY_REDUCE = 60,
    BH_MINIMUM_REDUCE = 61,
    BH_MAXIMUM_REDUCE = 62,
    BH_LOGICAL_AND_REDUCE = 63,
    BH_BITWISE_AND_REDUCE = 64,
    BH_LOGICAL_OR_REDUCE = 65,
    BH_BITWISE_OR_REDUCE = 66,
    BH_LOGICAL_XOR_REDUCE = 67,
    BH_BITWISE_XOR_REDUCE = 68,
    BH_RANDOM = 71,
    BH_RANGE = 72,
    BH_REAL = 73,
    BH_IMAG = 74,
    BH_ADD_ACCUMULATE = 75,
    BH_MULTIPLY_ACCUMULATE = 76,
    BH_SIGN = 77,
    BH_GATHER = 79,
    BH_SCATTER = 80,
    BH_REMAINDER = 81,
    BH_COND_SCATTER = 82,
    BH_ISFINITE = 83,
    BH_CONJ = 84,

    BH_NO_OPCODES = 79,    // number of opcodes
    BH_MAX_OPCODE_ID = 84  // extension methods get ids above this
};

const char *bh_opcode_text(bh_opcode opcode);
int bh_opcode_nop(bh_opcode opcode); // number of operands (incl. the constant slot), -1 if unknown
bool bh_opcode_is_system(bh_opcode opcode);
bool bh_opcode_is_reduction(bh_opcode opcode);
bool bh_opcode_is_accumulate(bh_opcode opcode);
bool bh_opcode_is_elementwise(bh_opcode opcode);
bool bh_opcode_is_sweep(bh_opcode opcode);

#ifdef __cplusplus
}
#endif
