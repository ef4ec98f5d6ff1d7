// expr.h — AdditionalCompute expressions compiled to a register-stack bytecode.
//
// The reference parses with cpp-peglib (grammar at source/granite/TrajectoryIntegrator.cpp:10-26),
// builds a tree (Language.hpp:91-140), flattens it pre-order (cpp:770-798) and walks it
// recursively on the device for every alive particle and step (TrajectoryIntegrator.hpp:539-627).
// Here the tree is compiled once into postfix code whose evaluation order keeps the operand
// stack at most GR_EXPR_MAX_STACK deep, so the device keeps the whole stack in registers.
#pragma once

#ifndef __CUDACC_RTC__
#include <cstdint>
#include <string>
#include <vector>
#endif

namespace granite_b200 {

constexpr int GR_EXPR_MAX_CODE = 256;
constexpr int GR_EXPR_MAX_STACK = 8;

// Reference-vector slots, the order of `ref` in TrajectoryIntegrator.tpp:381-439.
enum RefSlot : int16_t {
    REF_X = 0, REF_Y = 1, REF_Z = 2, REF_CV = 3, REF_F0 = 4, REF_C0 = 12,
    REF_U = 16, REF_V = 17, REF_W = 18, REF_COUNT = 19
};

enum Op : int16_t {
    OP_REF = 1,    // push ref[arg]
    OP_CONST,      // push value
    OP_ADD, OP_SUB, OP_MUL, OP_DIV,   // a op b, a pushed first
    OP_RSUB, OP_RDIV,                 // b op a (right operand was pushed first)
    OP_SQRT, OP_EXP, OP_LOG, OP_SIN, OP_COS, OP_TAN, OP_ASIN, OP_ACOS, OP_ATAN,
    OP_ATAN2, OP_RATAN2
};

struct Instr {
    int16_t op;
    int16_t arg;
    float value;
};

struct Program {
    int32_t len;
    int32_t depth;
    Instr code[GR_EXPR_MAX_CODE];
};

#ifndef __CUDACC_RTC__
// Compiles `code`.  volume_names[k] -> f_k, constant_names[k] -> c_k.  On failure returns
// false and sets `error` to the reference's message ("ERROR < USER INPUT | ... >").
bool compile_expression(const std::string &code, const std::vector<std::string> &volume_names,
                        const std::vector<std::string> &constant_names, int dim,
                        int curvature_mode, Program &out, std::string &error);

// Host evaluation of a compiled program (used by the engine's self-check and tests).
float evaluate(const Program &p, const float *ref);
#endif

}  // namespace granite_b200
