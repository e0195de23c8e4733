// expression.h -- the scalar-expression program shared by the host compiler
// (expression.cpp) and the device evaluator (classic.cu).
//
// The instruction set, its SSA ordering rule and the float semantics of
// every op are those of the reference's XgenFloatExpressionProgram
// (include/nanoxgen/xgen_expression.h:12-100, evaluated by
// src/xgen_expression.cpp:984-1148).  The op numbering is kept identical so a
// compiled program can be compared instruction by instruction with the
// reference compiler's output.
#pragma once

#include <cstdint>

namespace nxg {

enum ExprOp : uint8_t {
    kOpConstant = 0,
    kOpInput,
    kOpNegate,
    kOpLogicalNot,
    kOpAdd,
    kOpSubtract,
    kOpMultiply,
    kOpDivide,
    kOpLess,
    kOpLessEqual,
    kOpGreater,
    kOpGreaterEqual,
    kOpEqual,
    kOpNotEqual,
    kOpLogicalAnd,
    kOpLogicalOr,
    kOpSelect,
    kOpHash,
    kOpRandom,
    kOpMinimum,
    kOpMaximum,
    kOpClamp,
    kOpFit,
    kOpGamma,
    kOpContrast,
    kOpSmoothstep,
    kOpRamp,
    kOpCount
};

// How a program input is bound for a root (the Classic runtime's
// input_value, src/xgen_classic_runtime.cpp:503-556, plus $u/$v bound to the
// root's texture coordinate).
enum ExprBinding : uint8_t {
    kBindPrefNoise = 0,  // xgen_classic_noise_float(rest root * frequency)
    kBindId,             // primitive id = strand index
    kBindU,              // root uv.x
    kBindV,              // root uv.y
    kBindCLength,        // spline length of the generated curve
    kBindCWidth,         // 0 while length and width are evaluated
};

// Device form limits.  A program above them is refused at launch with
// NXG_ERROR_EXPRESSION_LIMIT; they keep two programs inside one kernel
// parameter block (constant bank, broadcast to every lane).
constexpr uint32_t kExprMaxInstructions = 128u;
constexpr uint32_t kExprMaxOperands = 320u;
constexpr uint32_t kExprMaxInputs = 16u;
constexpr uint32_t kExprMaxRampPoints = 32u;
constexpr uint32_t kExprMaxRamps = 8u;

struct ExprInstruction {
    uint8_t op;
    uint8_t reserved;
    uint16_t operand_count;
    uint32_t operand_offset;
    uint32_t auxiliary;
    float immediate;
};
static_assert(sizeof(ExprInstruction) == 16u, "packed instruction");

struct ExprRampPoint {
    float position;
    float value;
    uint32_t interpolation;
};

struct ExprRamp {
    uint32_t point_offset;
    uint32_t point_count;
};

struct DeviceExpression {
    uint32_t instruction_count;
    uint32_t operand_count;
    uint32_t input_count;
    uint32_t ramp_count;
    uint32_t ramp_point_count;
    uint32_t result;
    uint32_t uses_clength;
    uint32_t uses_random;   // rand() needs the root's face seed
    uint32_t present;
    uint32_t reserved;
    ExprInstruction instructions[kExprMaxInstructions];
    uint16_t operands[kExprMaxOperands];
    uint8_t input_binding[kExprMaxInputs];
    float input_frequency[kExprMaxInputs];
    ExprRampPoint ramp_points[kExprMaxRampPoints];
    ExprRamp ramps[kExprMaxRamps];
};

} // namespace nxg

struct nxg_expression;

namespace nxg {

// Fills the device form of a compiled expression (expression.cpp).  Returns
// NXG_ERROR_EXPRESSION_LIMIT when it does not fit the limits above and
// NXG_ERROR_EXPRESSION_INPUT when an input has no per-root binding.
uint32_t pack_device_expression(const nxg_expression *expression, DeviceExpression &device);

} // namespace nxg
