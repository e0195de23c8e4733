// classic_eval.cuh -- the exact scalar-expression evaluator for one root,
// shared by the exact runtime (classic.cu) and the surrogate's per-batch
// spot checks and exact re-runs (surrogate.cu).
//
// Semantics of the reference's evaluate_xgen_scalar_expression_float
// (src/xgen_expression.cpp:984-1148) with IEEE-rounded, never-contracted
// arithmetic, and xgen_classic_noise_float (src/xgen_classic_runtime.cpp:
// 803-837) for the noise($Prefg*k) inputs.
#pragma once

#include "expression.h"
#include "nxg_classic.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <cstdint>

namespace nxg {
namespace dev {

// The SeExpr gradient table the Classic runtime compiles in
// (xgen_classic_runtime.cpp:803-837 reads detail::kSeExprNoiseGradients).
static __constant__ float c_gradients[256][3] = {
#include "seexpr_gradients.inc"
};

static __constant__ uint8_t c_permutation[256] = {
#include "seexpr_permutation.inc"
};


// xgen_classic_noise_float (xgen_classic_runtime.cpp:803-837) with the
// reference's operation order and rounding.
__device__ inline float classic_noise(const float4 *table, float x, float y, float z) {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const uint32_t ix = static_cast<uint32_t>(static_cast<int32_t>(fx));
    const uint32_t iy = static_cast<uint32_t>(static_cast<int32_t>(fy));
    const uint32_t iz = static_cast<uint32_t>(static_cast<int32_t>(fz));
    const float wx = __fsub_rn(x, fx), wy = __fsub_rn(y, fy), wz = __fsub_rn(z, fz);
    const uint32_t base = ix * kLcgA2 + iy * kLcgA + iz + kLcgK;
    float v[8];
#pragma unroll
    for (uint32_t corner = 0u; corner < 8u; ++corner) {
        const uint32_t ox = corner & 1u, oy = (corner >> 1u) & 1u, oz = (corner >> 2u) & 1u;
        const float4 g = table[temper_index(base + (ox ? kLcgA2 : 0u) + (oy ? kLcgA : 0u) + oz)];
        v[corner] = __fadd_rn(__fadd_rn(__fmul_rn(g.x, __fsub_rn(wx, static_cast<float>(ox))),
                                        __fmul_rn(g.y, __fsub_rn(wy, static_cast<float>(oy)))),
                              __fmul_rn(g.z, __fsub_rn(wz, static_cast<float>(oz))));
    }
    const auto fade = [](float t) {  // t*t*t*(t*(t*6-15)+10), left to right
        return __fmul_rn(__fmul_rn(__fmul_rn(t, t), t),
                         __fadd_rn(__fmul_rn(t, __fsub_rn(__fmul_rn(t, 6.0f), 15.0f)), 10.0f));
    };
    const auto lerp = [](float a, float lo, float hi) {
        return __fadd_rn(__fmul_rn(__fsub_rn(1.0f, a), lo), __fmul_rn(a, hi));
    };
    const float ax = fade(wx), ay = fade(wy), az = fade(wz);
    v[0] = lerp(ax, v[0], v[1]);
    v[2] = lerp(ax, v[2], v[3]);
    v[4] = lerp(ax, v[4], v[5]);
    v[6] = lerp(ax, v[6], v[7]);
    v[0] = lerp(ay, v[0], v[2]);
    v[4] = lerp(ay, v[4], v[6]);
    v[0] = lerp(az, v[0], v[4]);
    return __fadd_rn(__fmul_rn(0.5f, v[0]), 0.5f);
}

// The 32 fraction bits and binary exponent of double(x) * 8.539734222673566
// in integer arithmetic (xgen_expression.cpp:648-690): the float's 24-bit
// significand times the constant's 53-bit significand as a 77-bit product,
// truncated to its top 32 bits with the reference's rounding correction.
__device__ inline uint32_t hash_component(float argument) {
    constexpr uint64_t kMantissa = 0x001114580b45d474ull;
    const uint32_t bits = __float_as_uint(argument);
    const uint32_t magnitude = bits & 0x7fffffffu;
    if (magnitude == 0u) { return 0u; }
    const uint32_t exponent_bits = magnitude >> 23u;
    const uint32_t significand = exponent_bits == 0u ? (magnitude & 0x7fffffu) : ((magnitude & 0x7fffffu) | 0x800000u);
    const uint64_t lo_product = static_cast<uint64_t>(significand) * static_cast<uint32_t>(kMantissa);
    const uint64_t hi_product = static_cast<uint64_t>(significand) * static_cast<uint32_t>(kMantissa >> 32u);
    const uint64_t low = lo_product + (hi_product << 32u);
    const uint64_t high = (hi_product >> 32u) + (low < lo_product ? 1u : 0u);
    const uint32_t length = high != 0u ? 128u - static_cast<uint32_t>(__clzll(static_cast<long long>(high)))
                                       : 64u - static_cast<uint32_t>(__clzll(static_cast<long long>(low)));
    const uint32_t shift = length - 32u;  // the product has at least 53 bits
    const uint32_t top = static_cast<uint32_t>((low >> shift) | (high << (64u - shift)));
    const uint64_t remainder = low & ((uint64_t{1} << shift) - 1u);
    const uint64_t ceil_high = ((low >> 32u) | (high << 32u)) + ((low & 0xffffffffu) != 0u ? 1u : 0u);
    const uint32_t fraction = top - (remainder < ceil_high ? 1u : 0u);
    const int32_t value_exponent = exponent_bits == 0u ? -149 : static_cast<int32_t>(exponent_bits) - 150;
    const uint32_t exponent = static_cast<uint32_t>(static_cast<int32_t>(length) + value_exponent - 49);
    return ((bits >> 31u) != 0u ? 0u - fraction : fraction) ^ exponent;
}

__device__ __forceinline__ uint32_t hash_step(uint32_t state, float argument) {
    return state * kLcgA + hash_component(argument) + kLcgC;
}

// Tempering then the byte permutation, as a float in [0, 1)
// (xgen_expression.cpp:628-646).
__device__ inline float hash_finish(uint32_t s, const uint8_t *perm) {
    s ^= s >> 11u;
    s ^= (s << 7u) & 0x9d2c5680u;
    s ^= (s << 15u) & 0xefc60000u;
    s ^= s >> 18u;
    const uint32_t b3 = perm[s & 0xffu];
    const uint32_t b2 = perm[((s >> 8u) + b3) & 0xffu];
    const uint32_t b1 = perm[((s >> 16u) + b2) & 0xffu];
    const uint32_t b0 = perm[((s >> 24u) + b1) & 0xffu];
    return __fmul_rn(__uint2float_rn(b0 | (b1 << 8u) | (b2 << 16u) | (b3 << 24u)), 0x1p-32f);
}

// std::min / std::max / std::clamp as libstdc++ defines them.
__device__ __forceinline__ float std_min(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float std_max(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float std_clamp(float v, float lo, float hi) { return std_min(std_max(v, lo), hi); }

// evaluate_ramp_points<float> (xgen_expression.cpp:559-612).
__device__ inline float ramp_value(const ExprRampPoint *pts, uint32_t n, float t) {
    if (t <= pts[0].position) { return std_clamp(pts[0].value, 0.0f, 1.0f); }
    if (t >= pts[n - 1].position) { return std_clamp(pts[n - 1].value, 0.0f, 1.0f); }
    uint32_t upper = 1u;
    while (upper < n && t >= pts[upper].position) { ++upper; }
    const uint32_t lower = upper - 1u;
    const float p0 = pts[lower].position, p1 = pts[upper].position;
    const float k0 = pts[lower].value, k1 = pts[upper].value;
    const float u = __fdiv_rn(__fsub_rn(t, p0), __fsub_rn(p1, p0));
    const float um1 = __fsub_rn(u, 1.0f);
    const float hermite = __fadd_rn(
        __fmul_rn(__fmul_rn(__fmul_rn(k0, um1), um1), __fadd_rn(__fmul_rn(2.0f, u), 1.0f)),
        __fmul_rn(__fmul_rn(__fmul_rn(k1, u), u), __fsub_rn(3.0f, __fmul_rn(2.0f, u))));
    float value;
    switch (pts[lower].interpolation) {
        case 0u: value = k0; break;
        case 1u: value = __fadd_rn(k0, __fmul_rn(u, __fsub_rn(k1, k0))); break;
        case 2u: value = hermite; break;
        default: {
            const float scale = __fdiv_rn(1.0f, __fsub_rn(p1, p0));
            const float end_slope = __fdiv_rn(__fsub_rn(k1, k0),
                                              __fmul_rn(scale, __fsub_rn(__fmul_rn(2.0f, p1), __fmul_rn(2.0f, p0))));
            const float d0 = lower == 0u ? end_slope
                : __fdiv_rn(__fsub_rn(k1, pts[lower - 1u].value),
                            __fmul_rn(scale, __fsub_rn(p1, pts[lower - 1u].position)));
            const float d1 = upper + 1u == n ? end_slope
                : __fdiv_rn(__fsub_rn(pts[upper + 1u].value, k0),
                            __fmul_rn(scale, __fsub_rn(pts[upper + 1u].position, p0)));
            value = __fadd_rn(__fadd_rn(hermite, __fmul_rn(__fmul_rn(__fmul_rn(d0, u), um1), um1)),
                              __fmul_rn(__fmul_rn(__fmul_rn(d1, u), u), um1));
        }
    }
    return std_clamp(value, 0.0f, 1.0f);
}

// has_prefix: rand() draws from a per-primitive SeExpr prefix (the Classic
// runtime's random_prefixes) instead of (u, v, face seed).
struct RootContext {
    float u, v, face_seed, t;
    uint32_t prefix = 0u;
    uint32_t has_prefix = 0u;
};

// One SSA program for one root.  Returns false where the reference throws
// (a non-finite input or intermediate value).
__device__ inline bool evaluate(const DeviceExpression &e, const float *inputs, const RootContext &c, const uint8_t *perm,
                         float *result) {
    float vals[kExprMaxInstructions];
    for (uint32_t i = 0; i < e.input_count; ++i) {
        if (!isfinite(inputs[i])) { return false; }
    }
    if (!isfinite(c.u) || !isfinite(c.v) || !isfinite(c.face_seed) || !isfinite(c.t)) { return false; }
    for (uint32_t pc = 0; pc < e.instruction_count; ++pc) {
        const ExprInstruction in = e.instructions[pc];
        const uint16_t *arg = e.operands + in.operand_offset;
        const int n = in.operand_count;
        float value = 0.0f;
        switch (in.op) {
            case kOpConstant: value = in.immediate; break;
            case kOpInput: value = inputs[in.auxiliary]; break;
            case kOpNegate: value = -vals[arg[0]]; break;
            case kOpLogicalNot: value = vals[arg[0]] == 0.0f ? 1.0f : 0.0f; break;
            case kOpAdd: value = __fadd_rn(vals[arg[0]], vals[arg[1]]); break;
            case kOpSubtract: value = __fsub_rn(vals[arg[0]], vals[arg[1]]); break;
            case kOpMultiply: value = __fmul_rn(vals[arg[0]], vals[arg[1]]); break;
            case kOpDivide: value = __fdiv_rn(vals[arg[0]], vals[arg[1]]); break;
            case kOpLess: value = vals[arg[0]] < vals[arg[1]] ? 1.0f : 0.0f; break;
            case kOpLessEqual: value = vals[arg[0]] <= vals[arg[1]] ? 1.0f : 0.0f; break;
            case kOpGreater: value = vals[arg[0]] > vals[arg[1]] ? 1.0f : 0.0f; break;
            case kOpGreaterEqual: value = vals[arg[0]] >= vals[arg[1]] ? 1.0f : 0.0f; break;
            case kOpEqual: value = vals[arg[0]] == vals[arg[1]] ? 1.0f : 0.0f; break;
            case kOpNotEqual: value = vals[arg[0]] != vals[arg[1]] ? 1.0f : 0.0f; break;
            case kOpLogicalAnd: value = (vals[arg[0]] != 0.0f && vals[arg[1]] != 0.0f) ? 1.0f : 0.0f; break;
            case kOpLogicalOr: value = (vals[arg[0]] != 0.0f || vals[arg[1]] != 0.0f) ? 1.0f : 0.0f; break;
            case kOpSelect: value = vals[arg[0]] != 0.0f ? vals[arg[1]] : vals[arg[2]]; break;
            case kOpHash: {
                uint32_t state = 0u;
                for (int k = 0; k < n; ++k) { state = hash_step(state, vals[arg[k]]); }
                value = hash_finish(state, perm);
                break;
            }
            case kOpRandom: {
                // With a SeExpr prefix: the LCG over (prefix, the site's
                // component); without: hash(u, v, face seed, site seed)
                // (xgen_expression.cpp:1063-1088); then the explicit seed.
                const bool seeded = n == 1 || n == 3;
                uint32_t state = c.has_prefix
                    ? c.prefix * kLcgA + in.auxiliary + kLcgC
                    : hash_step(hash_step(hash_step(hash_step(0u, c.u), c.v), c.face_seed), in.immediate);
                if (seeded) { state = hash_step(state, vals[arg[n - 1]]); }
                value = hash_finish(state, perm);
                if (n >= 2) {
                    value = __fadd_rn(__fmul_rn(__fsub_rn(vals[arg[1]], vals[arg[0]]), value), vals[arg[0]]);
                }
                break;
            }
            case kOpMinimum: value = std_min(vals[arg[0]], vals[arg[1]]); break;
            case kOpMaximum: value = std_max(vals[arg[0]], vals[arg[1]]); break;
            case kOpClamp: value = std_clamp(vals[arg[0]], vals[arg[1]], vals[arg[2]]); break;
            case kOpFit: {
                const float x = vals[arg[0]], a = vals[arg[1]], b = vals[arg[2]], lo = vals[arg[3]], hi = vals[arg[4]];
                value = __fadd_rn(lo, __fdiv_rn(__fmul_rn(__fsub_rn(x, a), __fsub_rn(hi, lo)), __fsub_rn(b, a)));
                break;
            }
            case kOpGamma: value = powf(vals[arg[0]], __fdiv_rn(1.0f, vals[arg[1]])); break;
            case kOpContrast: {
                const float x = vals[arg[0]];
                const float exponent = -log2f(x < 0.5f ? __fmul_rn(2.0f, x) : __fsub_rn(2.0f, __fmul_rn(2.0f, x)));
                const float shaped = __fmul_rn(0.5f, powf(__fsub_rn(1.0f, vals[arg[1]]), exponent));
                value = x < 0.5f ? shaped : __fsub_rn(1.0f, shaped);
                break;
            }
            case kOpSmoothstep: {
                const float t = std_clamp(__fdiv_rn(__fsub_rn(vals[arg[0]], vals[arg[1]]),
                                                    __fsub_rn(vals[arg[2]], vals[arg[1]])),
                                          0.0f, 1.0f);
                value = __fmul_rn(__fmul_rn(t, t), __fsub_rn(3.0f, __fmul_rn(2.0f, t)));
                break;
            }
            case kOpRamp: {
                const ExprRamp r = e.ramps[in.auxiliary];
                value = ramp_value(e.ramp_points + r.point_offset, r.point_count, c.t);
                break;
            }
            default: return false;
        }
        if (!isfinite(value)) { return false; }
        vals[pc] = value;
    }
    *result = vals[e.result];
    return true;
}

// Inputs of one program for one root (xgen_classic_runtime.cpp:503-556).
__device__ inline void bind_inputs(const DeviceExpression &e, const float4 *table, F3 pref, float id, float u, float v,
                            float *inputs) {
    for (uint32_t i = 0; i < e.input_count; ++i) {
        float x = 0.0f;
        switch (e.input_binding[i]) {
            case kBindPrefNoise: {
                const float f = e.input_frequency[i];
                x = classic_noise(table, __fmul_rn(pref.x, f), __fmul_rn(pref.y, f), __fmul_rn(pref.z, f));
                break;
            }
            case kBindId: x = id; break;
            case kBindU: x = u; break;
            case kBindV: x = v; break;
            default: x = 0.0f;  // cWidth is 0 while length and width are evaluated
        }
        inputs[i] = x;
    }
}

// Stages the gradient table and the hash permutation in shared memory
// (every thread of the block calls it; a __syncthreads must follow).
__device__ inline void stage_classic_tables(float4 *table, uint8_t *perm) {
    for (int i = threadIdx.x; i < 256; i += blockDim.x) {
        table[i] = make_float4(c_gradients[i][0], c_gradients[i][1], c_gradients[i][2], 0.0f);
        perm[i] = c_permutation[i];
    }
}

// rand() face seed of a root (xgen_runtime_face_seed over description id,
// patch seed and triangle).
__device__ inline float classic_face_seed(float description_id, float patch_seed, uint32_t triangle,
                                          const uint8_t *perm) {
    const uint32_t state = hash_step(hash_step(0u, description_id), patch_seed);
    return hash_finish(hash_step(state, __uint2float_rn(triangle)), perm);
}

// Length scale and width of one root under the given programs (scale 1 and
// width 0 where a program is absent).  Returns false where the reference
// throws (non-finite value, negative length).
__device__ inline bool classic_root_scalars(const DeviceExpression &length_program,
                                            const DeviceExpression &width_program, const float4 *table,
                                            const uint8_t *perm, const Root &root, uint32_t strand,
                                            float face_seed, float *length, float *width) {
    const RootContext c{root.u, root.v, face_seed, 0.0f};
    const float id = __uint2float_rn(strand);
    float inputs[kExprMaxInputs];
    *length = 1.0f;
    *width = 0.0f;
    bool ok = true;
    if (length_program.present) {
        bind_inputs(length_program, table, root.position, id, root.u, root.v, inputs);
        ok = evaluate(length_program, inputs, c, perm, length) && *length >= 0.0f;
    }
    if (ok && width_program.present) {
        bind_inputs(width_program, table, root.position, id, root.u, root.v, inputs);
        ok = evaluate(width_program, inputs, c, perm, width);
    }
    return ok;
}

} // namespace dev

// The exact per-root scalar kernel over strands [first, first + count)
// (classic.cu).  With `distrust`, it skips the batches a surrogate launch
// serves (see nxg_surrogate_root_scalars, adaptive mode).
uint32_t launch_classic_root_scalars(const nxg_device_asset_desc &asset, const nxg_generation_params &params,
                                     const nxg_classic_scalar_plan &plan, uint32_t first, uint32_t count,
                                     float *scalars, uint32_t *status, cudaStream_t stream,
                                     const uint32_t *distrust, uint32_t probe_period);
} // namespace nxg
