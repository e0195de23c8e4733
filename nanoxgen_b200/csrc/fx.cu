// fx.cu -- the Classic FX passes on sm_100a (nxg_classic_fx_*).
//
// A pass over a generated packed curve set that applies a description's
// Classic runtime plan per strand, in the order of
// apply_xgen_classic_float_runtime_plan_cpu (src/xgen_classic_runtime.cpp:
// 1420-1919): the SplinePrimitive length (scale about the root) and width,
// the drop rule on cLength and the width, the FX modules in the
// description's order -- NoiseFX mode 0 (apply_noise, :897-1040), CutFX
// rebuild type 1 (cut_from_tip_and_rebuild, :692-748) -- then the width
// profile (taper, taperStart, widthRamp).  One thread carries one strand
// through every step, as the reference's per-strand loop does; the strand's
// points live in the thread's local arrays (at most NXG_CLASSIC_MAX_FX_CVS).
// Arithmetic keeps the reference's order and IEEE rounding (uncontracted
// intrinsics), except the rotation's acos/cos/sin, which come from CUDA's
// math library, so the frame matches to rounding rather than bit for bit.
// The packed plan (every program in the device form the exact runtime uses)
// lives in a caller-owned device buffer, uploaded once.
#include "classic_eval.cuh"
#include "expression.h"
#include "generator_core.cuh"
#include "nxg_classic.h"
#include "nxg_internal.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace nxg {
namespace dev {

constexpr int kFxMaxCvs = static_cast<int>(NXG_CLASSIC_MAX_FX_CVS);
constexpr int kFxMaxEffects = static_cast<int>(NXG_CLASSIC_MAX_FX);

// Programs of one effect: NoiseFX mask, magnitude, magnitudeScale,
// frequency, correlation, preserveLength; CutFX amount in slot 0;
// ClumpingFX mask, clump, clumpScale, noise, noiseScale, noiseFrequency,
// noiseCorrelation.
enum : int { kFxMask = 0, kFxMagnitude, kFxMagnitudeScale, kFxFrequency, kFxCorrelation, kFxPreserve };
enum : int { kClumpMask = 0, kClumpAmount, kClumpScale, kClumpNoise, kClumpNoiseScale, kClumpNoiseFrequency,
             kClumpNoiseCorrelation, kFxSlots };

struct FxPlan {
    uint32_t effect_count;
    uint32_t effect_type[kFxMaxEffects];
    uint32_t length_after[kFxMaxEffects];  // a later program binds cLength
    uint32_t guide_noise_shared[kFxMaxEffects];  // ClumpingFX guide noise reads no per-strand input
    uint32_t uses_random;
    float description_id;   // rand() face seed inputs
    float patch_seed;
    DeviceExpression length, width, taper, taper_start, width_ramp;
    DeviceExpression effect[kFxMaxEffects][kFxSlots];
};

struct FxArgs {
    const FxPlan *plan;
    float4 *points;
    uint32_t *point_counts;
    const uint32_t *roots;        // 12 words per strand
    const float *surface_tangents;
    const float *noise_domains;
    uint32_t count, P, first_id;
    float radius_scale;
    uint32_t *status;
    const uint32_t *random_prefixes;
    uint32_t clump_count;
    nxg_classic_clump_guides clumps[kFxMaxEffects];
};

// The runtime context of one strand (ClassicFloatRuntimeContext,
// xgen_classic_runtime.h:157-170) for the variables this runtime binds.
struct FxContext {
    F3 pref;            // noise($Prefg*k) is evaluated at the root's position
    float id, u, v, face_seed, c_length, c_width, t;
    uint32_t prefix, has_prefix;  // rand()'s SeExpr prefix
};

// Inputs of one program (input_value, xgen_classic_runtime.cpp:503-556).
__device__ inline void fx_bind(const DeviceExpression &e, const float4 *table, const FxContext &c, float *inputs) {
    for (uint32_t i = 0; i < e.input_count; ++i) {
        float x = 0.0f;
        switch (e.input_binding[i]) {
            case kBindPrefNoise: {
                const float f = e.input_frequency[i];
                x = classic_noise(table, __fmul_rn(c.pref.x, f), __fmul_rn(c.pref.y, f), __fmul_rn(c.pref.z, f));
                break;
            }
            case kBindId: x = c.id; break;
            case kBindU: x = c.u; break;
            case kBindV: x = c.v; break;
            case kBindCLength: x = c.c_length; break;
            case kBindCWidth: x = c.c_width; break;
            default: x = 0.0f;
        }
        inputs[i] = x;
    }
}

// evaluate_runtime_expression for one strand's context; false where the
// reference throws (non-finite value).  One out-of-line copy: the
// interpreter is large and is called from a dozen places.
__device__ __noinline__ bool fx_eval(const DeviceExpression &e, const float4 *table, const uint8_t *perm,
                                     const FxContext &c, float *value) {
    float inputs[kExprMaxInputs];
    fx_bind(e, table, c, inputs);
    return evaluate(e, inputs, RootContext{c.u, c.v, c.face_seed, c.t, c.prefix, c.has_prefix}, perm, value);
}

// One strand's curve: positions in local arrays.
struct FxCurve {
    F3 p[kFxMaxCvs];
};

// Strand-independent tables of one launch (P is uniform): the spline
// length's sample weights, and t = cv / (P - 1) per CV.
struct FxTables {
    float4 length_weights[2 * kFxMaxCvs + 4];  // (b0, b1, b2, f^3) at t = k / (2P + 4)
    int length_span[2 * kFxMaxCvs + 4];
    float t[kFxMaxCvs];
};

// The cubic B-spline weights of curve_eval_classic at parameter t in the
// reference's rounding (the arithmetic of classic_curve_eval_by).
__device__ inline float4 fx_weights(float t, int P, int &span) {
    const float scaled = __fmul_rn(t, static_cast<float>(P - 1));
    span = static_cast<int>(static_cast<uint32_t>(scaled));
    const float f = __fsub_rn(scaled, static_cast<float>(span));
    const float f2 = __fmul_rn(f, f);
    const float f3 = __fmul_rn(f2, f);
    const float omf = __fsub_rn(1.0f, f);
    return make_float4(
        __fmul_rn(__fmul_rn(omf, omf), omf), __fadd_rn(__fsub_rn(__fmul_rn(3.0f, f3), __fmul_rn(6.0f, f2)), 4.0f),
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(-3.0f, f3), __fmul_rn(3.0f, f2)), __fmul_rn(3.0f, f)), 1.0f), f3);
}

// Filled by the block before its first strand.  Every length sample has
// 1/132 <= t <= 131/132, away from the end clamps of curve_eval_classic.
__device__ inline void fx_fill_tables(FxTables &tb, int P) {
    const int intervals = 2 * P + 4;
    const float step = __fdiv_rn(1.0f, static_cast<float>(intervals));
    for (int k = 1 + static_cast<int>(threadIdx.x); k < intervals; k += static_cast<int>(blockDim.x)) {
        int span = 0;
        tb.length_weights[k] = fx_weights(__fmul_rn(step, static_cast<float>(k)), P, span);
        tb.length_span[k] = span;
    }
    for (int cv = static_cast<int>(threadIdx.x); cv < P; cv += static_cast<int>(blockDim.x)) {
        tb.t[cv] = __fdiv_rn(static_cast<float>(cv), static_cast<float>(P - 1));
    }
}

// The four control points of span s (the end spans extrapolated), moved
// along the curve one span at a time as the parameter grows.
struct FxWindow {
    F3 p0, p1, p2, p3;
    int s;
    __device__ void start(const FxCurve &k, int P) {
        s = 0;
        p0 = xsub(xmul(k.p[0], 2.0f), k.p[1]);
        p1 = k.p[0];
        p2 = k.p[1];
        p3 = P == 2 ? xsub(xmul(k.p[1], 2.0f), k.p[0]) : k.p[2];
    }
    __device__ void seek(const FxCurve &k, int P, int span) {
        while (s < span) {
            p0 = p1;
            p1 = p2;
            p2 = p3;
            ++s;
            p3 = s + 2 == P ? xsub(xmul(k.p[P - 1], 2.0f), k.p[P - 2]) : k.p[s + 2];
        }
    }
    __device__ F3 at(float4 w) const {
        return xmul(xadd(xadd(xadd(xmul(p0, w.x), xmul(p1, w.y)), xmul(p2, w.z)), xmul(p3, w.w)), 1.0f / 6.0f);
    }
};

// spline_length_classic: 2P + 4 chords of the B-spline, summed in order.
__device__ inline float fx_spline_length(const FxCurve &k, int P, const FxTables &tb) {
    const int intervals = 2 * P + 4;
    FxWindow w;
    w.start(k, P);
    F3 previous = k.p[0];
    float length = 0.0f;
    for (int j = 1; j < intervals; ++j) {
        w.seek(k, P, tb.length_span[j]);
        const F3 current = w.at(tb.length_weights[j]);
        const F3 d = xsub(current, previous);
        length = __fadd_rn(length, __fsqrt_rn(xdot(d, d)));
        previous = current;
    }
    const F3 d = xsub(k.p[P - 1], previous);
    return __fadd_rn(length, __fsqrt_rn(xdot(d, d)));
}

// curve_polyline_length (xgen_classic_runtime.cpp:681-690).
__device__ inline float fx_polyline_length(const FxCurve &k, int P) {
    float length = 0.0f;
    for (int i = 1; i < P; ++i) {
        const F3 d = xsub(k.p[i], k.p[i - 1]);
        length = __fadd_rn(length, __fsqrt_rn(xdot(d, d)));
    }
    return length;
}

// scale_curve (xgen_classic_runtime.cpp:576-585): about the first point.
__device__ inline void fx_scale(FxCurve &k, int P, float s) {
    const F3 root = k.p[0];
    for (int i = 0; i < P; ++i) { k.p[i] = xadd(root, xmul(xsub(k.p[i], root), s)); }
}

__device__ inline F3 fx_normalize_or(F3 v, F3 fallback) {
    return xdot(v, v) >= 1.0e-12f ? xnormalize(v) : fallback;
}

// fallback_surface_u (generate.h:312-316) in the reference's rounding.
__device__ inline F3 fx_fallback_surface_u(F3 n) {
    const F3 axis = (n.z > -0.999f && n.z < 0.999f) ? F3{0.0f, 0.0f, 1.0f} : F3{0.0f, 1.0f, 0.0f};
    return xnormalize(xcross(n, axis));
}

// apply_noise (xgen_classic_runtime.cpp:897-1040) on one strand: the
// module's parameters, then the SgCurve frame transported from the surface
// normal along the current curve with gradient-noise displacement of every
// CV after the root, then preserveLength.  `c.t` is left at the last CV's t,
// as the reference's context is.  False where the reference throws.
__device__ inline bool fx_noise(FxCurve &k, int P, const DeviceExpression *m, const float4 *table,
                                const uint8_t *perm, const FxTables &tb, FxContext &c, F3 domain_position,
                                F3 surface_normal, F3 surface_tangent) {
    float raw = 0.0f;
    if (!fx_eval(m[kFxMask], table, perm, c, &raw)) { return false; }
    const float mask = std_clamp(raw, 0.0f, 1.0f);
    if (!(mask > 1.0e-6f)) { return true; }
    float frequency = 0.0f, correlation = 0.0f, preserve = 0.0f;
    if (!fx_eval(m[kFxFrequency], table, perm, c, &raw)) { return false; }
    frequency = std_max(raw, 0.0f);
    if (!fx_eval(m[kFxCorrelation], table, perm, c, &raw)) { return false; }
    correlation = std_clamp(__fmul_rn(raw, 0.01f), 0.0f, 1.0f);
    if (!fx_eval(m[kFxPreserve], table, perm, c, &raw)) { return false; }
    preserve = std_clamp(__fmul_rn(raw, 0.01f), 0.0f, 1.0f);
    if (!isfinite(frequency) || !isfinite(correlation) || !isfinite(preserve)) { return false; }
    const float original_length = fx_polyline_length(k, P);
    const float effective_frequency =
        original_length > 0.0f ? std_max(__fdiv_rn(0.5f, original_length), frequency) : frequency;
    const float decorrelation = __fsub_rn(1.0f, correlation);
    const float domain_scale = __fmul_rn(__fmul_rn(100.0f, decorrelation), decorrelation);
    const F3 domain = xmul(xadd(domain_position, F3{0.419276f, 0.184247f, 0.805721f}), domain_scale);
    constexpr float kMin = 1.0e-12f;
    surface_tangent = xdot(surface_tangent, surface_tangent) >= kMin ? xnormalize(surface_tangent)
                                                                    : fx_fallback_surface_u(surface_normal);
    // magnitude and magnitudeScale depend on the CV only through a ramp of
    // t; without one their value is the same at every CV and is taken once.
    const bool per_cv = m[kFxMagnitude].ramp_count != 0u || m[kFxMagnitudeScale].ramp_count != 0u;
    float magnitude = 0.0f;
    if (!per_cv) {
        float scale = 0.0f;
        c.t = 0.0f;
        if (!fx_eval(m[kFxMagnitude], table, perm, c, &magnitude)) { return false; }
        if (!fx_eval(m[kFxMagnitudeScale], table, perm, c, &scale)) { return false; }
        magnitude = __fmul_rn(__fmul_rn(std_max(magnitude, 0.0f), std_max(scale, 0.0f)), mask);
        if (!isfinite(magnitude)) { return false; }
    }
    F3 previous_base = k.p[0], current_base = k.p[0], next_base = k.p[1];
    F3 prior_tangent = fx_normalize_or(surface_normal, F3{0.0f, 1.0f, 0.0f});
    F3 transported = surface_tangent;
    float travelled = 0.0f;
    for (int cv = 0; cv < P; ++cv) {
        if (cv > 0) {
            const F3 d = xsub(current_base, previous_base);
            travelled = __fadd_rn(travelled, __fsqrt_rn(xdot(d, d)));
        }
        F3 next_tangent = prior_tangent;
        if (cv + 1 < P) {
            const F3 segment = xsub(next_base, current_base);
            if (xdot(segment, segment) >= kMin) { next_tangent = xnormalize(segment); }
        }
        const F3 axis = xcross(prior_tangent, next_tangent);
        const float axis_l2 = xdot(axis, axis);
        const float tangent_dot = std_clamp(xdot(prior_tangent, next_tangent), -1.0f, 1.0f);
        if (axis_l2 >= kMin) {
            const F3 rotation_axis = xmul(axis, __fdiv_rn(1.0f, __fsqrt_rn(axis_l2)));
            const float angle = acosf(tangent_dot);
            const float cosine = cosf(angle);
            const float sine = sinf(angle);
            const F3 rotated = xadd(xadd(xmul(transported, cosine), xmul(xcross(rotation_axis, transported), sine)),
                                    xmul(rotation_axis, __fmul_rn(xdot(rotation_axis, transported),
                                                                  __fsub_rn(1.0f, cosine))));
            transported = fx_normalize_or(rotated, F3{0.0f, 0.0f, 0.0f});
        }
        const F3 normal = transported;
        const F3 binormal = fx_normalize_or(xcross(normal, next_tangent), F3{0.0f, 0.0f, 0.0f});
        const F3 tangent = xcross(binormal, normal);
        c.t = tb.t[cv];
        if (per_cv) {
            float scale = 0.0f;
            if (!fx_eval(m[kFxMagnitude], table, perm, c, &magnitude)) { return false; }
            if (!fx_eval(m[kFxMagnitudeScale], table, perm, c, &scale)) { return false; }
            magnitude = __fmul_rn(__fmul_rn(std_max(magnitude, 0.0f), std_max(scale, 0.0f)), mask);
            if (!isfinite(magnitude)) { return false; }
        }
        if (cv > 0) {
            const float distance = __fmul_rn(travelled, effective_frequency);
            const float lx = __fmul_rn(
                __fsub_rn(classic_noise(table, __fadd_rn(domain.x, distance), domain.y, domain.z), 0.5f), magnitude);
            const float ly = __fmul_rn(
                __fsub_rn(classic_noise(table, domain.x, __fadd_rn(domain.y, distance), domain.z), 0.5f), magnitude);
            const float lz = __fmul_rn(
                __fsub_rn(classic_noise(table, domain.x, domain.y, __fadd_rn(domain.z, distance)), 0.5f), magnitude);
            k.p[cv] = xadd(xadd(xadd(current_base, xmul(normal, lx)), xmul(binormal, ly)), xmul(tangent, lz));
        }
        prior_tangent = next_tangent;
        previous_base = current_base;
        if (cv + 1 < P) {
            current_base = next_base;
            if (cv + 2 < P) { next_base = k.p[cv + 2]; }
        }
    }
    if (preserve > 0.001f) {
        const float noisy = fx_polyline_length(k, P);
        if (noisy > 0.0f) {
            const float target = __fadd_rn(__fmul_rn(original_length, preserve),
                                           __fmul_rn(noisy, __fsub_rn(1.0f, preserve)));
            if (fabsf(__fsub_rn(noisy, target)) >= 0.0001f) { fx_scale(k, P, __fdiv_rn(target, noisy)); }
        }
    }
    return true;
}

// The rebuild of both cuts: `source` resampled to P CVs at parameters
// i * cut / (P - 1), increasing, so the span window moves forward only.
__device__ inline void fx_resample(FxCurve &k, const FxCurve &source, int P, float cut) {
    const float step = __fdiv_rn(cut, static_cast<float>(P - 1));
    FxWindow w;
    w.start(source, P);
    k.p[0] = source.p[0];
    for (int i = 1; i < P; ++i) {
        const float t = __fmul_rn(step, static_cast<float>(i));
        if (t < 1.0e-7f) {
            k.p[i] = source.p[0];
        } else if (t > 1.0f - 1.0e-7f) {
            k.p[i] = source.p[P - 1];
        } else {
            int span = 0;
            const float4 weights = fx_weights(t, P, span);
            w.seek(source, P, span);
            k.p[i] = w.at(weights);
        }
    }
}

// cut_from_tip_and_rebuild (xgen_classic_runtime.cpp:692-748): walks the
// curve's spline back from the tip in 2P + 4 steps until `amount` of length
// is behind, then resamples the remaining span to P CVs.  Returns the cut
// parameter (0 when the whole curve is cut).
__device__ inline float fx_cut(FxCurve &k, FxCurve &scratch, int P, float amount) {
    for (int i = 0; i < P; ++i) { scratch.p[i] = k.p[i]; }
    const auto source = [&scratch](int i) { return scratch.p[i]; };
    float cut_parameter = 1.0f;
    bool collapsed = false;
    if (amount >= 1.0e-10f) {
        const float step = __fdiv_rn(1.0f, __fadd_rn(__fmul_rn(2.0f, static_cast<float>(P)), 4.0f));
        float previous_parameter = 1.0f;
        F3 previous = scratch.p[P - 1];
        float accumulated = 0.0f;
        // The walk ends within 2P + 5 steps (the parameter reaches 0).
        for (int guard = 0; guard < 4 * kFxMaxCvs + 16; ++guard) {
            const float parameter = std_max(__fsub_rn(previous_parameter, step), 0.0f);
            const F3 current = classic_curve_eval_by(source, P, parameter);
            const F3 d = xsub(previous, current);
            const float segment = __fsqrt_rn(xdot(d, d));
            accumulated = __fadd_rn(accumulated, segment);
            if (accumulated >= amount && segment > 0.0f) {
                cut_parameter = __fadd_rn(parameter, __fmul_rn(__fdiv_rn(__fsub_rn(accumulated, amount), segment),
                                                               __fsub_rn(previous_parameter, parameter)));
                break;
            }
            if (parameter <= 1.0e-10f) {
                cut_parameter = 0.0f;
                collapsed = true;
                break;
            }
            previous_parameter = parameter;
            previous = current;
        }
    }
    if (collapsed) {
        for (int i = 0; i < P; ++i) { k.p[i] = scratch.p[0]; }
    } else if (cut_parameter > 0.0f) {
        fx_resample(k, scratch, P, cut_parameter);
    }
    return cut_parameter;
}

// rotate_between (xgen_classic_runtime.cpp:1106-1118): `value` turned about
// from x to by `fraction` of the angle between them.
__device__ inline F3 fx_rotate_between(F3 value, F3 from, F3 to, float fraction) {
    F3 axis = xcross(from, to);
    const float axis_l2 = xdot(axis, axis);
    if (!(axis_l2 >= 1.0e-12f)) { return value; }
    axis = xmul(axis, __fdiv_rn(1.0f, __fsqrt_rn(axis_l2)));
    const float angle = __fmul_rn(acosf(std_clamp(xdot(from, to), -1.0f, 1.0f)), fraction);
    const float cosine = cosf(angle);
    const float sine = sinf(angle);
    return xadd(xadd(xmul(value, cosine), xmul(xcross(axis, value), sine)),
                xmul(axis, __fmul_rn(xdot(axis, value), __fsub_rn(1.0f, cosine))));
}

// cut_to_length_and_rebuild (xgen_classic_runtime.cpp:749-800): keeps the
// curve up to `target` of its length measured from the root, searching the
// 2P + 4 spline samples of the length measure, then rebuilds P CVs on
// [0, cut].  The curve is rebuilt even when the whole of it is kept.
__device__ inline void fx_cut_to_length(FxCurve &k, FxCurve &scratch, int P, float target, const FxTables &tb) {
    for (int i = 0; i < P; ++i) { scratch.p[i] = k.p[i]; }
    if (target <= 1.0e-10f) {
        for (int i = 1; i < P; ++i) { k.p[i] = scratch.p[0]; }
        return;
    }
    const int intervals = 2 * P + 4;
    const float step = __fdiv_rn(1.0f, static_cast<float>(intervals));
    float previous_parameter = 0.0f, accumulated = 0.0f, cut = 1.0f;
    F3 previous = scratch.p[0];
    FxWindow w;
    w.start(scratch, P);
    for (int sample = 1; sample <= intervals; ++sample) {
        const bool last = sample == intervals;
        const float parameter = last ? 1.0f : __fmul_rn(step, static_cast<float>(sample));
        F3 current = scratch.p[P - 1];
        if (!last) {
            w.seek(scratch, P, tb.length_span[sample]);
            current = w.at(tb.length_weights[sample]);
        }
        const F3 d = xsub(current, previous);
        const float segment = __fsqrt_rn(xdot(d, d));
        accumulated = __fadd_rn(accumulated, segment);
        if (accumulated >= target && segment > 0.0f) {
            cut = __fsub_rn(parameter, __fmul_rn(__fdiv_rn(__fsub_rn(accumulated, target), segment),
                                                 __fsub_rn(parameter, previous_parameter)));
            break;
        }
        previous_parameter = parameter;
        previous = current;
    }
    fx_resample(k, scratch, P, cut);
}

// The guide-noise axis of build_clump_noise_axis (xgen_classic_runtime.cpp:
// 1041-1181) after its early-out, for a guide with render CVs `axis` and
// source CVs `source`: begin() sets up the domain, the effective frequency
// and the frame transported from the guide's normal and tangent; step(cv)
// returns CV cv's displacement before the magnitude,
// sample_u * first + sample_v * second, and moves the frame on.
struct FxGuideNoise {
    F3 domain, tu, tv, ct;
    float frequency, travelled;

    __device__ void begin(const nxg_classic_clump_guides &cg, uint32_t g, const float *axis, const float *source,
                          int P, float raw_frequency, float raw_correlation) {
        const float f = std_max(raw_frequency, 0.0f);
        const float correlation = std_clamp(__fmul_rn(raw_correlation, 0.01f), 0.0f, 1.0f);
        float polyline = 0.0f;
        for (int cv = 1; cv < P; ++cv) {
            const F3 d = xsub(ld3(source, cv), ld3(source, cv - 1));
            polyline = __fadd_rn(polyline, __fsqrt_rn(xdot(d, d)));
        }
        frequency = polyline > 0.0f ? std_max(__fdiv_rn(0.5f, polyline), f) : f;
        const float decorrelation = __fsub_rn(1.0f, correlation);
        const float domain_scale = __fmul_rn(__fmul_rn(100.0f, decorrelation), decorrelation);
        const F3 position = cg.reference_positions ? ld3(cg.reference_positions, g) : ld3(source, 0);
        domain = xmul(xadd(position, F3{0.419276f, 0.184247f, 0.805721f}), domain_scale);
        F3 normal = ld3(cg.normals, g), tangent = ld3(cg.tangents, g);
        normal = xdot(normal, normal) > 1.0e-20f ? xnormalize(normal) : F3{0.0f, 1.0f, 0.0f};
        tangent = xdot(tangent, tangent) > 1.0e-20f ? xnormalize(tangent) : fx_fallback_surface_u(normal);
        tu = tangent;
        tv = xcross(normal, tangent);
        ct = normal;
        const F3 first_segment = xsub(ld3(axis, 1), ld3(axis, 0));
        if (xdot(first_segment, first_segment) > 1.0e-20f) { ct = xnormalize(first_segment); }
        if (xdot(normal, ct) < 0.99999f) {
            tu = fx_rotate_between(tu, normal, ct, 1.0f);
            tv = fx_rotate_between(tv, normal, ct, 1.0f);
        }
        travelled = 0.0f;
    }

    __device__ F3 step(const float *axis, const float *source, int P, int cv, const float4 *table) {
        const F3 d = xsub(ld3(source, cv), ld3(source, cv - 1));
        travelled = __fadd_rn(travelled, __fsqrt_rn(xdot(d, d)));
        F3 su = tu, sv = tv, nt = ct;
        bool advance = false;
        if (cv + 1 < P) {
            const F3 segment = xsub(ld3(axis, cv + 1), ld3(axis, cv));
            if (xdot(segment, segment) > 1.0e-20f) {
                nt = xnormalize(segment);
                if (fabsf(xdot(ct, nt)) < 0.99999f) {
                    su = fx_rotate_between(tu, ct, nt, 0.5f);
                    sv = fx_rotate_between(tv, ct, nt, 0.5f);
                    advance = true;
                } else {
                    ct = nt;
                }
            }
        }
        const float distance = __fmul_rn(travelled, frequency);
        const float first = __fsub_rn(classic_noise(table, __fadd_rn(domain.x, distance), domain.y, domain.z), 0.5f);
        const float second = __fsub_rn(classic_noise(table, domain.x, domain.y, __fadd_rn(domain.z, distance)), 0.5f);
        const F3 unit = xadd(xmul(su, first), xmul(sv, second));
        if (advance) {
            tu = fx_rotate_between(tu, ct, nt, 1.0f);
            tv = fx_rotate_between(tv, ct, nt, 1.0f);
            ct = nt;
        }
        return unit;
    }
};

// Guide-noise table entries: CV 0 of each guide holds (noise, flags), CVs
// 1.. hold (the unit displacement, the raw noiseScale).
enum : uint32_t { kGuideNoiseFailed = 1u, kGuideRestFailed = 2u };

// The guide's context for its noise programs: its uv and SeExpr prefix.
__device__ inline void fx_guide_context(FxContext &gc, const nxg_classic_clump_guides &cg, uint32_t g) {
    gc.u = cg.uvs[2u * g];
    gc.v = cg.uvs[2u * g + 1u];
    gc.prefix = cg.random_prefixes[g];
    gc.has_prefix = 1u;
}

// The ClumpingFX step for one strand (xgen_classic_runtime.cpp:1680-1788),
// with world-space guides: the mask; the guide-noise axis (from the
// module's per-guide table when `shared`, else evaluated here in the guide's
// context); the cut to the guide's length; the pull of every CV after the
// root toward the guide's rebuilt CV by mask * clump * (1 - 2 clumpScale);
// the guide noise, times (mask * noise) * max(noiseScale, 0), added on top.
// The noise axis depends only on the guide, so it is taken in the same pass
// over the CVs as the pull.  `clumped` reports whether the curve changed
// (the reference recomputes cLength only then).  False where the reference
// throws; *code says why.
__device__ __noinline__ bool fx_clump(FxCurve &k, FxCurve &scratch, int P, const DeviceExpression *m,
                                      const nxg_classic_clump_guides &cg, bool shared, uint32_t strand,
                                      const float4 *table, const uint8_t *perm, const FxTables &tb, FxContext &c,
                                      uint32_t *code, bool *clumped) {
    *clumped = false;
    const uint32_t g = cg.strand_guides[strand];
    if (g == kInvalid) { return true; }
    if (g >= cg.guide_count) {
        *code = NXG_ERROR_INVALID_ARGUMENT;
        return false;
    }
    const float *axis = cg.render_axes + 3u * static_cast<uint64_t>(g) * static_cast<uint32_t>(P);
    const float *source = cg.axes + 3u * static_cast<uint64_t>(g) * static_cast<uint32_t>(P);
    const float4 *entries = shared ? reinterpret_cast<const float4 *>(cg.noise_table) +
                                         static_cast<uint64_t>(g) * static_cast<uint32_t>(P)
                                   : nullptr;
    c.t = 0.0f;
    float raw = 0.0f;
    if (!fx_eval(m[kClumpMask], table, perm, c, &raw)) { return false; }
    const float mask = std_clamp(raw, 0.0f, 1.0f);
    if (mask <= 0.0f) { return true; }
    FxContext gc = c;
    fx_guide_context(gc, cg, g);
    float noise = 0.0f;
    uint32_t flags = 0u;
    if (shared) {
        const float4 head = entries[0];
        noise = head.x;
        flags = __float_as_uint(head.y);
        if (flags & kGuideNoiseFailed) { return false; }
    } else {
        if (!fx_eval(m[kClumpNoise], table, perm, gc, &raw)) { return false; }
        noise = std_max(raw, 0.0f);
    }
    const bool noisy = noise > 1.0e-5f && mask > 1.0e-4f;
    FxGuideNoise gn;
    if (noisy) {
        if (shared) {
            if (flags & kGuideRestFailed) { return false; }
        } else {
            float raw_frequency = 0.0f, raw_correlation = 0.0f;
            if (!fx_eval(m[kClumpNoiseFrequency], table, perm, gc, &raw_frequency) ||
                !fx_eval(m[kClumpNoiseCorrelation], table, perm, gc, &raw_correlation)) {
                return false;
            }
            gn.begin(cg, g, axis, source, P, raw_frequency, raw_correlation);
        }
    }
    fx_cut_to_length(k, scratch, P, cg.spline_lengths[g], tb);
    c.c_length = fx_spline_length(k, P, tb);
    if (!fx_eval(m[kClumpAmount], table, perm, c, &raw)) { return false; }
    const float pull = __fmul_rn(mask, std_clamp(raw, 0.0f, 1.0f));
    const float strength = __fmul_rn(mask, noise);
    // clumpScale depends on the CV only through a ramp of t; without one it
    // is taken once.
    const bool scale_per_cv = m[kClumpScale].ramp_count != 0u;
    float factor = 0.0f;
    if (!scale_per_cv) {
        float scale = 0.0f;
        c.t = tb.t[1];
        if (!fx_eval(m[kClumpScale], table, perm, c, &scale)) { return false; }
        factor = __fmul_rn(pull, __fsub_rn(1.0f, __fmul_rn(2.0f, scale)));
    }
    for (int cv = 1; cv < P; ++cv) {
        F3 displacement{0.0f, 0.0f, 0.0f};
        if (noisy) {
            F3 unit;
            float raw_scale = 0.0f;
            if (shared) {
                const float4 e = entries[cv];
                unit = F3{e.x, e.y, e.z};
                raw_scale = e.w;
            } else {
                gc.t = tb.t[cv];
                if (!fx_eval(m[kClumpNoiseScale], table, perm, gc, &raw_scale)) { return false; }
                unit = gn.step(axis, source, P, cv, table);
            }
            const float magnitude = __fmul_rn(strength, std_max(raw_scale, 0.0f));
            if (!isfinite(magnitude)) { return false; }
            displacement = xmul(unit, magnitude);
        }
        c.t = tb.t[cv];
        if (scale_per_cv) {
            float scale = 0.0f;
            if (!fx_eval(m[kClumpScale], table, perm, c, &scale)) { return false; }
            factor = __fmul_rn(pull, __fsub_rn(1.0f, __fmul_rn(2.0f, scale)));
        }
        const F3 current = k.p[cv];
        k.p[cv] = xadd(xadd(current, xmul(xsub(ld3(axis, cv), current), factor)), displacement);
    }
    *clumped = true;
    return true;
}

__device__ inline void fx_fail(uint32_t *status, uint32_t code = NXG_ERROR_EXPRESSION_DOMAIN) {
    atomicCAS(status, 0u, code);
    atomicAdd(status + 1, 1u);
}

// One thread per strand (the per-strand body of
// apply_xgen_classic_float_runtime_plan_cpu, xgen_classic_runtime.cpp:
// 1614-1868).  A strand whose point count is not P is left alone; a dropped
// strand's count becomes 0 and its points stay as they were.
__global__ void __launch_bounds__(128, 5) classic_fx_kernel(const FxArgs k) {
    __shared__ float4 table[256];
    __shared__ uint8_t perm[256];
    __shared__ FxTables tb;
    const int P = static_cast<int>(k.P);
    stage_classic_tables(table, perm);
    fx_fill_tables(tb, P);
    __syncthreads();
    const FxPlan &plan = *k.plan;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k.count; i += gridDim.x * blockDim.x) {
        if (k.point_counts[i] != k.P) { continue; }
        const uint32_t *rw = k.roots + 12u * static_cast<uint64_t>(i);
        const F3 root_position = {__uint_as_float(rw[0]), __uint_as_float(rw[1]), __uint_as_float(rw[2])};
        const F3 root_normal = {__uint_as_float(rw[3]), __uint_as_float(rw[4]), __uint_as_float(rw[5])};
        FxContext c;
        c.pref = root_position;
        c.id = static_cast<float>(k.first_id + i);
        c.u = __uint_as_float(rw[6]);
        c.v = __uint_as_float(rw[7]);
        const uint32_t face = rw[11] == kInvalid ? rw[8] : rw[11];  // surface_face_id, else the triangle
        c.face_seed = plan.uses_random ? classic_face_seed(plan.description_id, plan.patch_seed, face, perm) : 0.0f;
        c.c_length = 0.0f;
        c.c_width = 0.0f;
        c.t = 0.0f;
        c.prefix = k.random_prefixes ? k.random_prefixes[i] : 0u;
        c.has_prefix = k.random_prefixes != nullptr;
        if (plan.uses_random && !k.random_prefixes) {  // rand() needs the strands' SeExpr prefixes
            fx_fail(k.status, NXG_ERROR_INVALID_ARGUMENT);
            continue;
        }
        float4 *pts = k.points + static_cast<uint64_t>(i) * k.P;
        FxCurve curve, scratch;
        for (int j = 0; j < P; ++j) { curve.p[j] = xyz(pts[j]); }
        const float first_radius = pts[0].w;
        c.c_length = fx_spline_length(curve, P, tb);
        bool ok = true;
        if (plan.length.present) {
            float s = 0.0f;
            ok = fx_eval(plan.length, table, perm, c, &s) && s >= 0.0f;
            if (ok) {
                fx_scale(curve, P, s);
                c.c_length = __fmul_rn(c.c_length, s);
            }
        }
        float raw_width = 0.0f;
        if (ok) {
            if (plan.width.present) {
                ok = fx_eval(plan.width, table, perm, c, &raw_width);
            } else {
                raw_width = k.radius_scale > 0.0f ? __fdiv_rn(__fmul_rn(2.0f, first_radius), k.radius_scale) : 0.0f;
            }
        }
        if (!ok) {
            fx_fail(k.status);
            continue;
        }
        // XgSplinePrimitive::mkGeometry's rejection before any FX.
        if (c.c_length < 1.0e-4f || raw_width < 1.0e-4f) {
            k.point_counts[i] = 0u;
            continue;
        }
        c.c_width = raw_width;
        bool keep = true;
        uint32_t code = NXG_ERROR_EXPRESSION_DOMAIN;
        uint32_t clump = 0u;
        for (uint32_t e = 0; ok && e < plan.effect_count; ++e) {
            bool changed = true;
            if (plan.effect_type[e] == NXG_CLASSIC_FX_CLUMP) {
                if (clump >= k.clump_count || P < 3) {  // the module's guides, of at least 3 CVs
                    ok = false;
                    code = NXG_ERROR_INVALID_ARGUMENT;
                } else {
                    const nxg_classic_clump_guides guides = k.clumps[clump];
                    const bool shared = guides.noise_table != nullptr && plan.guide_noise_shared[e] != 0u;
                    ok = fx_clump(curve, scratch, P, plan.effect[e], guides, shared, i, table, perm, tb, c, &code,
                                  &changed);
                }
                ++clump;
            } else if (plan.effect_type[e] == NXG_CLASSIC_FX_NOISE && k.surface_tangents == nullptr) {
                ok = false;  // NoiseFX needs the strand's surface tangent
                code = NXG_ERROR_INVALID_ARGUMENT;
            } else if (plan.effect_type[e] == NXG_CLASSIC_FX_NOISE) {
                const F3 domain = k.noise_domains
                    ? F3{k.noise_domains[3u * i], k.noise_domains[3u * i + 1u], k.noise_domains[3u * i + 2u]}
                    : curve.p[0];
                const F3 tangent = {k.surface_tangents[3u * i], k.surface_tangents[3u * i + 1u],
                                    k.surface_tangents[3u * i + 2u]};
                ok = fx_noise(curve, P, plan.effect[e], table, perm, tb, c, domain, root_normal, tangent);
            } else {
                float amount = 0.0f;
                ok = fx_eval(plan.effect[e][0], table, perm, c, &amount);
                if (ok && fx_cut(curve, scratch, P, std_max(amount, 0.0f)) < 1.0e-4f) { keep = false; }
            }
            // cLength after this effect, where a later program reads it.
            if (ok && changed && plan.length_after[e]) { c.c_length = fx_spline_length(curve, P, tb); }
        }
        float taper = 0.0f, taper_start = 0.0f;
        if (ok && plan.taper.present) { ok = fx_eval(plan.taper, table, perm, c, &taper); }
        if (ok && plan.taper_start.present) { ok = fx_eval(plan.taper_start, table, perm, c, &taper_start); }
        const bool profile = plan.width.present || plan.taper.present || plan.taper_start.present ||
                             plan.width_ramp.present;
        float radii[kFxMaxCvs];
        for (int j = 0; ok && j < P; ++j) {
            float radius = pts[j].w;
            if (profile) {
                c.t = tb.t[j];
                float scale = 1.0f;
                if (c.t > taper_start && taper_start < 1.0f) {
                    scale = __fmul_rn(scale, __fsub_rn(1.0f, __fmul_rn(taper, __fdiv_rn(__fsub_rn(c.t, taper_start),
                                                                                          __fsub_rn(1.0f, taper_start)))));
                }
                if (plan.width_ramp.present) {
                    float ramp = 0.0f;
                    ok = fx_eval(plan.width_ramp, table, perm, c, &ramp);
                    scale = __fmul_rn(scale, ramp);
                }
                const float raw_diameter = __fmul_rn(c.c_width, scale);
                ok = ok && isfinite(raw_diameter);
                radius = __fmul_rn(__fmul_rn(0.5f, std_max(raw_diameter, 0.0f)), k.radius_scale);
            }
            radii[j] = radius;
        }
        if (!ok) {
            fx_fail(k.status, code);
            continue;
        }
        for (int j = 0; j < P; ++j) { pts[j] = make_float4(curve.p[j].x, curve.p[j].y, curve.p[j].z, radii[j]); }
        if (!keep) { k.point_counts[i] = 0u; }
    }
}

// The guide-noise table of the plan's ClumpingFX module number `module`,
// one thread per guide: the guide noise evaluated once per guide instead of
// once per strand, when the module's guide-noise programs read no per-strand
// input.  Entry 0 holds (noise, failure flags); entries 1.. the unit
// displacement and the raw noiseScale.  The early-outs and failures of
// build_clump_noise_axis are kept as flags, for the strands to apply with
// their own mask.
__global__ void __launch_bounds__(128) clump_guide_noise_kernel(const FxPlan *plan_ptr, uint32_t module,
                                                                const nxg_classic_clump_guides cg, uint32_t P) {
    __shared__ float4 table[256];
    __shared__ uint8_t perm[256];
    __shared__ FxTables tb;
    stage_classic_tables(table, perm);
    fx_fill_tables(tb, static_cast<int>(P));
    __syncthreads();
    const FxPlan &plan = *plan_ptr;
    int effect = -1;
    for (uint32_t e = 0, seen = 0; e < plan.effect_count; ++e) {
        if (plan.effect_type[e] == NXG_CLASSIC_FX_CLUMP && seen++ == module) { effect = static_cast<int>(e); }
    }
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (effect < 0 || !plan.guide_noise_shared[effect] || g >= cg.guide_count) { return; }
    const DeviceExpression *m = plan.effect[effect];
    const int n = static_cast<int>(P);
    const float *axis = cg.render_axes + 3u * static_cast<uint64_t>(g) * P;
    const float *source = cg.axes + 3u * static_cast<uint64_t>(g) * P;
    float4 *out = reinterpret_cast<float4 *>(cg.noise_table) + static_cast<uint64_t>(g) * P;
    FxContext gc{};
    fx_guide_context(gc, cg, g);
    uint32_t flags = 0u;
    float raw = 0.0f, noise = 0.0f;
    if (!fx_eval(m[kClumpNoise], table, perm, gc, &raw)) {
        flags = kGuideNoiseFailed;
    } else {
        noise = std_max(raw, 0.0f);
    }
    if (flags == 0u && noise > 1.0e-5f) {
        float raw_frequency = 0.0f, raw_correlation = 0.0f;
        if (!fx_eval(m[kClumpNoiseFrequency], table, perm, gc, &raw_frequency) ||
            !fx_eval(m[kClumpNoiseCorrelation], table, perm, gc, &raw_correlation)) {
            flags = kGuideRestFailed;
        } else {
            FxGuideNoise gn;
            gn.begin(cg, g, axis, source, n, raw_frequency, raw_correlation);
            for (int cv = 1; cv < n; ++cv) {
                gc.t = tb.t[cv];
                float raw_scale = 0.0f;
                if (!fx_eval(m[kClumpNoiseScale], table, perm, gc, &raw_scale)) {
                    flags = kGuideRestFailed;
                    break;
                }
                const F3 unit = gn.step(axis, source, n, cv, table);
                out[cv] = make_float4(unit.x, unit.y, unit.z, raw_scale);
            }
        }
    }
    out[0] = make_float4(noise, __uint_as_float(flags), 0.0f, 0.0f);
}

// prepare_xgen_classic_clump_runtime_data (xgen_classic_runtime.cpp:839-892)
// for world-space guides: one thread per guide.
__global__ void __launch_bounds__(128) clump_prepare_kernel(const float *axes, uint32_t guides, uint32_t P,
                                                            float *render_axes, float *lengths) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= guides) { return; }
    const float *src = axes + 3u * static_cast<uint64_t>(g) * P;
    float *out = render_axes + 3u * static_cast<uint64_t>(g) * P;
    const auto source = [src](int i) { return ld3(src, static_cast<uint32_t>(i)); };
    const int n = static_cast<int>(P);
    const auto put = [out](int i, F3 v) {
        out[3 * i] = v.x;
        out[3 * i + 1] = v.y;
        out[3 * i + 2] = v.z;
    };
    put(0, source(0));
    for (int cv = 1; cv + 1 < n; ++cv) {
        put(cv, classic_curve_eval_by(source, n, __fdiv_rn(static_cast<float>(cv), static_cast<float>(n - 1))));
    }
    put(n - 1, source(n - 1));
    lengths[g] = classic_spline_length_by(source, n);
}

} // namespace dev
} // namespace nxg

namespace nxg {
namespace {

uint32_t pack_optional(const nxg_expression *e, DeviceExpression &d) {
    std::memset(&d, 0, sizeof d);
    return e ? pack_device_expression(e, d) : NXG_ERROR_NONE;
}

// xgen_runtime_face_seed's name seed: the text after the last ':'.
float name_seed(const char *name) {
    const char *text = name ? name : "";
    for (const char *p = text; *p; ++p) {
        if (*p == ':') { text = p + 1; }
    }
    return static_cast<float>(nxg_xgen_string_seed(text));
}

} // namespace
} // namespace nxg

extern "C" {

uint64_t nxg_classic_fx_plan_bytes(void) { return (sizeof(nxg::dev::FxPlan) + 255u) / 256u * 256u; }

uint32_t nxg_classic_fx_plan_upload(const nxg_classic_fx_plan *plan, void *device_plan, uint64_t bytes,
                                    void *stream) {
    using nxg::dev::FxPlan;
    if (!plan || !device_plan || bytes < sizeof(FxPlan) || plan->effect_count > NXG_CLASSIC_MAX_FX ||
        (plan->effect_count && !plan->effects)) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    std::vector<unsigned char> storage(sizeof(FxPlan));
    FxPlan &host = *reinterpret_cast<FxPlan *>(storage.data());
    uint32_t error = NXG_ERROR_NONE;
    if ((error = nxg::pack_optional(plan->length, host.length)) ||
        (error = nxg::pack_optional(plan->width, host.width)) ||
        (error = nxg::pack_optional(plan->taper, host.taper)) ||
        (error = nxg::pack_optional(plan->taper_start, host.taper_start)) ||
        (error = nxg::pack_optional(plan->width_ramp, host.width_ramp))) {
        return error;
    }
    host.effect_count = plan->effect_count;
    for (uint32_t e = 0; e < plan->effect_count; ++e) {
        const nxg_classic_fx &fx = plan->effects[e];
        host.effect_type[e] = fx.type;
        if (fx.type == NXG_CLASSIC_FX_NOISE) {
            const nxg_expression *programs[] = {fx.mask, fx.magnitude, fx.magnitude_scale,
                                                fx.frequency, fx.correlation, fx.preserve_length};
            for (int k = 0; k < 6; ++k) {
                if (!programs[k]) { return NXG_ERROR_INVALID_ARGUMENT; }
                if ((error = nxg::pack_optional(programs[k], host.effect[e][k]))) { return error; }
            }
        } else if (fx.type == NXG_CLASSIC_FX_CUT) {
            if (!fx.amount) { return NXG_ERROR_INVALID_ARGUMENT; }
            if ((error = nxg::pack_optional(fx.amount, host.effect[e][0]))) { return error; }
        } else if (fx.type == NXG_CLASSIC_FX_CLUMP) {
            const nxg_expression *programs[nxg::dev::kFxSlots] = {fx.mask, fx.clump, fx.clump_scale, fx.noise,
                                                                 fx.noise_scale, fx.noise_frequency,
                                                                 fx.noise_correlation};
            for (int k = 0; k < nxg::dev::kFxSlots; ++k) {
                if (!programs[k]) { return NXG_ERROR_INVALID_ARGUMENT; }
                if ((error = nxg::pack_optional(programs[k], host.effect[e][k]))) { return error; }
            }
        } else {
            return NXG_ERROR_INVALID_ARGUMENT;
        }
    }
    // A ClumpingFX module's guide noise is shared by the strands of a guide
    // when its programs bind none of $id, $cLength, $cWidth, noise($Prefg).
    for (uint32_t e = 0; e < plan->effect_count; ++e) {
        if (host.effect_type[e] != NXG_CLASSIC_FX_CLUMP) { continue; }
        bool shared = true;
        for (int slot : {nxg::dev::kClumpNoise, nxg::dev::kClumpNoiseScale, nxg::dev::kClumpNoiseFrequency,
                         nxg::dev::kClumpNoiseCorrelation}) {
            const nxg::DeviceExpression &d = host.effect[e][slot];
            for (uint32_t i = 0; i < d.input_count; ++i) {
                const uint8_t b = d.input_binding[i];
                shared = shared && b != nxg::kBindPrefNoise && b != nxg::kBindId && b != nxg::kBindCLength &&
                         b != nxg::kBindCWidth;
            }
        }
        host.guide_noise_shared[e] = shared ? 1u : 0u;
    }
    // cLength is recomputed after an effect only for a program that follows
    // it: a later effect's, or the width profile's.
    uint32_t later = host.taper.uses_clength | host.taper_start.uses_clength | host.width_ramp.uses_clength;
    for (uint32_t e = plan->effect_count; e-- > 0u;) {
        host.length_after[e] = later;
        for (int k = 0; k < nxg::dev::kFxSlots; ++k) { later |= host.effect[e][k].uses_clength; }
    }
    uint32_t random = host.length.uses_random | host.width.uses_random | host.taper.uses_random |
                      host.taper_start.uses_random | host.width_ramp.uses_random;
    for (uint32_t e = 0; e < plan->effect_count; ++e) {
        for (int k = 0; k < nxg::dev::kFxSlots; ++k) { random |= host.effect[e][k].uses_random; }
    }
    host.uses_random = random;
    host.description_id = static_cast<float>(plan->description_id);
    host.patch_seed = nxg::name_seed(plan->description_name);
    nxg::set_last_cuda_error(0);
    // From pageable memory: the copy is staged before the call returns.
    return nxg::record_cuda(cudaMemcpyAsync(device_plan, storage.data(), sizeof(FxPlan), cudaMemcpyHostToDevice,
                                            static_cast<cudaStream_t>(stream)));
}

uint32_t nxg_classic_fx_apply(const void *device_plan, const nxg_classic_fx_curves *curves,
                              uint32_t *device_status, void *stream) {
    if (!device_plan || !curves || !device_status || !curves->points || !curves->point_counts || !curves->roots) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    if (curves->cvs_per_strand < 2u || curves->cvs_per_strand > NXG_CLASSIC_MAX_FX_CVS ||
        !std::isfinite(curves->radius_scale) || curves->radius_scale < 0.0f) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    if (reinterpret_cast<std::uintptr_t>(curves->points) % 16u != 0u ||
        reinterpret_cast<std::uintptr_t>(curves->roots) % 4u != 0u ||
        reinterpret_cast<std::uintptr_t>(device_plan) % 256u != 0u) {
        return NXG_ERROR_MISALIGNED_OUTPUT;
    }
    if (curves->clump_count > NXG_CLASSIC_MAX_FX || (curves->clump_count && !curves->clumps)) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    for (uint32_t m = 0; m < curves->clump_count; ++m) {
        const nxg_classic_clump_guides &g = curves->clumps[m];
        if (!g.strand_guides ||
            (g.guide_count && (!g.axes || !g.render_axes || !g.spline_lengths || !g.normals || !g.tangents ||
                               !g.uvs || !g.random_prefixes))) {
            return NXG_ERROR_INVALID_ARGUMENT;
        }
    }
    if (curves->strand_count == 0u) { return NXG_ERROR_NONE; }
    nxg::dev::FxArgs k{};
    k.random_prefixes = curves->random_prefixes;
    k.clump_count = curves->clump_count;
    for (uint32_t m = 0; m < curves->clump_count; ++m) { k.clumps[m] = curves->clumps[m]; }
    k.plan = static_cast<const nxg::dev::FxPlan *>(device_plan);
    k.points = reinterpret_cast<float4 *>(curves->points);
    k.point_counts = curves->point_counts;
    k.roots = static_cast<const uint32_t *>(curves->roots);
    k.surface_tangents = curves->surface_tangents;
    k.noise_domains = curves->noise_domains;
    k.count = curves->strand_count;
    k.P = curves->cvs_per_strand;
    k.first_id = curves->first_id;
    k.radius_scale = curves->radius_scale;
    k.status = device_status;
    nxg::set_last_cuda_error(0);
    const uint32_t threads = 128u;
    const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>(
        (uint64_t{k.count} + threads - 1u) / threads, static_cast<uint64_t>(nxg::device_sm_count()) * 16u));
    for (uint32_t m = 0; m < curves->clump_count; ++m) {
        const nxg_classic_clump_guides &g = curves->clumps[m];
        if (!g.noise_table || g.guide_count == 0u) { continue; }
        nxg::dev::clump_guide_noise_kernel<<<(g.guide_count + 127u) / 128u, 128u, 0,
                                             static_cast<cudaStream_t>(stream)>>>(k.plan, m, g, k.P);
    }
    nxg::dev::classic_fx_kernel<<<blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(k);
    return nxg::record_cuda(cudaGetLastError());
}

uint32_t nxg_classic_clump_prepare(const float *axes, uint32_t guide_count, uint32_t cvs_per_guide,
                                   float *render_axes, float *spline_lengths, void *stream) {
    if (cvs_per_guide < 3u || cvs_per_guide > NXG_CLASSIC_MAX_FX_CVS ||
        (guide_count && (!axes || !render_axes || !spline_lengths))) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    if (guide_count == 0u) { return NXG_ERROR_NONE; }
    nxg::set_last_cuda_error(0);
    nxg::dev::clump_prepare_kernel<<<(guide_count + 127u) / 128u, 128u, 0, static_cast<cudaStream_t>(stream)>>>(
        axes, guide_count, cvs_per_guide, render_axes, spline_lengths);
    return nxg::record_cuda(cudaGetLastError());
}

} // extern "C"
