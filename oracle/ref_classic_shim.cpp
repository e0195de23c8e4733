// ref_classic_shim.cpp -- extern "C" shim over the reference's scalar
// expression compiler/evaluator and its Classic float runtime.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile links this file with the
// unmodified reference sources src/xgen_expression.cpp,
// src/xgen_classic_runtime.cpp and their support files (xgen_classic.cpp,
// context.cpp, task_executor.cpp) into oracle/_ref/libnxg_ref.so.  Tests pin
// the product's compiler, device evaluator and fused Classic application
// against it; make_permutation_table.py derives the SeExpr permutation from
// ref_seexpr_hash_finish.  Nothing here is product code.
#include "nanoxgen/asset.h"
#include "nanoxgen/context.h"
#include "nanoxgen/xgen_classic.h"
#include "nanoxgen/xgen_classic_runtime.h"
#include "nanoxgen/xgen_expression.h"

#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

using namespace nanoxgen;

namespace {

void copy_text(const std::string &text, char *out, std::uint64_t cap) {
    if (!out || cap == 0u) { return; }
    const std::size_t n = std::min<std::size_t>(text.size(), static_cast<std::size_t>(cap - 1u));
    std::memcpy(out, text.data(), n);
    out[n] = '\0';
}

const XgenFloatExpressionProgram *program_of(const void *p) {
    return static_cast<const XgenFloatExpressionProgram *>(p);
}

} // namespace

extern "C" {

// compile_xgen_scalar_expression + make_xgen_float_expression_program.
void *ref_expr_compile(const char *source, const char *name, const char *type, char *msg, std::uint64_t cap) {
    try {
        XgenExpressionCompileOptions options{};
        options.expression_name = name ? name : "";
        options.object_type = type ? type : "";
        auto *p = new XgenFloatExpressionProgram(
            make_xgen_float_expression_program(compile_xgen_scalar_expression(source, options)));
        copy_text("", msg, cap);
        return p;
    } catch (const std::exception &e) {
        copy_text(e.what(), msg, cap);
        return nullptr;
    }
}

void ref_expr_free(void *p) { delete static_cast<XgenFloatExpressionProgram *>(p); }

// instructions, operands, inputs, ramps, ramp points, result, seed, rand calls
void ref_expr_info(const void *p, std::uint32_t *out) {
    const XgenFloatExpressionProgram &g = *program_of(p);
    out[0] = static_cast<std::uint32_t>(g.instructions.size());
    out[1] = static_cast<std::uint32_t>(g.operands.size());
    out[2] = static_cast<std::uint32_t>(g.inputs.size());
    out[3] = static_cast<std::uint32_t>(g.ramps.size());
    out[4] = static_cast<std::uint32_t>(g.ramp_points.size());
    out[5] = g.result;
    out[6] = g.expression_seed;
    out[7] = g.random_call_count;
}

// op, operand offset, operand count, auxiliary; immediate separately.
void ref_expr_instruction(const void *p, std::uint32_t index, std::uint32_t *out, float *immediate) {
    const XgenFloatScalarInstruction &in = program_of(p)->instructions.at(index);
    out[0] = static_cast<std::uint32_t>(in.op);
    out[1] = in.operand_offset;
    out[2] = in.operand_count;
    out[3] = in.auxiliary;
    *immediate = in.immediate;
}

std::uint32_t ref_expr_operand(const void *p, std::uint32_t index) { return program_of(p)->operands.at(index); }

void ref_expr_ramp_point(const void *p, std::uint32_t index, float *position, float *value, std::uint32_t *interp) {
    const XgenFloatRampPoint &rp = program_of(p)->ramp_points.at(index);
    *position = rp.position;
    *value = rp.value;
    *interp = rp.interpolation;
}

const char *ref_expr_input(const void *p, std::uint32_t index) { return program_of(p)->inputs.at(index).c_str(); }

// evaluate_xgen_scalar_expression_float over `count` rows; inputs is
// row-major [count x input_count].  ok[i] = 0 where the reference throws.
void ref_expr_eval_batch(const void *p, const float *inputs, std::uint32_t input_count, std::uint64_t count,
                         const float *u, const float *v, const float *face_seed, float t,
                         const std::uint32_t *random_prefix, float *out, std::uint8_t *ok) {
    const XgenFloatExpressionProgram &g = *program_of(p);
    std::vector<float> scratch(g.instructions.size());
    for (std::uint64_t i = 0; i < count; ++i) {
        XgenExpressionFloatContext context{};
        context.inputs = std::span<const float>(inputs + i * input_count, input_count);
        context.u = u ? u[i] : 0.0f;
        context.v = v ? v[i] : 0.0f;
        context.face_seed = face_seed ? face_seed[i] : 0.0f;
        context.t = t;
        context.random_prefix = random_prefix ? random_prefix[i] : 0u;
        context.has_random_prefix = random_prefix != nullptr;
        try {
            out[i] = evaluate_xgen_scalar_expression_float(g, context, scratch);
            ok[i] = 1u;
        } catch (const std::exception &) {
            out[i] = 0.0f;
            ok[i] = 0u;
        }
    }
}

std::uint32_t ref_seexpr_hash_finish(std::uint32_t state) { return xgen_seexpr_hash_finish(state); }

std::uint32_t ref_runtime_hash_component(float argument) { return xgen_runtime_hash_component(argument); }

float ref_runtime_hash(const float *arguments, std::uint32_t count) {
    return xgen_runtime_hash(std::span<const float>(arguments, count));
}

float ref_runtime_face_seed(std::uint32_t description_id, const char *patch, std::uint32_t face) {
    return xgen_runtime_face_seed(description_id, patch ? patch : "", face);
}

std::uint32_t ref_string_seed(const char *text) { return xgen_string_seed(text ? text : ""); }

// xgen_classic_noise_float(p * frequency) for n points (xyz interleaved).
void ref_classic_noise_batch(const float *xyz, std::uint64_t n, float frequency, float *out) {
    for (std::uint64_t i = 0; i < n; ++i) {
        const Vec3 p{xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
        out[i] = xgen_classic_noise_float(p * frequency);
    }
}

// compile_xgen_classic_float_runtime_plan for a description whose
// SplinePrimitive carries the given length / width expressions (either may
// be NULL).  msg receives the fallback reasons joined by '\n'.
void *ref_classic_plan(const char *length, const char *width, std::uint32_t description_id,
                       const char *description_name, char *msg, std::uint64_t cap) {
    try {
        ClassicDescription description{};
        description.name = description_name ? description_name : "description";
        description.attributes.push_back({"descriptionId", std::to_string(description_id), 0u});
        ClassicObject primitive{};
        primitive.type = "SplinePrimitive";
        if (length) { primitive.attributes.push_back({"length", length, 0u}); }
        if (width) { primitive.attributes.push_back({"width", width, 0u}); }
        description.objects.push_back(primitive);
        auto *plan = new ClassicFloatRuntimePlan(compile_xgen_classic_float_runtime_plan(description, {}));
        std::string reasons;
        for (const std::string &r : plan->fallback_reasons) { reasons += r + "\n"; }
        copy_text(reasons, msg, cap);
        return plan;
    } catch (const std::exception &e) {
        copy_text(e.what(), msg, cap);
        return nullptr;
    }
}

void ref_classic_plan_free(void *plan) { delete static_cast<ClassicFloatRuntimePlan *>(plan); }

// has length, has width, PTEX paths, pref-noise inputs; frequencies out.
void ref_classic_plan_info(const void *plan, std::uint32_t *out, float *frequencies) {
    const ClassicFloatRuntimePlan &p = *static_cast<const ClassicFloatRuntimePlan *>(plan);
    out[0] = p.length.has_value();
    out[1] = p.width.has_value();
    out[2] = static_cast<std::uint32_t>(p.ptex_paths.size());
    out[3] = static_cast<std::uint32_t>(p.pref_noise_inputs.size());
    for (std::size_t i = 0; i < p.pref_noise_inputs.size(); ++i) { frequencies[i] = p.pref_noise_inputs[i].frequency; }
}

// The compiled float program of the plan's length (0) or width (1).
const void *ref_classic_plan_program(const void *plan, std::uint32_t which) {
    const ClassicFloatRuntimePlan &p = *static_cast<const ClassicFloatRuntimePlan *>(plan);
    const auto &e = which == 0u ? p.length : p.width;
    return e ? &e->program : nullptr;
}

// apply_xgen_classic_float_runtime_plan_cpu on a packed curve set.  points
// is [S*P] PackedCurvePoint, roots [S] RootSample, root_uvs [S] Vec2 (may be
// NULL); runtime_inputs is [S x (PTEX + pref-noise)] in the plan's order.
// The surviving strands are compacted to the front; *kept receives their
// number.  Returns 0, or 1 with the exception text in msg.
std::uint32_t ref_classic_apply(const void *plan, float *points, std::uint32_t *counts, void *roots,
                                float *root_uvs, std::uint32_t strands, std::uint32_t cvs, float radius_scale,
                                const float *runtime_inputs, std::uint64_t runtime_input_count,
                                std::uint32_t workers, std::uint32_t *kept, char *msg, std::uint64_t cap) {
    try {
        const ClassicFloatRuntimePlan &p = *static_cast<const ClassicFloatRuntimePlan *>(plan);
        PackedGeneratedCurves curves{};
        curves.strand_count = strands;
        curves.cvs_per_strand = cvs;
        const auto *pts = reinterpret_cast<const PackedCurvePoint *>(points);
        curves.points.assign(pts, pts + static_cast<std::size_t>(strands) * cvs);
        curves.point_counts.assign(counts, counts + strands);
        const auto *rs = static_cast<const RootSample *>(roots);
        curves.roots.assign(rs, rs + strands);
        if (root_uvs) {
            const auto *uv = reinterpret_cast<const Vec2 *>(root_uvs);
            curves.root_uvs.assign(uv, uv + strands);
        }
        NanoXGenContext context(workers == 0u ? 1u : workers);
        apply_xgen_classic_float_runtime_plan_cpu(
            curves, p, radius_scale, {}, {}, {}, {},
            std::span<const float>(runtime_inputs, runtime_inputs ? runtime_input_count : 0u), {}, false,
            &context);
        std::memcpy(points, curves.points.data(), curves.points.size() * sizeof(PackedCurvePoint));
        std::memcpy(counts, curves.point_counts.data(), curves.point_counts.size() * 4u);
        std::memcpy(roots, curves.roots.data(), curves.roots.size() * sizeof(RootSample));
        if (root_uvs) { std::memcpy(root_uvs, curves.root_uvs.data(), curves.root_uvs.size() * sizeof(Vec2)); }
        *kept = curves.strand_count;
        copy_text("", msg, cap);
        return 0u;
    } catch (const std::exception &e) {
        copy_text(e.what(), msg, cap);
        return 1u;
    }
}

// compile_xgen_classic_float_runtime_plan for a description with the given
// SplinePrimitive attributes (length, width, taper, taperStart, widthRamp;
// NULL = absent) and FX modules in order: type 0 NoiseFXModule (mode 0;
// attributes mask, magnitude, magnitudeScale, frequency, correlation,
// preserveLength from six strings) or type 1 CutFXModule (rebuildType 1;
// amount from the first string).  Fallback reasons go to msg.
void *ref_classic_plan_fx(const char *const *primitive, std::uint32_t effect_count, const std::uint32_t *types,
                          const char *const *effect_attributes, std::uint32_t description_id,
                          const char *description_name, char *msg, std::uint64_t cap) {
    try {
        ClassicDescription description{};
        description.name = description_name ? description_name : "description";
        description.attributes.push_back({"descriptionId", std::to_string(description_id), 0u});
        ClassicObject spline{};
        spline.type = "SplinePrimitive";
        const char *names[5] = {"length", "width", "taper", "taperStart", "widthRamp"};
        for (int k = 0; k < 5; ++k) {
            if (primitive[k]) { spline.attributes.push_back({names[k], primitive[k], 0u}); }
        }
        description.objects.push_back(spline);
        const char *noise_names[6] = {"mask", "magnitude", "magnitudeScale", "frequency", "correlation",
                                      "preserveLength"};
        const char *clump_names[7] = {"mask", "clump", "clumpScale", "noise", "noiseScale", "noiseFrequency",
                                      "noiseCorrelation"};
        for (std::uint32_t e = 0; e < effect_count; ++e) {
            ClassicObject fx{};
            const char *const *a = effect_attributes + 7u * e;
            fx.attributes.push_back({"name", "fx" + std::to_string(e), 0u});
            if (types[e] == 0u) {
                fx.type = "NoiseFXModule";
                fx.attributes.push_back({"mode", "0", 0u});
                for (int k = 0; k < 6; ++k) { fx.attributes.push_back({noise_names[k], a[k], 0u}); }
            } else if (types[e] == 2u) {
                fx.type = "ClumpingFXModule";
                for (int k = 0; k < 7; ++k) { fx.attributes.push_back({clump_names[k], a[k], 0u}); }
            } else {
                fx.type = "CutFXModule";
                fx.attributes.push_back({"rebuildType", "1", 0u});
                fx.attributes.push_back({"amount", a[0], 0u});
            }
            description.objects.push_back(fx);
        }
        auto *plan = new ClassicFloatRuntimePlan(compile_xgen_classic_float_runtime_plan(description, {}));
        std::string reasons;
        for (const std::string &r : plan->fallback_reasons) { reasons += r + "\n"; }
        copy_text(reasons, msg, cap);
        return plan;
    } catch (const std::exception &e) {
        copy_text(e.what(), msg, cap);
        return nullptr;
    }
}

// Effects compiled into a plan: count of NoiseFX, CutFX, of all effects and
// of ClumpingFX.
void ref_classic_plan_effects(const void *plan, std::uint32_t *out) {
    const ClassicFloatRuntimePlan &p = *static_cast<const ClassicFloatRuntimePlan *>(plan);
    out[0] = static_cast<std::uint32_t>(p.noises.size());
    out[1] = static_cast<std::uint32_t>(p.cuts.size());
    out[2] = static_cast<std::uint32_t>(p.effects.size());
    out[3] = static_cast<std::uint32_t>(p.clumps.size());
}

// prepare_xgen_classic_clump_runtime_data on world-space guides: [G*P] Vec3
// axes in, [G*P] Vec3 render axes and [G] spline lengths out.
std::uint32_t ref_classic_clump_prepare(const float *axes, std::uint32_t guides, std::uint32_t cvs,
                                        float *render_axes, float *lengths, char *msg, std::uint64_t cap) {
    try {
        ClassicClumpRuntimeData data{};
        data.cvs_per_guide = cvs;
        const auto *a = reinterpret_cast<const Vec3 *>(axes);
        data.guide_axes.assign(a, a + static_cast<std::size_t>(guides) * cvs);
        prepare_xgen_classic_clump_runtime_data(data);
        std::memcpy(render_axes, data.guide_render_axes.data(), data.guide_render_axes.size() * sizeof(Vec3));
        std::memcpy(lengths, data.guide_spline_lengths.data(), data.guide_spline_lengths.size() * sizeof(float));
        copy_text("", msg, cap);
        return 0u;
    } catch (const std::exception &e) {
        copy_text(e.what(), msg, cap);
        return 1u;
    }
}

// ref_classic_apply with one surface tangent per strand ([S] Vec3, may be
// NULL when the plan has no NoiseFX).
// random_prefixes: [S] or NULL.  Clump module m (in plan order) has
// guide_counts[m] world-space guides: axes [G*P] Vec3, normals, tangents
// [G] Vec3, uvs [G] Vec2, SeExpr prefixes [G], reference positions [G] Vec3
// or NULL, and strand_guides [S]; the reference prepares the render axes.
std::uint32_t ref_classic_apply_fx(const void *plan, float *points, std::uint32_t *counts, void *roots,
                                   float *root_uvs, std::uint32_t strands, std::uint32_t cvs, float radius_scale,
                                   const float *runtime_inputs, std::uint64_t runtime_input_count,
                                   const float *surface_tangents, const std::uint32_t *random_prefixes,
                                   std::uint32_t clump_count, const std::uint32_t *guide_counts,
                                   const float *const *clump_axes, const float *const *clump_normals,
                                   const float *const *clump_tangents, const float *const *clump_uvs,
                                   const std::uint32_t *const *clump_prefixes,
                                   const float *const *clump_reference_positions,
                                   const std::uint32_t *const *clump_strand_guides, std::uint32_t workers,
                                   std::uint32_t *kept, char *msg, std::uint64_t cap) {
    try {
        const ClassicFloatRuntimePlan &p = *static_cast<const ClassicFloatRuntimePlan *>(plan);
        std::vector<ClassicClumpRuntimeData> clumps(clump_count);
        for (std::uint32_t m = 0; m < clump_count; ++m) {
            ClassicClumpRuntimeData &d = clumps[m];
            const std::size_t G = guide_counts[m];
            d.module_name = m < p.clumps.size() ? p.clumps[m].name : std::string();
            d.cvs_per_guide = cvs;
            const auto *axes = reinterpret_cast<const Vec3 *>(clump_axes[m]);
            d.guide_axes.assign(axes, axes + G * cvs);
            const auto *n = reinterpret_cast<const Vec3 *>(clump_normals[m]);
            d.guide_normals.assign(n, n + G);
            const auto *t = reinterpret_cast<const Vec3 *>(clump_tangents[m]);
            d.guide_tangents.assign(t, t + G);
            const auto *uv = reinterpret_cast<const Vec2 *>(clump_uvs[m]);
            d.guide_uvs.assign(uv, uv + G);
            d.guide_face_ids.assign(G, 0u);
            d.guide_random_prefixes.assign(clump_prefixes[m], clump_prefixes[m] + G);
            if (clump_reference_positions[m]) {
                const auto *r = reinterpret_cast<const Vec3 *>(clump_reference_positions[m]);
                d.guide_reference_positions.assign(r, r + G);
            }
            d.strand_guide_indices.assign(clump_strand_guides[m], clump_strand_guides[m] + strands);
        }
        PackedGeneratedCurves curves{};
        curves.strand_count = strands;
        curves.cvs_per_strand = cvs;
        const auto *pts = reinterpret_cast<const PackedCurvePoint *>(points);
        curves.points.assign(pts, pts + static_cast<std::size_t>(strands) * cvs);
        curves.point_counts.assign(counts, counts + strands);
        const auto *rs = static_cast<const RootSample *>(roots);
        curves.roots.assign(rs, rs + strands);
        if (root_uvs) {
            const auto *uv = reinterpret_cast<const Vec2 *>(root_uvs);
            curves.root_uvs.assign(uv, uv + strands);
        }
        std::span<const Vec3> tangents;
        if (surface_tangents) { tangents = std::span<const Vec3>(reinterpret_cast<const Vec3 *>(surface_tangents), strands); }
        std::span<const std::uint32_t> prefixes;
        if (random_prefixes) { prefixes = std::span<const std::uint32_t>(random_prefixes, strands); }
        NanoXGenContext context(workers == 0u ? 1u : workers);
        apply_xgen_classic_float_runtime_plan_cpu(
            curves, p, radius_scale, tangents, prefixes, {}, clumps,
            std::span<const float>(runtime_inputs, runtime_inputs ? runtime_input_count : 0u), {}, false,
            &context);
        std::memcpy(points, curves.points.data(), curves.points.size() * sizeof(PackedCurvePoint));
        std::memcpy(counts, curves.point_counts.data(), curves.point_counts.size() * 4u);
        std::memcpy(roots, curves.roots.data(), curves.roots.size() * sizeof(RootSample));
        if (root_uvs) { std::memcpy(root_uvs, curves.root_uvs.data(), curves.root_uvs.size() * sizeof(Vec2)); }
        *kept = curves.strand_count;
        copy_text("", msg, cap);
        return 0u;
    } catch (const std::exception &e) {
        copy_text(e.what(), msg, cap);
        return 1u;
    }
}

} // extern "C"
