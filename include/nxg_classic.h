/*
 * nxg_classic.h -- Classic-expression per-root scalars on the GPU.
 *
 * Part of libnxg_b200.so; include after nxg.h.  Three layers:
 *
 *  1. The scalar-expression compiler.  nxg_expression_compile replaces the
 *     reference's compile_xgen_scalar_expression + make_xgen_float_expression_program
 *     (src/xgen_expression.cpp:771-818) and, with NXG_EXPRESSION_CLASSIC, the
 *     Classic runtime's comment stripping and noise($Prefg*k) rewrite
 *     (src/xgen_classic_runtime.cpp:138-347).  Same language, same SSA
 *     program, same error texts.
 *
 *  2. The exact runtime.  nxg_classic_root_scalars evaluates a description's
 *     SplinePrimitive length and width expressions for every root on the
 *     device with the float semantics of evaluate_xgen_scalar_expression_float
 *     (src/xgen_expression.cpp:984-1148) and xgen_classic_noise_float
 *     (src/xgen_classic_runtime.cpp:803-837).  nxg_generate_packed_classic
 *     applies the scalars inside the generator, as the reference's
 *     apply_xgen_classic_float_runtime_plan_cpu does afterwards on the host
 *     (src/xgen_classic_runtime.cpp:1650-1678 length, :1827-1858 width profile,
 *     :1670-1675 the drop rule).
 *
 *  3. The learned surrogate (no reference counterpart): a 3x64 MLP over the
 *     root's position, normal and uv, BF16 weights on the tcgen05 tensor cores
 *     with FP32 accumulation, trained on the device by the library's own
 *     forward/backward/Adam kernels on samples of the exact runtime, and
 *     spot-checked against the exact runtime on every batch with an exact
 *     re-run of any batch whose check exceeds the tolerance.
 */
#ifndef NXG_CLASSIC_H
#define NXG_CLASSIC_H

#include "nxg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- compiler */

typedef struct nxg_expression nxg_expression; /* opaque, host memory */

#define NXG_EXPRESSION_CLASSIC 1u /* apply the Classic source rewrites first */
#define NXG_EXPRESSION_MAX_INPUTS 16u

typedef struct nxg_expression_info {
    uint32_t instruction_count;
    uint32_t operand_count;
    uint32_t input_count;
    uint32_t ramp_count;
    uint32_t ramp_point_count;
    uint32_t result;
    uint32_t expression_seed;   /* xgen_expression_seed(name, object type) */
    uint32_t random_call_count;
    uint32_t pref_noise_count;  /* distinct noise($Prefg*k) frequencies */
    float pref_noise_frequencies[NXG_EXPRESSION_MAX_INPUTS];
} nxg_expression_info;

/* One SSA instruction of the float program (XgenFloatScalarInstruction,
 * xgen_expression.h:84-90); op numbers follow XgenScalarOp (:12-40). */
typedef struct nxg_expression_instruction {
    uint32_t op;
    uint32_t operand_offset;
    uint32_t operand_count;
    uint32_t auxiliary;
    float immediate;
} nxg_expression_instruction;

typedef struct nxg_expression_ramp_point {
    float position;
    float value;
    uint32_t interpolation;
} nxg_expression_ramp_point;

/* Compiles `source`.  expression_name / object_type seed rand() exactly as
 * xgen_expression_seed (xgen_expression.cpp:730-737); the Classic runtime
 * passes the attribute name ("length", "width") and the object type
 * ("SplinePrimitive").  On failure returns NXG_ERROR_EXPRESSION_SYNTAX and
 * writes the reference's message text to `message`. */
uint32_t nxg_expression_compile(const char *source, const char *expression_name, const char *object_type,
                                uint32_t flags, nxg_expression **out, char *message, size_t message_capacity);
void nxg_expression_destroy(nxg_expression *expression);
uint32_t nxg_expression_get_info(const nxg_expression *expression, nxg_expression_info *info);
uint32_t nxg_expression_get_instruction(const nxg_expression *expression, uint32_t index,
                                        nxg_expression_instruction *instruction);
uint32_t nxg_expression_get_operand(const nxg_expression *expression, uint32_t index, uint32_t *operand);
uint32_t nxg_expression_get_ramp_point(const nxg_expression *expression, uint32_t index,
                                       nxg_expression_ramp_point *point);
/* Name of input `index` (without '$'), or NULL. */
const char *nxg_expression_input_name(const nxg_expression *expression, uint32_t index);

/* xgen_string_seed (xgen_expression.cpp:716-728). */
uint32_t nxg_xgen_string_seed(const char *text);

/* ------------------------------------------------------------ exact runtime */

/* A description's per-root scalar expressions.  Bound inputs:
 * $__nxg_pref_noise_<k> (from noise($Prefg*k)), $id (strand index), $u/$v
 * (root uv), $cWidth (0, as in the reference while length and width are
 * evaluated).  $cLength needs the generated curve and is refused here. */
typedef struct nxg_classic_scalar_plan {
    const nxg_expression *length; /* SplinePrimitive.length or NULL (scale 1) */
    const nxg_expression *width;  /* SplinePrimitive.width or NULL */
    uint32_t description_id;      /* rand() face seed (xgen_expression.cpp:702-714) */
    uint32_t reserved;
    const char *patch_name;       /* rand() face seed; NULL = "" */
} nxg_classic_scalar_plan;

/* scalars[2*i] = length scale, scalars[2*i+1] = width of strand first+i
 * (float2 per strand, 8-byte aligned).  device_status (2 x uint32, zeroed
 * by the caller) receives NXG_ERROR_EXPRESSION_DOMAIN in [0] and the number
 * of failing strands in [1] when an expression yields a non-finite value or
 * a negative length (the reference throws there). */
uint32_t nxg_classic_root_scalars(const nxg_device_asset_desc *asset, const nxg_generation_params *params,
                                  const nxg_classic_scalar_plan *plan, uint32_t first_strand,
                                  uint32_t strand_count, float *scalars, uint32_t *device_status,
                                  void *stream);

/* Classic application fused into generation.  With apply_length the strand
 * is scaled about its first point by scalars[2i]; with apply_width every
 * radius becomes 0.5 * max(scalars[2i+1], 0) * radius_scale; a strand whose
 * scaled spline length or width is below 1e-4 gets point_counts = 0 (the
 * reference removes it from the set instead). */
typedef struct nxg_classic_apply_desc {
    const float *root_scalars; /* from nxg_classic_root_scalars or the surrogate */
    uint32_t apply_length;
    uint32_t apply_width;
} nxg_classic_apply_desc;

uint32_t nxg_generate_packed_classic(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                     const nxg_generation_params *params, const nxg_packed_output_desc *output,
                                     const nxg_classic_apply_desc *classic, const nxg_launch_config *config,
                                     uint32_t first_strand, uint32_t strand_count, void *workspace,
                                     uint64_t workspace_bytes, void *stream);

/* nxg_generate_batched (nxg.h) with per-description Classic scalars:
 * classic[d].root_scalars may be NULL for descriptions without them. */
uint32_t nxg_generate_batched_classic(const nxg_device_asset_desc *assets, const nxg_deformed_desc *deformed,
                                      const nxg_generation_params *params, const nxg_packed_output_desc *outputs,
                                      const nxg_classic_apply_desc *classic, uint32_t count,
                                      const nxg_launch_config *config, void *workspace, uint64_t workspace_bytes,
                                      void *stream);

/* -------------------------------------------------------------- FX passes */

/* The Classic FX pipeline of apply_xgen_classic_float_runtime_plan_cpu
 * (src/xgen_classic_runtime.cpp:1420-1919) on the GPU, as a pass over a
 * generated packed curve set: per strand, the SplinePrimitive length and
 * width with the drop rule, the description's FX modules in order -- NoiseFX
 * mode 0 (apply_noise, :897-1040) and CutFX rebuild type 1
 * (cut_from_tip_and_rebuild, :692-748) -- then the width profile (taper,
 * taperStart, widthRamp).  ClumpingFX is not supported.  Expressions are
 * compiled with NXG_EXPRESSION_CLASSIC and the attribute's own name and
 * object type; they may read $id, $cLength, $cWidth, $u, $v and
 * noise($Prefg*k) (evaluated at the root's position). */
#define NXG_CLASSIC_MAX_FX 8u
#define NXG_CLASSIC_MAX_FX_CVS 64u

enum { NXG_CLASSIC_FX_NOISE = 0, NXG_CLASSIC_FX_CUT = 1, NXG_CLASSIC_FX_CLUMP = 2 };

typedef struct nxg_classic_fx {
    uint32_t type;                         /* NXG_CLASSIC_FX_NOISE, _CUT or _CLUMP */
    uint32_t reserved;
    /* NoiseFXModule attributes (type NOISE), all required; `mask` is also
       ClumpingFXModule.mask */
    const nxg_expression *mask, *magnitude, *magnitude_scale, *frequency, *correlation, *preserve_length;
    const nxg_expression *amount;          /* CutFXModule.amount (type CUT) */
    /* ClumpingFXModule attributes (type CLUMP, with mask), all required */
    const nxg_expression *clump, *clump_scale, *noise, *noise_scale, *noise_frequency, *noise_correlation;
} nxg_classic_fx;

typedef struct nxg_classic_fx_plan {
    /* SplinePrimitive attributes, NULL when absent */
    const nxg_expression *length, *width, *taper, *taper_start, *width_ramp;
    const nxg_classic_fx *effects;         /* in the description's order */
    uint32_t effect_count;                 /* <= NXG_CLASSIC_MAX_FX */
    uint32_t description_id;               /* rand() face seed */
    const char *description_name;          /* rand() face seed (text after its last ':'); NULL = "" */
} nxg_classic_fx_plan;

/* Device bytes of a plan's packed form (constant; 256-byte aligned buffer). */
uint64_t nxg_classic_fx_plan_bytes(void);

/* Packs `plan` and copies it into `device_plan` on `stream` (a host-to-device
 * copy from library-owned host memory, complete when the call returns).
 * Returns NXG_ERROR_EXPRESSION_LIMIT / _INPUT when a program does not fit
 * the device form or reads an unbound variable, NXG_ERROR_INVALID_ARGUMENT
 * for a malformed plan. */
uint32_t nxg_classic_fx_plan_upload(const nxg_classic_fx_plan *plan, void *device_plan, uint64_t bytes,
                                    void *stream);

/* The clump guides of one ClumpingFXModule (ClassicClumpRuntimeData,
 * xgen_classic_runtime.h:59-88, without the root-relative copies), all
 * device arrays.  Each guide has cvs_per_strand CVs. */
typedef struct nxg_classic_clump_guides {
    const float *axes;                /* guide_count x P x 3: the guide CVs (before the rebuild) */
    const float *render_axes;         /* guide_count x P x 3: from nxg_classic_clump_prepare */
    const float *spline_lengths;      /* guide_count: from nxg_classic_clump_prepare */
    const float *normals;             /* guide_count x 3 */
    const float *tangents;            /* guide_count x 3 */
    const float *reference_positions; /* guide_count x 3 guide-noise domains, or NULL (the first CV) */
    const float *uvs;                 /* guide_count x 2 */
    const uint32_t *random_prefixes;  /* guide_count SeExpr prefixes (rand() in the guide noise) */
    const uint32_t *strand_guides;    /* strand_count: the strand's guide, or NXG_INVALID_INDEX */
    float *noise_table;               /* guide_count x P float4 scratch, or NULL: when the module's
                                         guide-noise programs read no per-strand input ($id, $cLength,
                                         $cWidth, noise($Prefg)), the apply computes each guide's
                                         noise axis once into it instead of once per strand */
    uint32_t guide_count;
    uint32_t reserved;
} nxg_classic_clump_guides;

/* prepare_xgen_classic_clump_runtime_data (xgen_classic_runtime.cpp:839-892)
 * on the device: each guide's CVs resampled at cv/(P-1) (the ends kept) into
 * render_axes, and its spline length.  P >= 3; enqueue only. */
uint32_t nxg_classic_clump_prepare(const float *axes, uint32_t guide_count, uint32_t cvs_per_guide,
                                   float *render_axes, float *spline_lengths, void *stream);

typedef struct nxg_classic_fx_curves {
    float *points;                 /* strand_count x cvs_per_strand float4 (position, radius), in/out */
    uint32_t *point_counts;        /* in/out; a strand whose count is not cvs_per_strand is skipped, a
                                      dropped strand gets 0 (its points are left as they were) */
    const void *roots;             /* nxg_root_sample[strand_count] of the curves */
    const float *surface_tangents; /* strand_count x 3 (the frame's cU per strand); required with NoiseFX */
    const float *noise_domains;    /* strand_count x 3 NoiseFX domain positions, or NULL (the curve's root) */
    uint32_t strand_count;
    uint32_t cvs_per_strand;       /* 2 .. NXG_CLASSIC_MAX_FX_CVS */
    uint32_t first_id;             /* $id of strand 0 */
    float radius_scale;
    const uint32_t *random_prefixes;          /* strand_count SeExpr prefixes; required when a program
                                                 calls rand() */
    const nxg_classic_clump_guides *clumps;   /* host array, one per CLUMP effect in plan order */
    uint32_t clump_count;
    uint32_t reserved;
} nxg_classic_fx_curves;

/* Applies the uploaded plan to `curves` on `stream` (enqueue only).
 * device_status (2 x uint32, zeroed by the caller) receives
 * NXG_ERROR_EXPRESSION_DOMAIN and the number of failing strands where an
 * expression yields a non-finite value or a negative length (the reference
 * throws there), or NXG_ERROR_INVALID_ARGUMENT where a strand needs an
 * input that was not given (surface tangents for NoiseFX, random prefixes
 * for rand(), a clump guide index beyond guide_count). */
uint32_t nxg_classic_fx_apply(const void *device_plan, const nxg_classic_fx_curves *curves,
                              uint32_t *device_status, void *stream);

/* ---------------------------------------------------------------- surrogate */

/* The model is one caller-owned device buffer of nxg_surrogate_model_bytes()
 * bytes (256-byte aligned): header (input/output normalisation, Adam step),
 * FP32 parameters, Adam moments and the BF16 weight tiles the kernels copy
 * into shared memory.  Parameters are the augmented matrices W1a 64x16,
 * W2a 64x80, W3a 64x80, W4a 16x80 (row-major, concatenated; the bias is the
 * column after the inputs: 8 for W1a, 64 for the others; W4a rows 0-1 are
 * the length and width outputs). */
#define NXG_SURROGATE_INPUTS 8u        /* rest position xyz, normal xyz, u, v */
#define NXG_SURROGATE_HIDDEN 64u
#define NXG_SURROGATE_PARAMETERS 12544u

typedef struct nxg_surrogate_config {
    float input_offset[NXG_SURROGATE_INPUTS]; /* the network sees (feature - offset) * scale */
    float input_scale[NXG_SURROGATE_INPUTS];
    uint32_t seed;                            /* initial weights */
    uint32_t reserved;
} nxg_surrogate_config;

typedef struct nxg_surrogate_train_config {
    uint32_t epochs;
    uint32_t batch;          /* samples per Adam step, a multiple of 128 */
    float learning_rate;
    float lr_decay;          /* learning-rate factor per epoch (0 = 1) */
    float beta1, beta2, epsilon; /* Adam (0 = 0.9, 0.999, 1e-8) */
    uint32_t seed;           /* sample order */
} nxg_surrogate_train_config;

/* Per-batch judge.  A batch is one 128-root tile: `checks_per_batch` of its
 * roots are evaluated by the exact runtime and, if any relative error
 * exceeds its tolerance (or the exact runtime fails there), every root of
 * the tile is re-run exactly.  mode 0 = checked surrogate, 1 = exact
 * runtime only, 2 = surrogate without checks, 3 = adaptive: as 0 while the
 * model is trusted; after a launch in which a check failed, the next launch
 * runs the network (checked) on one batch in 16 and the exact kernel on the
 * rest, and trust returns when those probes pass.  Adaptive launches update
 * state in the model buffer, so they are ordered on one stream. */
typedef struct nxg_surrogate_check {
    float length_tolerance;
    float width_tolerance;
    uint32_t checks_per_batch; /* 0..128 */
    uint32_t mode;
} nxg_surrogate_check;

uint64_t nxg_surrogate_model_bytes(void);
uint64_t nxg_surrogate_workspace_bytes(void);

/* Header, He-uniform weights, zero Adam state; synchronises `stream`. */
uint32_t nxg_surrogate_init(void *model, const nxg_surrogate_config *config, void *stream);

/* Raw features of strands [first, first + count): count x 8 floats. */
uint32_t nxg_surrogate_features(const nxg_device_asset_desc *asset, const nxg_generation_params *params,
                                uint32_t first_strand, uint32_t count, float *features, void *stream);

/* Output normalisation from training targets (count x 2: length, width). */
uint32_t nxg_surrogate_fit_outputs(void *model, const float *targets, uint32_t count, void *stream);

/* Mini-batch Adam on the squared error of the normalised outputs, forward,
 * backward and weight gradients on the tensor cores.  loss_history (device,
 * `epochs` floats, optional) receives per epoch the sum over its steps of
 * the step's mean loss.  A set-up call: synchronises `stream`. */
uint32_t nxg_surrogate_train(void *model, const float *features, const float *targets, uint32_t count,
                             const nxg_surrogate_train_config *config, void *workspace, uint64_t workspace_bytes,
                             float *loss_history, void *stream);

/* Gradient of the mean loss over all `count` samples with respect to every
 * parameter (NXG_SURROGATE_PARAMETERS floats, device) and the loss itself;
 * the same kernels as training, without the update. */
uint32_t nxg_surrogate_gradients(const void *model, const float *features, const float *targets, uint32_t count,
                                 float *gradients, float *loss, void *stream);

/* Network outputs (length, width) for raw features (count x 2 floats). */
uint32_t nxg_surrogate_forward(const void *model, const float *features, uint32_t count, float *outputs,
                               void *stream);

/* Per-root (length scale, width) of strands [first, first + count) by the
 * surrogate, judged per batch by the exact runtime of `plan`.
 * device_status (4 x uint32, zeroed by the caller): [0] error code, [1]
 * roots whose exact evaluation failed, [2] batches re-run exactly, [3]
 * batches checked. */
uint32_t nxg_surrogate_root_scalars(void *model, const nxg_device_asset_desc *asset,
                                    const nxg_generation_params *params, const nxg_classic_scalar_plan *plan,
                                    const nxg_surrogate_check *check, uint32_t first_strand, uint32_t count,
                                    float *scalars, uint32_t *device_status, void *stream);

/* Device address of the FP32 parameter array inside the model. */
uint32_t nxg_surrogate_parameters(void *model, float **parameters);

#ifdef __cplusplus
}
#endif

#endif /* NXG_CLASSIC_H */
