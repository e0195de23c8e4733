/* nxg_payload.h -- renderer payload batches (build_curve_batches,
 * src/curve_payload.cpp) on sm_100a.
 *
 * A curve set (the reference's CurveSetView, include/nanoxgen/curve_payload.h:
 * 28-39) of fixed or variable CV counts, with optional per-point widths and
 * per-strand root uvs, plus motion samples of the same strands, becomes the
 * renderer's payload: float4 points (position after the affine transform,
 * 0.5 * width * radius_scale), per-strand point counts and root uvs, and
 * sample-major motion positions, optionally resampled to a fixed CV count
 * (linear in normalised index space).  The reference cuts the payload into
 * batches of at most max_strands_per_batch strands (CurveBatch); here all
 * batches are written in one pass into one set of arrays, batch after batch
 * (so points and counts are in strand order), with the batch boundaries in
 * batch_first_point.  Batch b holds strands [b * M, min(S, (b + 1) * M)),
 * its points [batch_first_point[b], batch_first_point[b + 1]), and its motion
 * positions, sample-major within the batch, at
 * motion_points[samples * batch_first_point[b] ...] -- exactly the
 * reference's batches concatenated.  Uniform primvars are per-strand arrays
 * whose batch slice is [b * M, ...): the caller takes views, no copy is made.
 *
 * Every array is on the device; entry points enqueue only.
 */
#ifndef NXG_PAYLOAD_H
#define NXG_PAYLOAD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nxg_curve_set {
    uint32_t strand_count;
    uint32_t fixed_cvs_per_strand;  /* used when point_counts is NULL */
    const uint32_t *point_counts;   /* strand_count, or NULL */
    const float *points;            /* point_count x 3 */
    uint64_t point_count;           /* elements of points */
    const float *widths;            /* point_count full diameters, or NULL (constant_width) */
    const float *root_uvs;          /* strand_count x 2, or NULL */
    const void *roots;              /* nxg_root_sample[strand_count] (uv used when root_uvs is NULL), or NULL */
    float constant_width;
    uint32_t reserved;
} nxg_curve_set;

#define NXG_PAYLOAD_MAX_SAMPLES 32u

typedef struct nxg_motion_set {
    float time;
    uint32_t reserved;
    nxg_curve_set curves;
} nxg_motion_set;

typedef struct nxg_payload_options {
    uint32_t max_strands_per_batch;  /* > 0 (the reference's default: 65536) */
    uint32_t resample_cv_count;      /* 0 keeps the source counts, else >= 2 */
    float radius_scale;              /* finite, >= 0 */
    float transform[12];             /* row-major 3x4 affine transform */
} nxg_payload_options;

typedef struct nxg_payload_output {
    uint32_t *point_counts;          /* strand_count */
    float *points;                   /* nxg_payload_point_count float4, 16-byte aligned */
    float *root_uvs;                 /* strand_count x 2, or NULL (needed when the base has root uvs or roots) */
    float *motion_points;            /* samples x nxg_payload_point_count x 3, or NULL without samples */
    uint64_t *batch_first_point;     /* batch count + 1 */
} nxg_payload_output;

/* Errors reported in the device status (code, failing strands) or returned
 * by the host checks; nxg_payload_error_message gives the reference's text
 * (the curve-set label is "base curves" or "motion curves"). */
typedef enum nxg_payload_error {
    NXG_PAYLOAD_OK = 0,
    NXG_PAYLOAD_NO_STRAND_LIMIT,       /* curve batches need a positive strand limit */
    NXG_PAYLOAD_RESAMPLE_ONE,          /* curve resampling needs at least two CVs */
    NXG_PAYLOAD_BAD_RADIUS_SCALE,
    NXG_PAYLOAD_BASE_NO_STRANDS,
    NXG_PAYLOAD_BASE_NO_COUNTS,        /* needs fixed or variable CV counts */
    NXG_PAYLOAD_BASE_SHORT_CURVE,      /* curve has fewer than two CVs (device) */
    NXG_PAYLOAD_BASE_POINT_SIZE,       /* point array size mismatch (device with variable counts) */
    NXG_PAYLOAD_BASE_BAD_WIDTH,        /* invalid constant width */
    NXG_PAYLOAD_MOTION_BAD_TIME,       /* motion sample time must be finite */
    NXG_PAYLOAD_MOTION_STRANDS,        /* motion sample strand-count mismatch */
    NXG_PAYLOAD_MOTION_NO_STRANDS,
    NXG_PAYLOAD_MOTION_NO_COUNTS,
    NXG_PAYLOAD_MOTION_SHORT_CURVE,
    NXG_PAYLOAD_MOTION_POINT_SIZE,
    NXG_PAYLOAD_MOTION_BAD_WIDTH,
    NXG_PAYLOAD_BAD_TRANSFORM,         /* curve transform must contain finite values */
    NXG_PAYLOAD_ERROR_COUNT
} nxg_payload_error;

const char *nxg_payload_error_message(uint32_t code);

/* Points of the payload: strand_count * resample_cv_count, or the base's
 * point_count when not resampling. */
uint64_t nxg_payload_point_count(const nxg_curve_set *base, const nxg_payload_options *options);
uint32_t nxg_payload_batch_count(const nxg_curve_set *base, const nxg_payload_options *options);

/* Device scratch for the point offsets of the variable-count sets. */
uint64_t nxg_payload_workspace_size(const nxg_curve_set *base, const nxg_motion_set *samples, uint32_t sample_count);

/* build_curve_batches on the device.  The host checks (the reference's, in
 * its order, for what the host can see) return NXG_ERROR_INVALID_ARGUMENT
 * with their nxg_payload_error in *host_error; the count checks of variable
 * sets run on the device into device_status (2 x uint32: the first error in
 * the reference's order, and the failing strands; zeroed by the caller), in
 * which case the outputs are not meaningful.  At most NXG_PAYLOAD_MAX_SAMPLES
 * motion samples. */
uint32_t nxg_build_curve_batches(const nxg_curve_set *base, const nxg_motion_set *samples, uint32_t sample_count,
                                 const nxg_payload_options *options, const nxg_payload_output *output,
                                 void *workspace, uint64_t workspace_bytes, uint32_t *device_status,
                                 uint32_t *host_error, void *stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* NXG_PAYLOAD_H */
