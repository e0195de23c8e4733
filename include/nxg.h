/*
 * nxg.h -- C ABI of the B200 strand generator (nanoxgen_b200/libnxg_b200.so).
 *
 * This boundary replaces NanoXGen's checked device contract
 * (include/nanoxgen/device_contract.h) and the packed CPU drivers
 * (src/asset.cpp:412-449, include/nanoxgen/asset.h:119-153) for renderers
 * that own CUDA device memory and streams.  Every struct below keeps the
 * byte layout of the reference type it mirrors, so a renderer that already
 * fills the reference's descriptors can pass the same bytes.
 *
 * Conventions
 *   - All functions are callable from C, C++ (cgo/JNI/ctypes) and never throw.
 *   - Status-returning functions return an nxg_error code; 0 means success.
 *     Codes 0..20 are the reference's DeviceGenerationError values in the
 *     same order (device_contract.h:58-80); codes >= 64 are additions.
 *   - Device-side entry points take `stream` as a cudaStream_t passed as
 *     `void *` (NULL is the legacy default stream).  They only enqueue work:
 *     no allocation, no host synchronisation, no readback.  All device
 *     buffers (asset, outputs, workspace) are owned by the caller.
 */
#ifndef NXG_H
#define NXG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NXG_ABI_VERSION 1u

/* Format constants, include/nanoxgen/types.h:18-23 and :74-77. */
#define NXG_MAGIC 0x4e4547584f4e414eull
#define NXG_VERSION_MAJOR 0u
#define NXG_VERSION_MINOR 2u
#define NXG_GUIDE_STENCIL_SIZE 8u
#define NXG_NOISE_GRADIENT_COUNT 256u
#define NXG_INVALID_INDEX 0xffffffffu
#define NXG_ASSET_HAS_NORMALS 1u
#define NXG_ASSET_HAS_TEXCOORDS 2u

#if defined(__GNUC__) || defined(__clang__) || defined(__CUDACC__)
#define NXG_ALIGN(n) __attribute__((aligned(n)))
#else
#define NXG_ALIGN(n)
#endif

/* types.h:25-40 */
typedef struct nxg_vec2 { float x, y; } nxg_vec2;
typedef struct nxg_vec3 { float x, y, z; } nxg_vec3;
typedef struct nxg_uint3 { uint32_t x, y, z; } nxg_uint3;

/* types.h:53-56 Walker alias entry. */
typedef struct nxg_alias_entry {
    float probability;
    uint32_t alias;
} nxg_alias_entry;

/* types.h:58-69 GuideRecord, 56 bytes. */
typedef struct nxg_guide_record {
    uint32_t first_cv;
    uint16_t cv_count;
    uint16_t flags;
    uint32_t triangle_index;
    float support_radius;
    nxg_vec2 barycentric; /* weights of triangle vertices y and z */
    nxg_vec2 root_uv;
    nxg_vec3 root_position;
    nxg_vec3 root_normal;
} nxg_guide_record;

/* types.h:76-101 AssetHeader, 128 bytes, 64-byte aligned.  Offsets are byte
 * offsets from the first header byte; 0 means "section absent". */
typedef struct NXG_ALIGN(64) nxg_asset_header {
    uint64_t magic;
    uint16_t version_major;
    uint16_t version_minor;
    uint32_t flags;
    uint64_t byte_size;
    uint64_t content_hash; /* FNV-1a 64 of every byte after the header */
    uint32_t vertex_count;
    uint32_t triangle_count;
    uint32_t guide_count;
    uint32_t guide_cv_count;
    uint32_t guide_stencil_size;
    uint32_t noise_gradient_count;
    uint64_t positions_offset;
    uint64_t normals_offset;
    uint64_t texcoords_offset;
    uint64_t triangles_offset;
    uint64_t alias_table_offset;
    uint64_t guides_offset;
    uint64_t guide_cvs_offset;
    uint64_t triangle_guides_offset;
    uint64_t noise_gradients_offset;
} nxg_asset_header;

/* types.h:108-124 GenerationParams (same defaults documented there). */
typedef struct nxg_generation_params {
    uint32_t strand_count;
    uint32_t cvs_per_strand;
    uint32_t seed;
    uint32_t reserved;
    float guide_support_scale;
    float guide_weight_power;
    float normal_rejection_cos;
    float length_scale;
    float root_width;
    float tip_width;
    float noise_amplitude;
    float noise_frequency;
    float noise_mask;
    float noise_correlation;
    float noise_preserve_length;
} nxg_generation_params;

/* types.h:126-136 RootSample, 48 bytes. */
typedef struct nxg_root_sample {
    nxg_vec3 position;
    nxg_vec3 normal;
    nxg_vec2 uv;
    uint32_t triangle_index;
    nxg_vec2 barycentric;
    uint32_t surface_face_id;
} nxg_root_sample;

/* types.h:138-147 PackedCurvePoint: float4(position, radius), 16 bytes. */
typedef struct NXG_ALIGN(16) nxg_packed_point {
    float x, y, z, radius;
} nxg_packed_point;

/* device_contract.h:14-18 DeviceAssetDescriptor: the device copy of a
 * validated asset plus its host-validated header mirror.  Kernels take every
 * count and offset from `header`, never from device memory. */
typedef struct NXG_ALIGN(64) nxg_device_asset_desc {
    const void *asset; /* device pointer, 64-byte aligned */
    nxg_asset_header header;
    uint64_t byte_capacity;
} nxg_device_asset_desc;

/* device_contract.h:20-25 DeviceDeformedGeometryDescriptor.  NULL pointers
 * select the asset's rest arrays; a non-NULL pointer needs a count equal to
 * the header's vertex (positions, normals) or guide-CV count. */
typedef struct nxg_deformed_desc {
    const nxg_vec3 *positions;
    const nxg_vec3 *normals;
    const nxg_vec3 *guide_cvs;
    uint64_t position_count;
    uint64_t normal_count;
    uint64_t guide_cv_count;
} nxg_deformed_desc;

/* device_contract.h:27-32 DeviceGeneratedOutputDescriptor (SoA layout). */
typedef struct nxg_generated_output_desc {
    nxg_vec3 *points;
    float *widths;
    nxg_root_sample *roots;
    uint64_t point_capacity;
    uint64_t width_capacity;
    uint64_t root_capacity;
} nxg_generated_output_desc;

/* device_contract.h:34-40 DevicePackedCurveOutputDescriptor with the
 * DevicePackedCurveOutputView of types.h:164-170.  `points` is required;
 * the others are optional (NULL with capacity 0). */
typedef struct nxg_packed_output_desc {
    nxg_packed_point *points;
    nxg_root_sample *roots;
    nxg_vec2 *root_uvs;
    float radius_scale;
    uint32_t *point_counts;
    uint64_t point_capacity;
    uint64_t root_capacity;
    uint64_t root_uv_capacity;
    uint64_t point_count_capacity;
} nxg_packed_output_desc;

/* device_contract.h:42-45 */
typedef struct nxg_motion_sample_desc {
    nxg_deformed_desc deformation;
    float time;
} nxg_motion_sample_desc;

/* device_contract.h:47-52: sample-major absolute Vec3 positions. */
typedef struct nxg_motion_output_desc {
    nxg_vec3 *points;
    uint64_t point_capacity;
} nxg_motion_output_desc;

/* device_contract.h:54-56.  block_size must lie in [1, 1024]; the generator
 * rounds it up to whole warps and uses it as its CTA size. */
typedef struct nxg_launch_config {
    uint32_t block_size;
} nxg_launch_config;

/* device_contract.h:58-80 DeviceGenerationError, then additions (>= 64). */
typedef enum nxg_error {
    NXG_ERROR_NONE = 0,
    NXG_ERROR_NULL_ASSET = 1,
    NXG_ERROR_MISALIGNED_ASSET = 2,
    NXG_ERROR_INVALID_ASSET_METADATA = 3,
    NXG_ERROR_ASSET_CAPACITY_TOO_SMALL = 4,
    NXG_ERROR_INVALID_GENERATION_PARAMETERS = 5,
    NXG_ERROR_INVALID_BLOCK_SIZE = 6,
    NXG_ERROR_DEFORMED_POSITION_COUNT_MISMATCH = 7,
    NXG_ERROR_DEFORMED_NORMAL_COUNT_MISMATCH = 8,
    NXG_ERROR_DEFORMED_GUIDE_CV_COUNT_MISMATCH = 9,
    NXG_ERROR_MISSING_OUTPUT = 10,
    NXG_ERROR_POINT_CAPACITY_TOO_SMALL = 11,
    NXG_ERROR_WIDTH_CAPACITY_TOO_SMALL = 12,
    NXG_ERROR_ROOT_CAPACITY_TOO_SMALL = 13,
    NXG_ERROR_ROOT_UV_CAPACITY_TOO_SMALL = 14,
    NXG_ERROR_POINT_COUNT_CAPACITY_TOO_SMALL = 15,
    NXG_ERROR_INVALID_RADIUS_SCALE = 16,
    NXG_ERROR_MISSING_MOTION_SAMPLES = 17,
    NXG_ERROR_INVALID_MOTION_TIMES = 18,
    NXG_ERROR_MOTION_POINT_CAPACITY_TOO_SMALL = 19,
    NXG_ERROR_OUTPUT_SIZE_OVERFLOW = 20,
    /* additions of this library */
    NXG_ERROR_INVALID_ARGUMENT = 64,      /* a required descriptor pointer is NULL */
    NXG_ERROR_INVALID_STRAND_RANGE = 65,  /* first + count exceeds strand_count */
    NXG_ERROR_WORKSPACE_TOO_SMALL = 66,   /* workspace missing or below the queried size */
    NXG_ERROR_MISALIGNED_OUTPUT = 67,     /* points not 16-byte aligned, or workspace not 256-byte aligned */
    NXG_ERROR_STATIC_SCRATCH_LIMIT = 68,  /* request needs more than NXG_STATIC_SCRATCH_BYTES of scratch */
    NXG_ERROR_EXPRESSION_SYNTAX = 69,     /* expression did not compile; see the message buffer */
    NXG_ERROR_EXPRESSION_LIMIT = 70,      /* program exceeds the device form's limits */
    NXG_ERROR_EXPRESSION_INPUT = 71,      /* expression uses a variable this runtime cannot bind */
    NXG_ERROR_EXPRESSION_DOMAIN = 72,     /* device evaluation gave a non-finite value or negative length */
    NXG_ERROR_SURROGATE = 73,             /* surrogate model missing, untrained or misconfigured */
    NXG_ERROR_CUDA = 96                   /* a CUDA runtime call failed; see nxg_last_cuda_error */
} nxg_error;

/* --------------------------------------------------------------------- */
/* Errors and version                                                     */
/* --------------------------------------------------------------------- */

/* device_contract.h:82-116 device_generation_error_message. */
const char *nxg_error_message(uint32_t code);

/* ABI version (NXG_ABI_VERSION of the built library). */
uint32_t nxg_abi_version(void);

/* Last CUDA runtime error seen by this library on the calling thread
 * (a cudaError_t value, 0 when none); cleared by the next successful call. */
int32_t nxg_last_cuda_error(void);

/* --------------------------------------------------------------------- */
/* Host asset utilities (no device work)                                  */
/* --------------------------------------------------------------------- */

/* Replaces asset.h:120 / asset.cpp:295-338 validate_asset.  Returns 0 for a
 * valid blob, else 1 and copies the reference's message into `message`.
 * Beyond the reference's checks it rejects stencil entries that are neither
 * < guide_count nor NXG_INVALID_INDEX, and alias entries >= triangle_count,
 * because a device kernel would read out of bounds on them. */
int nxg_validate_asset(const void *bytes, uint64_t size, char *message, uint64_t message_capacity);

/* Replaces asset.h:125-128 / asset.cpp:364-378 make_device_asset_descriptor:
 * validates the host blob, then checks the device pointer (non-NULL,
 * 64-byte aligned) and capacity (>= blob size).  Returns an nxg_error code:
 * INVALID_ASSET_METADATA for a blob that fails validation (message set),
 * NULL_ASSET, MISALIGNED_ASSET or ASSET_CAPACITY_TOO_SMALL for the pointer. */
uint32_t nxg_make_device_asset_descriptor(const void *host_bytes, uint64_t host_size,
                                          const void *device_data, uint64_t device_capacity,
                                          nxg_device_asset_desc *out, char *message,
                                          uint64_t message_capacity);

/* Input of nxg_build_asset, the flattened AssetBuildInput of asset.h:14-44. */
typedef struct nxg_asset_build_input {
    const nxg_vec3 *positions;
    uint32_t vertex_count;
    const nxg_vec3 *normals;       /* NULL: area-weighted normals (asset.cpp:75-86) */
    const nxg_vec2 *texcoords;     /* NULL: no texcoords */
    const nxg_uint3 *triangles;
    uint32_t triangle_count;
    uint32_t guide_count;
    const uint32_t *guide_cv_counts;    /* [guide_count], each in [2, 65535] */
    const nxg_vec3 *guide_cvs;          /* concatenated CVs; CV 0 is the guide root */
    const nxg_vec3 *guide_root_normals; /* [guide_count] */
    const nxg_vec2 *guide_root_uvs;     /* [guide_count] */
    const uint32_t *guide_triangles;    /* [guide_count], NXG_INVALID_INDEX if unbound */
    const nxg_vec2 *guide_barycentrics; /* [guide_count] */
    const float *guide_support_radii;   /* [guide_count], 0 selects the automatic radius */
    uint32_t stencil_slots;  /* 1..8: slots >= this are NXG_INVALID_INDEX; 0 or 8 = reference */
    uint32_t worker_count;   /* host threads for the stencil search; 0 = all cores */
} nxg_asset_build_input;

/* Replaces asset.h:119 / asset.cpp:229-293 build_asset.  Produces a
 * byte-identical blob to the reference for stencil_slots 8.  On success
 * *out_bytes is a 64-byte aligned buffer to release with nxg_free. */
int nxg_build_asset(const nxg_asset_build_input *input, void **out_bytes, uint64_t *out_size,
                    char *message, uint64_t message_capacity);
void nxg_free(void *pointer);

/* nxg_build_asset with its two all-pairs searches run on the current CUDA
 * device: the per-triangle stencil search (asset.cpp:252-269, triangle_count
 * x guide_count candidates) and the nearest other root of each guide behind
 * the automatic support radius (asset.cpp:88-97, guide_count^2 distances);
 * worker_count is ignored.  The blob
 * is byte-identical to nxg_build_asset's for the same input.  Copies the
 * mesh and guide roots to the device, copies the rows back and synchronizes
 * `stream` (a cudaStream_t as void *, NULL = legacy default stream) before
 * returning.  A CUDA failure returns 1 with the CUDA error text in
 * `message` (and the code in nxg_last_cuda_error). */
int nxg_build_asset_device(const nxg_asset_build_input *input, void *stream, void **out_bytes,
                           uint64_t *out_size, char *message, uint64_t message_capacity);

/* The stencil search alone on device buffers; enqueues one kernel on
 * `stream`.  positions [vertex_count] and triangles [triangle_count] are the
 * mesh; guide_roots [guide_count] are the guides' first CVs and
 * guide_normals their root normals normalized as the asset's guide records
 * hold them (nxg_guide_record.root_normal).  Writes stencil [triangle_count
 * x 8] (16-byte aligned): per triangle the min(8, guide_count) guides of
 * smallest |centroid - root|^2 (+1e20 where dot(face normal, root normal) <
 * -0.25), ascending by (score, guide index), slots >= stencil_slots (1..8;
 * 0 = 8) NXG_INVALID_INDEX.  A triangle with a vertex index >= vertex_count
 * gets an all-invalid row.  Returns INVALID_ARGUMENT (NULL pointer, zero
 * count, stencil_slots > 8), MISALIGNED_OUTPUT, CUDA or NONE. */
uint32_t nxg_build_stencils_device(const nxg_vec3 *positions, uint32_t vertex_count,
                                   const nxg_uint3 *triangles, uint32_t triangle_count,
                                   const nxg_vec3 *guide_roots, const nxg_vec3 *guide_normals,
                                   uint32_t guide_count, uint32_t stencil_slots, uint32_t *stencil,
                                   void *stream);

/* FNV-1a 64 over a byte range (asset.cpp:34-41). */
uint64_t nxg_fnv1a(const void *bytes, uint64_t size);

/* --------------------------------------------------------------------- */
/* Checked boundary: pure validators (no device access)                   */
/* --------------------------------------------------------------------- */

/* device_contract.h:190-219 validate_device_generation_request. */
uint32_t nxg_validate_generation_request(const nxg_device_asset_desc *asset,
                                         const nxg_deformed_desc *deformed,
                                         const nxg_generation_params *params,
                                         const nxg_generated_output_desc *output,
                                         const nxg_launch_config *config);

/* device_contract.h:221-254 validate_device_packed_generation_request.
 * `deformed` and `config` may be NULL (no deformation, block size 128). */
uint32_t nxg_validate_packed_request(const nxg_device_asset_desc *asset,
                                     const nxg_deformed_desc *deformed,
                                     const nxg_generation_params *params,
                                     const nxg_packed_output_desc *output,
                                     const nxg_launch_config *config);

/* device_contract.h:256-288 validate_device_motion_generation_request. */
uint32_t nxg_validate_motion_request(const nxg_device_asset_desc *asset,
                                     const nxg_motion_sample_desc *samples,
                                     uint32_t sample_count,
                                     const nxg_generation_params *params,
                                     const nxg_motion_output_desc *output,
                                     const nxg_launch_config *config);

/* --------------------------------------------------------------------- */
/* Generation (enqueue-only, caller-owned buffers)                         */
/* --------------------------------------------------------------------- */

/* Bytes of device workspace nxg_generate_packed needs for `strand_count`
 * strands of this asset at params->cvs_per_strand CVs: the strand-locality
 * sort (keys, permutation, per-guide bins) and the per-frame guide-offset
 * table (guide_count x cvs_per_strand float4, then 2 guide records per guide
 * and 32 zero entries).  The workspace must be
 * 256-byte aligned; its contents need no initialisation. */
uint64_t nxg_packed_workspace_size(const nxg_device_asset_desc *asset, const nxg_generation_params *params,
                                   uint32_t strand_count);

/* The device form of asset.cpp:412-449 generate_packed_cpu /
 * generate_packed_deformed_cpu over generate.h:612-642
 * generate_packed_strand: validates exactly as nxg_validate_packed_request,
 * then enqueues the generator on `stream`.  Writes, for every strand s,
 * points[s*P .. s*P+P-1] = float4(position, 0.5*width*radius_scale) and the
 * optional roots[s], root_uvs[s], point_counts[s] = P. */
uint32_t nxg_generate_packed(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                             const nxg_generation_params *params,
                             const nxg_packed_output_desc *output,
                             const nxg_launch_config *config, void *workspace,
                             uint64_t workspace_bytes, void *stream);

/* Same as nxg_generate_packed for the strands [first_strand, first_strand +
 * strand_count) of a params->strand_count-strand description; strand s
 * writes output record s - first_strand.  This is the shard unit when
 * several GPUs split one description (strand identity stays global). */
uint32_t nxg_generate_packed_range(const nxg_device_asset_desc *asset,
                                   const nxg_deformed_desc *deformed,
                                   const nxg_generation_params *params,
                                   const nxg_packed_output_desc *output,
                                   const nxg_launch_config *config, uint32_t first_strand,
                                   uint32_t strand_count, void *workspace,
                                   uint64_t workspace_bytes, void *stream);

/* Phase 1 of nxg_generate_packed_range, for callers that reuse one strand
 * order across several generations of the same strands (motion samples,
 * repeated frames): sorts strands [first_strand, first_strand+strand_count)
 * by the first stencil guide of their root triangle into `workspace`.  The
 * order depends only on the asset, params->seed and the range. */
uint32_t nxg_prepare_strand_order(const nxg_device_asset_desc *asset, const nxg_generation_params *params,
                                  uint32_t first_strand, uint32_t strand_count, void *workspace,
                                  uint64_t workspace_bytes, void *stream);

/* Phase 2: rebuilds the frame's guide-offset table in `workspace` and runs
 * the generator over the order nxg_prepare_strand_order left there (same
 * asset, seed and range).  The order only decides which strands share a CTA
 * (cache locality); the output does not depend on it. */
uint32_t nxg_generate_packed_ordered(const nxg_device_asset_desc *asset,
                                     const nxg_deformed_desc *deformed,
                                     const nxg_generation_params *params,
                                     const nxg_packed_output_desc *output,
                                     const nxg_launch_config *config, uint32_t first_strand,
                                     uint32_t strand_count, void *workspace,
                                     uint64_t workspace_bytes, void *stream);

/* Tile of the warp-parallel generator: a group of `lanes_per_strand` lanes
 * (2, 4, 8, 16 or 32) owns one strand, each lane `cvs_per_lane` consecutive
 * CVs (1, 2 or 4; lanes * cvs <= 128 and >= the strand's CVs); a CTA has
 * `block_size` threads (0: take nxg_launch_config::block_size).
 * lanes_per_strand 1 (with cvs_per_lane 1, strands of 2..32 CVs) selects the
 * lane-walk generator: base curve and stores lane-parallel, one lane walking
 * each strand's noise frame; with noise and block_size 64 (or below) its
 * CTAs are producer/consumer warp pairs; with noise, CTAs of eleven warps
 * keep ten noise-lattice columns per axis and strand, smaller CTAs twelve (a
 * warp holding a strand whose noise needs more evaluates gradient noise
 * directly).  It is the built-in choice for 2..32 CVs (352-thread CTAs with
 * noise, 256 without). */
typedef struct nxg_tile {
    uint32_t lanes_per_strand;
    uint32_t cvs_per_lane;
    uint32_t block_size;
} nxg_tile;

/* Registers, for this process, the tile used for strands of
 * `cvs_per_strand` CVs with noise off (0) or on (1); NULL restores the
 * built-in choice.  Thread-safe; takes effect at the next launch. */
uint32_t nxg_set_tile(uint32_t cvs_per_strand, uint32_t noise, const nxg_tile *tile);

/* The tile the next launch for this CV count and noise setting will use. */
uint32_t nxg_get_tile(uint32_t cvs_per_strand, uint32_t noise, nxg_tile *tile);

/* Autotuner: prepares the strand order, then times every admissible tile
 * (lane groups and CVs per lane that hold the strand, CTAs of
 * 64/128/256/320/352 threads) over `repeats` launches of nxg_generate_packed_ordered with CUDA
 * events on `stream`, registers the fastest with nxg_set_tile and returns
 * it.  It writes the outputs and synchronises the stream, so it is a
 * set-up call, not part of the enqueue-only path. */
uint32_t nxg_autotune_packed(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                             const nxg_generation_params *params, const nxg_packed_output_desc *output,
                             uint32_t first_strand, uint32_t strand_count, void *workspace,
                             uint64_t workspace_bytes, uint32_t repeats, void *stream, nxg_tile *best,
                             float *best_ms);

/* Motion samples of one description in one enqueue (the device form of one
 * generate_packed_deformed_cpu call per shutter sample, asset.cpp:421-449):
 * sample i (strictly increasing finite times, each deformation validated as
 * in device_contract.h:256-288) is written to outputs[i], a packed output
 * with the same contract as nxg_generate_packed's.  The strand order is
 * prepared once for all samples; strand identities are shared. */
uint32_t nxg_generate_motion_packed(const nxg_device_asset_desc *asset,
                                    const nxg_motion_sample_desc *samples, uint32_t sample_count,
                                    const nxg_generation_params *params,
                                    const nxg_packed_output_desc *outputs,
                                    const nxg_launch_config *config, void *workspace,
                                    uint64_t workspace_bytes, void *stream);

/* The reference's motion contract (device_contract.h:42-53, :256-288):
 * validated exactly as nxg_validate_motion_request, then writes sample-major
 * absolute Vec3 positions, strand_count * cvs_per_strand per sample. */
uint32_t nxg_generate_motion(const nxg_device_asset_desc *asset, const nxg_motion_sample_desc *samples,
                             uint32_t sample_count, const nxg_generation_params *params,
                             const nxg_motion_output_desc *output, const nxg_launch_config *config,
                             void *workspace, uint64_t workspace_bytes, void *stream);

/* Descriptions per nxg_generate_batched call. */
#define NXG_MAX_BATCH 32u

/* Workspace bytes of nxg_generate_batched for these descriptions. */
uint64_t nxg_batched_workspace_size(const nxg_device_asset_desc *assets, const nxg_generation_params *params,
                                    uint32_t count);

/* Several descriptions -- each its own asset, strand count, CV count (<= 128),
 * stencil and noise settings -- in one persistent generate launch per work
 * class (noisy descriptions on the lane walk, noise-free descriptions, noisy
 * descriptions on lane-group tiles): CTAs pull (description, strand range)
 * work items from an atomic counter, costliest descriptions first, and run
 * each with its description's registered tile (nxg_set_tile /
 * nxg_autotune_packed).  Each class launch after the first is a programmatic
 * dependent launch of the one before (the classes share no output), so its
 * CTAs start on the SMs the earlier class leaves idle.  Every description is
 * validated as by nxg_validate_packed_request and written as by
 * nxg_generate_packed; `deformed` is NULL or an array of `count`.  Five
 * set-up launches plus one per class with work, all enqueue-only (capturable
 * as one graph, where the chaining becomes programmatic edges). */
uint32_t nxg_generate_batched(const nxg_device_asset_desc *assets, const nxg_deformed_desc *deformed,
                              const nxg_generation_params *params, const nxg_packed_output_desc *outputs,
                              uint32_t count, const nxg_launch_config *config, void *workspace,
                              uint64_t workspace_bytes, void *stream);

/* Size of the library-owned device scratch used by
 * nxg_generate_packed_static_scratch (4 MiB, held on every device that
 * loads the library until the process exits). */
#define NXG_STATIC_SCRATCH_BYTES (4ull << 20)

/* No counterpart in the reference.  nxg_generate_packed for callers that
 * cannot allocate device memory -- a plugin whose host application owns all
 * allocations and their budget, or a frame loop where cudaMalloc would
 * synchronise the device -- using the library's own fixed scratch instead
 * of a caller workspace.  Same validation and output as
 * nxg_generate_packed; returns NXG_ERROR_STATIC_SCRATCH_LIMIT, before
 * touching the device, when nxg_packed_workspace_size for the request
 * exceeds NXG_STATIC_SCRATCH_BYTES (for a 4,096-guide description at 32
 * CVs, about 240,000 strands fit and a million do not).  Allocates
 * nothing.  The first call on each device looks up the scratch's device
 * address (once per device, and again after a device reset gives the device
 * a new context), so make that first call before any stream capture.  Every
 * call shares the one scratch: calls that can overlap on the GPU (different
 * streams without ordering between them) race on it. */
uint32_t nxg_generate_packed_static_scratch(const nxg_device_asset_desc *asset,
                                            const nxg_deformed_desc *deformed,
                                            const nxg_generation_params *params,
                                            const nxg_packed_output_desc *output,
                                            const nxg_launch_config *config, void *stream);

/* Per-strand blend state: the RootSample of generate.h:101-135, the
 * GuideBlendState of generate.h:207-244 and the noise-frame inputs of
 * generate.h:543-552, for stencil parity checks and renderer debugging. */
typedef struct nxg_strand_state {
    nxg_root_sample root;
    uint32_t indices[8];    /* guide blended in each stencil slot, else NXG_INVALID_INDEX */
    float weights[8];       /* its weight, else 0 */
    float weight_sum;
    uint32_t nearest;       /* nearest non-rejected guide, else NXG_INVALID_INDEX */
    nxg_vec3 surface_u;     /* zero unless noise is enabled */
    nxg_vec3 noise_domain;  /* zero unless noise is enabled */
} nxg_strand_state;

/* Evaluates the state above for `count` global strand ids (device array)
 * into `out` (device array), on `stream`.  Uses the device functions of the
 * lane-group and serial generators (strands of more than 32 CVs), so its
 * indices are the ones those generators blend; the lane walk's own choices
 * are reported by nxg_query_walk_states. */
uint32_t nxg_query_strand_states(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                 const nxg_generation_params *params, const uint32_t *strands,
                                 uint32_t count, nxg_strand_state *out, void *stream);

/* The lane-walk generator's own per-strand stencil decisions (the walk
 * generates every strand of 2..32 CVs).  No reference counterpart as an
 * entry point: it exposes, for parity checks, the choices the reference makes
 * inside make_guide_blend_state and interpolate_offset (generate.h:214-266).
 * mode: 0 blend (weight_sum > 1e-12), 1 nearest guide, 2 root normal. */
typedef struct nxg_walk_state {
    uint32_t mode;
    uint32_t nearest;       /* nearest non-rejected guide, else NXG_INVALID_INDEX */
    float weight_sum;       /* the sum the mode was decided on */
    uint32_t slot_count;    /* weighted slots the base step reads */
    uint32_t guides[8];     /* their guides in stencil-slot order, else NXG_INVALID_INDEX */
    float weights[8];       /* their weights (1 for the nearest guide), else 0 */
} nxg_walk_state;

/* Runs the lane walk's setup step for `count` global strand ids (device
 * array) into `out` (device array), on `stream`.  `workspace` (256-byte
 * aligned, at least nxg_packed_workspace_size(asset, params, count) bytes)
 * receives the frame's guide records first, as in generation. */
uint32_t nxg_query_walk_states(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                               const nxg_generation_params *params, const uint32_t *strands, uint32_t count,
                               nxg_walk_state *out, void *workspace, uint64_t workspace_bytes, void *stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* NXG_H */
