/* nxg_cache.h -- NanoXGen's renderer curve cache (.nxc) on the host and on
 * sm_100a.
 *
 * The blob layout is the reference's CurveCacheHeader + sections
 * (include/nanoxgen/curve_cache.h:19-52, src/curve_cache.cpp): a 128-byte,
 * 64-byte aligned header, then each present section at a 16-byte aligned
 * offset from the header's start, in the order point counts, points
 * (float4 position + radius), motion times, motion points (sample-major
 * xyz), texcoords (per point), patch uvs, face uvs, face ids (per strand);
 * content_hash covers every byte after the header.
 *
 * Entry points and the reference functions they replace:
 *   nxg_curve_cache_build         build_curve_cache     (src/curve_cache.cpp:104-171)
 *   nxg_curve_cache_validate      validate_curve_cache  (src/curve_cache.cpp:173-251)
 *   nxg_curve_cache_content_hash  content_hash          (src/curve_cache.cpp:35-54)
 *   nxg_curve_cache_validate_device   validate_curve_cache's element checks on
 *                                 a device copy, plus a point sum and a bit checksum
 */
#ifndef NXG_CACHE_H
#define NXG_CACHE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NXG_CURVE_CACHE_MAGIC 0x454843414347584eull /* "NXGCACHE" */
#define NXG_CURVE_CACHE_VERSION_MAJOR 1u

enum {
    NXG_CURVE_CACHE_HAS_TEXCOORDS = 1u << 0,
    NXG_CURVE_CACHE_HAS_PATCH_UVS = 1u << 1,
    NXG_CURVE_CACHE_HAS_FACE_UVS = 1u << 2,
    NXG_CURVE_CACHE_HAS_FACE_IDS = 1u << 3,
    NXG_CURVE_CACHE_HAS_MOTION = 1u << 4
};

/* CurveCacheHeader, byte for byte (128 bytes). */
typedef struct nxg_curve_cache_header {
    uint64_t magic;
    uint16_t version_major;
    uint16_t version_minor;
    uint32_t flags;
    uint64_t byte_size;
    uint64_t content_hash;
    uint32_t strand_count;
    uint32_t point_count;
    uint32_t motion_sample_count;
    uint32_t reserved;
    uint64_t point_counts_offset;
    uint64_t points_offset;
    uint64_t motion_times_offset;
    uint64_t motion_points_offset;
    uint64_t texcoords_offset;
    uint64_t patch_uvs_offset;
    uint64_t face_uvs_offset;
    uint64_t face_ids_offset;
    uint8_t padding[16];
} nxg_curve_cache_header;

/* Validation results, in the reference's order of checks.  Their texts are
 * validate_curve_cache's messages (nxg_curve_cache_error_message). */
typedef enum nxg_curve_cache_error {
    NXG_CACHE_OK = 0,
    NXG_CACHE_TOO_SMALL,            /* blob is smaller than CurveCacheHeader */
    NXG_CACHE_MISALIGNED,           /* curve-cache base is not 64-byte aligned */
    NXG_CACHE_BAD_MAGIC,
    NXG_CACHE_BAD_VERSION,
    NXG_CACHE_UNKNOWN_FLAGS,
    NXG_CACHE_SIZE_MISMATCH,
    NXG_CACHE_EMPTY,
    NXG_CACHE_MOTION_MISMATCH,
    NXG_CACHE_SECTION_BOUNDS,
    NXG_CACHE_HASH_MISMATCH,
    NXG_CACHE_SHORT_CURVE,          /* a curve with fewer than two CVs */
    NXG_CACHE_POINT_SUM,
    NXG_CACHE_BAD_POINT,            /* non-finite point or radius, or negative radius */
    NXG_CACHE_BAD_TEXCOORD,
    NXG_CACHE_BAD_MOTION_TIMES,
    NXG_CACHE_BAD_MOTION_POINT,
    NXG_CACHE_BAD_PATCH_UV,
    NXG_CACHE_BAD_FACE_UV,
    NXG_CACHE_ERROR_COUNT
} nxg_curve_cache_error;

const char *nxg_curve_cache_error_message(uint32_t code);

/* The arrays of CurveCacheBuildInput; an optional array has count 0. */
typedef struct nxg_curve_cache_input {
    const uint32_t *point_counts; uint64_t strand_count;
    const float *points;          uint64_t point_count;          /* float4 per point */
    const float *texcoords;       uint64_t texcoord_count;       /* float2 per point */
    const float *patch_uvs;       uint64_t patch_uv_count;       /* float2 per strand */
    const float *face_uvs;        uint64_t face_uv_count;        /* float2 per strand */
    const uint32_t *face_ids;     uint64_t face_id_count;        /* per strand */
    const float *motion_times;    uint64_t motion_sample_count;
    const float *motion_points;   uint64_t motion_point_count;   /* xyz, sample-major */
} nxg_curve_cache_input;

/* build_curve_cache: *blob (64-byte aligned, release with nxg_free) and
 * *size.  Returns 0, or NXG_ERROR_INVALID_ARGUMENT with the reference's
 * exception text in msg. */
uint32_t nxg_curve_cache_build(const nxg_curve_cache_input *input, void **blob, uint64_t *size, char *msg,
                               uint64_t msg_capacity);

/* validate_curve_cache on the host, every check including the content hash:
 * an nxg_curve_cache_error. */
uint32_t nxg_curve_cache_validate(const void *blob, uint64_t size);

/* content_hash over `size` bytes (the blob's bytes after the header). */
uint64_t nxg_curve_cache_content_hash(const void *bytes, uint64_t size);

/* The bit checksum of the device check, on the host: over the points, the
 * sum modulo 2^64 of mix64((xy ^ i * 0x9e3779b97f4a7c15) + zw *
 * 0xd6e8feb86659fd93), with xy and zw point i's two little-endian 64-bit
 * words and mix64 the SplitMix64 finaliser (Steele, Lea and Flood, 2014). */
uint64_t nxg_curve_cache_point_checksum(const void *blob, uint64_t size);

typedef struct nxg_curve_cache_check {
    uint32_t error;          /* nxg_curve_cache_error */
    uint32_t reserved;
    uint64_t point_sum;      /* sum of the point counts */
    uint64_t checksum;       /* nxg_curve_cache_point_checksum of the device copy */
    uint64_t first_bad[8];   /* scratch: first failing index per element check */
} nxg_curve_cache_check;

/* validate_curve_cache on a device copy of a blob, except the serial
 * content hash (the host's nxg_curve_cache_content_hash covers it): the
 * header checks on the host copy `header`, then one pass over the device
 * blob for the element checks, whose first failure in the reference's order
 * lands in device_result->error, with the point sum and the bit checksum.
 * device_result is overwritten (no zeroing needed).  Returns
 * NXG_ERROR_INVALID_ARGUMENT (with the header check's code in *header_error)
 * when the header alone fails; enqueue only otherwise. */
uint32_t nxg_curve_cache_validate_device(const nxg_curve_cache_header *header, const void *device_blob,
                                         uint64_t size, nxg_curve_cache_check *device_result,
                                         uint32_t *header_error, void *stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* NXG_CACHE_H */
