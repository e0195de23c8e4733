// curve_cache.cu -- the renderer curve cache (.nxc): building and validating
// blobs on the host, and validating a device copy on sm_100a.
//
// The host functions restate src/curve_cache.cpp: the same blob layout
// (CurveCacheHeader + 16-byte aligned sections in a fixed order), the same
// word-serial content hash, the same checks in the same order with the same
// messages.  The device check runs every element check of
// validate_curve_cache in one pass over the device copy -- count bounds and
// their sum, finite points and non-negative radii, finite texcoords, motion
// samples and strand uvs -- and reports the first failure in the reference's
// order from per-check minimum indices; it also sums a bit checksum of the
// points.  The content hash is a serial chain over 64-bit words (each step
// multiplies the previous hash), so it has no parallel form and stays on the
// host.
#include "nxg.h"
#include "nxg_cache.h"
#include "nxg_internal.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

static_assert(sizeof(nxg_curve_cache_header) == 128u, "CurveCacheHeader is 128 bytes");

namespace nxg {

// The launch helpers of generate.cu (declared with the generator's kernels).
uint32_t record_cuda(cudaError_t e);
int device_sm_count();

namespace cache {

constexpr uint32_t kKnownFlags = NXG_CURVE_CACHE_HAS_TEXCOORDS | NXG_CURVE_CACHE_HAS_PATCH_UVS |
                                 NXG_CURVE_CACHE_HAS_FACE_UVS | NXG_CURVE_CACHE_HAS_FACE_IDS |
                                 NXG_CURVE_CACHE_HAS_MOTION;
constexpr uint64_t kSectionAlignment = 16u;

const char *const kMessages[NXG_CACHE_ERROR_COUNT] = {
    "",
    "blob is smaller than CurveCacheHeader",
    "curve-cache base is not 64-byte aligned",
    "bad curve-cache magic",
    "unsupported curve-cache major version",
    "curve cache has unknown flags",
    "curve-cache byte_size mismatch",
    "curve cache is empty",
    "curve-cache motion flag/count mismatch",
    "one or more curve-cache sections are out of bounds",
    "curve-cache content hash mismatch",
    "curve cache contains a curve with fewer than two CVs",
    "curve-cache point counts do not sum to point_count",
    "curve cache contains an invalid point or radius",
    "curve cache contains an invalid texcoord",
    "curve cache contains invalid motion times",
    "curve cache contains an invalid motion position",
    "curve cache contains an invalid patch UV",
    "curve cache contains an invalid face UV",
};

// content_hash (src/curve_cache.cpp:35-54): per 64-bit little-endian word
// xor, multiply, xor-shift; the tail bytes zero-extended into one word.
uint64_t content_hash(const unsigned char *bytes, uint64_t size) {
    constexpr uint64_t prime = 0x9e3779b185ebca87ull;
    uint64_t hash = 0x243f6a8885a308d3ull ^ size;
    uint64_t offset = 0u;
    for (; offset + 8u <= size; offset += 8u) {
        uint64_t word;
        std::memcpy(&word, bytes + offset, 8u);
        hash ^= word;
        hash *= prime;
        hash ^= hash >> 29u;
    }
    uint64_t tail = 0u;
    if (size > offset) { std::memcpy(&tail, bytes + offset, static_cast<size_t>(size - offset)); }
    hash ^= tail + prime;
    hash *= 0xc2b2ae3d27d4eb4full;
    hash ^= hash >> 32u;
    return hash;
}

// section_fits (src/curve_cache.cpp:56-64).
bool section_fits(const nxg_curve_cache_header &h, uint64_t offset, uint64_t count, uint64_t element,
                  uint64_t alignment) {
    if (count == 0u) { return offset == 0u; }
    if (offset < sizeof(nxg_curve_cache_header) || offset > h.byte_size) { return false; }
    if (count > std::numeric_limits<uint64_t>::max() / element) { return false; }
    return count * element <= h.byte_size - offset && offset % alignment == 0u;
}

// The checks of validate_curve_cache that read only the header, in its
// order (src/curve_cache.cpp:173-211).
uint32_t check_header(const nxg_curve_cache_header &h, uint64_t size) {
    if (h.magic != NXG_CURVE_CACHE_MAGIC) { return NXG_CACHE_BAD_MAGIC; }
    if (h.version_major != NXG_CURVE_CACHE_VERSION_MAJOR) { return NXG_CACHE_BAD_VERSION; }
    if ((h.flags & ~kKnownFlags) != 0u) { return NXG_CACHE_UNKNOWN_FLAGS; }
    if (h.byte_size != size) { return NXG_CACHE_SIZE_MISMATCH; }
    if (h.strand_count == 0u || h.point_count == 0u) { return NXG_CACHE_EMPTY; }
    if (((h.flags & NXG_CURVE_CACHE_HAS_MOTION) != 0u) != (h.motion_sample_count != 0u)) {
        return NXG_CACHE_MOTION_MISMATCH;
    }
    const uint64_t motion_points = uint64_t{h.motion_sample_count} * h.point_count;
    const auto optional = [&h](uint32_t flag, uint64_t count) { return (h.flags & flag) ? count : 0u; };
    if (!section_fits(h, h.point_counts_offset, h.strand_count, 4u, 4u) ||
        !section_fits(h, h.points_offset, h.point_count, 16u, 16u) ||
        !section_fits(h, h.motion_times_offset, h.motion_sample_count, 4u, 4u) ||
        !section_fits(h, h.motion_points_offset, motion_points, 12u, 4u) ||
        !section_fits(h, h.texcoords_offset, optional(NXG_CURVE_CACHE_HAS_TEXCOORDS, h.point_count), 8u, 4u) ||
        !section_fits(h, h.patch_uvs_offset, optional(NXG_CURVE_CACHE_HAS_PATCH_UVS, h.strand_count), 8u, 4u) ||
        !section_fits(h, h.face_uvs_offset, optional(NXG_CURVE_CACHE_HAS_FACE_UVS, h.strand_count), 8u, 4u) ||
        !section_fits(h, h.face_ids_offset, optional(NXG_CURVE_CACHE_HAS_FACE_IDS, h.strand_count), 4u, 4u)) {
        return NXG_CACHE_SECTION_BOUNDS;
    }
    return NXG_CACHE_OK;
}

bool finite2(const float *v) { return std::isfinite(v[0]) && std::isfinite(v[1]); }

template <class T>
const T *section(const unsigned char *blob, uint64_t offset) {
    return offset ? reinterpret_cast<const T *>(blob + offset) : nullptr;
}

// validate_curve_cache (src/curve_cache.cpp:173-251).
uint32_t validate(const unsigned char *blob, uint64_t size) {
    if (size < sizeof(nxg_curve_cache_header)) { return NXG_CACHE_TOO_SMALL; }
    if (reinterpret_cast<uintptr_t>(blob) % 64u != 0u) { return NXG_CACHE_MISALIGNED; }
    nxg_curve_cache_header h;
    std::memcpy(&h, blob, sizeof h);
    if (const uint32_t e = check_header(h, size)) { return e; }
    if (content_hash(blob + sizeof h, size - sizeof h) != h.content_hash) { return NXG_CACHE_HASH_MISMATCH; }
    const uint32_t *counts = section<uint32_t>(blob, h.point_counts_offset);
    uint64_t sum = 0u;
    for (uint32_t s = 0; s < h.strand_count; ++s) {
        if (counts[s] < 2u) { return NXG_CACHE_SHORT_CURVE; }
        sum += counts[s];
    }
    if (sum != h.point_count) { return NXG_CACHE_POINT_SUM; }
    const float *points = section<float>(blob, h.points_offset);
    const float *texcoords = section<float>(blob, h.texcoords_offset);
    for (uint32_t i = 0; i < h.point_count; ++i) {
        const float *p = points + 4u * uint64_t{i};
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]) || !std::isfinite(p[3]) ||
            p[3] < 0.0f) {
            return NXG_CACHE_BAD_POINT;
        }
        if (texcoords && !finite2(texcoords + 2u * uint64_t{i})) { return NXG_CACHE_BAD_TEXCOORD; }
    }
    const float *times = section<float>(blob, h.motion_times_offset);
    float previous = -std::numeric_limits<float>::infinity();
    for (uint32_t k = 0; k < h.motion_sample_count; ++k) {
        if (!std::isfinite(times[k]) || times[k] <= previous) { return NXG_CACHE_BAD_MOTION_TIMES; }
        previous = times[k];
    }
    const float *motion = section<float>(blob, h.motion_points_offset);
    const uint64_t motion_count = uint64_t{h.motion_sample_count} * h.point_count;
    for (uint64_t i = 0; i < motion_count; ++i) {
        const float *p = motion + 3u * i;
        if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) {
            return NXG_CACHE_BAD_MOTION_POINT;
        }
    }
    const float *patch = section<float>(blob, h.patch_uvs_offset);
    const float *face = section<float>(blob, h.face_uvs_offset);
    for (uint32_t s = 0; s < h.strand_count; ++s) {
        if (patch && !finite2(patch + 2u * uint64_t{s})) { return NXG_CACHE_BAD_PATCH_UV; }
        if (face && !finite2(face + 2u * uint64_t{s})) { return NXG_CACHE_BAD_FACE_UV; }
    }
    return NXG_CACHE_OK;
}

// SplitMix64's finaliser (Steele, Lea and Flood, "Fast splittable
// pseudorandom number generators", OOPSLA 2014).
__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30u)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27u)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31u);
}

// The checksum term of point `index` from its two 64-bit words (x, y) and
// (z, radius): one SplitMix64 finalisation of (xy ^ index * G) + zw * K, with
// G the golden-ratio constant and K odd (so every bit of either word reaches
// the mix).
__host__ __device__ inline uint64_t point_term(uint64_t xy, uint64_t zw, uint64_t index) {
    return mix64((xy ^ (index * 0x9e3779b97f4a7c15ull)) + zw * 0xd6e8feb86659fd93ull);
}

// build_curve_cache (src/curve_cache.cpp:104-171): the input checks with the
// reference's messages, then header + sections, each at a 16-byte aligned
// offset (zero gaps), and the content hash.  Throws std::invalid_argument.
std::vector<unsigned char> build(const nxg_curve_cache_input &in) {
    const auto fail = [](const std::string &m) { throw std::invalid_argument(m); };
    if (in.strand_count == 0u || in.point_count == 0u || !in.point_counts || !in.points) {
        fail("curve cache needs curves and points");
    }
    if (in.strand_count > std::numeric_limits<uint32_t>::max() ||
        in.point_count > std::numeric_limits<uint32_t>::max()) {
        fail("curve cache v1 count exceeds uint32");
    }
    uint64_t sum = 0u;
    for (uint64_t s = 0; s < in.strand_count; ++s) {
        if (in.point_counts[s] < 2u) { fail("curve cache curve has fewer than two CVs"); }
        sum += in.point_counts[s];
    }
    if (sum != in.point_count) { fail("curve cache point counts do not match point array"); }
    const auto optional = [&fail](uint64_t n, uint64_t expected, const char *name) {
        if (n != 0u && n != expected) { fail(std::string("curve cache ") + name + " size mismatch"); }
    };
    optional(in.texcoord_count, in.point_count, "texcoord");
    optional(in.patch_uv_count, in.strand_count, "patch-UV");
    optional(in.face_uv_count, in.strand_count, "face-UV");
    optional(in.face_id_count, in.strand_count, "face-ID");
    if (in.motion_sample_count > std::numeric_limits<uint32_t>::max()) {
        fail("curve cache has too many motion samples");
    }
    if ((in.motion_sample_count == 0u) != (in.motion_point_count == 0u)) {
        fail("curve cache motion times and positions must both be present");
    }
    if (in.motion_sample_count != 0u && in.motion_point_count != in.point_count * in.motion_sample_count) {
        fail("curve cache motion-position size mismatch");
    }
    float previous = -std::numeric_limits<float>::infinity();
    for (uint64_t k = 0; k < in.motion_sample_count; ++k) {
        if (!std::isfinite(in.motion_times[k]) || in.motion_times[k] <= previous) {
            fail("curve cache motion times must be finite and increasing");
        }
        previous = in.motion_times[k];
    }
    std::vector<unsigned char> blob(sizeof(nxg_curve_cache_header), 0u);
    nxg_curve_cache_header h{};
    h.magic = NXG_CURVE_CACHE_MAGIC;
    h.version_major = NXG_CURVE_CACHE_VERSION_MAJOR;
    h.strand_count = static_cast<uint32_t>(in.strand_count);
    h.point_count = static_cast<uint32_t>(in.point_count);
    h.motion_sample_count = static_cast<uint32_t>(in.motion_sample_count);
    if (in.texcoord_count) { h.flags |= NXG_CURVE_CACHE_HAS_TEXCOORDS; }
    if (in.patch_uv_count) { h.flags |= NXG_CURVE_CACHE_HAS_PATCH_UVS; }
    if (in.face_uv_count) { h.flags |= NXG_CURVE_CACHE_HAS_FACE_UVS; }
    if (in.face_id_count) { h.flags |= NXG_CURVE_CACHE_HAS_FACE_IDS; }
    if (in.motion_sample_count) { h.flags |= NXG_CURVE_CACHE_HAS_MOTION; }
    const auto append = [&blob](const void *data, uint64_t bytes) -> uint64_t {
        if (bytes == 0u) { return 0u; }
        const uint64_t offset = (blob.size() + kSectionAlignment - 1u) / kSectionAlignment * kSectionAlignment;
        blob.resize(offset + bytes, 0u);
        std::memcpy(blob.data() + offset, data, bytes);
        return offset;
    };
    h.point_counts_offset = append(in.point_counts, 4u * in.strand_count);
    h.points_offset = append(in.points, 16u * in.point_count);
    h.motion_times_offset = append(in.motion_times, 4u * in.motion_sample_count);
    h.motion_points_offset = append(in.motion_points, 12u * in.motion_point_count);
    h.texcoords_offset = append(in.texcoords, 8u * in.texcoord_count);
    h.patch_uvs_offset = append(in.patch_uvs, 8u * in.patch_uv_count);
    h.face_uvs_offset = append(in.face_uvs, 8u * in.face_uv_count);
    h.face_ids_offset = append(in.face_ids, 4u * in.face_id_count);
    h.byte_size = blob.size();
    h.content_hash = content_hash(blob.data() + sizeof h, blob.size() - sizeof h);
    std::memcpy(blob.data(), &h, sizeof h);
    return blob;
}

// ---------------------------------------------------------------- device

struct CheckArgs {
    const unsigned char *blob;
    nxg_curve_cache_check *result;
    uint64_t counts_offset, points_offset, texcoords_offset, motion_points_offset, patch_offset, face_offset,
        times_offset;
    uint64_t motion_count;
    uint32_t strands, points, samples;
};

// first_bad slots, one per element check.
enum : int { kBadCount = 0, kBadPoint, kBadTexcoord, kBadMotion, kBadPatch, kBadFace };

__global__ void check_init_kernel(nxg_curve_cache_check *r) {
    if (threadIdx.x < 8u) { r->first_bad[threadIdx.x] = ~0ull; }
    if (threadIdx.x == 0u) {
        r->error = NXG_CACHE_OK;
        r->reserved = 0u;
        r->point_sum = 0u;
        r->checksum = 0u;
    }
}

__device__ __forceinline__ uint64_t warp_sum(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { v += __shfl_xor_sync(0xffffffffu, v, o); }
    return v;
}

__device__ __forceinline__ bool finite_f(float x) { return isfinite(x); }

// One pass over the device copy: every element check records its first
// failing index (atomicMin, taken only on a failure); the counts and the bit
// checksum accumulate per thread across the grid-stride loops and leave as
// one warp sum and one atomicAdd per warp.
__global__ void __launch_bounds__(256) check_kernel(const CheckArgs a) {
    nxg_curve_cache_check *r = a.result;
    const uint64_t stride = uint64_t{gridDim.x} * blockDim.x;
    const uint64_t start = uint64_t{blockIdx.x} * blockDim.x + threadIdx.x;
    uint64_t count_sum = 0u, checksum = 0u;
    // point counts
    const uint32_t *counts = reinterpret_cast<const uint32_t *>(a.blob + a.counts_offset);
    for (uint64_t s = start; s < a.strands; s += stride) {
        const uint32_t c = __ldcs(counts + s);
        if (c < 2u) { atomicMin(reinterpret_cast<unsigned long long *>(&r->first_bad[kBadCount]), s); }
        count_sum += c;
    }
    // points (with their texcoords) and the bit checksum: four points per
    // thread and pass, their loads issued before any is used
    const float4 *points = reinterpret_cast<const float4 *>(a.blob + a.points_offset);
    const float2 *tex = a.texcoords_offset ? reinterpret_cast<const float2 *>(a.blob + a.texcoords_offset) : nullptr;
    constexpr int kUnroll = 4;
    for (uint64_t base = start; base < a.points; base += kUnroll * stride) {
        float4 p[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t i = base + u * stride;
            p[u] = i < a.points ? __ldcs(points + i) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const uint64_t i = base + u * stride;
            if (i >= a.points) { break; }
            if (!finite_f(p[u].x) || !finite_f(p[u].y) || !finite_f(p[u].z) || !finite_f(p[u].w) ||
                p[u].w < 0.0f) {
                atomicMin(reinterpret_cast<unsigned long long *>(&r->first_bad[kBadPoint]), i);
            }
            if (tex) {
                const float2 t = __ldcs(tex + i);
                if (!finite_f(t.x) || !finite_f(t.y)) {
                    atomicMin(reinterpret_cast<unsigned long long *>(&r->first_bad[kBadTexcoord]), i);
                }
            }
            const uint64_t xy = uint64_t{__float_as_uint(p[u].x)} | (uint64_t{__float_as_uint(p[u].y)} << 32u);
            const uint64_t zw = uint64_t{__float_as_uint(p[u].z)} | (uint64_t{__float_as_uint(p[u].w)} << 32u);
            checksum += point_term(xy, zw, i);
        }
    }
    count_sum = warp_sum(count_sum);
    checksum = warp_sum(checksum);
    if ((threadIdx.x & 31u) == 0u) {
        if (count_sum) { atomicAdd(reinterpret_cast<unsigned long long *>(&r->point_sum), count_sum); }
        atomicAdd(reinterpret_cast<unsigned long long *>(&r->checksum), checksum);
    }
    const uint64_t first = uint64_t{blockIdx.x} * blockDim.x;
    // motion points (xyz, 4-byte aligned)
    const float *motion = reinterpret_cast<const float *>(a.blob + a.motion_points_offset);
    for (uint64_t i = first + threadIdx.x; i < a.motion_count; i += stride) {
        const float x = __ldcs(motion + 3u * i), y = __ldcs(motion + 3u * i + 1u), z = __ldcs(motion + 3u * i + 2u);
        if (!finite_f(x) || !finite_f(y) || !finite_f(z)) {
            atomicMin(reinterpret_cast<unsigned long long *>(&r->first_bad[kBadMotion]), i);
        }
    }
    // strand uvs
    const float2 *patch = a.patch_offset ? reinterpret_cast<const float2 *>(a.blob + a.patch_offset) : nullptr;
    const float2 *face = a.face_offset ? reinterpret_cast<const float2 *>(a.blob + a.face_offset) : nullptr;
    if (patch || face) {
        for (uint64_t s = first + threadIdx.x; s < a.strands; s += stride) {
            if (patch) {
                const float2 t = __ldcs(patch + s);
                if (!finite_f(t.x) || !finite_f(t.y)) {
                    atomicMin(reinterpret_cast<unsigned long long *>(&r->first_bad[kBadPatch]), s);
                }
            }
            if (face) {
                const float2 t = __ldcs(face + s);
                if (!finite_f(t.x) || !finite_f(t.y)) {
                    atomicMin(reinterpret_cast<unsigned long long *>(&r->first_bad[kBadFace]), s);
                }
            }
        }
    }
}

// The first failure in validate_curve_cache's order (after its content
// hash): counts, their sum, the point loop (point before texcoord at one
// index), motion times (serial, here), motion points, the strand loop
// (patch uv before face uv at one index).
__global__ void check_finish_kernel(const CheckArgs a) {
    nxg_curve_cache_check *r = a.result;
    const uint64_t *b = r->first_bad;
    uint32_t e = NXG_CACHE_OK;
    bool times_bad = false;
    const float *times = reinterpret_cast<const float *>(a.blob + a.times_offset);
    float previous = -INFINITY;
    for (uint32_t k = 0; k < a.samples; ++k) {
        const float t = times[k];
        if (!isfinite(t) || t <= previous) {
            times_bad = true;
            break;
        }
        previous = t;
    }
    if (b[kBadCount] != ~0ull) {
        e = NXG_CACHE_SHORT_CURVE;
    } else if (r->point_sum != a.points) {
        e = NXG_CACHE_POINT_SUM;
    } else if (min(b[kBadPoint], b[kBadTexcoord]) != ~0ull) {
        e = b[kBadPoint] <= b[kBadTexcoord] ? NXG_CACHE_BAD_POINT : NXG_CACHE_BAD_TEXCOORD;
    } else if (times_bad) {
        e = NXG_CACHE_BAD_MOTION_TIMES;
    } else if (b[kBadMotion] != ~0ull) {
        e = NXG_CACHE_BAD_MOTION_POINT;
    } else if (min(b[kBadPatch], b[kBadFace]) != ~0ull) {
        e = b[kBadPatch] <= b[kBadFace] ? NXG_CACHE_BAD_PATCH_UV : NXG_CACHE_BAD_FACE_UV;
    }
    r->error = e;
}

} // namespace cache
} // namespace nxg

extern "C" {

const char *nxg_curve_cache_error_message(uint32_t code) {
    return code < NXG_CACHE_ERROR_COUNT ? nxg::cache::kMessages[code] : "unknown curve-cache error";
}

uint32_t nxg_curve_cache_build(const nxg_curve_cache_input *input, void **blob, uint64_t *size, char *msg,
                               uint64_t msg_capacity) {
    const auto message = [msg, msg_capacity](const std::string &text) {
        if (msg && msg_capacity) {
            const size_t n = std::min<size_t>(text.size(), static_cast<size_t>(msg_capacity - 1u));
            std::memcpy(msg, text.data(), n);
            msg[n] = '\0';
        }
    };
    if (!input || !blob || !size) { return NXG_ERROR_INVALID_ARGUMENT; }
    *blob = nullptr;
    *size = 0u;
    try {
        const std::vector<unsigned char> bytes = nxg::cache::build(*input);
        void *out = std::aligned_alloc(64u, (bytes.size() + 63u) / 64u * 64u);
        if (!out) {
            message("out of host memory");
            return NXG_ERROR_INVALID_ARGUMENT;
        }
        std::memcpy(out, bytes.data(), bytes.size());
        const uint32_t e = nxg::cache::validate(static_cast<const unsigned char *>(out), bytes.size());
        if (e != NXG_CACHE_OK) {
            std::free(out);
            message(std::string("built an invalid curve cache: ") + nxg::cache::kMessages[e]);
            return NXG_ERROR_INVALID_ARGUMENT;
        }
        *blob = out;
        *size = bytes.size();
        message("");
        return NXG_ERROR_NONE;
    } catch (const std::exception &error) {
        message(error.what());
        return NXG_ERROR_INVALID_ARGUMENT;
    }
}

uint32_t nxg_curve_cache_validate(const void *blob, uint64_t size) {
    if (!blob) { return NXG_CACHE_TOO_SMALL; }
    return nxg::cache::validate(static_cast<const unsigned char *>(blob), size);
}

uint64_t nxg_curve_cache_content_hash(const void *bytes, uint64_t size) {
    return nxg::cache::content_hash(static_cast<const unsigned char *>(bytes), size);
}

uint64_t nxg_curve_cache_point_checksum(const void *blob, uint64_t size) {
    if (!blob || size < sizeof(nxg_curve_cache_header)) { return 0u; }
    nxg_curve_cache_header h;
    std::memcpy(&h, blob, sizeof h);
    if (!h.points_offset || !nxg::cache::section_fits(h, h.points_offset, h.point_count, 16u, 16u) ||
        h.byte_size != size) {
        return 0u;
    }
    const unsigned char *p = static_cast<const unsigned char *>(blob) + h.points_offset;
    uint64_t sum = 0u;
    for (uint64_t i = 0; i < h.point_count; ++i) {
        uint64_t xy, zw;
        std::memcpy(&xy, p + 16u * i, 8u);
        std::memcpy(&zw, p + 16u * i + 8u, 8u);
        sum += nxg::cache::point_term(xy, zw, i);
    }
    return sum;
}

uint32_t nxg_curve_cache_validate_device(const nxg_curve_cache_header *header, const void *device_blob,
                                         uint64_t size, nxg_curve_cache_check *device_result,
                                         uint32_t *header_error, void *stream) {
    if (header_error) { *header_error = NXG_CACHE_OK; }
    if (!header || !device_blob || !device_result ||
        reinterpret_cast<uintptr_t>(device_result) % 8u != 0u) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    uint32_t e = NXG_CACHE_OK;
    if (size < sizeof(nxg_curve_cache_header)) {
        e = NXG_CACHE_TOO_SMALL;
    } else if (reinterpret_cast<uintptr_t>(device_blob) % 64u != 0u) {
        e = NXG_CACHE_MISALIGNED;
    } else {
        e = nxg::cache::check_header(*header, size);
    }
    if (e != NXG_CACHE_OK) {
        if (header_error) { *header_error = e; }
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    const nxg_curve_cache_header &h = *header;
    nxg::cache::CheckArgs a{};
    a.blob = static_cast<const unsigned char *>(device_blob);
    a.result = device_result;
    a.counts_offset = h.point_counts_offset;
    a.points_offset = h.points_offset;
    a.texcoords_offset = (h.flags & NXG_CURVE_CACHE_HAS_TEXCOORDS) ? h.texcoords_offset : 0u;
    a.motion_points_offset = h.motion_points_offset;
    a.patch_offset = (h.flags & NXG_CURVE_CACHE_HAS_PATCH_UVS) ? h.patch_uvs_offset : 0u;
    a.face_offset = (h.flags & NXG_CURVE_CACHE_HAS_FACE_UVS) ? h.face_uvs_offset : 0u;
    a.times_offset = h.motion_times_offset;
    a.motion_count = uint64_t{h.motion_sample_count} * h.point_count;
    a.strands = h.strand_count;
    a.points = h.point_count;
    a.samples = h.motion_sample_count;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    nxg::set_last_cuda_error(0);
    nxg::cache::check_init_kernel<<<1, 32, 0, s>>>(device_result);
    int per_sm = 0;
    if (const uint32_t st = nxg::record_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, nxg::cache::check_kernel, 256, 0))) {
        return st;
    }
    const uint64_t largest = std::max<uint64_t>({a.points, a.motion_count, a.strands});
    const uint64_t needed = (largest + 255u) / 256u;
    const uint32_t grid = static_cast<uint32_t>(
        std::max<uint64_t>(1u, std::min<uint64_t>(needed, uint64_t(nxg::device_sm_count()) * std::max(per_sm, 1))));
    nxg::cache::check_kernel<<<grid, 256, 0, s>>>(a);
    nxg::cache::check_finish_kernel<<<1, 1, 0, s>>>(a);
    return nxg::record_cuda(cudaGetLastError());
}

} // extern "C"
