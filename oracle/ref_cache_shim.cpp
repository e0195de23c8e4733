// ref_cache_shim.cpp -- test-only extern "C" entry points over the
// reference's curve cache (src/curve_cache.cpp) and renderer payload
// batching (src/curve_payload.cpp), compiled with the reference's own
// sources into oracle/_ref/libnxg_ref.so.  The checker (oracle/checker.py)
// calls them to pin this library's host restatement and device kernels.
#include "nanoxgen/curve_cache.h"
#include "nanoxgen/curve_payload.h"

#include <cstdint>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

using namespace nanoxgen;

namespace {

void put_text(const std::string &text, char *msg, std::uint64_t cap) {
    if (!msg || cap == 0u) { return; }
    const std::size_t n = std::min<std::size_t>(text.size(), static_cast<std::size_t>(cap - 1u));
    std::memcpy(msg, text.data(), n);
    msg[n] = '\0';
}

template <class T>
std::span<const T> span_of(const void *p, std::uint64_t n) {
    return n ? std::span<const T>(static_cast<const T *>(p), static_cast<std::size_t>(n)) : std::span<const T>{};
}

} // namespace

extern "C" {

// build_curve_cache.  Counts are element counts (points: PackedCurvePoint,
// uvs: Vec2, motion points: Vec3).  Returns the blob size (0 on error, with
// the exception text in msg); copies the blob into `out` when out_capacity
// allows.
std::uint64_t ref_curve_cache_build(const std::uint32_t *counts, std::uint64_t strands, const float *points,
                                    std::uint64_t point_count, const float *texcoords, std::uint64_t texcoord_count,
                                    const float *patch_uvs, std::uint64_t patch_count, const float *face_uvs,
                                    std::uint64_t face_count, const std::uint32_t *face_ids,
                                    std::uint64_t face_id_count, const float *motion_times,
                                    std::uint64_t sample_count, const float *motion_points,
                                    std::uint64_t motion_point_count, void *out, std::uint64_t out_capacity,
                                    char *msg, std::uint64_t cap) {
    try {
        const CurveCache cache = build_curve_cache(
            {span_of<std::uint32_t>(counts, strands), span_of<PackedCurvePoint>(points, point_count),
             span_of<Vec2>(texcoords, texcoord_count), span_of<Vec2>(patch_uvs, patch_count),
             span_of<Vec2>(face_uvs, face_count), span_of<std::uint32_t>(face_ids, face_id_count),
             span_of<float>(motion_times, sample_count), span_of<Vec3>(motion_points, motion_point_count)});
        const std::span<const std::byte> bytes = cache.bytes();
        if (out && out_capacity >= bytes.size()) { std::memcpy(out, bytes.data(), bytes.size()); }
        put_text("", msg, cap);
        return bytes.size();
    } catch (const std::exception &e) {
        put_text(e.what(), msg, cap);
        return 0u;
    }
}

// validate_curve_cache's message ("" when valid).
void ref_curve_cache_validate(const void *bytes, std::uint64_t size, char *msg, std::uint64_t cap) {
    put_text(validate_curve_cache(std::span<const std::byte>(static_cast<const std::byte *>(bytes),
                                                             static_cast<std::size_t>(size))),
             msg, cap);
}

} // extern "C"
