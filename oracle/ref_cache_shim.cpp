// ref_cache_shim.cpp -- test-only extern "C" entry points over the
// reference's curve cache (src/curve_cache.cpp) and renderer payload
// batching (src/curve_payload.cpp), compiled with the reference's own
// sources into oracle/_ref/libnxg_ref.so.  The checker (oracle/checker.py)
// calls them to pin this library's host restatement and device kernels.
#include "nanoxgen/curve_cache.h"
#include "nanoxgen/curve_payload.h"

#include <algorithm>
#include <cstdint>
#include <stdexcept>
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

// build_curve_batches over host arrays, with the batches concatenated.
// A curve set is (strands, fixed CVs, counts or NULL, points [N x 3],
// point count, widths or NULL, root uvs [S x 2] or NULL, roots or NULL,
// constant width); samples are `sample_count` such sets with their times.
// Outputs (capacities in elements): point counts [S], points [total x 4],
// root uvs [S x 2] (written when the batches carry them; *has_uvs says),
// motion points [samples * total x 3], batch first points [batches + 1].
// Returns the total points (0 on error, with the exception text in msg).
struct RefCurveSet {
    std::uint32_t strands, fixed;
    const std::uint32_t *counts;
    const float *points;
    std::uint64_t point_count;
    const float *widths;
    const float *root_uvs;
    const void *roots;
    float constant_width;
};

std::uint64_t ref_build_curve_batches(const RefCurveSet *base, const RefCurveSet *samples, const float *times,
                                      std::uint32_t sample_count, std::uint32_t per_batch, std::uint32_t resample,
                                      float radius_scale, const float *transform, std::uint32_t *out_counts,
                                      float *out_points, float *out_uvs, std::uint32_t *has_uvs, float *out_motion,
                                      std::uint64_t *out_first, std::uint64_t capacity, char *msg,
                                      std::uint64_t cap) {
    try {
        const auto view = [](const RefCurveSet &v) {
            CurveSetView out{};
            out.strand_count = v.strands;
            out.fixed_cvs_per_strand = v.fixed;
            out.point_counts = v.counts ? std::span<const std::uint32_t>(v.counts, v.strands)
                                        : std::span<const std::uint32_t>{};
            out.points = std::span<const Vec3>(reinterpret_cast<const Vec3 *>(v.points), v.point_count);
            out.widths = v.widths ? std::span<const float>(v.widths, v.point_count) : std::span<const float>{};
            out.root_uvs = v.root_uvs ? std::span<const Vec2>(reinterpret_cast<const Vec2 *>(v.root_uvs), v.strands)
                                      : std::span<const Vec2>{};
            out.roots = v.roots ? std::span<const RootSample>(static_cast<const RootSample *>(v.roots), v.strands)
                                : std::span<const RootSample>{};
            out.constant_width = v.constant_width;
            return out;
        };
        std::vector<MotionSampleView> motion;
        for (std::uint32_t k = 0; k < sample_count; ++k) { motion.push_back({times[k], view(samples[k])}); }
        CurvePayloadOptions options{};
        options.max_strands_per_batch = per_batch;
        options.resample_cv_count = resample;
        options.radius_scale = radius_scale;
        std::copy(transform, transform + 12, options.transform.values.begin());
        const std::vector<CurveBatch> batches = build_curve_batches(view(*base), motion, {}, {}, options);
        std::uint64_t strand = 0u, point = 0u, motion_at = 0u;
        *has_uvs = 0u;
        for (std::size_t b = 0; b < batches.size(); ++b) {
            const CurveBatch &batch = batches[b];
            out_first[b] = point;
            if (point + batch.points.size() > capacity) { throw std::runtime_error("shim capacity"); }
            std::memcpy(out_counts + strand, batch.point_counts.data(), batch.point_counts.size() * 4u);
            std::memcpy(out_points + 4u * point, batch.points.data(), batch.points.size() * 16u);
            if (!batch.root_uvs.empty()) {
                *has_uvs = 1u;
                std::memcpy(out_uvs + 2u * strand, batch.root_uvs.data(), batch.root_uvs.size() * 8u);
            }
            std::memcpy(out_motion + 3u * motion_at, batch.motion_points.data(), batch.motion_points.size() * 12u);
            strand += batch.point_counts.size();
            point += batch.points.size();
            motion_at += batch.motion_points.size();
        }
        out_first[batches.size()] = point;
        put_text("", msg, cap);
        return point;
    } catch (const std::exception &e) {
        put_text(e.what(), msg, cap);
        return 0u;
    }
}

} // extern "C"
