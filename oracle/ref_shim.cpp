// ref_shim.cpp -- extern "C" shim over the reference's own public API.
//
// TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with
// the unmodified reference source src/asset.cpp (from the reference checkout)
// into oracle/_ref/libnxg_ref.so.  Tests use it to pin the C restatement in
// nxg_oracle.c and the product's asset builder; bench.py's reference arm times
// generate_packed_cpu through it.  Nothing here is product code.
#include "nanoxgen/asset.h"
#include "nanoxgen/device_contract.h"

#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <span>
#include <string>
#include <vector>

using namespace nanoxgen;

namespace {

void copy_message(const std::string &text, char *out, std::uint64_t cap) {
    if (!out || cap == 0u) { return; }
    const std::size_t n = std::min<std::size_t>(text.size(), static_cast<std::size_t>(cap - 1u));
    std::memcpy(out, text.data(), n);
    out[n] = '\0';
}

DeformedGeometryView deformed_view(const Vec3 *positions, std::uint64_t position_count,
                                   const Vec3 *normals, std::uint64_t normal_count,
                                   const Vec3 *guide_cvs, std::uint64_t guide_cv_count) {
    DeformedGeometryView view{};
    if (positions) { view.positions = std::span<const Vec3>(positions, position_count); }
    if (normals) { view.normals = std::span<const Vec3>(normals, normal_count); }
    if (guide_cvs) { view.guide_cvs = std::span<const Vec3>(guide_cvs, guide_cv_count); }
    return view;
}

} // namespace

extern "C" {

struct RefStrandState {
    RootSample root;
    std::uint32_t indices[8];
    float weights[8];
    float weight_sum;
    std::uint32_t nearest;
    Vec3 surface_u;
    Vec3 noise_domain;
    float original_length;
    float effective_noise_frequency;
    float preserve_scale;
};

// asset.h:119 build_asset.  Returns a malloc'd copy of the blob (ref_free).
int ref_build_asset(const Vec3 *positions, std::uint32_t vertex_count, const Vec3 *normals,
                    const Vec2 *texcoords, const UInt3 *triangles, std::uint32_t triangle_count,
                    std::uint32_t guide_count, const std::uint32_t *guide_cv_counts,
                    const Vec3 *guide_cvs, const Vec3 *guide_root_normals,
                    const Vec2 *guide_root_uvs, const std::uint32_t *guide_triangles,
                    const Vec2 *guide_barycentrics, const float *guide_support_radii,
                    void **out_bytes, std::uint64_t *out_size, char *msg, std::uint64_t cap) {
    try {
        AssetBuildInput input{};
        input.positions.assign(positions, positions + vertex_count);
        if (normals) { input.normals.assign(normals, normals + vertex_count); }
        if (texcoords) { input.texcoords.assign(texcoords, texcoords + vertex_count); }
        input.triangles.assign(triangles, triangles + triangle_count);
        std::size_t cursor = 0u;
        for (std::uint32_t g = 0; g < guide_count; ++g) {
            GuideInput guide{};
            guide.cvs.assign(guide_cvs + cursor, guide_cvs + cursor + guide_cv_counts[g]);
            cursor += guide_cv_counts[g];
            guide.root_normal = guide_root_normals[g];
            guide.root_uv = guide_root_uvs[g];
            guide.triangle_index = guide_triangles[g];
            guide.barycentric = guide_barycentrics[g];
            guide.support_radius = guide_support_radii[g];
            input.guides.push_back(std::move(guide));
        }
        const Asset asset = build_asset(input);
        void *copy = std::malloc(asset.bytes().size());
        std::memcpy(copy, asset.bytes().data(), asset.bytes().size());
        *out_bytes = copy;
        *out_size = asset.bytes().size();
        copy_message("", msg, cap);
        return 0;
    } catch (const std::exception &error) {
        copy_message(error.what(), msg, cap);
        return 1;
    }
}

void ref_free(void *pointer) { std::free(pointer); }

// asset.cpp:295 validate_asset on a caller buffer (must be 64-byte aligned).
int ref_validate_asset(const void *bytes, std::uint64_t size, char *msg, std::uint64_t cap) {
    const std::string error = validate_asset(
        std::span<const std::byte>(static_cast<const std::byte *>(bytes), size));
    copy_message(error, msg, cap);
    return error.empty() ? 0 : 1;
}

void *ref_asset_create(const void *bytes, std::uint64_t size) {
    const auto *b = static_cast<const std::byte *>(bytes);
    return new Asset(AlignedByteVector(b, b + size));
}

void ref_asset_destroy(void *asset) { delete static_cast<Asset *>(asset); }

// asset.cpp:421-449 generate_packed_deformed_cpu.  *elapsed_ms covers the
// reference call alone (its own validation, allocation and generation), not
// the copy into the caller's arrays.
int ref_generate_packed(const void *asset_handle, const GenerationParams *params,
                        float radius_scale, std::uint32_t workers, std::uint32_t tile,
                        const Vec3 *def_positions, std::uint64_t def_position_count,
                        const Vec3 *def_normals, std::uint64_t def_normal_count,
                        const Vec3 *def_guide_cvs, std::uint64_t def_guide_cv_count,
                        PackedCurvePoint *points, RootSample *roots, Vec2 *root_uvs,
                        std::uint32_t *point_counts, double *elapsed_ms, char *msg,
                        std::uint64_t cap) {
    try {
        const Asset &asset = *static_cast<const Asset *>(asset_handle);
        const DeformedGeometryView deformed = deformed_view(
            def_positions, def_position_count, def_normals, def_normal_count, def_guide_cvs,
            def_guide_cv_count);
        const auto begin = std::chrono::steady_clock::now();
        const PackedGeneratedCurves curves = generate_packed_deformed_cpu(
            asset, *params, deformed, radius_scale, CpuGenerationOptions{workers, tile});
        const auto end = std::chrono::steady_clock::now();
        if (elapsed_ms) {
            *elapsed_ms = std::chrono::duration<double, std::milli>(end - begin).count();
        }
        if (points) {
            std::memcpy(points, curves.points.data(), curves.points.size() * sizeof(PackedCurvePoint));
        }
        if (roots) {
            std::memcpy(roots, curves.roots.data(), curves.roots.size() * sizeof(RootSample));
        }
        if (root_uvs) {
            std::memcpy(root_uvs, curves.root_uvs.data(), curves.root_uvs.size() * sizeof(Vec2));
        }
        if (point_counts) {
            std::memcpy(point_counts, curves.point_counts.data(),
                        curves.point_counts.size() * sizeof(std::uint32_t));
        }
        copy_message("", msg, cap);
        return 0;
    } catch (const std::exception &error) {
        copy_message(error.what(), msg, cap);
        return 1;
    }
}

// generate.h:568-575 make_strand_generation_state, exported field by field.
void ref_strand_state(const void *asset_handle, const Vec3 *def_positions, const Vec3 *def_normals,
                      const Vec3 *def_guide_cvs, const GenerationParams *params,
                      std::uint32_t strand, RefStrandState *out) {
    const Asset &asset = *static_cast<const Asset *>(asset_handle);
    const DeviceDeformedGeometryView deformed{def_positions, def_normals, def_guide_cvs};
    const StrandGenerationState state =
        make_strand_generation_state(asset.view(), deformed, *params, strand);
    out->root = state.root;
    std::memcpy(out->indices, state.guide_blend.indices, sizeof out->indices);
    std::memcpy(out->weights, state.guide_blend.weights, sizeof out->weights);
    out->weight_sum = state.guide_blend.weight_sum;
    out->nearest = state.guide_blend.nearest;
    out->surface_u = state.surface_u;
    out->noise_domain = state.noise_domain;
    out->original_length = state.original_length;
    out->effective_noise_frequency = state.effective_noise_frequency;
    out->preserve_scale = state.preserve_scale;
}

float ref_gradient_noise(const void *asset_handle, float x, float y, float z) {
    const Asset &asset = *static_cast<const Asset *>(asset_handle);
    return gradient_noise(asset.view(), Vec3{x, y, z});
}

// device_contract.h:221-254, on host memory standing in for device memory
// (the pattern of the reference's own tests/test_main.cpp:483-588).
std::uint32_t ref_validate_packed_request(
    const void *asset_data, const AssetHeader *header, std::uint64_t asset_capacity,
    const Vec3 *def_positions, std::uint64_t def_position_count, const Vec3 *def_normals,
    std::uint64_t def_normal_count, const Vec3 *def_guide_cvs, std::uint64_t def_guide_cv_count,
    const GenerationParams *params, PackedCurvePoint *points, RootSample *roots, Vec2 *root_uvs,
    float radius_scale, std::uint32_t *point_counts, std::uint64_t point_capacity,
    std::uint64_t root_capacity, std::uint64_t root_uv_capacity,
    std::uint64_t point_count_capacity, std::uint32_t block_size) {
    const DeviceAssetDescriptor asset{DeviceAssetView{asset_data}, *header, asset_capacity};
    DeviceDeformedGeometryDescriptor deformed{};
    deformed.geometry = {def_positions, def_normals, def_guide_cvs};
    deformed.position_count = def_position_count;
    deformed.normal_count = def_normal_count;
    deformed.guide_cv_count = def_guide_cv_count;
    DevicePackedCurveOutputDescriptor output{};
    output.output = {points, roots, root_uvs, radius_scale, point_counts};
    output.point_capacity = point_capacity;
    output.root_capacity = root_capacity;
    output.root_uv_capacity = root_uv_capacity;
    output.point_count_capacity = point_count_capacity;
    DeviceLaunchConfig config{};
    config.block_size = block_size;
    return static_cast<std::uint32_t>(
        validate_device_packed_generation_request(asset, deformed, *params, output, config));
}

// device_contract.h:256-288 with every sample sharing one deformation.
std::uint32_t ref_validate_motion_request(
    const void *asset_data, const AssetHeader *header, std::uint64_t asset_capacity,
    const float *times, std::uint32_t sample_count, const GenerationParams *params,
    Vec3 *points, std::uint64_t point_capacity, std::uint32_t block_size) {
    const DeviceAssetDescriptor asset{DeviceAssetView{asset_data}, *header, asset_capacity};
    std::vector<DeviceMotionSampleDescriptor> samples(sample_count);
    for (std::uint32_t i = 0; i < sample_count; ++i) { samples[i].time = times[i]; }
    DeviceMotionOutputDescriptor output{points, point_capacity};
    DeviceLaunchConfig config{};
    config.block_size = block_size;
    return static_cast<std::uint32_t>(validate_device_motion_generation_request(
        asset, times ? samples.data() : nullptr, sample_count, *params, output, config));
}

const char *ref_error_message(std::uint32_t code) {
    return device_generation_error_message(static_cast<DeviceGenerationError>(code));
}

} // extern "C"
