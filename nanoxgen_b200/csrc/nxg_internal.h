// nxg_internal.h -- declarations shared by the host translation unit
// (host.cpp) and the CUDA translation units of libnxg_b200.so.
#pragma once

#include "nxg.h"

#include <cstdint>

namespace nxg {

static_assert(sizeof(nxg_vec3) == 12u, "Vec3 layout (types.h:30-34)");
static_assert(sizeof(nxg_uint3) == 12u, "UInt3 layout (types.h:36-40)");
static_assert(sizeof(nxg_guide_record) == 56u, "GuideRecord layout (src/luisa/generate.cpp:26)");
static_assert(sizeof(nxg_asset_header) == 128u, "AssetHeader layout (types.h:76-101)");
static_assert(alignof(nxg_asset_header) == 64u, "AssetHeader alignment (types.h:106)");
static_assert(sizeof(nxg_root_sample) == 48u, "RootSample layout (src/luisa/generate.cpp:32)");
static_assert(sizeof(nxg_packed_point) == 16u, "PackedCurvePoint layout (types.h:145)");
static_assert(sizeof(nxg_generation_params) == 60u, "GenerationParams layout (types.h:108-124)");
static_assert(sizeof(nxg_device_asset_desc) == 256u, "DeviceAssetDescriptor layout");

// Records the last CUDA error for nxg_last_cuda_error().
void set_last_cuda_error(int32_t code) noexcept;

// device_contract.h:137-181 (common part of every request).
uint32_t validate_common(const nxg_device_asset_desc &asset, const nxg_deformed_desc &deformed,
                         const nxg_generation_params &params, const nxg_launch_config &config) noexcept;

// Header-only bounds check of every section a kernel dereferences.  The
// reference validator leaves these to validate_asset; the launch path
// repeats them so that a hand-built descriptor cannot steer a kernel out of
// the asset allocation.
bool sections_in_bounds(const nxg_asset_header &header) noexcept;

// The two all-pairs searches of build_asset on the current CUDA device
// (stencil.cu): the per-triangle stencil rows (src/asset.cpp:252-269) and
// each guide's nearest other root (the automatic support radius, before its
// 1.75 scale).  Copies the mesh and guide roots/normals/CV counts from host
// memory, runs both kernels, copies the triangle_count x 8 rows into the host
// array `stencil` and the guide_count distances into `nearest`, and
// synchronizes `stream`.  Returns 0 or the CUDA error code, with its text in
// `what`.
int device_guide_search(const nxg_vec3 *positions, uint32_t vertex_count, const nxg_uint3 *triangles,
                        uint32_t triangle_count, const nxg_vec3 *guide_roots, const nxg_vec3 *guide_normals,
                        const uint32_t *guide_cv_counts, uint32_t guide_count, uint32_t stencil_slots,
                        uint32_t *stencil, float *nearest, void *stream, const char **what) noexcept;

} // namespace nxg
