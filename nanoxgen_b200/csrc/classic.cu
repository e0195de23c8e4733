// classic.cu -- the exact Classic-expression runtime on sm_100a.
//
// nxg_classic_root_scalars evaluates a description's SplinePrimitive length
// and width expressions once per root, one thread per root, with the float
// semantics of the reference's evaluate_xgen_scalar_expression_float
// (src/xgen_expression.cpp:984-1148): every arithmetic op is an IEEE-rounded
// intrinsic that nvcc never contracts, so results are bit-identical to the
// CPU runtime built with -ffp-contract=off (gamma and contrast call powf and
// log2f, whose last bit may differ from the host libm).  The program lives in
// the kernel's parameter block: every lane executes the same instruction at
// the same time, read from the constant bank.
//
// nxg_generate_packed_classic runs the generator with the scalars applied
// inside it (generator_core.cuh, emit_strand).
#include "classic_eval.cuh"
#include "expression.h"
#include "generator_core.cuh"
#include "nxg_classic.h"
#include "nxg_internal.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

namespace nxg {
namespace dev {

struct ScalarArgs {
    AssetArgs a;
    FrameArgs f;
    uint32_t seed, first, count;
    float description_id;   // rand() face seed inputs
    float patch_seed;
    float2 *out;
    uint32_t *status;
    const uint32_t *distrust;  // surrogate split: skip the network's batches (see surrogate.cu)
    uint32_t probe_period;
    DeviceExpression length;
    DeviceExpression width;
};

__global__ void __launch_bounds__(256) classic_scalars_kernel(const __grid_constant__ ScalarArgs k) {
    __shared__ float4 table[256];
    __shared__ uint8_t perm[256];
    stage_classic_tables(table, perm);
    __syncthreads();
    const bool random = k.length.uses_random || k.width.uses_random;
    // With a surrogate split, this kernel takes the 128-root batches the
    // network does not: none while the model is trusted, else all but the
    // probes (every probe_period-th batch).
    const bool split = k.distrust != nullptr;
    if (split && *k.distrust == 0u) { return; }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k.count; i += gridDim.x * blockDim.x) {
        if (split && (i / 128u) % k.probe_period == 0u) { continue; }
        const uint32_t strand = k.first + i;
        const Root root = sample_root(k.a, k.f, k.seed, strand);
        const float face_seed = random ? classic_face_seed(k.description_id, k.patch_seed, root.triangle, perm) : 0.0f;
        float length, width;
        const bool ok = classic_root_scalars(k.length, k.width, table, perm, root, strand, face_seed, &length, &width);
        k.out[i] = make_float2(length, width);
        if (!ok) {
            atomicCAS(k.status, 0u, static_cast<uint32_t>(NXG_ERROR_EXPRESSION_DOMAIN));
            atomicAdd(k.status + 1, 1u);
        }
    }
}

} // namespace dev
} // namespace nxg

namespace nxg {

uint32_t launch_classic_root_scalars(const nxg_device_asset_desc &asset, const nxg_generation_params &params,
                                     const nxg_classic_scalar_plan &plan, uint32_t first, uint32_t count,
                                     float *scalars, uint32_t *status, cudaStream_t stream,
                                     const uint32_t *distrust, uint32_t probe_period) {
    dev::ScalarArgs k{};
    uint32_t error = NXG_ERROR_NONE;
    if (plan.length && (error = pack_device_expression(plan.length, k.length))) { return error; }
    if (plan.width && (error = pack_device_expression(plan.width, k.width))) { return error; }
    if (k.length.uses_clength || k.width.uses_clength) { return NXG_ERROR_EXPRESSION_INPUT; }
    if (count == 0u) { return NXG_ERROR_NONE; }
    const nxg_deformed_desc none{};
    k.a = resolve_asset(asset);
    k.f = resolve_frame(k.a, none);
    k.seed = params.seed;
    k.first = first;
    k.count = count;
    k.description_id = static_cast<float>(plan.description_id);
    // xgen_runtime_face_seed keeps the patch name after its last ':'
    const char *patch = plan.patch_name ? plan.patch_name : "";
    for (const char *p = patch; *p; ++p) {
        if (*p == ':') { patch = p + 1; }
    }
    k.patch_seed = static_cast<float>(nxg_xgen_string_seed(patch));
    k.out = reinterpret_cast<float2 *>(scalars);
    k.status = status;
    k.distrust = distrust;
    k.probe_period = probe_period;
    set_last_cuda_error(0);
    const uint32_t threads = 256u;
    const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>(
        (uint64_t{count} + threads - 1u) / threads, static_cast<uint64_t>(device_sm_count()) * 8u));
    dev::classic_scalars_kernel<<<blocks, threads, 0, stream>>>(k);
    return record_cuda(cudaGetLastError());
}

} // namespace nxg

extern "C" {

uint32_t nxg_classic_root_scalars(const nxg_device_asset_desc *asset, const nxg_generation_params *params,
                                  const nxg_classic_scalar_plan *plan, uint32_t first_strand,
                                  uint32_t strand_count, float *scalars, uint32_t *device_status, void *stream) {
    if (!asset || !params || !plan) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    uint32_t error = nxg::validate_common(*asset, none, *params, default_config);
    if (error != NXG_ERROR_NONE) { return error; }
    if (first_strand > params->strand_count || strand_count > params->strand_count - first_strand) {
        return NXG_ERROR_INVALID_STRAND_RANGE;
    }
    if (!scalars || !device_status) { return NXG_ERROR_MISSING_OUTPUT; }
    if (reinterpret_cast<std::uintptr_t>(scalars) % 8u != 0u ||
        reinterpret_cast<std::uintptr_t>(device_status) % 4u != 0u) {
        return NXG_ERROR_MISALIGNED_OUTPUT;
    }
    if ((error = nxg::check_launch_inputs(*asset, nullptr)) != NXG_ERROR_NONE) { return error; }
    return nxg::launch_classic_root_scalars(*asset, *params, *plan, first_strand, strand_count, scalars,
                                            device_status, static_cast<cudaStream_t>(stream), nullptr, 0u);
}

uint32_t nxg_generate_packed_classic(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                     const nxg_generation_params *params, const nxg_packed_output_desc *output,
                                     const nxg_classic_apply_desc *classic, const nxg_launch_config *config,
                                     uint32_t first_strand, uint32_t strand_count, void *workspace,
                                     uint64_t workspace_bytes, void *stream) {
    uint32_t error =
        nxg::validate_range_request(asset, deformed, params, output, config, first_strand, strand_count);
    if (error != NXG_ERROR_NONE) { return error; }
    if (!classic || !classic->root_scalars) { return NXG_ERROR_INVALID_ARGUMENT; }
    if (reinterpret_cast<std::uintptr_t>(classic->root_scalars) % 8u != 0u) { return NXG_ERROR_MISALIGNED_OUTPUT; }
    if ((error = nxg::check_launch_inputs(*asset, output)) != NXG_ERROR_NONE) { return error; }
    if (strand_count == 0u) { return NXG_ERROR_NONE; }
    if ((error = nxg::check_workspace(*asset, strand_count, params->cvs_per_strand, workspace, workspace_bytes)) !=
        NXG_ERROR_NONE) {
        return error;
    }
    const auto s = static_cast<cudaStream_t>(stream);
    nxg::set_last_cuda_error(0);
    if ((error = nxg::launch_order(*asset, params->seed, first_strand, strand_count, params->cvs_per_strand,
                                   workspace, s))) {
        return error;
    }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    return nxg::launch_generate(*asset, deformed ? *deformed : none, *params, *output,
                                config ? *config : default_config, first_strand, strand_count, workspace, s,
                                nullptr, classic);
}

} // extern "C"
