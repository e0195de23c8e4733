// payload.cu -- renderer payload batches (build_curve_batches,
// src/curve_payload.cpp:142-302) on sm_100a.
//
// One pass writes every batch: a warp takes a strand at a time (lanes over
// its output CVs, so point and motion stores are coalesced runs), copying
// or resampling its CVs, applying the affine transform and the radius scale
// with the reference's operation order in IEEE rounding (uncontracted
// intrinsics), so the payload is bit-identical to the reference's.
// Variable-count curve sets first get their point offsets from a three-step
// scan (tile sums, a scan of the tile sums, tile scans), which also runs the
// reference's count checks; a one-thread finish kernel reports the first
// failure in the reference's order, and the payload kernel reads that status
// and does nothing when a check failed.
#include "nxg.h"
#include "nxg_internal.h"
#include "nxg_payload.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace nxg {

uint32_t record_cuda(cudaError_t e);
int device_sm_count();

namespace payload {

const char *const kMessages[NXG_PAYLOAD_ERROR_COUNT] = {
    "",
    "curve batches need a positive strand limit",
    "curve resampling needs at least two CVs",
    "curve radius scale must be finite and non-negative",
    "base curves has no strands",
    "base curves needs fixed or variable CV counts",
    "base curves curve has fewer than two CVs",
    "base curves point array size mismatch",
    "base curves has an invalid constant width",
    "motion sample time must be finite",
    "motion sample strand-count mismatch",
    "motion curves has no strands",
    "motion curves needs fixed or variable CV counts",
    "motion curves curve has fewer than two CVs",
    "motion curves point array size mismatch",
    "motion curves has an invalid constant width",
    "curve transform must contain finite values",
};

constexpr uint32_t kTile = 4096u;       // counts per scan tile
constexpr uint32_t kScanThreads = 256u;  // 16 counts per thread

// One curve set on the device: fixed counts (counts == nullptr) or counts
// with their exclusive prefix offsets (strand_count + 1 entries).
struct SetArgs {
    const float *points;
    const uint32_t *counts;
    const uint64_t *offsets;
    const float *widths;
    uint32_t fixed;
    float constant_width;
    __device__ __forceinline__ uint32_t count(uint32_t s) const { return counts ? counts[s] : fixed; }
    __device__ __forceinline__ uint64_t offset(uint32_t s) const {
        return counts ? offsets[s] : uint64_t{s} * fixed;
    }
};

// Per variable set: the first short strand, the short-strand count.
struct SetCheck {
    unsigned long long first_short;
    unsigned int short_count;
    unsigned int reserved;
};

__device__ __forceinline__ float3 load3(const float *p, uint64_t i) {
    return make_float3(p[3u * i], p[3u * i + 1u], p[3u * i + 2u]);
}

// lerp (curve_payload.cpp:65): a * (1 - f) + b * f per component.
__device__ __forceinline__ float lerp1(float a, float b, float f) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, f)), __fmul_rn(b, f));
}

// sample_point / sample_width (curve_payload.cpp:67-87) for the strand at
// offset `off` with `count` CVs.
__device__ __forceinline__ float3 sample_point(const float *pts, uint64_t off, uint32_t count, float t) {
    const float x = __fmul_rn(fminf(fmaxf(t, 0.0f), 1.0f), static_cast<float>(count - 1u));
    const uint32_t first = static_cast<uint32_t>(x);
    if (first >= count - 1u) { return load3(pts, off + count - 1u); }
    const float f = __fsub_rn(x, static_cast<float>(first));
    const float3 a = load3(pts, off + first), b = load3(pts, off + first + 1u);
    return make_float3(lerp1(a.x, b.x, f), lerp1(a.y, b.y, f), lerp1(a.z, b.z, f));
}

__device__ __forceinline__ float sample_width(const SetArgs &v, uint64_t off, uint32_t count, float t) {
    if (!v.widths) { return v.constant_width; }
    const float x = __fmul_rn(fminf(fmaxf(t, 0.0f), 1.0f), static_cast<float>(count - 1u));
    const uint32_t first = static_cast<uint32_t>(x);
    if (first >= count - 1u) { return v.widths[off + count - 1u]; }
    const float f = __fsub_rn(x, static_cast<float>(first));
    return lerp1(v.widths[off + first], v.widths[off + first + 1u], f);
}

// AffineTransform::apply_point (curve_payload.cpp:127-133).
__device__ __forceinline__ float3 transform_point(const float *m, float3 p) {
    return make_float3(
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[0], p.x), __fmul_rn(m[1], p.y)), __fmul_rn(m[2], p.z)), m[3]),
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[4], p.x), __fmul_rn(m[5], p.y)), __fmul_rn(m[6], p.z)), m[7]),
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(m[8], p.x), __fmul_rn(m[9], p.y)), __fmul_rn(m[10], p.z)), m[11]));
}

__device__ __forceinline__ uint64_t block_sum(uint64_t v, uint64_t *scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { v += __shfl_xor_sync(0xffffffffu, v, o); }
    if ((threadIdx.x & 31u) == 0u) { scratch[threadIdx.x >> 5u] = v; }
    __syncthreads();
    uint64_t total = 0u;
    for (uint32_t w = 0; w < blockDim.x / 32u; ++w) { total += scratch[w]; }
    __syncthreads();
    return total;
}

// Scan step 1: tile sums of the counts, with the short-strand check
// (validate_view's count < 2, curve_payload.cpp:38-44).
__global__ void __launch_bounds__(kScanThreads) tile_sums_kernel(const uint32_t *counts, uint32_t n, uint64_t *sums,
                                                                 SetCheck *check) {
    __shared__ uint64_t scratch[kScanThreads / 32u];
    const uint64_t base = uint64_t{blockIdx.x} * kTile;
    uint64_t sum = 0u;
    for (uint32_t k = threadIdx.x; k < kTile; k += kScanThreads) {
        const uint64_t s = base + k;
        if (s < n) {
            const uint32_t c = counts[s];
            if (c < 2u) {
                atomicMin(&check->first_short, static_cast<unsigned long long>(s));
                atomicAdd(&check->short_count, 1u);
            }
            sum += c;
        }
    }
    sum = block_sum(sum, scratch);
    if (threadIdx.x == 0u) { sums[blockIdx.x] = sum; }
}

// Scan step 2: exclusive scan of the tile sums in place (one block), the
// total after the last tile.
__global__ void __launch_bounds__(1024) tile_scan_kernel(uint64_t *sums, uint32_t tiles) {
    __shared__ uint64_t warp_totals[32];
    __shared__ uint64_t carry;
    if (threadIdx.x == 0u) { carry = 0u; }
    __syncthreads();
    for (uint32_t base = 0; base <= tiles; base += 1024u) {
        const uint32_t i = base + threadIdx.x;
        const uint64_t v = i < tiles ? sums[i] : 0u;
        uint64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if ((threadIdx.x & 31u) >= static_cast<uint32_t>(o)) { x += y; }
        }
        if ((threadIdx.x & 31u) == 31u) { warp_totals[threadIdx.x >> 5u] = x; }
        __syncthreads();
        if (threadIdx.x < 32u) {
            uint64_t t = warp_totals[threadIdx.x];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, t, o);
                if (threadIdx.x >= static_cast<uint32_t>(o)) { t += y; }
            }
            warp_totals[threadIdx.x] = t;
        }
        __syncthreads();
        const uint64_t inclusive = x + (threadIdx.x >= 32u ? warp_totals[(threadIdx.x >> 5u) - 1u] : 0u) + carry;
        if (i <= tiles) { sums[i] = inclusive - v; }
        __syncthreads();
        if (threadIdx.x == 1023u) { carry = inclusive; }
        __syncthreads();
    }
}

// Scan step 3: exclusive offsets within each tile from the tile's base;
// offsets[n] = the total.
__global__ void __launch_bounds__(kScanThreads) tile_offsets_kernel(const uint32_t *counts, uint32_t n,
                                                                    const uint64_t *sums, uint64_t *offsets) {
    __shared__ uint64_t warp_totals[kScanThreads / 32u];
    constexpr uint32_t kPer = kTile / kScanThreads;  // consecutive counts per thread
    const uint64_t first = uint64_t{blockIdx.x} * kTile + uint64_t{threadIdx.x} * kPer;
    uint32_t c[kPer];
    uint64_t local = 0u;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        c[k] = first + k < n ? counts[first + k] : 0u;
        local += c[k];
    }
    uint64_t x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31u) >= static_cast<uint32_t>(o)) { x += y; }
    }
    if ((threadIdx.x & 31u) == 31u) { warp_totals[threadIdx.x >> 5u] = x; }
    __syncthreads();
    uint64_t before = sums[blockIdx.x];
    for (uint32_t w = 0; w < (threadIdx.x >> 5u); ++w) { before += warp_totals[w]; }
    uint64_t running = before + x - local;
#pragma unroll
    for (uint32_t k = 0; k < kPer; ++k) {
        if (first + k < n) { offsets[first + k] = running; }
        running += c[k];
    }
    if (first < n && first + kPer >= n) { offsets[n] = running; }
}

// One check in the reference's order: a device check of set `set` (kind 0
// short curve, 1 point size) or the host's first failure (set = -1).
struct OrderedCheck {
    int set;
    uint32_t kind;
    uint32_t code;
};

constexpr int kMaxChecks = 2 * (1 + static_cast<int>(NXG_PAYLOAD_MAX_SAMPLES)) + 1;

struct FinishArgs {
    const SetCheck *checks;          // per variable set
    uint64_t point_counts[1 + NXG_PAYLOAD_MAX_SAMPLES];
    const uint64_t *offsets_end[1 + NXG_PAYLOAD_MAX_SAMPLES];  // &offsets[n] per variable set
    OrderedCheck order[kMaxChecks];
    uint32_t order_count;
    uint32_t *status;
};

// The first failing check in order: status[0] its code, status[1] the
// failing strands (short-curve checks) or 1.
__global__ void finish_kernel(const FinishArgs a) {
    for (uint32_t k = 0; k < a.order_count; ++k) {
        const OrderedCheck c = a.order[k];
        if (c.set < 0) {
            a.status[0] = c.code;
            a.status[1] = 1u;
            return;
        }
        if (c.kind == 0u && a.checks[c.set].short_count != 0u) {
            a.status[0] = c.code;
            a.status[1] = a.checks[c.set].short_count;
            return;
        }
        if (c.kind == 1u && *a.offsets_end[c.set] != a.point_counts[c.set]) {
            a.status[0] = c.code;
            a.status[1] = 1u;
            return;
        }
    }
}

struct BatchArgs {
    SetArgs base;
    SetArgs samples[NXG_PAYLOAD_MAX_SAMPLES];
    uint32_t sample_count;
    uint32_t strands;
    uint32_t per_batch;       // M
    uint32_t resample;        // R, 0 = keep
    uint32_t identity;
    float radius_scale;
    float radius_factor;      // 0.5f * radius_scale (the copy path's factor)
    float transform[12];
    const float *root_uvs;    // base root uvs, or nullptr
    const uint32_t *roots;    // base RootSample words (12 per strand), or nullptr
    uint64_t total;           // payload points
    const uint32_t *status;   // nonzero: a check failed, nothing is written
    nxg_payload_output out;
};

// The payload of one strand per warp at a time; lanes over its output CVs.
__global__ void __launch_bounds__(256) batches_kernel(const BatchArgs a) {
    if (a.status && a.status[0] != 0u) { return; }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5u);
    const uint32_t S = a.strands, M = a.per_batch, R = a.resample;
    const auto out_offset = [&a, R](uint32_t s) { return R ? uint64_t{s} * R : a.base.offset(s); };
    for (uint32_t s = blockIdx.x * (blockDim.x >> 5u) + (threadIdx.x >> 5u); s < S; s += warps) {
        const uint32_t count_src = a.base.count(s);
        const uint64_t src = a.base.offset(s);
        const uint32_t count = R ? R : count_src;
        const uint64_t dst = out_offset(s);
        const uint32_t b = s / M;
        if (lane == 0u) {
            a.out.point_counts[s] = count;
            if (a.out.root_uvs && (a.root_uvs || a.roots)) {
                float2 uv;
                if (a.root_uvs) {
                    uv = make_float2(a.root_uvs[2u * uint64_t{s}], a.root_uvs[2u * uint64_t{s} + 1u]);
                } else {
                    uv = make_float2(__uint_as_float(a.roots[12u * uint64_t{s} + 6u]),
                                     __uint_as_float(a.roots[12u * uint64_t{s} + 7u]));
                }
                reinterpret_cast<float2 *>(a.out.root_uvs)[s] = uv;
            }
            if (s == b * M) { a.out.batch_first_point[b] = dst; }
            if (s + 1u == S) { a.out.batch_first_point[b + 1u] = a.total; }
        }
        float4 *points = reinterpret_cast<float4 *>(a.out.points);
        const float last = static_cast<float>(count - 1u);
        for (uint32_t c = lane; c < count; c += 32u) {
            float3 p;
            float radius;
            if (R == 0u) {
                p = load3(a.base.points, src + c);
                const float w = a.base.widths ? a.base.widths[src + c] : a.base.constant_width;
                radius = __fmul_rn(w, a.radius_factor);
            } else {
                const float t = __fdiv_rn(static_cast<float>(c), last);
                p = sample_point(a.base.points, src, count_src, t);
                radius = __fmul_rn(__fmul_rn(0.5f, sample_width(a.base, src, count_src, t)), a.radius_scale);
            }
            if (!a.identity) { p = transform_point(a.transform, p); }
            __stcs(points + dst + c, make_float4(p.x, p.y, p.z, radius));
        }
        if (a.sample_count == 0u) { continue; }
        // This batch's points: [first, end); its motion block is sample-major.
        const uint64_t first = out_offset(b * M);
        const uint64_t end = (b + 1u) * uint64_t{M} >= S ? a.total : out_offset((b + 1u) * M);
        const uint64_t batch_points = end - first;
        float *motion = a.out.motion_points + 3u * (uint64_t{a.sample_count} * first + (dst - first));
        for (uint32_t k = 0; k < a.sample_count; ++k) {
            const SetArgs &v = a.samples[k];
            const uint32_t count_k = v.count(s);
            const uint64_t off_k = v.offset(s);
            const bool direct = R == 0u && count_k == count;
            float *row = motion + 3u * uint64_t{k} * batch_points;
            for (uint32_t c = lane; c < count; c += 32u) {
                float3 p = direct ? load3(v.points, off_k + c)
                                  : sample_point(v.points, off_k, count_k, __fdiv_rn(static_cast<float>(c), last));
                if (!a.identity) { p = transform_point(a.transform, p); }
                row[3u * c] = p.x;
                row[3u * c + 1u] = p.y;
                row[3u * c + 2u] = p.z;
            }
        }
    }
}

// The per-strand outputs alone (point counts, root uvs, batch boundaries),
// for the flat path.
__global__ void __launch_bounds__(256) strand_outputs_kernel(const BatchArgs a) {
    const uint32_t S = a.strands, M = a.per_batch, P = a.base.fixed;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        a.out.point_counts[s] = P;
        if (a.out.root_uvs && (a.root_uvs || a.roots)) {
            float2 uv;
            if (a.root_uvs) {
                uv = make_float2(a.root_uvs[2u * uint64_t{s}], a.root_uvs[2u * uint64_t{s} + 1u]);
            } else {
                uv = make_float2(__uint_as_float(a.roots[12u * uint64_t{s} + 6u]),
                                 __uint_as_float(a.roots[12u * uint64_t{s} + 7u]));
            }
            reinterpret_cast<float2 *>(a.out.root_uvs)[s] = uv;
        }
        const uint32_t b = s / M;
        if (s == b * M) { a.out.batch_first_point[b] = uint64_t{s} * P; }
        if (s + 1u == S) { a.out.batch_first_point[b + 1u] = a.total; }
    }
}

// Flat path: every set has the same fixed CV count P and nothing is
// resampled, so output point i is input point i of each set, and its motion
// position goes to K * first + k * bp + (i - first) of its batch (first
// point `first`, bp points).  A thread takes four consecutive points: three
// 16-byte loads of their xyz (48 bytes), one of their widths, four float4
// stores, and per motion sample three loads and three stores when the four
// share a batch and the addresses are 16-byte aligned; otherwise point by
// point.
__global__ void __launch_bounds__(256) flat_points_kernel(const BatchArgs a) {
    const uint64_t total = a.total;
    const uint64_t batch_points = uint64_t{a.per_batch} * a.base.fixed;
    const uint32_t K = a.sample_count;
    float4 *points = reinterpret_cast<float4 *>(a.out.points);
    const bool vector_widths = a.base.widths && (reinterpret_cast<uintptr_t>(a.base.widths) & 15u) == 0u;
    const bool vector_xyz = (reinterpret_cast<uintptr_t>(a.base.points) & 15u) == 0u;
    for (uint64_t i0 = (uint64_t{blockIdx.x} * blockDim.x + threadIdx.x) * 4u; i0 < total;
         i0 += uint64_t{gridDim.x} * blockDim.x * 4u) {
        const bool four = i0 + 4u <= total;
        float3 p[4];
        float w[4];
        if (four && vector_xyz) {
            const float4 *src = reinterpret_cast<const float4 *>(a.base.points + 3u * i0);
            const float4 q0 = __ldcs(src), q1 = __ldcs(src + 1), q2 = __ldcs(src + 2);
            p[0] = make_float3(q0.x, q0.y, q0.z);
            p[1] = make_float3(q0.w, q1.x, q1.y);
            p[2] = make_float3(q1.z, q1.w, q2.x);
            p[3] = make_float3(q2.y, q2.z, q2.w);
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                p[u] = i0 + u < total ? load3(a.base.points, i0 + u) : make_float3(0.0f, 0.0f, 0.0f);
            }
        }
        if (four && vector_widths) {
            const float4 q = __ldcs(reinterpret_cast<const float4 *>(a.base.widths + i0));
            w[0] = q.x;
            w[1] = q.y;
            w[2] = q.z;
            w[3] = q.w;
        } else {
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                w[u] = a.base.widths ? (i0 + u < total ? a.base.widths[i0 + u] : 0.0f) : a.base.constant_width;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (i0 + u >= total) { break; }
            float3 q = p[u];
            if (!a.identity) { q = transform_point(a.transform, q); }
            __stcs(points + i0 + u, make_float4(q.x, q.y, q.z, __fmul_rn(w[u], a.radius_factor)));
        }
        if (K == 0u) { continue; }
        const uint64_t b = i0 / batch_points;
        const bool one_batch = four && (i0 + 3u) / batch_points == b;
        for (uint32_t k = 0; k < K; ++k) {
            const float *sp = a.samples[k].points;
            if (one_batch) {
                const uint64_t first = b * batch_points;
                const uint64_t bp = min(first + batch_points, total) - first;
                float *mo = a.out.motion_points + 3u * (uint64_t{K} * first + uint64_t{k} * bp + (i0 - first));
                const float *in = sp + 3u * i0;
                if ((reinterpret_cast<uintptr_t>(in) & 15u) == 0u && (reinterpret_cast<uintptr_t>(mo) & 15u) == 0u) {
                    const float4 *src = reinterpret_cast<const float4 *>(in);
                    float4 q0 = __ldcs(src), q1 = __ldcs(src + 1), q2 = __ldcs(src + 2);
                    if (!a.identity) {
                        const float3 r0 = transform_point(a.transform, make_float3(q0.x, q0.y, q0.z));
                        const float3 r1 = transform_point(a.transform, make_float3(q0.w, q1.x, q1.y));
                        const float3 r2 = transform_point(a.transform, make_float3(q1.z, q1.w, q2.x));
                        const float3 r3 = transform_point(a.transform, make_float3(q2.y, q2.z, q2.w));
                        q0 = make_float4(r0.x, r0.y, r0.z, r1.x);
                        q1 = make_float4(r1.y, r1.z, r2.x, r2.y);
                        q2 = make_float4(r2.z, r3.x, r3.y, r3.z);
                    }
                    float4 *d = reinterpret_cast<float4 *>(mo);
                    __stcs(d, q0);
                    __stcs(d + 1, q1);
                    __stcs(d + 2, q2);
                    continue;
                }
            }
            for (int u = 0; u < 4; ++u) {
                const uint64_t i = i0 + u;
                if (i >= total) { break; }
                const uint64_t bu = i / batch_points;
                const uint64_t first = bu * batch_points;
                const uint64_t bp = min(first + batch_points, total) - first;
                float3 q = load3(sp, i);
                if (!a.identity) { q = transform_point(a.transform, q); }
                float *mo = a.out.motion_points + 3u * (uint64_t{K} * first + uint64_t{k} * bp + (i - first));
                mo[0] = q.x;
                mo[1] = q.y;
                mo[2] = q.z;
            }
        }
    }
}

} // namespace payload
} // namespace nxg

namespace {

using nxg::payload::kTile;

bool is_identity(const float *m) {
    static const float identity[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    return std::memcmp(m, identity, sizeof identity) == 0;
}

uint64_t tiles_of(uint32_t strands) { return (uint64_t{strands} + kTile - 1u) / kTile; }

// The check records of the variable sets, first in the workspace.
uint64_t checks_bytes(uint32_t sample_count) {
    return (sizeof(nxg::payload::SetCheck) * (1u + uint64_t{sample_count}) + 255u) / 256u * 256u;
}

// Workspace of one variable set: offsets (n + 1), tile sums (tiles + 1), its
// check record; 256-byte aligned pieces.
uint64_t set_bytes(uint32_t strands) {
    const auto up = [](uint64_t b) { return (b + 255u) / 256u * 256u; };
    return up(8u * (uint64_t{strands} + 1u)) + up(8u * (tiles_of(strands) + 1u)) + 256u;
}

} // namespace

extern "C" {

const char *nxg_payload_error_message(uint32_t code) {
    return code < NXG_PAYLOAD_ERROR_COUNT ? nxg::payload::kMessages[code] : "unknown curve payload error";
}

uint64_t nxg_payload_point_count(const nxg_curve_set *base, const nxg_payload_options *options) {
    if (!base || !options) { return 0u; }
    return options->resample_cv_count ? uint64_t{base->strand_count} * options->resample_cv_count
                                      : base->point_count;
}

uint32_t nxg_payload_batch_count(const nxg_curve_set *base, const nxg_payload_options *options) {
    if (!base || !options || options->max_strands_per_batch == 0u) { return 0u; }
    return static_cast<uint32_t>((uint64_t{base->strand_count} + options->max_strands_per_batch - 1u) /
                                 options->max_strands_per_batch);
}

uint64_t nxg_payload_workspace_size(const nxg_curve_set *base, const nxg_motion_set *samples, uint32_t sample_count) {
    uint64_t bytes = checks_bytes(sample_count);
    if (base && base->point_counts) { bytes += set_bytes(base->strand_count); }
    for (uint32_t k = 0; samples && k < sample_count; ++k) {
        if (samples[k].curves.point_counts) { bytes += set_bytes(samples[k].curves.strand_count); }
    }
    return bytes;
}

uint32_t nxg_build_curve_batches(const nxg_curve_set *base, const nxg_motion_set *samples, uint32_t sample_count,
                                 const nxg_payload_options *options, const nxg_payload_output *output,
                                 void *workspace, uint64_t workspace_bytes, uint32_t *device_status,
                                 uint32_t *host_error, void *stream) {
    using namespace nxg::payload;
    if (host_error) { *host_error = NXG_PAYLOAD_OK; }
    if (!base || !options || !output || !device_status || (sample_count && !samples) ||
        sample_count > NXG_PAYLOAD_MAX_SAMPLES) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    // The reference's checks in its order (curve_payload.cpp:148-211); a
    // count check of a variable set is the device's, in its place.
    std::vector<OrderedCheck> order;
    uint32_t host_first = NXG_PAYLOAD_OK;
    const auto host = [&](bool failed, uint32_t code) {
        if (failed && host_first == NXG_PAYLOAD_OK) {
            host_first = code;
            order.push_back({-1, 0u, code});
        }
    };
    int variable_sets = 0;
    std::array<int, 1 + NXG_PAYLOAD_MAX_SAMPLES> set_index{};
    const auto view = [&](const nxg_curve_set &v, int which, bool motion) {
        const uint32_t d = motion ? NXG_PAYLOAD_MOTION_NO_STRANDS - NXG_PAYLOAD_BASE_NO_STRANDS : 0u;
        host(v.strand_count == 0u, NXG_PAYLOAD_BASE_NO_STRANDS + d);
        host(!v.point_counts && v.fixed_cvs_per_strand < 2u, NXG_PAYLOAD_BASE_NO_COUNTS + d);
        set_index[which] = -1;
        if (v.point_counts && host_first == NXG_PAYLOAD_OK) {
            set_index[which] = variable_sets++;
            order.push_back({set_index[which], 0u, NXG_PAYLOAD_BASE_SHORT_CURVE + d});
            order.push_back({set_index[which], 1u, NXG_PAYLOAD_BASE_POINT_SIZE + d});
        } else if (v.point_counts) {
            set_index[which] = variable_sets++;
        } else {
            host(uint64_t{v.strand_count} * v.fixed_cvs_per_strand != v.point_count, NXG_PAYLOAD_BASE_POINT_SIZE + d);
        }
        host(!v.widths && (!std::isfinite(v.constant_width) || v.constant_width < 0.0f),
             NXG_PAYLOAD_BASE_BAD_WIDTH + d);
    };
    host(options->max_strands_per_batch == 0u, NXG_PAYLOAD_NO_STRAND_LIMIT);
    host(options->resample_cv_count == 1u, NXG_PAYLOAD_RESAMPLE_ONE);
    host(!std::isfinite(options->radius_scale) || options->radius_scale < 0.0f, NXG_PAYLOAD_BAD_RADIUS_SCALE);
    view(*base, 0, false);
    for (uint32_t k = 0; k < sample_count; ++k) {
        host(!std::isfinite(samples[k].time), NXG_PAYLOAD_MOTION_BAD_TIME);
        host(samples[k].curves.strand_count != base->strand_count, NXG_PAYLOAD_MOTION_STRANDS);
        view(samples[k].curves, 1 + static_cast<int>(k), true);
    }
    for (float v : options->transform) { host(!std::isfinite(v), NXG_PAYLOAD_BAD_TRANSFORM); }
    const bool device_checks_first = !order.empty() && order.front().set >= 0;
    if (host_first != NXG_PAYLOAD_OK && !device_checks_first) {
        if (host_error) { *host_error = host_first; }
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    const uint64_t total = nxg_payload_point_count(base, options);
    if (!output->points || !output->point_counts || !output->batch_first_point ||
        reinterpret_cast<uintptr_t>(output->points) % 16u != 0u || (sample_count && !output->motion_points) ||
        (!output->root_uvs && (base->root_uvs || base->roots))) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    if (workspace_bytes < nxg_payload_workspace_size(base, samples, sample_count) ||
        (variable_sets && (!workspace || reinterpret_cast<uintptr_t>(workspace) % 256u != 0u))) {
        return NXG_ERROR_WORKSPACE_TOO_SMALL;
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    nxg::set_last_cuda_error(0);
    // Variable sets: offsets and count checks.
    unsigned char *ws = static_cast<unsigned char *>(workspace);
    SetCheck *checks = reinterpret_cast<SetCheck *>(ws);
    uint64_t cursor = checks_bytes(sample_count);
    FinishArgs fin{};
    fin.checks = checks;
    fin.status = device_status;
    BatchArgs a{};
    const auto make_set = [&](const nxg_curve_set &v, int which) -> SetArgs {
        SetArgs out{v.points, v.point_counts, nullptr, v.widths, v.fixed_cvs_per_strand, v.constant_width};
        const int idx = set_index[which];
        if (idx < 0) { return out; }
        const auto up = [](uint64_t b) { return (b + 255u) / 256u * 256u; };
        uint64_t *offsets = reinterpret_cast<uint64_t *>(ws + cursor);
        cursor += up(8u * (uint64_t{v.strand_count} + 1u));
        uint64_t *sums = reinterpret_cast<uint64_t *>(ws + cursor);
        cursor += up(8u * (tiles_of(v.strand_count) + 1u)) + 256u;
        out.offsets = offsets;
        fin.point_counts[idx] = v.point_count;
        fin.offsets_end[idx] = offsets + v.strand_count;
        const uint32_t tiles = static_cast<uint32_t>(tiles_of(v.strand_count));
        tile_sums_kernel<<<tiles, kScanThreads, 0, st>>>(v.point_counts, v.strand_count, sums, checks + idx);
        tile_scan_kernel<<<1, 1024, 0, st>>>(sums, tiles);
        tile_offsets_kernel<<<tiles, kScanThreads, 0, st>>>(v.point_counts, v.strand_count, sums, offsets);
        return out;
    };
    if (variable_sets) {
        // check records: no short strand yet
        std::vector<SetCheck> init(static_cast<size_t>(variable_sets), SetCheck{~0ull, 0u, 0u});
        if (const uint32_t e = nxg::record_cuda(cudaMemcpyAsync(checks, init.data(), init.size() * sizeof(SetCheck),
                                                                cudaMemcpyHostToDevice, st))) {
            return e;
        }
    }
    a.base = make_set(*base, 0);
    for (uint32_t k = 0; k < sample_count; ++k) { a.samples[k] = make_set(samples[k].curves, 1 + static_cast<int>(k)); }
    if (variable_sets) {
        fin.order_count = static_cast<uint32_t>(std::min<size_t>(order.size(), kMaxChecks));
        std::copy(order.begin(), order.begin() + fin.order_count, fin.order);
        finish_kernel<<<1, 1, 0, st>>>(fin);
    }
    if (host_first != NXG_PAYLOAD_OK) {  // reported through the status, after the device checks before it
        return nxg::record_cuda(cudaGetLastError());
    }
    a.sample_count = sample_count;
    a.strands = base->strand_count;
    a.per_batch = options->max_strands_per_batch;
    a.resample = options->resample_cv_count;
    a.identity = is_identity(options->transform) ? 1u : 0u;
    a.radius_scale = options->radius_scale;
    a.radius_factor = 0.5f * options->radius_scale;
    std::memcpy(a.transform, options->transform, sizeof a.transform);
    a.root_uvs = base->root_uvs;
    a.roots = static_cast<const uint32_t *>(base->roots);
    a.total = total;
    a.status = variable_sets ? device_status : nullptr;
    a.out = *output;
    // Flat path: one fixed CV count everywhere and no resampling.
    bool flat = !base->point_counts && options->resample_cv_count == 0u;
    for (uint32_t k = 0; flat && k < sample_count; ++k) {
        flat = !samples[k].curves.point_counts &&
               samples[k].curves.fixed_cvs_per_strand == base->fixed_cvs_per_strand;
    }
    if (flat) {
        const uint64_t quads = (total + 3u) / 4u;
        const uint32_t sgrid = static_cast<uint32_t>(std::max<uint64_t>(
            1u, std::min<uint64_t>((uint64_t{base->strand_count} + 255u) / 256u, uint64_t(nxg::device_sm_count()) * 8u)));
        strand_outputs_kernel<<<sgrid, 256, 0, st>>>(a);
        const uint32_t pgrid = static_cast<uint32_t>(std::max<uint64_t>(
            1u, std::min<uint64_t>((quads + 255u) / 256u, uint64_t(nxg::device_sm_count()) * 8u)));
        flat_points_kernel<<<pgrid, 256, 0, st>>>(a);
        return nxg::record_cuda(cudaGetLastError());
    }
    int per_sm = 0;
    if (const uint32_t e = nxg::record_cuda(
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batches_kernel, 256, 0))) {
        return e;
    }
    const uint64_t needed = (uint64_t{base->strand_count} + 7u) / 8u;
    const uint32_t grid = static_cast<uint32_t>(std::max<uint64_t>(
        1u, std::min<uint64_t>(needed, uint64_t(nxg::device_sm_count()) * std::max(per_sm, 1))));
    batches_kernel<<<grid, 256, 0, st>>>(a);
    return nxg::record_cuda(cudaGetLastError());
}

} // extern "C"
