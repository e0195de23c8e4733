// generate.cu -- the packed strand generator for sm_100a and its C-ABI entry
// points (nxg_generate_packed, nxg_generate_packed_range,
// nxg_packed_workspace_size, nxg_query_strand_states).
//
// Pipeline per call, all enqueued on the caller's stream:
//   1. strand_keys     : alias-sample every strand's root triangle and bin the
//                        strand by its triangle's nearest stencil guide
//                        (a counting sort's histogram pass);
//   2. exclusive_scan  : bin offsets;
//   3. scatter_order   : the permutation that groups strands sharing guides,
//                        so one CTA's strands read the same guide CVs from L1
//                        (ranks in shared memory per block, one global atomic
//                        per block and bin);
//   4. guide_offsets   : the frame's guide-offset table and guide frame
//                        records;
//   5. generate        : persistent CTAs walk contiguous ranges of the
//                        permutation.  For 2..32 CVs (the built-in tile) the
//                        lane-walk generator (walk.cuh): setup one lane per
//                        strand, the base curve one lane per CV, the noise
//                        frame one lane per strand walking the reference's
//                        cursor, coalesced streaming stores.  Otherwise the
//                        lane-group generator: a group of L lanes owns one
//                        strand, the transported frame as prefix scans over
//                        shuffles (generator_core.cuh), with a separate
//                        roots kernel.
// Strands longer than 128 CVs take a serial per-thread kernel that walks the
// reference's cursor directly.
#include "generator_core.cuh"
#include "walk.cuh"
#include "nxg_internal.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <cstring>

namespace nxg {
namespace dev {

// Persistent CTAs over contiguous ranges of the strand order.  Each warp
// takes 32 strands at a time: phase A sets them up one lane per strand,
// phase B emits them one L-lane group per strand.
template <int L, int PPT, bool NOISE, bool CLASSIC>
__global__ void generate_kernel(LaunchArgs g, const float4 *offsets) {
    extern __shared__ float4 smem[];
    constexpr int kGroups = 32 / L;
    constexpr int kLatticePerWarp = 384;                 // float2 columns per warp (3 axes)
    constexpr int kLatticeMax = kLatticePerWarp / 3 / kGroups;
    const int P = static_cast<int>(g.p.cvs_per_strand);
    const int warps = blockDim.x >> 5;
    // Layout: gradient table | t values | per warp: records, stage, lattice.
    float4 *table = smem;
    float *tvals = reinterpret_cast<float *>(smem + kTableFloat4);
    unsigned char *warp_base = reinterpret_cast<unsigned char *>(tvals + ((P + 3) & ~3));
    const size_t rec_bytes = sizeof(uint32_t) * kRecFields * 32;
    const size_t stage_bytes = sizeof(float4) * kGroups * L * PPT;
    const size_t lattice_bytes = NOISE ? sizeof(float2) * kLatticePerWarp : 0;
    const size_t per_warp = rec_bytes + stage_bytes + lattice_bytes;
    if constexpr (NOISE) {
        for (int i = threadIdx.x; i < kTableFloat4; i += blockDim.x) {
            table[i] = make_float4(__ldg(g.a.gradients + 3 * i), __ldg(g.a.gradients + 3 * i + 1),
                                   __ldg(g.a.gradients + 3 * i + 2), 0.0f);
        }
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x) {  // t = cv / (P - 1) (generate.h:295-298)
        tvals[i] = __fdiv_rn(static_cast<float>(i), static_cast<float>(P - 1));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int group = lane / L;
    const int gl = lane % L;
    unsigned char *mine = warp_base + per_warp * warp;
    const Records rec{reinterpret_cast<uint32_t *>(mine)};
    float4 *stage = reinterpret_cast<float4 *>(mine + rec_bytes) + group * (L * PPT);
    float2 *lattice = reinterpret_cast<float2 *>(mine + rec_bytes + stage_bytes) + group * (kLatticePerWarp / kGroups);
    const uint32_t begin = static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x) * g.count / gridDim.x);
    const uint32_t end = static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x + 1u) * g.count / gridDim.x);
    for (uint32_t batch = begin + static_cast<uint32_t>(warp) * 32u; batch < end;
         batch += static_cast<uint32_t>(warps) * 32u) {
        const uint32_t item = batch + static_cast<uint32_t>(lane);
        const bool valid = item < end;
        setup_strand<NOISE>(g, rec, lane, valid ? item : batch, valid);
        __syncwarp();
        const uint32_t in_batch = min(32u, end - batch);
#pragma unroll 1
        for (uint32_t r = 0; r < in_batch; r += kGroups) {
            emit_strand<L, PPT, NOISE, CLASSIC>(g, rec, static_cast<int>(r) + group, gl, table, offsets, tvals, stage,
                                       lattice, kLatticeMax);
        }
        __syncwarp();
    }
}

// Strands of 2..32 CVs: the lane-walk generator (walk.cuh).  Persistent CTAs
// over contiguous ranges of the strand order positions [range_begin,
// range_end); each warp takes 32 strands at a time through setup (which also
// writes the roots, root UVs and point counts), base, frame (with noise) and
// store.  Without noise the base step writes the output directly (no
// stage), applying Classic scalars itself when given.  Register budgets:
// the noise variant runs one CTA of up to eleven warps per SM (its shared
// memory allows no more: eleven-warp CTAs hold ten lattice columns per axis
// and strand, smaller ones twelve); the plain one three CTAs of eight warps
// (at most 80 registers), the plain Classic one two.
template <bool NOISE, bool CLASSIC>
__global__ void __launch_bounds__(NOISE ? 384 : 256, NOISE ? 1 : (CLASSIC ? 2 : 3))
    generate_walk_kernel(LaunchArgs g, const float4 *offsets) {
    constexpr bool kStaged = NOISE;
    constexpr bool kWalk = NOISE;  // noise walk inside this kernel
    extern __shared__ float4 smem[];
    const int P = static_cast<int>(g.p.cvs_per_strand);
    const int warps = blockDim.x >> 5;
    float4 *table = smem;
    float *tvals = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(smem) + walk_head_bytes(kWalk) -
                                             2u * sizeof(float) * kWalkMaxCvs);
    float *rvals = tvals + kWalkMaxCvs;
    unsigned char *warp_base = reinterpret_cast<unsigned char *>(rvals + kWalkMaxCvs);
    if constexpr (kWalk) {
        for (int i = threadIdx.x; i < kTableFloat4; i += blockDim.x) {
            table[i] = make_float4(__ldg(g.a.gradients + 3 * i), __ldg(g.a.gradients + 3 * i + 1),
                                   __ldg(g.a.gradients + 3 * i + 2), 0.0f);
        }
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x) {  // t = cv / (P - 1) (generate.h:295-298)
        tvals[i] = __fdiv_rn(static_cast<float>(i), static_cast<float>(P - 1));
        rvals[i] = strand_radius(g.p, tvals[i]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int columns = walk_lattice_columns(warps);
    const size_t warp_bytes = walk_warp_bytes(kWalk, kStaged, columns);
    unsigned char *mine = warp_base + warp_bytes * warp;
    float *stage = reinterpret_cast<float *>(mine);  // staged variants only
    float4 *records = reinterpret_cast<float4 *>(kStaged ? mine + kWalkStageBytes : mine);
    float2 *lattice = reinterpret_cast<float2 *>(mine + kWalkStageBytes);
    float4 *scratch = reinterpret_cast<float4 *>(mine + kWalkRecordBytes);  // plain Classic variant only
    uint32_t *locals = reinterpret_cast<uint32_t *>(mine + warp_bytes - kWalkLocalBytes);
    const uint32_t span = g.range_end - g.range_begin;
    const uint32_t begin = g.range_begin + static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x) * span / gridDim.x);
    const uint32_t end =
        g.range_begin + static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x + 1u) * span / gridDim.x);
    for (uint32_t batch = begin + static_cast<uint32_t>(warp) * 32u; batch < end;
         batch += static_cast<uint32_t>(warps) * 32u) {
        const uint32_t item = batch + static_cast<uint32_t>(lane);
        const bool valid = item < end;
        const int in_batch = static_cast<int>(min(32u, end - batch));
        const WalkRoot wr = walk_setup<NOISE>(g, records, locals, lane, valid ? item : batch, valid,
                                              static_cast<uint32_t>(P));
        __syncwarp();
        if constexpr (CLASSIC && !NOISE) {
            walk_classic_setup(g, records, lane, valid, locals[lane] & 0x7fffffffu, tvals, offsets, scratch, P);
            __syncwarp();
        }
        if constexpr (kStaged) {
            walk_base_direct<false, true>(g, records, locals, tvals, rvals, offsets, lane, in_batch, P, stage);
        } else {
            walk_base_direct<CLASSIC>(g, records, locals, tvals, rvals, offsets, lane, in_batch, P);
        }
        __syncwarp();
        if constexpr (kWalk) {
            walk_frame(g.p, wr, lane < in_batch, stage + lane * kWalkRowFloats, lattice + lane, tvals, table, P,
                       columns);
            __syncwarp();
        }
        if constexpr (kStaged) {
            if constexpr (CLASSIC) {
                walk_classic_strand(g, records, stage, locals, lane, in_batch, P);
                __syncwarp();
                walk_store8_classic(g, records, stage, locals, rvals, lane, in_batch, P);
            } else {
                walk_store8(g, stage, locals, rvals, lane, in_batch, P);
            }
            __syncwarp();
        }
    }
}

// Noise on strands of 2..32 CVs without Classic scalars: one producer warp
// and one consumer warp per 64-thread CTA over the CTA's contiguous range of
// the strand order, sharing two stage buffers.  The producer runs setup and
// base (the latency-bound gathers) into one buffer while the consumer runs
// the noise frame and the stores (the arithmetic) from the other; hardware
// named barriers hand the buffers over (1, 2: buffer full; 3, 4: buffer
// empty).  Both warps step through the same batches, so every bar.sync has
// its matching arrivals.
__device__ __forceinline__ void named_sync(uint32_t id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }
__device__ __forceinline__ void named_arrive(uint32_t id) {
    __threadfence_block();  // this warp's shared-memory reads and writes are done before the other warp proceeds
    asm volatile("bar.arrive %0, 64;" ::"r"(id) : "memory");
}

__global__ void __launch_bounds__(64, 1) generate_pipe_kernel(LaunchArgs g, const float4 *offsets) {
    extern __shared__ float4 smem[];
    const int P = static_cast<int>(g.p.cvs_per_strand);
    float4 *table = smem;
    float *tvals = reinterpret_cast<float *>(smem + kTableFloat4);
    float *rvals = tvals + kWalkMaxCvs;
    unsigned char *base = reinterpret_cast<unsigned char *>(rvals + kWalkMaxCvs);
    for (int i = threadIdx.x; i < kTableFloat4; i += blockDim.x) {
        table[i] = make_float4(__ldg(g.a.gradients + 3 * i), __ldg(g.a.gradients + 3 * i + 1),
                               __ldg(g.a.gradients + 3 * i + 2), 0.0f);
    }
    for (int i = threadIdx.x; i < P; i += blockDim.x) {  // t = cv / (P - 1) (generate.h:295-298)
        tvals[i] = __fdiv_rn(static_cast<float>(i), static_cast<float>(P - 1));
        rvals[i] = strand_radius(g.p, tvals[i]);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const bool producer = threadIdx.x < 32;
    unsigned char *tail = base + 2 * kPipeBufferBytes;
    float4 *records = reinterpret_cast<float4 *>(tail);                    // producer
    float2 *lattice = reinterpret_cast<float2 *>(tail + kWalkRecordBytes);  // consumer
    const float inv_p = 1.0f / static_cast<float>(P);
    const uint32_t span = g.range_end - g.range_begin;
    const uint32_t begin = g.range_begin + static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x) * span / gridDim.x);
    const uint32_t end =
        g.range_begin + static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x + 1u) * span / gridDim.x);
    const uint32_t iterations = (end - begin + 31u) / 32u;
    for (uint32_t it = 0; it < iterations; ++it) {
        const uint32_t batch = begin + it * 32u;
        const int in_batch = static_cast<int>(min(32u, end - batch));
        const int b = static_cast<int>(it & 1u);
        unsigned char *buf = base + b * kPipeBufferBytes;
        float *stage = reinterpret_cast<float *>(buf);
        float *fr = reinterpret_cast<float *>(buf + kWalkStageBytes);  // 12 x 32: root position, normal, surface_u, domain
        uint32_t *locals = reinterpret_cast<uint32_t *>(buf + kWalkStageBytes + kPipeFrameBytes);
        if (producer) {
            if (it >= 2u) { named_sync(3u + b); }
            const uint32_t item = batch + static_cast<uint32_t>(lane);
            const bool valid = item < end;
            const WalkRoot wr = walk_setup<true>(g, records, locals, lane, valid ? item : batch, valid,
                                                 static_cast<uint32_t>(P));
            fr[0 * 32 + lane] = wr.position.x;
            fr[1 * 32 + lane] = wr.position.y;
            fr[2 * 32 + lane] = wr.position.z;
            fr[3 * 32 + lane] = wr.normal.x;
            fr[4 * 32 + lane] = wr.normal.y;
            fr[5 * 32 + lane] = wr.normal.z;
            fr[6 * 32 + lane] = wr.surface_u.x;
            fr[7 * 32 + lane] = wr.surface_u.y;
            fr[8 * 32 + lane] = wr.surface_u.z;
            fr[9 * 32 + lane] = wr.domain.x;
            fr[10 * 32 + lane] = wr.domain.y;
            fr[11 * 32 + lane] = wr.domain.z;
            __syncwarp();
            walk_base<false>(g, records, stage, locals, tvals, rvals, offsets, lane, in_batch, P, inv_p);
            named_arrive(1u + b);
        } else {
            named_sync(1u + b);
            WalkRoot wr;
            wr.position = F3{fr[0 * 32 + lane], fr[1 * 32 + lane], fr[2 * 32 + lane]};
            wr.normal = F3{fr[3 * 32 + lane], fr[4 * 32 + lane], fr[5 * 32 + lane]};
            wr.surface_u = F3{fr[6 * 32 + lane], fr[7 * 32 + lane], fr[8 * 32 + lane]};
            wr.domain = F3{fr[9 * 32 + lane], fr[10 * 32 + lane], fr[11 * 32 + lane]};
            walk_frame(g.p, wr, lane < in_batch, stage + lane * kWalkRowFloats, lattice + lane, tvals, table, P,
                       kWalkAxisColumns);
            __syncwarp();
            walk_store8(g, stage, locals, rvals, lane, in_batch, P);
            if (it + 2u < iterations) { named_arrive(3u + b); }
        }
    }
}

// The Classic application for the serial generator (P > 128): one thread
// per strand re-reads its written points (xgen_classic_runtime.cpp:1650-1678,
// :1827-1858), measuring cLength for every strand.
__global__ void classic_serial_apply_kernel(LaunchArgs g) {
    const int P = static_cast<int>(g.p.cvs_per_strand);
    const float rs = g.p.radius_scale;
    for (uint32_t local = blockIdx.x * blockDim.x + threadIdx.x; local < g.count; local += gridDim.x * blockDim.x) {
        float4 *pts = g.points + static_cast<uint64_t>(local) * static_cast<uint32_t>(P);
        const float2 sc = g.scalars[local];
        const float s = g.classic_length ? sc.x : 1.0f;
        const float raw_width = g.classic_width ? sc.y : (rs > 0.0f ? __fdiv_rn(__fmul_rn(2.0f, pts[0].w), rs) : 0.0f);
        bool keep = !(raw_width < 1.0e-4f);
        if (keep) { keep = !(__fmul_rn(classic_spline_length(pts, P), s) < 1.0e-4f); }
        const F3 front = xyz(pts[0]);
        const float radius = __fmul_rn(__fmul_rn(0.5f, raw_width < 0.0f ? 0.0f : raw_width), rs);
        for (int cv = 0; cv < P; ++cv) {
            float4 q = pts[cv];
            if (g.classic_length) {
                const F3 v = xadd(front, xmul(xsub(xyz(q), front), s));
                q.x = v.x;
                q.y = v.y;
                q.z = v.z;
            }
            if (g.classic_width) { q.w = radius; }
            pts[cv] = q;
        }
        if (!keep && g.point_counts != nullptr) { g.point_counts[local] = 0u; }
    }
}

// RootSample, root UV and point count of every strand of the range, in
// output order (coalesced), for the frame (generate.h:101-135, :621-623).
__global__ void strand_roots_kernel(LaunchArgs g) {
    __shared__ uint32_t staged[8][32 * 12];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t P = g.p.cvs_per_strand;
    for (uint32_t base = (blockIdx.x * (blockDim.x >> 5) + warp) * 32u; base < g.count;
         base += gridDim.x * (blockDim.x >> 5) * 32u) {
        const uint32_t i = base + lane;
        const bool valid = i < g.count;
        const Root r = sample_root(g.a, g.f, g.p.seed, g.first_strand + (valid ? i : base));
        uint32_t *rec = staged[warp] + lane * 12;
        rec[0] = __float_as_uint(r.position.x);
        rec[1] = __float_as_uint(r.position.y);
        rec[2] = __float_as_uint(r.position.z);
        rec[3] = __float_as_uint(r.normal.x);
        rec[4] = __float_as_uint(r.normal.y);
        rec[5] = __float_as_uint(r.normal.z);
        rec[6] = __float_as_uint(r.u);
        rec[7] = __float_as_uint(r.v);
        rec[8] = r.triangle;
        rec[9] = __float_as_uint(r.b1);
        rec[10] = __float_as_uint(r.b2);
        rec[11] = r.triangle;  // surface_face_id == triangle_index (generate.h:134)
        __syncwarp();
        const uint32_t n = min(32u, g.count - base);
        if (g.roots) {
            uint32_t *dst = g.roots + static_cast<uint64_t>(base) * 12u;
            for (uint32_t w = lane; w < n * 12u; w += 32u) { dst[w] = staged[warp][w]; }
        }
        if (valid) {
            if (g.root_uvs) { g.root_uvs[i] = make_float2(r.u, r.v); }
            if (g.point_counts) { g.point_counts[i] = P; }
        }
        __syncwarp();
    }
}

// The frame's guide-offset table (G x P float4) and, after it, the guide
// frame records (2 float4 per guide) the lane-walk generator reads, then the
// zero row (kWalkMaxCvs zero entries) its unused stencil slots point at.
__global__ void guide_offsets_kernel(AssetArgs a, FrameArgs f, uint32_t P, float support_scale, float4 *offsets) {
    const uint64_t n = static_cast<uint64_t>(a.guide_count) * P;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    const uint64_t first = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    for (uint64_t k = first; k < static_cast<uint64_t>(kWalkMaxCvs); k += stride) {
        offsets[n + 2u * a.guide_count + k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    for (uint64_t idx = first; idx < n; idx += stride) {
        offsets[idx] = guide_offset_entry(a, f, P, static_cast<uint32_t>(idx / P), static_cast<uint32_t>(idx % P));
    }
    for (uint64_t gi = first; gi < a.guide_count; gi += stride) {
        guide_frame_entry(a, f, support_scale, static_cast<uint32_t>(gi), offsets + n + 2u * gi);
    }
}

// Strands longer than 128 CVs: one thread walks the reference's cursor
// (generate.h:445-642) directly.  Slot records live in registers.
__device__ F3 serial_base_cv(const LaunchArgs &g, const Root &root, const Slot *slots, float wsum,
                             int nearest, uint32_t cv) {
    const float t = __fdiv_rn(static_cast<float>(cv), static_cast<float>(g.p.cvs_per_strand - 1u));
    F3 off = {0.0f, 0.0f, 0.0f};
    if (wsum > 1.0e-12f) {
        for (uint32_t j = 0; j < kSlots; ++j) {
            if (slots[j].flags & kSlotBlended) { off = off + guide_offset(g.f.guide_cvs, slots[j], t) * slots[j].w; }
        }
        off = off * (1.0f / wsum);
    } else if (nearest >= 0) {
        off = guide_offset(g.f.guide_cvs, slots[nearest], t);
    } else {
        off = root.normal * t;
    }
    return root.position + off * g.p.length_scale;
}

struct SerialCursor {
    uint32_t cv;
    F3 previous_base, current_base, next_base, tangent, transported_normal;
    float arc_length;
};

__device__ F3 serial_advance(const LaunchArgs &g, const Root &root, const Slot *slots, float wsum, int nearest,
                             const F3 &domain, float f_eff, const float4 *table, SerialCursor &cur) {
    const ParamArgs &p = g.p;
    if (cur.cv > 0u) {
        const F3 d = cur.current_base - cur.previous_base;
        cur.arc_length += sqrtf(dot(d, d));
    }
    F3 next_tangent = cur.tangent;
    if (cur.cv + 1u < p.cvs_per_strand) {
        const F3 seg = xsub(cur.next_base, cur.current_base);
        if (xdot(seg, seg) > 0.0f) { next_tangent = xnormalize(seg); }
    }
    const F3 axis = xcross(cur.tangent, next_tangent);
    if (xdot(axis, axis) > 0.0f) {
        const float angle = acosf(fminf(fmaxf(dot(cur.tangent, next_tangent), -1.0f), 1.0f));
        cur.transported_normal = normalize(apply3(rotation3(axis, angle), cur.transported_normal));
    }
    const F3 n = cur.transported_normal;
    const F3 b = cross(n, next_tangent);
    const F3 t = cross(b, n);
    F3 point = cur.current_base;
    if (cur.cv > 0u) {
        const float distance = cur.arc_length * f_eff;
        const float magnitude = p.noise_mask * p.noise_amplitude *
                                __fdiv_rn(static_cast<float>(cur.cv), static_cast<float>(p.cvs_per_strand - 1u));
        const float lx = (gradient_noise(table, domain.x + distance, domain.y, domain.z) - 0.5f) * magnitude;
        const float ly = (gradient_noise(table, domain.x, domain.y + distance, domain.z) - 0.5f) * magnitude;
        const float lz = (gradient_noise(table, domain.x, domain.y, domain.z + distance) - 0.5f) * magnitude;
        point = point + n * lx + b * ly + t * lz;
    }
    cur.tangent = next_tangent;
    cur.previous_base = cur.current_base;
    if (cur.cv + 1u < p.cvs_per_strand) {
        cur.current_base = cur.next_base;
        if (cur.cv + 2u < p.cvs_per_strand) {
            cur.next_base = serial_base_cv(g, root, slots, wsum, nearest, cur.cv + 2u);
        }
    }
    ++cur.cv;
    return point;
}

__device__ __forceinline__ void serial_store(const LaunchArgs &g, uint32_t local, uint32_t cv, F3 q, float radius) {
    const uint64_t index = static_cast<uint64_t>(local) * g.p.cvs_per_strand + cv;
    if (g.vec3_points) {
        g.vec3_points[3u * index] = q.x;
        g.vec3_points[3u * index + 1u] = q.y;
        g.vec3_points[3u * index + 2u] = q.z;
    } else {
        g.points[index] = make_float4(q.x, q.y, q.z, radius);
    }
}

__global__ void generate_serial_kernel(LaunchArgs g) {
    __shared__ float4 table[kTableFloat4];
    for (int i = threadIdx.x; i < kTableFloat4; i += blockDim.x) {
        table[i] = make_float4(__ldg(g.a.gradients + 3 * i), __ldg(g.a.gradients + 3 * i + 1),
                               __ldg(g.a.gradients + 3 * i + 2), 0.0f);
    }
    __syncthreads();
    const ParamArgs &p = g.p;
    const uint32_t P = p.cvs_per_strand;
    for (uint32_t item = blockIdx.x * blockDim.x + threadIdx.x; item < g.count; item += gridDim.x * blockDim.x) {
        const uint32_t local = g.order ? min(__ldg(g.order + item), g.count - 1u) : item;
        const Root root = sample_root(g.a, g.f, p.seed, g.first_strand + local);
        Slot slots[kSlots];
        float wsum = 0.0f, nd2 = FLT_MAX;
        int nearest = -1;
        for (uint32_t j = 0; j < kSlots; ++j) {
            slots[j] = eval_slot(g.a, g.f, p, root, j);
            if ((slots[j].flags & kSlotEligible) && slots[j].d2 < nd2) {
                nd2 = slots[j].d2;
                nearest = static_cast<int>(j);
            }
            if (slots[j].flags & kSlotBlended) { wsum = __fadd_rn(wsum, slots[j].w); }
        }
        float scale = 1.0f;
        F3 domain = {0.0f, 0.0f, 0.0f};
        float f_eff = 0.0f;
        F3 surface_u = {0.0f, 0.0f, 0.0f};
        if (p.noise) {
            surface_u = root_surface_u(g.a, g.f, root);
            F3 prev = serial_base_cv(g, root, slots, wsum, nearest, 0u);
            float length = 0.0f;
            for (uint32_t cv = 1u; cv < P; ++cv) {
                const F3 cur = serial_base_cv(g, root, slots, wsum, nearest, cv);
                const F3 d = cur - prev;
                length += sqrtf(dot(d, d));
                prev = cur;
            }
            f_eff = length > 0.0f ? fmaxf(0.5f / length, p.noise_frequency) : p.noise_frequency;
            const float dec = 1.0f - p.noise_correlation;
            domain = (rest_root_position(g.a, root) + F3{0.419276f, 0.184247f, 0.805721f}) * (100.0f * dec * dec);
            if (p.noise_preserve_length > 0.001f) {
                SerialCursor c{0u, {}, {}, {}, root.normal, surface_u, 0.0f};
                c.current_base = serial_base_cv(g, root, slots, wsum, nearest, 0u);
                c.previous_base = c.current_base;
                c.next_base = serial_base_cv(g, root, slots, wsum, nearest, 1u);
                F3 pv = serial_advance(g, root, slots, wsum, nearest, domain, f_eff, table, c);
                float noisy = 0.0f;
                for (uint32_t cv = 1u; cv < P; ++cv) {
                    const F3 cur = serial_advance(g, root, slots, wsum, nearest, domain, f_eff, table, c);
                    const F3 d = cur - pv;
                    noisy += sqrtf(dot(d, d));
                    pv = cur;
                }
                if (noisy > 0.0f) {
                    const float target = length * p.noise_preserve_length + noisy * (1.0f - p.noise_preserve_length);
                    if (fabsf(noisy - target) >= 0.0001f) { scale = target / noisy; }
                }
            }
            SerialCursor c{0u, {}, {}, {}, root.normal, surface_u, 0.0f};
            c.current_base = serial_base_cv(g, root, slots, wsum, nearest, 0u);
            c.previous_base = c.current_base;
            c.next_base = serial_base_cv(g, root, slots, wsum, nearest, 1u);
            for (uint32_t cv = 0u; cv < P; ++cv) {
                F3 q = serial_advance(g, root, slots, wsum, nearest, domain, f_eff, table, c);
                if (scale != 1.0f) { q = root.position + (q - root.position) * scale; }
                const float t = __fdiv_rn(static_cast<float>(cv), static_cast<float>(P - 1u));
                serial_store(g, local, cv, q, strand_radius(p, t));
            }
        } else {
            for (uint32_t cv = 0u; cv < P; ++cv) {
                const F3 q = serial_base_cv(g, root, slots, wsum, nearest, cv);
                const float t = __fdiv_rn(static_cast<float>(cv), static_cast<float>(P - 1u));
                serial_store(g, local, cv, q, strand_radius(p, t));
            }
        }
        if (g.roots) {
            for (int w = 0; w < 12; ++w) { g.roots[static_cast<uint64_t>(local) * 12u + w] = root_word(root, w); }
        }
        if (g.root_uvs) { g.root_uvs[local] = make_float2(root.u, root.v); }
        if (g.point_counts) { g.point_counts[local] = P; }
    }
}

// ---------------------------------------------------------------------------
// Strand-locality counting sort.
// ---------------------------------------------------------------------------
constexpr uint32_t kPrivateBins = 8192u;

__global__ void strand_keys_kernel(AssetArgs a, uint32_t seed, uint32_t first, uint32_t count, uint32_t *keys,
                                   uint32_t *hist, uint32_t bins) {
    extern __shared__ uint32_t local_hist[];
    const bool priv = bins <= kPrivateBins;
    if (priv) {
        for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x) { local_hist[b] = 0u; }
        __syncthreads();
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t tri = sample_triangle(a, seed, first + i);
        const uint32_t gi = __ldg(a.stencil + static_cast<uint64_t>(tri) * kSlots);
        const uint32_t key = gi < a.guide_count ? gi : a.guide_count;
        keys[i] = key;
        if (priv) {
            atomicAdd(&local_hist[key], 1u);
        } else {
            atomicAdd(&hist[key], 1u);
        }
    }
    if (priv) {
        __syncthreads();
        for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x) {
            const uint32_t v = local_hist[b];
            if (v) { atomicAdd(&hist[b], v); }
        }
    }
}

// Exclusive scan of n words in place, one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(uint32_t *data, uint32_t n) {
    __shared__ uint32_t warp_sums[32];
    const uint32_t tid = threadIdx.x;
    const uint32_t per = (n + blockDim.x - 1u) / blockDim.x;
    const uint32_t lo = min(n, tid * per), hi = min(n, lo + per);
    uint32_t sum = 0u;
    for (uint32_t i = lo; i < hi; ++i) { sum += data[i]; }
    uint32_t incl = sum;
    const int lane = tid & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t u = __shfl_up_sync(kFull, incl, d);
        if (lane >= d) { incl += u; }
    }
    if (lane == 31) { warp_sums[tid >> 5] = incl; }
    __syncthreads();
    if (tid < 32) {
        uint32_t w = tid < (blockDim.x >> 5) ? warp_sums[tid] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t u = __shfl_up_sync(kFull, w, d);
            if (lane >= d) { w += u; }
        }
        warp_sums[tid] = w;
    }
    __syncthreads();
    uint32_t running = incl - sum + ((tid >> 5) ? warp_sums[(tid >> 5) - 1u] : 0u);
    for (uint32_t i = lo; i < hi; ++i) {
        const uint32_t v = data[i];
        data[i] = running;
        running += v;
    }
}

__global__ void scatter_order_kernel(const uint32_t *keys, uint32_t *offsets, uint32_t count, uint32_t bins,
                                     uint32_t *order) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t key = min(keys[i], bins - 1u);
        const uint32_t pos = atomicAdd(&offsets[key], 1u);
        if (pos < count) { order[pos] = i; }
    }
}

// The same scatter with one global atomic per (block, non-empty bin): block
// b owns strands [b * chunk, (b + 1) * chunk); it counts its keys in shared
// memory, reserves each bin's range of the order with one atomicAdd on the
// bin offset, then places each strand at that range plus its shared-memory
// rank.  For up to kPrivateBins bins (the count array is in shared memory).
__global__ void __launch_bounds__(1024) scatter_order_blocked_kernel(const uint32_t *keys, uint32_t *offsets,
                                                                     uint32_t count, uint32_t bins, uint32_t chunk,
                                                                     uint32_t *order) {
    extern __shared__ uint32_t slots[];  // per bin: count, then the next free position
    const uint32_t begin = blockIdx.x * chunk;
    const uint32_t end = min(count, begin + chunk);
    for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x) { slots[b] = 0u; }
    __syncthreads();
    for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) { atomicAdd(&slots[min(keys[i], bins - 1u)], 1u); }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < bins; b += blockDim.x) {
        const uint32_t n = slots[b];
        slots[b] = n ? atomicAdd(&offsets[b], n) : 0u;
    }
    __syncthreads();
    for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
        const uint32_t pos = atomicAdd(&slots[min(keys[i], bins - 1u)], 1u);
        if (pos < count) { order[pos] = i; }
    }
}

// Per-strand state for stencil/root parity checks (generate.h:568-575).
struct StrandStateOut {
    uint32_t root[12];
    uint32_t indices[8];
    float weights[8];
    float weight_sum;
    uint32_t nearest;
    float surface_u[3];
    float noise_domain[3];
};

__global__ void query_states_kernel(AssetArgs a, FrameArgs f, ParamArgs p, const uint32_t *strands,
                                    uint32_t count, StrandStateOut *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) { return; }
    const Root root = sample_root(a, f, p.seed, strands[i]);
    StrandStateOut s;
    for (int w = 0; w < 12; ++w) { s.root[w] = root_word(root, w); }
    s.weight_sum = 0.0f;
    s.nearest = kInvalid;
    float nd2 = FLT_MAX;
    for (uint32_t j = 0; j < kSlots; ++j) {
        const Slot slot = eval_slot(a, f, p, root, j);
        s.indices[j] = (slot.flags & kSlotBlended) ? slot.guide : kInvalid;
        s.weights[j] = (slot.flags & kSlotBlended) ? slot.w : 0.0f;
        if ((slot.flags & kSlotEligible) && slot.d2 < nd2) {
            nd2 = slot.d2;
            s.nearest = slot.guide;
        }
        if (slot.flags & kSlotBlended) { s.weight_sum = __fadd_rn(s.weight_sum, slot.w); }
    }
    F3 su = {0.0f, 0.0f, 0.0f}, dom = {0.0f, 0.0f, 0.0f};
    if (p.noise) {
        su = root_surface_u(a, f, root);
        const float dec = 1.0f - p.noise_correlation;
        dom = (rest_root_position(a, root) + F3{0.419276f, 0.184247f, 0.805721f}) * (100.0f * dec * dec);
    }
    s.surface_u[0] = su.x;
    s.surface_u[1] = su.y;
    s.surface_u[2] = su.z;
    s.noise_domain[0] = dom.x;
    s.noise_domain[1] = dom.y;
    s.noise_domain[2] = dom.z;
    out[i] = s;
}

// The lane walk's own setup decisions for listed strands (one warp per CTA,
// g.order = the strand ids, first_strand 0): walk_setup itself, with the
// frame's guide records already in g.guide_frames, outputs off.
__global__ void __launch_bounds__(32) walk_states_kernel(LaunchArgs g, uint32_t count, WalkDecision *out) {
    __shared__ float4 records[kWalkRecords * 32];
    __shared__ uint32_t locals[32];
    const int lane = threadIdx.x & 31;
    const uint32_t i = blockIdx.x * 32u + static_cast<uint32_t>(lane);
    const bool valid = i < count;
    WalkDecision d;
    walk_setup<false>(g, records, locals, lane, valid ? i : 0u, valid, g.p.cvs_per_strand, false, &d);
    if (valid) { out[i] = d; }
}

} // namespace dev

using dev::LaunchArgs;

namespace {

constexpr uint64_t kWorkspaceAlign = 256u;
inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1u) / a * a; }

struct WorkspaceLayout {
    uint64_t keys, order, hist, offsets, offset_bytes, total;
};

// Largest guide-offset table the warp-parallel generator stages; beyond it
// (or beyond 128 CVs) strands take the serial per-thread kernel.
constexpr uint64_t kMaxOffsetTableBytes = uint64_t{1} << 30;
constexpr uint32_t kMaxParallelCvs = 128u;

bool parallel_path(uint32_t guide_count, uint32_t P) {
    return P <= kMaxParallelCvs && uint64_t{guide_count} * P * 16u <= kMaxOffsetTableBytes;
}

// keys[count] | order[count] | bins[guides + 1] | offsets[guides * P] (float4)
// followed by the guide frame records [guides * 2] and the zero row
// [kWalkMaxCvs] (float4)
WorkspaceLayout workspace_layout(uint32_t guide_count, uint32_t count, uint32_t P) {
    WorkspaceLayout w{};
    w.keys = 0u;
    w.order = align_up(uint64_t{count} * 4u, kWorkspaceAlign);
    w.hist = w.order + align_up(uint64_t{count} * 4u, kWorkspaceAlign);
    w.offsets = w.hist + align_up((uint64_t{guide_count} + 1u) * 4u, kWorkspaceAlign);
    w.offset_bytes = parallel_path(guide_count, P) ? (uint64_t{guide_count} * (P + 2u) + dev::kWalkMaxCvs) * 16u : 0u;
    w.total = w.offsets + align_up(w.offset_bytes, kWorkspaceAlign);
    return w;
}

} // namespace

int device_sm_count() {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) { return 148; }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) {
        return 148;
    }
    return sms;
}

dev::AssetArgs resolve_asset(const nxg_device_asset_desc &desc) {
    const auto *base = static_cast<const unsigned char *>(desc.asset);
    const nxg_asset_header &h = desc.header;
    dev::AssetArgs a{};
    a.positions = reinterpret_cast<const float *>(base + h.positions_offset);
    a.normals = reinterpret_cast<const float *>(base + h.normals_offset);
    a.texcoords = (h.flags & NXG_ASSET_HAS_TEXCOORDS) && h.texcoords_offset
        ? reinterpret_cast<const float *>(base + h.texcoords_offset) : nullptr;
    a.triangles = reinterpret_cast<const uint32_t *>(base + h.triangles_offset);
    a.alias = reinterpret_cast<const uint2 *>(base + h.alias_table_offset);
    a.guides = reinterpret_cast<const uint32_t *>(base + h.guides_offset);
    a.guide_cvs = reinterpret_cast<const float *>(base + h.guide_cvs_offset);
    a.stencil = reinterpret_cast<const uint32_t *>(base + h.triangle_guides_offset);
    a.gradients = reinterpret_cast<const float *>(base + h.noise_gradients_offset);
    a.vertex_count = h.vertex_count;
    a.triangle_count = h.triangle_count;
    a.guide_count = h.guide_count;
    a.guide_cv_count = h.guide_cv_count;
    a.flags = h.flags;
    return a;
}

namespace {

} // namespace

dev::FrameArgs resolve_frame(const dev::AssetArgs &a, const nxg_deformed_desc &d) {
    dev::FrameArgs f{};
    f.positions = d.positions ? reinterpret_cast<const float *>(d.positions) : a.positions;
    f.normals = d.normals ? reinterpret_cast<const float *>(d.normals) : a.normals;
    f.guide_cvs = d.guide_cvs ? reinterpret_cast<const float *>(d.guide_cvs) : a.guide_cvs;
    f.deformed_positions = d.positions != nullptr;
    f.deformed_normals = d.normals != nullptr;
    f.deformed_guide_cvs = d.guide_cvs != nullptr;
    return f;
}

namespace {

} // namespace

dev::ParamArgs resolve_params(const nxg_generation_params &p, float radius_scale) {
    dev::ParamArgs r{};
    r.strand_count = p.strand_count;
    r.cvs_per_strand = p.cvs_per_strand;
    r.seed = p.seed;
    r.support_scale = p.guide_support_scale;
    r.weight_power = p.guide_weight_power > 0.0f ? p.guide_weight_power : 0.0f;
    r.rejection_cos = p.normal_rejection_cos;
    r.length_scale = p.length_scale;
    r.root_width = p.root_width;
    r.tip_width = p.tip_width;
    r.noise_amplitude = p.noise_amplitude;
    r.noise_frequency = p.noise_frequency;
    r.noise_mask = p.noise_mask;
    r.noise_correlation = p.noise_correlation;
    r.noise_preserve_length = p.noise_preserve_length;
    r.radius_scale = radius_scale;
    r.noise = (p.noise_amplitude != 0.0f && p.noise_mask != 0.0f) ? 1u : 0u;
    return r;
}

namespace {

using KernelFn = void (*)(LaunchArgs, const float4 *);

// Classic variants (scalars applied in the kernel) are separate
// instantiations, so the plain generator keeps its register budget.
template <int L, int PPT>
KernelFn pick_noise(bool noise, bool classic) {
    if (classic) {
        return noise ? dev::generate_kernel<L, PPT, true, true> : dev::generate_kernel<L, PPT, false, true>;
    }
    return noise ? dev::generate_kernel<L, PPT, true, false> : dev::generate_kernel<L, PPT, false, false>;
}

template <int PPT>
KernelFn pick_lanes(int lanes, bool noise, bool classic) {
    switch (lanes) {
        case 2: return pick_noise<2, PPT>(noise, classic);
        case 4: return pick_noise<4, PPT>(noise, classic);
        case 8: return pick_noise<8, PPT>(noise, classic);
        case 16: return pick_noise<16, PPT>(noise, classic);
        default: return pick_noise<32, PPT>(noise, classic);
    }
}

// Tile registry: the (lanes per strand, CVs per lane, CTA size) used for
// strands of P CVs with noise off/on, set by nxg_set_tile or the autotuner.
// Packed as lanes | ppt << 8 | (block / 32) << 16; 0 means "not set".
std::atomic<uint32_t> g_tiles[kMaxParallelCvs + 1][2];

bool valid_tile(uint32_t P, uint32_t lanes, uint32_t ppt) {
    if (lanes == 1u) { return ppt == 1u && P >= 2u && P <= static_cast<uint32_t>(dev::kWalkMaxCvs); }
    const bool lanes_ok = lanes == 2u || lanes == 4u || lanes == 8u || lanes == 16u || lanes == 32u;
    const bool ppt_ok = ppt == 1u || ppt == 2u || ppt == 4u;
    return lanes_ok && ppt_ok && lanes * ppt >= P && P >= 2u && P <= kMaxParallelCvs;
}

// Tile shape for P CVs: the registered one, else the lane-walk generator for
// 2..32 CVs (lanes_per_strand 1; CTAs of 352 threads with noise, 256
// without), else four CVs per lane on the narrowest power-of-two group that
// holds the strand.
void default_tile(uint32_t P, bool noise, int *lanes, int *ppt, uint32_t *block) {
    const uint32_t packed = P <= kMaxParallelCvs ? g_tiles[P][noise ? 1 : 0].load(std::memory_order_relaxed) : 0u;
    if (packed) {
        *lanes = static_cast<int>(packed & 0xffu);
        *ppt = static_cast<int>((packed >> 8) & 0xffu);
        *block = ((packed >> 16) & 0xffu) * 32u;
        return;
    }
    if (P >= 2u && P <= static_cast<uint32_t>(dev::kWalkMaxCvs)) {  // the lane-walk generator
        *lanes = 1;
        *ppt = 1;
        *block = noise ? 352u : 256u;  // with noise: eleven 20 KB warps fill the SM's shared memory
        return;
    }
    *ppt = 4;
    int l = 2;
    while (l < 32 && static_cast<uint32_t>(l * 4) < P) { l *= 2; }
    *lanes = l;
    *block = 0u;
}

KernelFn pick_kernel(int lanes, int ppt, bool noise, bool classic) {
    if (lanes == 1) {
        if (classic) { return noise ? dev::generate_walk_kernel<true, true> : dev::generate_walk_kernel<false, true>; }
        return noise ? dev::generate_walk_kernel<true, false> : dev::generate_walk_kernel<false, false>;
    }
    switch (ppt) {
        case 1: return pick_lanes<1>(lanes, noise, classic);
        case 2: return pick_lanes<2>(lanes, noise, classic);
        default: return pick_lanes<4>(lanes, noise, classic);
    }
}

// Dynamic shared memory of the generate kernels; for the lane-walk kernel,
// `staged` says whether its stage is used and `noise` whether it walks the
// noise frame itself.
uint32_t launch_kernel(void (*fn)(LaunchArgs, const float4 *), uint32_t grid, uint32_t block, size_t shm,
                       cudaStream_t stream, const LaunchArgs &g, const float4 *offsets) {
    fn<<<grid, block, shm, stream>>>(g, offsets);
    return record_cuda(cudaGetLastError());
}


size_t generate_smem_bytes(uint32_t P, int lanes, int ppt, bool noise, bool staged, uint32_t warps) {
    if (lanes == 1) {
        const bool walk = noise && staged;
        return dev::walk_head_bytes(walk) +
               dev::walk_warp_bytes(walk, staged, dev::walk_lattice_columns(static_cast<int>(warps))) * warps;
    }
    const size_t per_warp = sizeof(uint32_t) * dev::kRecFields * 32u + sizeof(float4) * 32u / lanes * lanes * ppt +
                            (noise ? sizeof(float2) * 384u : 0u);
    return sizeof(float4) * dev::kTableFloat4 + sizeof(float) * ((P + 3u) & ~3u) + per_warp * warps;
}

} // namespace

uint32_t record_cuda(cudaError_t e) {
    if (e == cudaSuccess) { return NXG_ERROR_NONE; }
    set_last_cuda_error(static_cast<int32_t>(e));
    return NXG_ERROR_CUDA;
}


uint32_t check_launch_inputs(const nxg_device_asset_desc &asset, const nxg_packed_output_desc *output) {
    if (!sections_in_bounds(asset.header)) { return NXG_ERROR_INVALID_ASSET_METADATA; }
    if (output && (reinterpret_cast<std::uintptr_t>(output->points) % 16u != 0u ||
                   reinterpret_cast<std::uintptr_t>(output->roots) % 4u != 0u ||
                   reinterpret_cast<std::uintptr_t>(output->root_uvs) % 8u != 0u ||
                   reinterpret_cast<std::uintptr_t>(output->point_counts) % 4u != 0u)) {
        return NXG_ERROR_MISALIGNED_OUTPUT;
    }
    return NXG_ERROR_NONE;
}

uint32_t check_workspace(const nxg_device_asset_desc &asset, uint32_t count, uint32_t P, const void *workspace,
                         uint64_t workspace_bytes) {
    const WorkspaceLayout ws = workspace_layout(asset.header.guide_count, count, P);
    if (!workspace || workspace_bytes < ws.total) { return NXG_ERROR_WORKSPACE_TOO_SMALL; }
    if (reinterpret_cast<std::uintptr_t>(workspace) % kWorkspaceAlign != 0u) { return NXG_ERROR_MISALIGNED_OUTPUT; }
    return NXG_ERROR_NONE;
}

// Counting sort of strands [first, first + count) by their triangle's first
// stencil guide; leaves the permutation in the workspace's order section.
uint32_t launch_order(const nxg_device_asset_desc &asset, uint32_t seed, uint32_t first, uint32_t count,
                      uint32_t P, void *workspace, cudaStream_t stream) {
    const WorkspaceLayout ws = workspace_layout(asset.header.guide_count, count, P);
    auto *wbase = static_cast<unsigned char *>(workspace);
    auto *keys = reinterpret_cast<uint32_t *>(wbase + ws.keys);
    auto *order = reinterpret_cast<uint32_t *>(wbase + ws.order);
    auto *hist = reinterpret_cast<uint32_t *>(wbase + ws.hist);
    const uint32_t bins = asset.header.guide_count + 1u;
    const int sms = device_sm_count();
    const dev::AssetArgs a = resolve_asset(asset);
    uint32_t status = record_cuda(cudaMemsetAsync(hist, 0, uint64_t{bins} * 4u, stream));
    if (status) { return status; }
    const uint32_t threads = 256u;
    const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((count + threads - 1u) / threads,
                                                                      static_cast<uint64_t>(sms) * 4u));
    const size_t shm = bins <= dev::kPrivateBins ? bins * 4u : 0u;
    dev::strand_keys_kernel<<<blocks, threads, shm, stream>>>(a, seed, first, count, keys, hist, bins);
    if ((status = record_cuda(cudaGetLastError()))) { return status; }
    dev::exclusive_scan_kernel<<<1, 1024, 0, stream>>>(hist, bins);
    if ((status = record_cuda(cudaGetLastError()))) { return status; }
    if (bins <= dev::kPrivateBins) {  // one block per SM, shared-memory ranks
        const uint32_t scatter_blocks = static_cast<uint32_t>(std::max(1, sms));
        const uint32_t chunk = (count + scatter_blocks - 1u) / scatter_blocks;
        const uint32_t used = (count + chunk - 1u) / chunk;
        if (bins * 4u > 48u * 1024u) {
            if ((status = record_cuda(cudaFuncSetAttribute(dev::scatter_order_blocked_kernel,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           static_cast<int>(bins * 4u))))) {
                return status;
            }
        }
        dev::scatter_order_blocked_kernel<<<used, 1024, bins * 4u, stream>>>(keys, hist, count, bins, chunk, order);
    } else {
        dev::scatter_order_kernel<<<blocks, threads, 0, stream>>>(keys, hist, count, bins, order);
    }
    return record_cuda(cudaGetLastError());
}

// The generator over the strand order prepared in `workspace`: the
// guide-offset table for this frame, then the persistent generate kernel.
uint32_t launch_generate(const nxg_device_asset_desc &asset, const nxg_deformed_desc &deformed,
                         const nxg_generation_params &params, const nxg_packed_output_desc &output,
                         const nxg_launch_config &config, uint32_t first, uint32_t count, void *workspace,
                         cudaStream_t stream, float *vec3_points, const nxg_classic_apply_desc *classic) {
    set_last_cuda_error(0);
    const uint32_t P = params.cvs_per_strand;
    const WorkspaceLayout ws = workspace_layout(asset.header.guide_count, count, P);
    auto *wbase = static_cast<unsigned char *>(workspace);
    LaunchArgs g{};
    g.a = resolve_asset(asset);
    g.f = resolve_frame(g.a, deformed);
    g.p = resolve_params(params, output.radius_scale);
    g.first_strand = first;
    g.count = count;
    g.points = reinterpret_cast<float4 *>(output.points);
    g.vec3_points = vec3_points;
    g.roots = reinterpret_cast<uint32_t *>(output.roots);
    g.root_uvs = reinterpret_cast<float2 *>(output.root_uvs);
    g.point_counts = output.point_counts;
    g.order = reinterpret_cast<const uint32_t *>(wbase + ws.order);
    if (classic != nullptr) {
        g.scalars = reinterpret_cast<const float2 *>(classic->root_scalars);
        g.classic_length = classic->apply_length != 0u;
        g.classic_width = classic->apply_width != 0u;
    }
    const int sms = device_sm_count();
    uint32_t status = NXG_ERROR_NONE;
    if (!parallel_path(asset.header.guide_count, P)) {
        const uint32_t threads = 128u;
        const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((count + threads - 1u) / threads,
                                                                          static_cast<uint64_t>(sms) * 8u));
        dev::generate_serial_kernel<<<blocks, threads, 0, stream>>>(g);
        if ((status = record_cuda(cudaGetLastError())) || g.scalars == nullptr) { return status; }
        dev::classic_serial_apply_kernel<<<blocks, threads, 0, stream>>>(g);
        return record_cuda(cudaGetLastError());
    }
    auto *offsets = reinterpret_cast<float4 *>(wbase + ws.offsets);
    g.guide_frames = offsets + uint64_t{asset.header.guide_count} * P;
    g.zero_row = asset.header.guide_count * (P + 2u);
    {
        const uint64_t n = uint64_t{asset.header.guide_count} * P;
        const uint32_t threads = 256u;
        const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((n + threads - 1u) / threads,
                                                                          static_cast<uint64_t>(sms) * 16u));
        dev::guide_offsets_kernel<<<blocks, threads, 0, stream>>>(g.a, g.f, P, g.p.support_scale, offsets);
        if ((status = record_cuda(cudaGetLastError()))) { return status; }
    }
    int lanes = 32, ppt = 4;
    uint32_t tile_block = 0u;
    const bool noise = g.p.noise != 0u;
    default_tile(P, noise, &lanes, &ppt, &tile_block);
    if (lanes != 1 && (g.roots || g.root_uvs || g.point_counts)) {  // the lane-walk kernel writes its own
        const uint32_t threads = 256u;
        const uint32_t per_block = threads;  // one strand per thread
        const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((count + per_block - 1u) / per_block,
                                                                          static_cast<uint64_t>(sms) * 8u));
        dev::strand_roots_kernel<<<blocks, threads, 0, stream>>>(g);
        if ((status = record_cuda(cudaGetLastError()))) { return status; }
    }
    g.range_begin = 0u;
    g.range_end = count;
    int device = 0, smem_optin = 48 * 1024;
    if (cudaGetDevice(&device) == cudaSuccess) {
        cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    }
    // Launches `fn` persistently over the order positions [g.range_begin,
    // g.range_end).  block_size in [1, 1024] is a request: rounded up to whole
    // warps, then capped at what the kernel's registers and shared memory
    // (smem(warps) bytes) can launch.
    auto launch = [&](auto fn, uint32_t requested, auto smem) -> uint32_t {
        cudaFuncAttributes attr{};
        uint32_t st = record_cuda(cudaFuncGetAttributes(&attr, reinterpret_cast<const void *>(fn)));
        if (st) { return st; }
        const uint32_t launchable =
            std::max<uint32_t>(32u, static_cast<uint32_t>(attr.maxThreadsPerBlock) / 32u * 32u);
        uint32_t block = std::min(launchable, std::max<uint32_t>(32u, (requested + 31u) / 32u * 32u));
        while (block > 32u && smem(block / 32u) > static_cast<size_t>(smem_optin)) { block -= 32u; }
        const uint32_t warps = block / 32u;
        const size_t shm = smem(warps);
        if (shm > 48u * 1024u) {
            st = record_cuda(cudaFuncSetAttribute(reinterpret_cast<const void *>(fn),
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(shm)));
            if (st) { return st; }
        }
        int per_sm = 0;
        st = record_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reinterpret_cast<const void *>(fn),
                                                                       static_cast<int>(block), shm));
        if (st) { return st; }
        per_sm = std::max(per_sm, 1);
        const uint64_t n = g.range_end - g.range_begin;
        const uint64_t needed = (n + 32u * warps - 1u) / (32u * warps);
        const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(needed, static_cast<uint64_t>(sms) * per_sm));
        return grid ? launch_kernel(fn, grid, block, shm, stream, g, offsets) : NXG_ERROR_NONE;
    };
    const uint32_t requested = tile_block ? tile_block : config.block_size;
    const bool classic_scalars = g.scalars != nullptr;
    if (lanes == 1 && noise && !classic_scalars && requested <= 64u) {  // producer/consumer warp pairs
        return launch(dev::generate_pipe_kernel, 64u, [](uint32_t) { return dev::kPipeSmemBytes; });
    }
    const bool staged = lanes == 1 ? noise : (noise || classic_scalars);
    return launch(pick_kernel(lanes, ppt, noise, classic_scalars), requested,
                  [&](uint32_t w) { return generate_smem_bytes(P, lanes, ppt, noise, staged, w); });
}

uint32_t validate_range_request(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                const nxg_generation_params *params, const nxg_packed_output_desc *output,
                                const nxg_launch_config *config, uint32_t first, uint32_t count) {
    if (!asset || !params || !output) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    const uint32_t error = validate_common(*asset, deformed ? *deformed : none, *params,
                                           config ? *config : default_config);
    if (error != NXG_ERROR_NONE) { return error; }
    if (first > params->strand_count || count > params->strand_count - first) {
        return NXG_ERROR_INVALID_STRAND_RANGE;
    }
    if (!output->points) { return NXG_ERROR_MISSING_OUTPUT; }
    if (!std::isfinite(output->radius_scale) || output->radius_scale < 0.0f) {
        return NXG_ERROR_INVALID_RADIUS_SCALE;
    }
    const uint64_t point_count = uint64_t{count} * params->cvs_per_strand;
    if (output->point_capacity < point_count) { return NXG_ERROR_POINT_CAPACITY_TOO_SMALL; }
    auto optional_ok = [](const void *ptr, uint64_t cap, uint64_t need) { return ptr ? cap >= need : cap == 0u; };
    if (!optional_ok(output->roots, output->root_capacity, count)) { return NXG_ERROR_ROOT_CAPACITY_TOO_SMALL; }
    if (!optional_ok(output->root_uvs, output->root_uv_capacity, count)) {
        return NXG_ERROR_ROOT_UV_CAPACITY_TOO_SMALL;
    }
    if (!optional_ok(output->point_counts, output->point_count_capacity, count)) {
        return NXG_ERROR_POINT_COUNT_CAPACITY_TOO_SMALL;
    }
    return NXG_ERROR_NONE;
}

} // namespace nxg

extern "C" {

uint64_t nxg_packed_workspace_size(const nxg_device_asset_desc *asset, const nxg_generation_params *params,
                                   uint32_t strand_count) {
    if (!asset || !params || strand_count == 0u) { return 0u; }
    return nxg::workspace_layout(asset->header.guide_count, strand_count, params->cvs_per_strand).total;
}

uint32_t nxg_generate_packed(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                             const nxg_generation_params *params, const nxg_packed_output_desc *output,
                             const nxg_launch_config *config, void *workspace, uint64_t workspace_bytes,
                             void *stream) {
    const uint32_t error = nxg_validate_packed_request(asset, deformed, params, output, config);
    if (error != NXG_ERROR_NONE) { return error; }
    return nxg_generate_packed_range(asset, deformed, params, output, config, 0u, params->strand_count,
                                     workspace, workspace_bytes, stream);
}

uint32_t nxg_generate_packed_range(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                   const nxg_generation_params *params, const nxg_packed_output_desc *output,
                                   const nxg_launch_config *config, uint32_t first_strand, uint32_t strand_count,
                                   void *workspace, uint64_t workspace_bytes, void *stream) {
    uint32_t error =
        nxg::validate_range_request(asset, deformed, params, output, config, first_strand, strand_count);
    if (error != NXG_ERROR_NONE) { return error; }
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
                                nullptr, nullptr);
}

uint32_t nxg_prepare_strand_order(const nxg_device_asset_desc *asset, const nxg_generation_params *params,
                                  uint32_t first_strand, uint32_t strand_count, void *workspace,
                                  uint64_t workspace_bytes, void *stream) {
    if (!asset || !params) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    uint32_t error = nxg::validate_common(*asset, none, *params, default_config);
    if (error != NXG_ERROR_NONE) { return error; }
    if (first_strand > params->strand_count || strand_count > params->strand_count - first_strand) {
        return NXG_ERROR_INVALID_STRAND_RANGE;
    }
    if ((error = nxg::check_launch_inputs(*asset, nullptr)) != NXG_ERROR_NONE) { return error; }
    if (strand_count == 0u) { return NXG_ERROR_NONE; }
    if ((error = nxg::check_workspace(*asset, strand_count, params->cvs_per_strand, workspace, workspace_bytes)) !=
        NXG_ERROR_NONE) {
        return error;
    }
    nxg::set_last_cuda_error(0);
    return nxg::launch_order(*asset, params->seed, first_strand, strand_count, params->cvs_per_strand, workspace,
                             static_cast<cudaStream_t>(stream));
}

uint32_t nxg_generate_packed_ordered(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                     const nxg_generation_params *params, const nxg_packed_output_desc *output,
                                     const nxg_launch_config *config, uint32_t first_strand,
                                     uint32_t strand_count, void *workspace, uint64_t workspace_bytes,
                                     void *stream) {
    uint32_t error =
        nxg::validate_range_request(asset, deformed, params, output, config, first_strand, strand_count);
    if (error != NXG_ERROR_NONE) { return error; }
    if ((error = nxg::check_launch_inputs(*asset, output)) != NXG_ERROR_NONE) { return error; }
    if (strand_count == 0u) { return NXG_ERROR_NONE; }
    if ((error = nxg::check_workspace(*asset, strand_count, params->cvs_per_strand, workspace, workspace_bytes)) !=
        NXG_ERROR_NONE) {
        return error;
    }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    return nxg::launch_generate(*asset, deformed ? *deformed : none, *params, *output,
                                config ? *config : default_config, first_strand, strand_count, workspace,
                                static_cast<cudaStream_t>(stream), nullptr, nullptr);
}

uint32_t nxg_query_strand_states(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                 const nxg_generation_params *params, const uint32_t *strands, uint32_t count,
                                 nxg_strand_state *out, void *stream) {
    if (!asset || !params || (count && (!strands || !out))) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    const uint32_t error = nxg::validate_common(*asset, deformed ? *deformed : none, *params, default_config);
    if (error != NXG_ERROR_NONE) { return error; }
    if (!nxg::sections_in_bounds(asset->header)) { return NXG_ERROR_INVALID_ASSET_METADATA; }
    if (count == 0u) { return NXG_ERROR_NONE; }
    const nxg::dev::AssetArgs a = nxg::resolve_asset(*asset);
    const nxg::dev::FrameArgs f = nxg::resolve_frame(a, deformed ? *deformed : none);
    const nxg::dev::ParamArgs p = nxg::resolve_params(*params, 1.0f);
    nxg::set_last_cuda_error(0);
    const uint32_t threads = 128u;
    nxg::dev::query_states_kernel<<<(count + threads - 1u) / threads, threads, 0,
                                    static_cast<cudaStream_t>(stream)>>>(
        a, f, p, strands, count, reinterpret_cast<nxg::dev::StrandStateOut *>(out));
    return nxg::record_cuda(cudaGetLastError());
}

uint32_t nxg_query_walk_states(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                               const nxg_generation_params *params, const uint32_t *strands, uint32_t count,
                               nxg_walk_state *out, void *workspace, uint64_t workspace_bytes, void *stream) {
    static_assert(sizeof(nxg_walk_state) == sizeof(nxg::dev::WalkDecision), "nxg_walk_state layout");
    if (!asset || !params || (count && (!strands || !out))) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    const nxg_deformed_desc &frame = deformed ? *deformed : none;
    uint32_t error = nxg::validate_common(*asset, frame, *params, default_config);
    if (error != NXG_ERROR_NONE) { return error; }
    if ((error = nxg::check_launch_inputs(*asset, nullptr)) != NXG_ERROR_NONE) { return error; }
    if (count == 0u) { return NXG_ERROR_NONE; }
    const uint32_t P = params->cvs_per_strand;
    if (!nxg::parallel_path(asset->header.guide_count, P)) { return NXG_ERROR_INVALID_ARGUMENT; }
    if ((error = nxg::check_workspace(*asset, count, P, workspace, workspace_bytes)) != NXG_ERROR_NONE) {
        return error;
    }
    const auto s = static_cast<cudaStream_t>(stream);
    const nxg::WorkspaceLayout ws = nxg::workspace_layout(asset->header.guide_count, count, P);
    auto *offsets = reinterpret_cast<float4 *>(static_cast<unsigned char *>(workspace) + ws.offsets);
    nxg::LaunchArgs g{};
    g.a = nxg::resolve_asset(*asset);
    g.f = nxg::resolve_frame(g.a, frame);
    g.p = nxg::resolve_params(*params, 1.0f);
    g.first_strand = 0u;
    g.count = 0xffffffffu;  // strand ids are global: every id is a valid order entry
    g.order = strands;
    g.guide_frames = offsets + uint64_t{asset->header.guide_count} * P;
    g.zero_row = asset->header.guide_count * (P + 2u);
    nxg::set_last_cuda_error(0);
    const uint64_t n = uint64_t{asset->header.guide_count} * P;
    const uint32_t threads = 256u;
    const uint32_t blocks = static_cast<uint32_t>(std::max<uint64_t>(1u, std::min<uint64_t>(
        (n + threads - 1u) / threads, static_cast<uint64_t>(nxg::device_sm_count()) * 16u)));
    nxg::dev::guide_offsets_kernel<<<blocks, threads, 0, s>>>(g.a, g.f, P, g.p.support_scale, offsets);
    if ((error = nxg::record_cuda(cudaGetLastError()))) { return error; }
    nxg::dev::walk_states_kernel<<<(count + 31u) / 32u, 32, 0, s>>>(g, count,
                                                                  reinterpret_cast<nxg::dev::WalkDecision *>(out));
    return nxg::record_cuda(cudaGetLastError());
}

uint32_t nxg_set_tile(uint32_t cvs_per_strand, uint32_t noise, const nxg_tile *tile) {
    if (cvs_per_strand < 2u || cvs_per_strand > nxg::kMaxParallelCvs) { return NXG_ERROR_INVALID_ARGUMENT; }
    std::atomic<uint32_t> &slot = nxg::g_tiles[cvs_per_strand][noise ? 1 : 0];
    if (!tile) {
        slot.store(0u, std::memory_order_relaxed);
        return NXG_ERROR_NONE;
    }
    if (!nxg::valid_tile(cvs_per_strand, tile->lanes_per_strand, tile->cvs_per_lane) || tile->block_size > 1024u) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    const uint32_t warps = (tile->block_size + 31u) / 32u;
    slot.store(tile->lanes_per_strand | (tile->cvs_per_lane << 8) | (warps << 16), std::memory_order_relaxed);
    return NXG_ERROR_NONE;
}

uint32_t nxg_get_tile(uint32_t cvs_per_strand, uint32_t noise, nxg_tile *tile) {
    if (!tile || cvs_per_strand < 2u || cvs_per_strand > nxg::kMaxParallelCvs) { return NXG_ERROR_INVALID_ARGUMENT; }
    int lanes = 0, ppt = 0;
    uint32_t block = 0u;
    nxg::default_tile(cvs_per_strand, noise != 0u, &lanes, &ppt, &block);
    tile->lanes_per_strand = static_cast<uint32_t>(lanes);
    tile->cvs_per_lane = static_cast<uint32_t>(ppt);
    tile->block_size = block;
    return NXG_ERROR_NONE;
}

uint32_t nxg_autotune_packed(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                             const nxg_generation_params *params, const nxg_packed_output_desc *output,
                             uint32_t first_strand, uint32_t strand_count, void *workspace, uint64_t workspace_bytes,
                             uint32_t repeats, void *stream, nxg_tile *best, float *best_ms) {
    const nxg_launch_config config{128u};
    uint32_t error =
        nxg::validate_range_request(asset, deformed, params, output, &config, first_strand, strand_count);
    if (error != NXG_ERROR_NONE) { return error; }
    const uint32_t P = params->cvs_per_strand;
    if (strand_count == 0u || P > nxg::kMaxParallelCvs ||
        !nxg::parallel_path(asset->header.guide_count, P)) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    if ((error = nxg_prepare_strand_order(asset, params, first_strand, strand_count, workspace, workspace_bytes,
                                          stream))) {
        return error;
    }
    const bool noise = params->noise_amplitude != 0.0f && params->noise_mask != 0.0f;
    const auto s = static_cast<cudaStream_t>(stream);
    cudaEvent_t start = nullptr, stop = nullptr;
    if ((error = nxg::record_cuda(cudaEventCreate(&start)))) { return error; }
    if ((error = nxg::record_cuda(cudaEventCreate(&stop)))) {
        cudaEventDestroy(start);
        return error;
    }
    const uint32_t saved = nxg::g_tiles[P][noise ? 1 : 0].load(std::memory_order_relaxed);
    nxg_tile winner{0u, 0u, 0u};
    float winner_ms = 0.0f;
    const uint32_t reps = std::max(1u, repeats);
    const uint32_t blocks[5] = {64u, 128u, 256u, 320u, 352u};
    for (uint32_t lanes = 1u; lanes <= 32u && !error; lanes *= 2u) {
        for (uint32_t ppt = 1u; ppt <= 4u && !error; ppt *= 2u) {
            // tiles that hold the strand without idling half of their lanes
            if (!nxg::valid_tile(P, lanes, ppt) || (lanes > 2u && lanes * ppt >= 2u * P)) { continue; }
            for (const uint32_t block : blocks) {
                const nxg_tile tile{lanes, ppt, block};
                nxg_set_tile(P, noise ? 1u : 0u, &tile);
                error = nxg_generate_packed_ordered(asset, deformed, params, output, &config, first_strand,
                                                    strand_count, workspace, workspace_bytes, stream);
                if (error) { break; }
                if ((error = nxg::record_cuda(cudaEventRecord(start, s)))) { break; }
                for (uint32_t r = 0; r < reps && !error; ++r) {
                    error = nxg_generate_packed_ordered(asset, deformed, params, output, &config, first_strand,
                                                        strand_count, workspace, workspace_bytes, stream);
                }
                if (error) { break; }
                if ((error = nxg::record_cuda(cudaEventRecord(stop, s)))) { break; }
                if ((error = nxg::record_cuda(cudaEventSynchronize(stop)))) { break; }
                float ms = 0.0f;
                if ((error = nxg::record_cuda(cudaEventElapsedTime(&ms, start, stop)))) { break; }
                ms /= static_cast<float>(reps);
                if (winner.lanes_per_strand == 0u || ms < winner_ms) {
                    winner = tile;
                    winner_ms = ms;
                }
            }
        }
    }
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    if (error || winner.lanes_per_strand == 0u) {
        nxg::g_tiles[P][noise ? 1 : 0].store(saved, std::memory_order_relaxed);
        return error ? error : NXG_ERROR_INVALID_ARGUMENT;
    }
    nxg_set_tile(P, noise ? 1u : 0u, &winner);
    if (best) { *best = winner; }
    if (best_ms) { *best_ms = winner_ms; }
    return NXG_ERROR_NONE;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Motion samples (device_contract.h:42-53, :256-288): one description at
// several deformed frames, strand identities shared.  The strand order depends
// only on rest data and the seed, so it is prepared once; each sample then
// rebuilds the offset table for its frame and runs the generator.
// ---------------------------------------------------------------------------
namespace nxg {
namespace {

uint32_t validate_motion_samples(const nxg_device_asset_desc &asset, const nxg_motion_sample_desc *samples,
                                 uint32_t sample_count, const nxg_generation_params &params,
                                 const nxg_launch_config &config) {
    if (!samples || sample_count == 0u) { return NXG_ERROR_MISSING_MOTION_SAMPLES; }
    float previous = -INFINITY;
    for (uint32_t i = 0; i < sample_count; ++i) {
        if (!std::isfinite(samples[i].time) || samples[i].time <= previous) { return NXG_ERROR_INVALID_MOTION_TIMES; }
        previous = samples[i].time;
        const uint32_t error = validate_common(asset, samples[i].deformation, params, config);
        if (error != NXG_ERROR_NONE) { return error; }
    }
    return NXG_ERROR_NONE;
}

} // namespace
} // namespace nxg

extern "C" uint32_t nxg_generate_motion_packed(const nxg_device_asset_desc *asset,
                                               const nxg_motion_sample_desc *samples, uint32_t sample_count,
                                               const nxg_generation_params *params,
                                               const nxg_packed_output_desc *outputs,
                                               const nxg_launch_config *config, void *workspace,
                                               uint64_t workspace_bytes, void *stream) {
    if (!asset || !params || !outputs) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_launch_config cfg = config ? *config : nxg_launch_config{128u};
    uint32_t error = nxg::validate_motion_samples(*asset, samples, sample_count, *params, cfg);
    if (error != NXG_ERROR_NONE) { return error; }
    for (uint32_t i = 0; i < sample_count; ++i) {
        error = nxg::validate_range_request(asset, &samples[i].deformation, params, &outputs[i], &cfg, 0u,
                                            params->strand_count);
        if (error == NXG_ERROR_NONE) { error = nxg::check_launch_inputs(*asset, &outputs[i]); }
        if (error != NXG_ERROR_NONE) { return error; }
    }
    if ((error = nxg::check_workspace(*asset, params->strand_count, params->cvs_per_strand, workspace,
                                      workspace_bytes)) != NXG_ERROR_NONE) {
        return error;
    }
    const auto s = static_cast<cudaStream_t>(stream);
    nxg::set_last_cuda_error(0);
    if ((error = nxg::launch_order(*asset, params->seed, 0u, params->strand_count, params->cvs_per_strand,
                                   workspace, s))) {
        return error;
    }
    for (uint32_t i = 0; i < sample_count && !error; ++i) {
        error = nxg::launch_generate(*asset, samples[i].deformation, *params, outputs[i], cfg, 0u,
                                     params->strand_count, workspace, s, nullptr, nullptr);
    }
    return error;
}

extern "C" uint32_t nxg_generate_motion(const nxg_device_asset_desc *asset, const nxg_motion_sample_desc *samples,
                                        uint32_t sample_count, const nxg_generation_params *params,
                                        const nxg_motion_output_desc *output, const nxg_launch_config *config,
                                        void *workspace, uint64_t workspace_bytes, void *stream) {
    uint32_t error = nxg_validate_motion_request(asset, samples, sample_count, params, output, config);
    if (error != NXG_ERROR_NONE) { return error; }
    if ((error = nxg::check_launch_inputs(*asset, nullptr)) != NXG_ERROR_NONE) { return error; }
    if (reinterpret_cast<std::uintptr_t>(output->points) % 4u != 0u) { return NXG_ERROR_MISALIGNED_OUTPUT; }
    if ((error = nxg::check_workspace(*asset, params->strand_count, params->cvs_per_strand, workspace,
                                      workspace_bytes)) != NXG_ERROR_NONE) {
        return error;
    }
    const nxg_launch_config cfg = config ? *config : nxg_launch_config{128u};
    const auto s = static_cast<cudaStream_t>(stream);
    nxg::set_last_cuda_error(0);
    if ((error = nxg::launch_order(*asset, params->seed, 0u, params->strand_count, params->cvs_per_strand,
                                   workspace, s))) {
        return error;
    }
    const uint64_t per_sample = uint64_t{params->strand_count} * params->cvs_per_strand * 3u;
    nxg_packed_output_desc none{};
    none.radius_scale = 1.0f;
    for (uint32_t i = 0; i < sample_count && !error; ++i) {
        float *dst = reinterpret_cast<float *>(output->points) + per_sample * i;
        error = nxg::launch_generate(*asset, samples[i].deformation, *params, none, cfg, 0u, params->strand_count,
                                     workspace, s, dst, nullptr);
    }
    return error;
}

// ---------------------------------------------------------------------------
// Generation without a caller-provided workspace.
//
// Some callers cannot allocate device memory themselves: a renderer plugin
// whose host application owns every allocation through its own pool and
// memory budget, or a frame loop that must not call cudaMalloc because it
// implicitly synchronises the device and stalls the frame.  For them the
// library keeps its own scratch in a fixed-size array in device memory
// (below), held by every GPU that loads the library until the process exits.
// ---------------------------------------------------------------------------
namespace nxg {
namespace {

__device__ __align__(256) unsigned char g_static_scratch[NXG_STATIC_SCRATCH_BYTES];

constexpr int kMaxScratchDevices = 64;

// Driver entry points for the identity of the current context, so that an
// address looked up before a device reset (which destroys the context and
// unloads this module's device memory) is never handed out after it.
using CtxGetCurrentFn = int (*)(void **context);
using CtxGetIdFn = int (*)(void *context, unsigned long long *id);

struct ScratchSlot {
    unsigned long long context_id;  // 0: not looked up on this device yet
    void *address;
};
ScratchSlot g_static_scratch_slots[kMaxScratchDevices];
std::mutex g_static_scratch_mutex;

// The id of the context current on this thread, or 0 when none is current or
// the driver cannot say.
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult found{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
        }
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &found) == cudaSuccess &&
            found == cudaDriverEntryPointSuccess) {
            get_id = reinterpret_cast<CtxGetIdFn>(fn);
        }
    });
    void *context = nullptr;
    unsigned long long id = 0u;
    if (!get_current || !get_id || get_current(&context) != 0 || context == nullptr || get_id(context, &id) != 0) {
        return 0u;
    }
    return id;
}

// The device address of g_static_scratch on the current device (host code
// may not use the array's name as a device pointer).  Looked up with
// cudaGetSymbolAddress once per device and context: again after a device
// reset, or whenever the current context's id cannot be read.
uint32_t static_scratch_address(void **out) {
    int device = 0;
    if (const uint32_t status = record_cuda(cudaGetDevice(&device))) { return status; }
    if (device < 0 || device >= kMaxScratchDevices) { return NXG_ERROR_INVALID_ARGUMENT; }
    std::lock_guard<std::mutex> lock(g_static_scratch_mutex);
    ScratchSlot &slot = g_static_scratch_slots[device];
    const unsigned long long id = current_context_id();
    if (id == 0u || id != slot.context_id || slot.address == nullptr) {
        void *address = nullptr;
        if (const uint32_t status = record_cuda(cudaGetSymbolAddress(&address, g_static_scratch))) {
            return status;
        }
        slot.address = address;
        slot.context_id = current_context_id();  // the lookup makes the device's context current
    }
    *out = slot.address;
    return NXG_ERROR_NONE;
}

} // namespace
} // namespace nxg

extern "C" uint32_t nxg_generate_packed_static_scratch(const nxg_device_asset_desc *asset,
                                                      const nxg_deformed_desc *deformed,
                                                      const nxg_generation_params *params,
                                                      const nxg_packed_output_desc *output,
                                                      const nxg_launch_config *config, void *stream) {
    const uint32_t error = nxg_validate_packed_request(asset, deformed, params, output, config);
    if (error != NXG_ERROR_NONE) { return error; }
    if (nxg_packed_workspace_size(asset, params, params->strand_count) > NXG_STATIC_SCRATCH_BYTES) {
        return NXG_ERROR_STATIC_SCRATCH_LIMIT;
    }
    void *scratch = nullptr;
    if (const uint32_t status = nxg::static_scratch_address(&scratch)) { return status; }
    return nxg_generate_packed(asset, deformed, params, output, config, scratch, NXG_STATIC_SCRATCH_BYTES, stream);
}
