// walk.cuh -- the lane-walk generator for strands of 2..32 CVs.
//
// A warp takes 32 strands of the strand order at a time, in four steps:
//
//   setup  (lane = strand)  root sample, the eight stencil slots and the
//                           blend mode, folded into one weighted-sum record;
//   base   (lane = CV)      the base curve from the guide-offset table, read
//                           as coalesced rows (consecutive lanes on
//                           consecutive CVs of one guide), into a stage in
//                           shared memory, one row of 32 xyz slots per strand;
//   frame  (lane = strand)  with noise: the arc-length prefix, the strand's
//                           noise lattice, then the reference's cursor walk
//                           (generate.h:445-502) over the staged row -- the
//                           transported normal is a serial recurrence, so a
//                           lane carries it CV by CV with the reference's
//                           rotation applied as a vector update, and no
//                           matrix products or cross-lane scans are needed;
//   store  (8 lanes/strand) the strands' float4s as coalesced streaming
//                           stores; with per-root Classic scalars, a step
//                           with lane = strand first takes each strand's
//                           Classic values (scale, width, drop rule) once.
//
// Stage rows are 97 words apart and a CV takes 3 words; both strides are odd,
// so a warp reading column c of 32 rows (frame step) and a warp reading one
// row are free of shared-memory bank conflicts, and the eight-lane base and
// store steps (four strands of eight CVs per access) meet at most two lanes
// to a bank (97 = 1 mod 32 shifts each strand's banks by one).
#pragma once

#include "generator_core.cuh"

namespace nxg {
namespace dev {

constexpr int kWalkMaxCvs = 32;
constexpr int kWalkRowFloats = 3 * kWalkMaxCvs + 1; // a row holds x, y, z per CV (97 words: an odd stride)
constexpr int kWalkAxisColumns = 12;           // noise lattice columns per axis and strand, at most
constexpr int kWalkRecords = 8;                // float4 setup records per strand

// Shared-memory bytes per warp.  Staged variants (noise or Classic scalars):
// stage | records (aliased by the lattice once the base step has read them) |
// output words; the RootSample words use the stage.  The plain variant has no
// stage -- its base step writes the output directly -- so: records | RootSample
// words | output words.
constexpr size_t kWalkStageBytes = sizeof(float) * 32u * kWalkRowFloats;
constexpr size_t kWalkRecordBytes = sizeof(float4) * kWalkRecords * 32u;
constexpr size_t kWalkLatticeBytes = sizeof(float2) * 3u * kWalkAxisColumns * 32u;
// Lattice columns per axis and strand for a CTA of `warps` noise warps:
// twelve up to ten warps; ten for eleven-warp CTAs, whose shared memory holds
// no more.  A strand needs floor(d + span) - floor(d) + 2 columns on an axis
// whose noise coordinate starts at d and advances by span over the strand
// (at most ceil(span) + 2); a warp with a strand that needs more takes direct
// noise.
__host__ __device__ constexpr int walk_lattice_columns(int warps) { return warps > 10 ? 10 : kWalkAxisColumns; }
__host__ __device__ constexpr size_t walk_lattice_bytes(int columns) {
    return sizeof(float2) * 3u * static_cast<size_t>(columns) * 32u;
}
constexpr size_t kWalkRootWordBytes = sizeof(uint32_t) * 12u * 32u;
constexpr size_t kWalkLocalBytes = sizeof(uint32_t) * 32u;
__host__ __device__ constexpr size_t walk_warp_bytes(bool noise, bool staged, int columns = kWalkAxisColumns) {
    return staged ? kWalkStageBytes +
                        (noise && walk_lattice_bytes(columns) > kWalkRecordBytes ? walk_lattice_bytes(columns)
                                                                                 : kWalkRecordBytes) +
                        kWalkLocalBytes
                  : kWalkRecordBytes + kWalkRootWordBytes + kWalkLocalBytes;
}
// Per CTA, before the warps: gradient table (noise) | t values | radii.
__host__ __device__ constexpr size_t walk_head_bytes(bool noise) {
    return (noise ? sizeof(float4) * kTableFloat4 : 0u) + 2u * sizeof(float) * kWalkMaxCvs;
}

// Record q of strand s lives at records[q * 32 + s]:
//   q = 0..3  (row of slot 2q, weight, row of slot 2q+1, weight); a row is
//             guide * P, the guide's first entry in the offset table
//   q = 4     (root position, 1 / weight sum)
//   q = 5     (root normal in normal mode else 0, slot count as bits)
//   q = 6, 7  Classic scalars without noise (walk_classic_setup): (first
//             point, length scale) and (width radius, width override flag)
// Nearest mode becomes one slot of weight 1 and normal mode zero slots, so
// the base step evaluates every strand as
//   base = root + (inv * sum_j w_j offsets[row_j + c] + normal' * t_c) * length_scale.
// Square root by the PTX approximate instruction (one MUFU operation, no
// special-case branch); its relative error (below 2^-22) is far inside the
// position tolerance where it is used (arc lengths, sin(acos x), blend weights).
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

struct WalkRoot {
    F3 position, normal, surface_u, domain;
};

// sample_root (generate.h:101-135) plus, with noise, the root's surface_u
// (generate.h:312-341) and rest position (generate.h:343-351), reusing the
// triangle's vertex data instead of loading it again.
template <bool NOISE>
__device__ __forceinline__ Root walk_root(const AssetArgs &a, const FrameArgs &f, uint32_t seed, uint32_t strand,
                                          F3 &surface_u, F3 &rest_position) {
    Root r;
    r.triangle = sample_triangle(a, seed, strand);
    const float r1 = random01(seed, strand, 2u);
    const float r2 = random01(seed, strand, 3u);
    const float s = __fsqrt_rn(r1);
    const float b0 = __fsub_rn(1.0f, s);
    r.b1 = __fmul_rn(s, __fsub_rn(1.0f, r2));
    r.b2 = __fmul_rn(s, r2);
    const uint3 t = load_triangle(a, r.triangle);
    const F3 p0 = ld3(f.positions, t.x), p1 = ld3(f.positions, t.y), p2 = ld3(f.positions, t.z);
    // A deformed frame's noise domain needs the rest-pose vertices too:
    // requested with the frame's, before any arithmetic waits on them.
    F3 q0 = p0, q1 = p1, q2 = p2;
    if (NOISE && f.positions != a.positions) {
        q0 = ld3(a.positions, t.x);
        q1 = ld3(a.positions, t.y);
        q2 = ld3(a.positions, t.z);
    }
    r.position = xbary(p0, p1, p2, b0, r.b1, r.b2);
    // The face normal only where the asset has no vertex normals (the
    // reference computes it first and then replaces it).
    if (a.flags & NXG_ASSET_HAS_NORMALS) {
        r.normal = xnormalize(xbary(ld3(f.normals, t.x), ld3(f.normals, t.y), ld3(f.normals, t.z),
                                    b0, r.b1, r.b2));
    } else {
        r.normal = xnormalize(xcross(xsub(p1, p0), xsub(p2, p0)));
    }
    r.u = 0.0f;
    r.v = 0.0f;
    const bool uvs = (a.flags & NXG_ASSET_HAS_TEXCOORDS) && a.texcoords;
    float2 uv0 = make_float2(0.0f, 0.0f), uv1 = uv0, uv2 = uv0;
    if (uvs) {
        uv0 = make_float2(__ldg(a.texcoords + 2u * static_cast<uint64_t>(t.x)),
                          __ldg(a.texcoords + 2u * static_cast<uint64_t>(t.x) + 1u));
        uv1 = make_float2(__ldg(a.texcoords + 2u * static_cast<uint64_t>(t.y)),
                          __ldg(a.texcoords + 2u * static_cast<uint64_t>(t.y) + 1u));
        uv2 = make_float2(__ldg(a.texcoords + 2u * static_cast<uint64_t>(t.z)),
                          __ldg(a.texcoords + 2u * static_cast<uint64_t>(t.z) + 1u));
        r.u = __fadd_rn(__fadd_rn(__fmul_rn(uv0.x, b0), __fmul_rn(uv1.x, r.b1)), __fmul_rn(uv2.x, r.b2));
        r.v = __fadd_rn(__fadd_rn(__fmul_rn(uv0.y, b0), __fmul_rn(uv1.y, r.b1)), __fmul_rn(uv2.y, r.b2));
    }
    if constexpr (NOISE) {
        F3 tangent = {0.0f, 0.0f, 0.0f};
        if (uvs) {
            const F3 e1 = p1 - p0;
            const F3 e2 = p2 - p0;
            const float du1 = uv1.x - uv0.x, dv1 = uv1.y - uv0.y;
            const float du2 = uv2.x - uv0.x, dv2 = uv2.y - uv0.y;
            const float det = du1 * dv2 - dv1 * du2;
            if (fabsf(det) > 1.0e-12f) {
                tangent = (e1 * dv2 - e2 * dv1) * (1.0f / det);
                tangent = tangent - r.normal * dot(tangent, r.normal);
            }
        }
        surface_u = dot(tangent, tangent) > 1.0e-20f ? normalize(tangent) : fallback_surface_u(r.normal);
        const float rb0 = __fsub_rn(__fsub_rn(1.0f, r.b1), r.b2);
        rest_position = xbary(q0, q1, q2, rb0, r.b1, r.b2);
    }
    return r;
}

// The blend weights of generate.h:226-241 in the reference's rounding: every
// value IEEE-rounded and uncontracted.  Rewrites the weights of the strand's
// blended slots (records in slot order, as the setup step staged them) and
// returns their sum in slot order.  For powers other than 2 the setup step
// takes the fast power; it calls this only for strands whose sum may lie on
// the other side of the 1e-12 threshold that chooses between blending and the
// nearest-guide fallback (generate.h:261), so that choice is the reference's
// (to the last-bit agreement of CUDA's powf with the host's).  The hot path
// rarely takes it: the noise walk calls the out-of-line copy below (inlined
// it costs that kernel more registers than the call), the noise-free walk
// this inlined one (the call's saved registers cost it more).
__device__ __forceinline__ float walk_exact_weights_inline(const LaunchArgs &g, uint32_t triangle, F3 position,
                                                          F3 normal, float *slot_words, int lane) {
    const AssetArgs &a = g.a;
    const ParamArgs &p = g.p;
    float wsum = 0.0f;
    uint32_t blended = 0u;
    for (uint32_t j = 0; j < kSlots; ++j) {
        const uint32_t gi = __ldg(a.stencil + static_cast<uint64_t>(triangle) * kSlots + j);
        if (gi == kInvalid || gi >= a.guide_count) { continue; }
        const float4 gr = __ldg(g.guide_frames + 2u * gi);
        const float4 gn = __ldg(g.guide_frames + 2u * gi + 1u);
        if (__float_as_uint(gn.w) == 0u) { continue; }
        const F3 delta = xsub(position, F3{gr.x, gr.y, gr.z});
        const float d2 = xdot(delta, delta);
        if (xdot(normal, F3{gn.x, gn.y, gn.z}) < p.rejection_cos) { continue; }
        const float radius = gr.w;
        if (radius <= 0.0f || d2 >= __fmul_rn(radius, radius)) { continue; }
        const float x = __fsub_rn(1.0f, __fdiv_rn(__fsqrt_rn(d2), radius));
        const float w = p.weight_power == 2.0f ? __fmul_rn(x, x) : powf(x, p.weight_power);
        slot_words[((blended >> 1) * 32u + static_cast<uint32_t>(lane)) * 4u + (blended & 1u) * 2u + 1u] = w;
        ++blended;
        wsum = __fadd_rn(wsum, w);
    }
    return wsum;
}

static __device__ __noinline__ float walk_exact_weights(const LaunchArgs &g, uint32_t triangle, F3 position,
                                                        F3 normal, float *slot_words, int lane) {
    return walk_exact_weights_inline(g, triangle, position, normal, slot_words, lane);
}

// Whether a weight sum from the fast power (__powf, within p * 4e-7 + 1e-5
// relative of powf for exact bases) may lie on the other side of the 1e-12
// blend threshold from the reference's; twice that bound is used.
__device__ __forceinline__ bool walk_blend_uncertain(float wsum, float power) {
    return fabsf(wsum - 1.0e-12f) <= 2.0f * (power * 4.0e-7f + 1.0e-5f) * wsum;
}

// The lane walk's own per-strand decisions, for inspection
// (nxg_query_walk_states): the blend mode (0 blend, 1 nearest guide,
// 2 root normal), the nearest eligible guide, the weight sum the decision
// was taken on, and the weighted slots in the order the base step reads
// them (guide index and weight; one slot of weight 1 in nearest mode).
struct WalkDecision {
    uint32_t mode;
    uint32_t nearest;
    float weight_sum;
    uint32_t slot_count;
    uint32_t guides[kSlots];
    float weights[kSlots];
};

// The strand's RootSample (types.h:126-136) at roots[local]: three 16-byte
// stores when the array is 16-byte aligned, else twelve word stores.
__device__ __forceinline__ void walk_store_root(uint32_t *roots, uint32_t local, const Root &r) {
    uint32_t *dst = roots + static_cast<uint64_t>(local) * 12u;
    if ((reinterpret_cast<std::uintptr_t>(roots) & 15u) == 0u) {
        uint4 *v = reinterpret_cast<uint4 *>(dst);
        v[0] = make_uint4(root_word(r, 0), root_word(r, 1), root_word(r, 2), root_word(r, 3));
        v[1] = make_uint4(root_word(r, 4), root_word(r, 5), root_word(r, 6), root_word(r, 7));
        v[2] = make_uint4(root_word(r, 8), root_word(r, 9), root_word(r, 10), root_word(r, 11));
    } else {
#pragma unroll
        for (int w = 0; w < 12; ++w) { dst[w] = root_word(r, w); }
    }
}

// Setup step for this lane's strand.  The stencil slots follow eval_slot and
// the loop of generate.h:214-244 with the frame's guide roots, normals and
// support radii read from the per-frame guide records.  With `outputs`,
// also writes the strand's RootSample, root UV and point count.  With
// `decision` (inspection only), also reports the choices made.  Slots past
// the strand's count point at the frame's zero row with weight 0, so the
// base step may read any slot of the four records.
template <bool NOISE>
__device__ __forceinline__ WalkRoot walk_setup(const LaunchArgs &g, float4 *records, uint32_t *locals, int lane,
                                               uint32_t pick, bool valid, uint32_t P, bool outputs = true,
                                               WalkDecision *decision = nullptr) {
    const AssetArgs &a = g.a;
    const FrameArgs &f = g.f;
    const ParamArgs &p = g.p;
    uint32_t local = __ldg(g.order + pick);
    if (local >= g.count) {
        local = 0u;
        valid = false;
    }
    WalkRoot r;
    r.surface_u = F3{0.0f, 0.0f, 0.0f};
    F3 rest_position = {0.0f, 0.0f, 0.0f};
    const Root root = walk_root<NOISE>(a, f, p.seed, g.first_strand + local, r.surface_u, rest_position);
    if (outputs && valid) {  // generate.h:621-623
        if (g.roots) { walk_store_root(g.roots, local, root); }
        if (g.root_uvs) { g.root_uvs[local] = make_float2(root.u, root.v); }
        if (g.point_counts) { g.point_counts[local] = P; }
    }
    const float zero_row = __uint_as_float(g.zero_row);
#pragma unroll
    for (int q = 0; q < 4; ++q) { records[q * 32 + lane] = make_float4(zero_row, 0.0f, zero_row, 0.0f); }
    uint32_t stencil[kSlots];
    const uint32_t *row = a.stencil + static_cast<uint64_t>(root.triangle) * kSlots;
    if ((reinterpret_cast<std::uintptr_t>(a.stencil) & 15u) == 0u) {
        const uint4 s0 = __ldg(reinterpret_cast<const uint4 *>(row));
        const uint4 s1 = __ldg(reinterpret_cast<const uint4 *>(row) + 1);
        stencil[0] = s0.x; stencil[1] = s0.y; stencil[2] = s0.z; stencil[3] = s0.w;
        stencil[4] = s1.x; stencil[5] = s1.y; stencil[6] = s1.z; stencil[7] = s1.w;
    } else {
#pragma unroll
        for (uint32_t j = 0; j < kSlots; ++j) { stencil[j] = __ldg(row + j); }
    }
    float *slot_words = reinterpret_cast<float *>(records);
    // Guide frame record of slot j (an out-of-range slot reads as a corrupt
    // record: no slot).  With noise (fewer warps per SM to hide latency) all
    // eight are requested before any is used; without, one at a time, which
    // keeps the register count and the occupancy of the plain kernel.
    float4 gr[kSlots], gn[kSlots];
    auto load_slot = [&](uint32_t j) {
        const bool in_range = stencil[j] != kInvalid && stencil[j] < a.guide_count;
        const uint32_t gi = in_range ? stencil[j] : 0u;
        gr[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        gn[j] = gr[j];
        if (a.guide_count != 0u) {
            gr[j] = __ldg(g.guide_frames + 2u * gi);
            gn[j] = __ldg(g.guide_frames + 2u * gi + 1u);
        }
        if (!in_range) { gn[j].w = 0.0f; }
    };
    if constexpr (NOISE) {
#pragma unroll
        for (uint32_t j = 0; j < kSlots; ++j) { load_slot(j); }
    }
    // Blend weights (1 - d / r)^power in fast arithmetic (they feed positions
    // only); d^2, the rejection test and the radius test that decide which
    // slots count stay in the reference's exact rounding.
    const bool square = p.weight_power == 2.0f;
    float wsum = 0.0f;
    float nearest_d2 = FLT_MAX;
    uint32_t nearest = kInvalid;
    uint32_t blended = 0u;
#pragma unroll
    for (uint32_t j = 0; j < kSlots; ++j) {
        if constexpr (!NOISE) { load_slot(j); }
        if (__float_as_uint(gn[j].w) == 0u) { continue; }  // out of range or corrupt record
        const F3 delta = xsub(root.position, F3{gr[j].x, gr[j].y, gr[j].z});
        const float d2 = xdot(delta, delta);
        if (xdot(root.normal, F3{gn[j].x, gn[j].y, gn[j].z}) < p.rejection_cos) { continue; }
        if (d2 < nearest_d2) {  // strict first minimum over eligible slots (generate.h:234)
            nearest_d2 = d2;
            nearest = stencil[j];
        }
        const float radius = gr[j].w;
        if (radius <= 0.0f || d2 >= __fmul_rn(radius, radius)) { continue; }
        // The base 1 - sqrt(d2) / r in the reference's rounding: near the
        // edge of the support radius it cancels, and a fast quotient would
        // change the weight there by a large fraction.  The square is then
        // the reference's weight bit for bit; other powers take __powf.
        const float x = __fsub_rn(1.0f, __fdiv_rn(__fsqrt_rn(d2), radius));
        const float w = square ? __fmul_rn(x, x)
                               : (x > 0.0f ? __powf(x, p.weight_power) : (p.weight_power > 0.0f ? 0.0f : 1.0f));
        float *dst = slot_words + ((blended >> 1) * 32u + lane) * 4u + (blended & 1u) * 2u;
        dst[0] = __uint_as_float(stencil[j] * P);
        dst[1] = w;
        ++blended;
        wsum = __fadd_rn(wsum, w);
    }
    if (!square && blended != 0u && walk_blend_uncertain(wsum, p.weight_power)) {
        if constexpr (NOISE) {
            wsum = walk_exact_weights(g, root.triangle, root.position, root.normal, slot_words, lane);
        } else {
            wsum = walk_exact_weights_inline(g, root.triangle, root.position, root.normal, slot_words, lane);
        }
    }
    float inv = 0.0f;
    F3 normal_term = {0.0f, 0.0f, 0.0f};
    uint32_t nb = blended;
    uint32_t mode = 0u;
    if (wsum > 1.0e-12f) {
        inv = 1.0f / wsum;
    } else if (nearest != kInvalid) {
        records[lane] = make_float4(__uint_as_float(nearest * P), 1.0f, zero_row, 0.0f);
        nb = 1u;
        inv = 1.0f;
        mode = 1u;
    } else {
        nb = 0u;
        normal_term = root.normal;
        mode = 2u;
    }
    if (decision != nullptr) {
        decision->mode = mode;
        decision->nearest = nearest;
        decision->weight_sum = wsum;
        decision->slot_count = nb;
        for (uint32_t j = 0; j < kSlots; ++j) {
            const float *src = slot_words + (((j >> 1) * 32u + lane) * 4u + (j & 1u) * 2u);
            decision->guides[j] = j < nb ? __float_as_uint(src[0]) / P : kInvalid;
            decision->weights[j] = j < nb ? src[1] : 0.0f;
        }
    }
    records[4 * 32 + lane] = make_float4(root.position.x, root.position.y, root.position.z, inv);
    records[5 * 32 + lane] = make_float4(normal_term.x, normal_term.y, normal_term.z, __uint_as_float(nb));
    locals[lane] = local | (valid ? 0u : 0x80000000u);
    r.position = root.position;
    r.normal = root.normal;
    r.domain = F3{0.0f, 0.0f, 0.0f};
    if constexpr (NOISE) {
        const float decorrelation = 1.0f - p.noise_correlation;
        const float domain_scale = 100.0f * decorrelation * decorrelation;
        r.domain = (rest_position + F3{0.419276f, 0.184247f, 0.805721f}) * domain_scale;
    }
    return r;
}

// One output point of the strand whose output word is `word` (skipped when
// the word is marked invalid): float4 (position, radius), or Vec3 positions,
// 3P consecutive floats per strand (device_contract.h:47-52).
__device__ __forceinline__ void walk_emit(const LaunchArgs &g, uint32_t word, int P, int c, float4 q) {
    if (word >> 31) { return; }
    const uint64_t index = static_cast<uint64_t>(word) * static_cast<uint32_t>(P) + static_cast<uint32_t>(c);
    if (g.vec3_points) {
        float *out3 = g.vec3_points + 3u * index;
        __stcs(out3, q.x);
        __stcs(out3 + 1, q.y);
        __stcs(out3 + 2, q.z);
    } else {
        __stcs(g.points + index, q);
    }
}

// CV c of a staged row.
__device__ __forceinline__ F3 stage_get(const float *row, int c) {
    return F3{row[3 * c], row[3 * c + 1], row[3 * c + 2]};
}
__device__ __forceinline__ void stage_put(float *row, int c, F3 v) {
    row[3 * c] = v.x;
    row[3 * c + 1] = v.y;
    row[3 * c + 2] = v.z;
}

// Strand of a flattened (strand, CV) item: floor((item + 0.5) / P), exact for
// item < 32 * 32 (the quotient is at least 0.5 / P from an integer).
__device__ __forceinline__ int walk_strand(int item, float inv_p) {
    return static_cast<int>((static_cast<float>(item) + 0.5f) * inv_p);
}

// Base point c of strand s from its records (generate.h:246-267, :300-310).
__device__ __forceinline__ F3 walk_base_point(const float4 *records, int s, int c, float t, float ls,
                                              const float4 *offsets) {
    const float4 head = records[4 * 32 + s];
    const float4 tail = records[5 * 32 + s];
    const uint32_t nb = __float_as_uint(tail.w);
    F3 acc = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const float4 gw = records[q * 32 + s];
        if (static_cast<uint32_t>(2 * q) < nb) {
            const float4 d = __ldg(offsets + (__float_as_uint(gw.x) + static_cast<uint32_t>(c)));
            acc = acc + F3{d.x, d.y, d.z} * gw.y;
        }
        if (static_cast<uint32_t>(2 * q + 1) < nb) {
            const float4 d = __ldg(offsets + (__float_as_uint(gw.z) + static_cast<uint32_t>(c)));
            acc = acc + F3{d.x, d.y, d.z} * gw.w;
        }
    }
    const F3 off = acc * head.w + F3{tail.x, tail.y, tail.z} * t;
    return F3{head.x, head.y, head.z} + off * ls;
}

// Classic scalars without noise (xgen_classic_runtime.cpp:1650-1678,
// :1827-1858), for this lane's strand before its base step: the first and
// last base points give the chord; a strand whose scaled chord is near the
// 1e-4 threshold measures its sampled spline (lanes that need it take turns
// on `scratch`, 32 float4); a dropped strand gets point count 0.  Leaves
// records 6 and 7 for walk_base.  Every lane of the warp calls it.
__device__ __forceinline__ void walk_classic_setup(const LaunchArgs &g, float4 *records, int lane, bool valid,
                                                   uint32_t local, const float *tvals, const float4 *offsets,
                                                   float4 *scratch, int P) {
    const ParamArgs &p = g.p;
    const float ls = p.length_scale;
    const float2 sc = __ldg(g.scalars + local);
    const F3 front = walk_base_point(records, lane, 0, tvals[0], ls, offsets);
    const F3 back = walk_base_point(records, lane, P - 1, tvals[P - 1], ls, offsets);
    const float scale = g.classic_length ? sc.x : 1.0f;
    const float raw_width = g.classic_width ? sc.y
        : (p.radius_scale > 0.0f ? __fdiv_rn(__fmul_rn(2.0f, strand_radius(p, 0.0f)), p.radius_scale) : 0.0f);
    bool keep = !(raw_width < 1.0e-4f);
    const F3 chord = back - front;
    const bool measure = keep && !(sqrtf(dot(chord, chord)) * scale > 1.01e-4f);
    for (unsigned todo = __ballot_sync(kFull, measure); todo != 0u; todo &= todo - 1u) {
        if (lane == __ffs(todo) - 1) {
            for (int c = 0; c < P; ++c) {
                const F3 b = walk_base_point(records, lane, c, tvals[c], ls, offsets);
                scratch[c] = make_float4(b.x, b.y, b.z, 0.0f);
            }
            keep = !(__fmul_rn(classic_spline_length(scratch, P), scale) < 1.0e-4f);
        }
        __syncwarp();
    }
    const float radius = __fmul_rn(__fmul_rn(0.5f, raw_width < 0.0f ? 0.0f : raw_width), p.radius_scale);
    records[6 * 32 + lane] = make_float4(front.x, front.y, front.z, scale);
    records[7 * 32 + lane] = make_float4(radius, g.classic_width ? 1.0f : 0.0f, 0.0f, 0.0f);
    if (!keep && valid && g.point_counts != nullptr) { g.point_counts[local] = 0u; }
}

// Base step: item = s * P + c over the batch, 32 consecutive items per pass,
// into the stage or (DIRECT) straight to the output; CLASSIC (with DIRECT)
// applies records 6 and 7: scale about the first point, width override.
template <bool DIRECT, bool CLASSIC = false>
__device__ __forceinline__ void walk_base(const LaunchArgs &g, const float4 *records, float *stage,
                                          const uint32_t *locals, const float *tvals, const float *rvals,
                                          const float4 *offsets, int lane, int in_batch, int P, float inv_p) {
    const int items = in_batch * P;
    const float ls = g.p.length_scale;
#pragma unroll 2
    for (int item = lane; item < items; item += 32) {
        const int s = walk_strand(item, inv_p);
        const int c = item - s * P;
        F3 base = walk_base_point(records, s, c, tvals[c], ls, offsets);
        float radius = rvals[c];
        if constexpr (CLASSIC) {
            const float4 front = records[6 * 32 + s];
            const float4 width = records[7 * 32 + s];
            if (g.classic_length) { base = xadd(xyz(front), xmul(xsub(base, xyz(front)), front.w)); }
            if (width.y != 0.0f) { radius = width.x; }
        }
        if constexpr (DIRECT) {
            walk_emit(g, locals[s], P, c, make_float4(base.x, base.y, base.z, radius));
        } else {
            stage_put(stage + s * kWalkRowFloats, c, base);  // radii come from the t table at the store
        }
    }
}

// Base step straight to the output (no noise).  Eight lanes per strand and
// four strands per pass: lane (s = pass * 4 + lane / 8, c = lane % 8)
// computes CVs c + 8m, m < ceil(P / 8).  One address per slot serves the
// lane's loads (the other CVs sit at fixed distances along the guide's
// offset row), every load of a warp instruction stays within one 128-byte
// line per strand, and a lane's t values are fixed for the whole kernel.  A
// pass runs as many slot pairs as its strands' largest count; a strand's
// loads past its own count are predicated off (no memory request), and its
// records there hold the zero row with weight 0, so the accumulation needs
// no predicate.  CLASSIC applies records 6 and 7 as walk_base does.  STAGED
// writes the base points into the strands' stage rows instead of the output
// (the noise walk reads them there); a stage row of 97 words keeps the
// four strands of a pass at most two lanes to a bank.  Every lane of the
// warp calls it.
template <bool CLASSIC, bool STAGED = false>
__device__ __forceinline__ void walk_base_direct(const LaunchArgs &g, const float4 *records, const uint32_t *locals,
                                                 const float *tvals, const float *rvals, const float4 *offsets,
                                                 int lane, int in_batch, int P, float *stage = nullptr) {
    static_assert(!(CLASSIC && STAGED), "staged strands take the Classic application at the store");
    constexpr int kPerLane = kWalkMaxCvs / 8;
    const int c = lane & 7;
    const int cpl = (P + 7) >> 3;
    float tv[kPerLane];
#pragma unroll
    for (int m = 0; m < kPerLane; ++m) { tv[m] = tvals[min(c + 8 * m, P - 1)]; }
    const float ls = g.p.length_scale;
    const float4 *column = offsets + c;
    for (int first = 0; first < in_batch; first += 4) {
        const int s = first + (lane >> 3);
        const bool live = s < in_batch;
        const float4 head = records[4 * 32 + s];
        const float4 tail = records[5 * 32 + s];
        const uint32_t nb = live ? __float_as_uint(tail.w) : 0u;
        const uint32_t pairs = __reduce_max_sync(kFull, (nb + 1u) >> 1);
        F3 acc[kPerLane];
        float4 da[kPerLane], db[kPerLane];
#pragma unroll
        for (int m = 0; m < kPerLane; ++m) {
            acc[m] = F3{0.0f, 0.0f, 0.0f};
            da[m] = db[m] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
        for (uint32_t q = 0; q < pairs; ++q) {
            // A strand loads only its own slots: past its count the registers
            // keep the last (finite) entries and the weights are zero.
            const float4 gw = records[q * 32 + s];
            const float4 *ra = column + __float_as_uint(gw.x);
            const float4 *rb = column + __float_as_uint(gw.z);
            const bool la = 2u * q < nb, lb = 2u * q + 1u < nb;
#pragma unroll
            for (int m = 0; m < kPerLane; ++m) {
                if (m < cpl) {
                    if (la) { da[m] = __ldg(ra + 8 * m); }
                    if (lb) { db[m] = __ldg(rb + 8 * m); }
                }
            }
#pragma unroll
            for (int m = 0; m < kPerLane; ++m) {
                if (m < cpl) { acc[m] = acc[m] + xyz(da[m]) * gw.y + xyz(db[m]) * gw.w; }
            }
        }
        if constexpr (STAGED) {
            float *row = stage + s * kWalkRowFloats;
#pragma unroll
            for (int m = 0; m < kPerLane; ++m) {
                const int cm = c + 8 * m;
                if (live && m < cpl && cm < P) {
                    stage_put(row, cm,
                              F3{head.x, head.y, head.z} + (acc[m] * head.w + F3{tail.x, tail.y, tail.z} * tv[m]) * ls);
                }
            }
            continue;
        }
        const uint32_t word = live ? locals[s] : 0x80000000u;
        float4 front = {0.0f, 0.0f, 0.0f, 1.0f}, width = {0.0f, 0.0f, 0.0f, 0.0f};
        if constexpr (CLASSIC) {
            front = records[6 * 32 + s];
            width = records[7 * 32 + s];
        }
#pragma unroll
        for (int m = 0; m < kPerLane; ++m) {
            const int cm = c + 8 * m;
            if (m < cpl && cm < P) {
                F3 base = F3{head.x, head.y, head.z} + (acc[m] * head.w + F3{tail.x, tail.y, tail.z} * tv[m]) * ls;
                float radius = rvals[cm];
                if constexpr (CLASSIC) {
                    if (g.classic_length) { base = xadd(xyz(front), xmul(xsub(base, xyz(front)), front.w)); }
                    if (width.y != 0.0f) { radius = width.x; }
                }
                walk_emit(g, word, P, cm, make_float4(base.x, base.y, base.z, radius));
            }
        }
    }
}

// Floor by a round-down add: for |x| < 2^22, x + 1.5 * 2^23 lies in
// [2^23, 2^24), where consecutive floats are consecutive integers, so the
// sum rounded toward minus infinity is 1.5 * 2^23 + floor(x) exactly.  Its
// bit pattern minus that of 1.5 * 2^23 is floor(x) as an integer, and the
// sum minus 1.5 * 2^23 is floor(x) as a float (an exact difference).  Two
// adds on the FMA pipe replace the rounding and conversion instructions.
constexpr float kFloorMagic = 12582912.0f;      // 1.5 * 2^23
constexpr uint32_t kFloorMagicBits = 0x4b400000u;
constexpr float kFloorMagicLimit = 4194304.0f;  // 2^22

// 2 (noise - 0.5) along one axis from the strand's lattice columns (the
// regrouped blend of lattice_noise); the caller folds the 1/2 into the
// magnitude, a product by an exact power of two.  The axis' columns start at
// column axis * columns of the strand's lattice; `bias` is the bit pattern
// of 1.5 * 2^23 plus the axis' first lattice coordinate minus that start, so
// the sum's bits minus `bias` index the lattice directly, and `kmax` (the
// axis' last pair) bounds the index (x never lies below the first column:
// the walk's distances are non-negative; lanes with no strand read some
// column of their own lattice).
__device__ __forceinline__ float walk_lattice_delta(const float2 *lat, uint32_t bias, uint32_t kmax, float x) {
    const float t = __fadd_rd(x, kFloorMagic);
    const float w = x - (t - kFloorMagic);
    const uint32_t k = min(__float_as_uint(t) - bias, kmax);
    const float2 *col = lat + static_cast<int>(k) * 32;
    const float2 c0 = col[0];
    const float2 c1 = col[32];
    const float s = s_curve(w);
    const float v0 = c0.x * w + c0.y;
    const float v1 = c1.x * (w - 1.0f) + c1.y;
    return v0 + s * (v1 - v0);
}

// Lattice columns (A, B) of the three noise axes for one strand (see
// lattice_noise): columns lo .. floor(d0 + span) + 1 cover every CV's X and
// X + 1 (the walk's noise coordinates d0 + arc * f are computed in the same
// IEEE operations as d0 + span, so none passes it).  `lat` is this lane's
// column 0 of axis 0; column k of axis a is at lat[(a * columns + k) * 32].
// fits is false when a strand needs more columns than the lattice holds, or
// has coordinates beyond the round-down floor's range (it then takes direct
// noise).  bias and kmax are the per-axis arguments of walk_lattice_delta.
struct WalkLattice {
    int lo[3], n[3];
    uint32_t bias[3], kmax[3];
    bool fits;
};

__device__ __forceinline__ WalkLattice walk_fill_lattice(F3 dom, float span, float2 *lat, const float4 *table,
                                                       int columns) {
    WalkLattice wl;
    wl.fits = true;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const float d0 = component(dom, ax);
        wl.lo[ax] = static_cast<int>(floorf(d0));
        wl.n[ax] = static_cast<int>(floorf(__fadd_rn(d0, span))) + 2 - wl.lo[ax];
        wl.fits = wl.fits && wl.n[ax] >= 2 && wl.n[ax] <= columns && fabsf(d0) + span < kFloorMagicLimit;
    }
    if (!wl.fits) {  // lattice reads stay in bounds (column 0 and 1) whatever the strand
        wl.n[0] = wl.n[1] = wl.n[2] = 2;
    }
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        wl.bias[ax] = kFloorMagicBits + static_cast<uint32_t>(wl.lo[ax]) - static_cast<uint32_t>(ax * columns);
        wl.kmax[ax] = static_cast<uint32_t>(ax * columns + wl.n[ax] - 2);
    }
    if (!wl.fits) { return wl; }
    // Columns 0 and 1 of every axis are faces of the unit lattice cube at
    // floor(dom): its eight corner gradients (corner o = ox + 2 oy + 4 oz)
    // serve all three axes, the gradients of columns 2.. are looked up.
    float4 cube[8];
    {
        const uint32_t base = static_cast<uint32_t>(wl.lo[0]) * kLcgA2 + static_cast<uint32_t>(wl.lo[1]) * kLcgA +
                              static_cast<uint32_t>(wl.lo[2]) + kLcgK;
#pragma unroll
        for (int o = 0; o < 8; ++o) {
            cube[o] = table[temper_index(base + ((o & 1) ? kLcgA2 : 0u) + ((o & 2) ? kLcgA : 0u) +
                                         ((o & 4) ? 1u : 0u))];
        }
    }
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const int ib = ax == 0 ? 1 : 0;  // the fixed axes, ascending
        const int ic = ax == 2 ? 1 : 2;
        const float db = component(dom, ib), dc = component(dom, ic);
        const float fb = floorf(db), fc = floorf(dc);
        const float wb = db - fb, wc = dc - fc;
        const float sb = s_curve(wb), sc = s_curve(wc);
        const int Yb = static_cast<int>(fb), Zc = static_cast<int>(fc);
        // The corner seed is linear in the moving coordinate X (noise_hash's
        // LCG chain): seed(X + 1) = seed(X) + step.
        const uint32_t step = ax == 0 ? kLcgA2 : (ax == 1 ? kLcgA : 1u);
        uint32_t seed[4];
        float wgt[4], wdb[4], wdc[4];
#pragma unroll
        for (int corner = 0; corner < 4; ++corner) {
            const int ob = corner & 1, oc = corner >> 1;
            const int X = wl.lo[ax];
            const int cx = ax == 0 ? X : Yb + ob;
            const int cy = ax == 1 ? X : (ax == 0 ? Yb + ob : Zc + oc);
            const int cz = ax == 2 ? X : Zc + oc;
            seed[corner] = static_cast<uint32_t>(cx) * kLcgA2 + static_cast<uint32_t>(cy) * kLcgA +
                           static_cast<uint32_t>(cz) + kLcgK;
            wgt[corner] = (ob ? sb : 1.0f - sb) * (oc ? sc : 1.0f - sc);
            wdb[corner] = wgt[corner] * (wb - static_cast<float>(ob));
            wdc[corner] = wgt[corner] * (wc - static_cast<float>(oc));
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            float A = 0.0f, B = 0.0f;
#pragma unroll
            for (int corner = 0; corner < 4; ++corner) {
                const float4 gr = cube[(k << ax) | ((corner & 1) << ib) | ((corner >> 1) << ic)];
                A += wgt[corner] * component4(gr, ax);
                B += component4(gr, ib) * wdb[corner] + component4(gr, ic) * wdc[corner];
            }
            lat[(ax * columns + k) * 32] = make_float2(A, B);
        }
#pragma unroll 2
        for (int k = 2; k < wl.n[ax]; ++k) {
            float A = 0.0f, B = 0.0f;
#pragma unroll
            for (int corner = 0; corner < 4; ++corner) {
                const float4 gr = table[temper_index(seed[corner] + static_cast<uint32_t>(k) * step)];
                A += wgt[corner] * component4(gr, ax);
                B += component4(gr, ib) * wdb[corner] + component4(gr, ic) * wdc[corner];
            }
            lat[(ax * columns + k) * 32] = make_float2(A, B);
        }
    }
    return wl;
}

__device__ __forceinline__ float walk_effective_frequency(const ParamArgs &p, float original_length) {
    return original_length > 0.0f ? fmaxf(0.5f / original_length, p.noise_frequency) : p.noise_frequency;
}

// |b - a| in fixed IEEE operations (no contraction left to the compiler), so
// the length pass and the cursor walk's arc-length prefix agree bit for bit.
__device__ __forceinline__ float walk_segment_length(F3 b, F3 a) {
    const F3 d = b - a;
    return sqrt_approx(__fmaf_rn(d.z, d.z, __fmaf_rn(d.y, d.y, __fmul_rn(d.x, d.x))));
}

// The cursor walk (generate.h:465-502) over base points base(0..P-1),
// handing each noisy point to emit(c, point) in CV order; returns the noisy
// length (generate.h:553-556) when PRESERVE, else 0.  Tangent after CV c: the
// next segment's direction, carried over zero-length segments and at the
// tip; the transported normal rotates by rotate_by(axis, acos(cos)) with
// cos(acos x) = x and sin(acos x) = sqrt(1 - x^2):
//   M v = cos v + (1 - cos)(axis . v) axis + sin (axis x v),
// and is left unchanged when the axis is zero (the axis and that test in
// ordinary arithmetic: where the reference's rounded cross product vanishes
// for nearly parallel tangents, the rotation left here is within rounding of
// the identity).  The body has no per-lane branches (each decision is a
// select), so the compiler can overlap the noise, tangent and frame chains of
// neighbouring CVs; noise at CV 0 is
// multiplied by t_0 = 0.  LATTICE: every lane of the warp reads lattice
// noise (else every lane evaluates gradient_noise).  Base points are
// requested three CVs before they are used.
template <bool LATTICE, bool PRESERVE, class Base, class Emit>
__device__ __forceinline__ float walk_cursor(const ParamArgs &p, const WalkRoot &wr, float f_eff,
                                             const WalkLattice &wl, const float2 *lat, const float *tvals,
                                             const float4 *table, int P, Base base, Emit emit) {
    // Lattice deltas come doubled (walk_lattice_delta): their magnitude takes
    // the 1/2, which leaves every product bit-identical.
    const float mscale = LATTICE ? 0.5f * (p.noise_mask * p.noise_amplitude) : p.noise_mask * p.noise_amplitude;
    const F3 dom = wr.domain;
    F3 tan = wr.normal;
    F3 v = wr.surface_u;
    F3 cur = base(0);
    F3 nxt = base(1);
    F3 ahead = P > 2 ? base(2) : nxt;
    F3 previous_base = cur;
    F3 previous_point = cur;
    float noisy = 0.0f;
    float arc = 0.0f;
#pragma unroll 2
    for (int c = 0; c < P; ++c) {
        // Past the strand's end the look-ahead repeats the last CV, which is
        // what `ahead` and `nxt` already hold there (the tip's tangent does
        // not read it).
        const F3 further = base(min(c + 3, P - 1));
        arc = __fadd_rn(arc, walk_segment_length(cur, previous_base));
        // The reference's length_squared(segment) > 0 holds exactly when some
        // component's square does not round to zero: the same test on the
        // fused sum (no flush to zero here).
        const F3 seg = nxt - cur;
        const F3 ntan = (c + 1 < P && dot(seg, seg) > 0.0f) ? normalize(seg) : tan;
        const F3 axis = cross(tan, ntan);
        // A zero axis leaves the normal as it is: cos 1, sin 0 (then k = 0
        // and the update below is v itself, exactly).
        const bool turn = dot(axis, axis) > 0.0f;
        const float d = fminf(fmaxf(dot(tan, ntan), -1.0f), 1.0f);
        const float cs = turn ? d : 1.0f;
        const float sn = turn ? sqrt_approx(fmaf(-d, d, 1.0f)) : 0.0f;
        const float k = (1.0f - cs) * dot(axis, v);
        const F3 axv = cross(axis, v);
        v = F3{v.x * cs + axis.x * k + axv.x * sn, v.y * cs + axis.y * k + axv.y * sn,
               v.z * cs + axis.z * k + axv.z * sn};
        // The update is linear in v and the reference renormalises after
        // every step, a positive factor each time: so the transported normal
        // is the direction of this unnormalised v, which is carried as it is
        // (each step keeps at least 0.86 of its length, so 32 steps neither
        // underflow nor overflow) and normalised here for the frame only.
        const F3 vu = v * rsqrtf(dot(v, v));
        const F3 bn = cross(vu, ntan);
        // The frame's third vector cross(bn, vu) is ntan - vu (vu . ntan) for
        // a unit vu; its part along vu joins vu's coefficient below.
        const float vn = dot(vu, ntan);
        const float distance = __fmul_rn(arc, f_eff);
        const float magnitude = mscale * tvals[c];
        float gx, gy, gz;
        if constexpr (LATTICE) {
            gx = walk_lattice_delta(lat, wl.bias[0], wl.kmax[0], __fadd_rn(dom.x, distance));
            gy = walk_lattice_delta(lat, wl.bias[1], wl.kmax[1], __fadd_rn(dom.y, distance));
            gz = walk_lattice_delta(lat, wl.bias[2], wl.kmax[2], __fadd_rn(dom.z, distance));
        } else {
            gx = gradient_noise(table, __fadd_rn(dom.x, distance), dom.y, dom.z) - 0.5f;
            gy = gradient_noise(table, dom.x, __fadd_rn(dom.y, distance), dom.z) - 0.5f;
            gz = gradient_noise(table, dom.x, dom.y, __fadd_rn(dom.z, distance)) - 0.5f;
        }
        const float gzm = gz * magnitude;
        const F3 q = cur + vu * fmaf(-gzm, vn, gx * magnitude) + bn * (gy * magnitude) + ntan * gzm;
        if constexpr (PRESERVE) {
            const F3 e = q - previous_point;
            noisy += sqrt_approx(dot(e, e));
            previous_point = q;
        }
        emit(c, q);
        tan = ntan;
        previous_base = cur;
        cur = nxt;
        nxt = ahead;
        ahead = further;
    }
    return noisy;
}

// walk_cursor with its warp-uniform variant: lattice noise when every lane
// whose strand counts (`counts`) fits its lattice.  Every lane of the warp
// calls it.
template <class Base, class Emit>
__device__ __forceinline__ float walk_cursor_any(const ParamArgs &p, const WalkRoot &wr, float f_eff,
                                                 const WalkLattice &wl, bool counts, const float2 *lat,
                                                 const float *tvals, const float4 *table, int P, Base base,
                                                 Emit emit) {
    const bool lattice = __all_sync(kFull, wl.fits || !counts);
    const bool preserve = p.noise_preserve_length > 0.001f;
    if (lattice) {
        return preserve ? walk_cursor<true, true>(p, wr, f_eff, wl, lat, tvals, table, P, base, emit)
                        : walk_cursor<true, false>(p, wr, f_eff, wl, lat, tvals, table, P, base, emit);
    }
    return preserve ? walk_cursor<false, true>(p, wr, f_eff, wl, lat, tvals, table, P, base, emit)
                    : walk_cursor<false, false>(p, wr, f_eff, wl, lat, tvals, table, P, base, emit);
}

// preserveLength scale (generate.h:553-563), or 1.
__device__ __forceinline__ float walk_preserve_scale(const ParamArgs &p, float original_length, float noisy) {
    if (!(p.noise_preserve_length > 0.001f) || !(noisy > 0.0f)) { return 1.0f; }
    const float target = original_length * p.noise_preserve_length + noisy * (1.0f - p.noise_preserve_length);
    return fabsf(noisy - target) >= 0.0001f ? target / noisy : 1.0f;
}

// Frame step for the strand whose staged row is `row` (this lane's strand):
// the base curve's length, the lattice, then the cursor walk, leaving the
// noisy points in the row.  The walk reads CV c + 3 after
// writing CV c, so it never reads a point it has replaced.  Every lane of the
// warp calls it; lanes whose strand does not count (past the batch) work on
// whatever their row holds and are ignored.
__device__ __forceinline__ void walk_frame(const ParamArgs &p, const WalkRoot &wr, bool counts, float *row,
                                           float2 *lat, const float *tvals, const float4 *table, int P,
                                           int columns) {
    // Length of the base curve (generate.h:420-433); the walk accumulates the
    // same prefix again as its arc length, in the same operations.
    float original_length = 0.0f;
    {
        F3 prev = stage_get(row, 0);
#pragma unroll 8
        for (int c = 1; c < P; ++c) {
            const F3 cur = stage_get(row, c);
            original_length = __fadd_rn(original_length, walk_segment_length(cur, prev));
            prev = cur;
        }
    }
    const float f_eff = walk_effective_frequency(p, original_length);
    const WalkLattice wl = walk_fill_lattice(wr.domain, __fmul_rn(original_length, f_eff), lat, table, columns);
    const float noisy = walk_cursor_any(
        p, wr, f_eff, wl, counts, lat, tvals, table, P, [&](int c) { return stage_get(row, c); },
        [&](int c, F3 q) { stage_put(row, c, q); });
    const float scale = walk_preserve_scale(p, original_length, noisy);
    if (scale != 1.0f) {
        const F3 root = wr.position;
        for (int c = 0; c < P; ++c) { stage_put(row, c, root + (stage_get(row, c) - root) * scale); }
    }
}

// generate_pipe_kernel shared memory: table | t values | radii | two buffers
// (stage, 12 x 32 frame floats, 32 output words) | producer records |
// consumer lattice.
constexpr size_t kPipeFrameBytes = sizeof(float) * 12u * 32u;
constexpr size_t kPipeBufferBytes = kWalkStageBytes + kPipeFrameBytes + kWalkLocalBytes;
constexpr size_t kPipeSmemBytes = sizeof(float4) * kTableFloat4 + 2u * sizeof(float) * kWalkMaxCvs +
                                  2u * kPipeBufferBytes + kWalkRecordBytes + kWalkLatticeBytes;

// Store step without Classic scalars, eight lanes per strand as in
// walk_base_direct: lane (s = pass * 4 + lane / 8, c = lane % 8) stores CVs
// c + 8m of its strand's staged row, so each store instruction writes four
// strands' runs of eight consecutive float4s, and a lane's radii are fixed
// for the whole kernel.  Every lane of the warp calls it.
__device__ __forceinline__ void walk_store8(const LaunchArgs &g, const float *stage, const uint32_t *locals,
                                            const float *rvals, int lane, int in_batch, int P) {
    constexpr int kPerLane = kWalkMaxCvs / 8;
    const int c = lane & 7;
    const int cpl = (P + 7) >> 3;
    float rv[kPerLane];
#pragma unroll
    for (int m = 0; m < kPerLane; ++m) { rv[m] = rvals[min(c + 8 * m, P - 1)]; }
    for (int first = 0; first < in_batch; first += 4) {
        const int s = first + (lane >> 3);  // at most 31
        const uint32_t word = s < in_batch ? locals[s] : 0x80000000u;
        const float *row = stage + s * kWalkRowFloats;
#pragma unroll
        for (int m = 0; m < kPerLane; ++m) {
            const int cm = c + 8 * m;
            if (m < cpl && cm < P) {
                const F3 q = stage_get(row, cm);
                walk_emit(g, word, P, cm, make_float4(q.x, q.y, q.z, rv[m]));
            }
        }
    }
}

// The Classic application's per-strand values for the noisy walk, once per
// strand after the walk (lane = strand; the rules of emit_strand: scale about
// the first point, width override, the drop rule with its chord bound and
// sampled-spline measure): records 6 and 7 take (first point, length scale)
// and (width radius); a dropped strand's point count becomes 0.  The records
// are free again once the walk is done (the lattice aliased them).  Every
// lane of the warp calls it.
__device__ __forceinline__ void walk_classic_strand(const LaunchArgs &g, float4 *records, const float *stage,
                                                    const uint32_t *locals, int lane, int in_batch, int P) {
    const ParamArgs &p = g.p;
    const uint32_t word = locals[lane];
    if (lane >= in_batch || (word >> 31)) { return; }
    const float *row = stage + lane * kWalkRowFloats;
    const float2 sc = __ldg(g.scalars + word);
    const F3 front = stage_get(row, 0);
    const F3 back = stage_get(row, P - 1);
    const float scale = g.classic_length ? sc.x : 1.0f;
    const float raw_width = g.classic_width ? sc.y
        : (p.radius_scale > 0.0f ? __fdiv_rn(__fmul_rn(2.0f, strand_radius(p, 0.0f)), p.radius_scale) : 0.0f);
    bool keep = !(raw_width < 1.0e-4f);
    const F3 chord = back - front;
    if (keep && !(sqrtf(dot(chord, chord)) * scale > 1.01e-4f)) {
        keep = !(__fmul_rn(classic_spline_length_by([row](int i) { return stage_get(row, i); }, P), scale) <
                 1.0e-4f);
    }
    records[6 * 32 + lane] = make_float4(front.x, front.y, front.z, scale);
    records[7 * 32 + lane] =
        make_float4(__fmul_rn(__fmul_rn(0.5f, raw_width < 0.0f ? 0.0f : raw_width), p.radius_scale), 0.0f, 0.0f, 0.0f);
    if (!keep && g.point_counts != nullptr) { g.point_counts[word] = 0u; }
}

// Store step with the Classic application of records 6 and 7
// (walk_classic_strand), eight lanes per strand as in walk_store8.  Every
// lane of the warp calls it.
__device__ __forceinline__ void walk_store8_classic(const LaunchArgs &g, const float4 *records, const float *stage,
                                                    const uint32_t *locals, const float *rvals, int lane,
                                                    int in_batch, int P) {
    constexpr int kPerLane = kWalkMaxCvs / 8;
    const int c = lane & 7;
    const int cpl = (P + 7) >> 3;
    float rv[kPerLane];
#pragma unroll
    for (int m = 0; m < kPerLane; ++m) { rv[m] = rvals[min(c + 8 * m, P - 1)]; }
    for (int first = 0; first < in_batch; first += 4) {
        const int s = first + (lane >> 3);  // at most 31
        const uint32_t word = s < in_batch ? locals[s] : 0x80000000u;
        const float *row = stage + s * kWalkRowFloats;
        const float4 front = records[6 * 32 + s];
        const float width = records[7 * 32 + s].x;
#pragma unroll
        for (int m = 0; m < kPerLane; ++m) {
            const int cm = c + 8 * m;
            if (m < cpl && cm < P) {
                F3 q = stage_get(row, cm);
                if (g.classic_length) { q = xadd(xyz(front), xmul(xsub(q, xyz(front)), front.w)); }
                walk_emit(g, word, P, cm, make_float4(q.x, q.y, q.z, g.classic_width ? width : rv[m]));
            }
        }
    }
}

} // namespace dev
} // namespace nxg
