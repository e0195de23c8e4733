// walk.cuh -- the lane-walk generator for strands of 2..32 CVs.
//
// A warp takes 32 strands of the strand order at a time, in four steps:
//
//   setup  (lane = strand)  root sample, the eight stencil slots and the
//                           blend mode, folded into one weighted-sum record;
//   base   (lane = CV)      the base curve from the guide-offset table, read
//                           as coalesced rows (consecutive lanes on
//                           consecutive CVs of one guide), into a stage in
//                           shared memory, one 33-float4 row per strand;
//   frame  (lane = strand)  with noise: the arc-length prefix, the strand's
//                           noise lattice, then the reference's cursor walk
//                           (generate.h:445-502) over the staged row -- the
//                           transported normal is a serial recurrence, so a
//                           lane carries it CV by CV with the reference's
//                           rotation applied as a vector update, and no
//                           matrix products or cross-lane scans are needed;
//   store  (lane = CV)      the strand's float4s as coalesced streaming
//                           stores, with the Classic application when
//                           per-root scalars are given.
//
// Stage rows are 33 float4 apart, so a warp reading column c of 32 rows
// (frame step) and a warp reading one row (base/store steps) are both free of
// shared-memory bank conflicts.
#pragma once

#include "generator_core.cuh"

namespace nxg {
namespace dev {

constexpr int kWalkMaxCvs = 32;
constexpr int kWalkStride = kWalkMaxCvs + 1;   // float4 per staged strand row
constexpr int kWalkAxisColumns = 12;           // noise lattice columns per axis and strand
constexpr int kWalkRecords = 6;                // float4 setup records per strand

// Shared-memory bytes per warp: stage | records (aliased by the lattice once
// the base step has read them) | output words.
constexpr size_t kWalkStageBytes = sizeof(float4) * 32u * kWalkStride;
constexpr size_t kWalkRecordBytes = sizeof(float4) * kWalkRecords * 32u;
constexpr size_t kWalkLatticeBytes = sizeof(float2) * 3u * kWalkAxisColumns * 32u;
constexpr size_t kWalkLocalBytes = sizeof(uint32_t) * 32u;
__host__ __device__ constexpr size_t walk_warp_bytes(bool noise) {
    return kWalkStageBytes + (noise && kWalkLatticeBytes > kWalkRecordBytes ? kWalkLatticeBytes : kWalkRecordBytes) +
           kWalkLocalBytes;
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
// Nearest mode becomes one slot of weight 1 and normal mode zero slots, so
// the base step evaluates every strand as
//   base = root + (inv * sum_j w_j offsets[row_j + c] + normal' * t_c) * length_scale.
struct WalkRoot {
    F3 position, normal, surface_u, domain;
};

// Also writes the strand's root UV and point count, and stages its twelve
// RootSample words at root_words[lane * 12] for walk_store_roots.
template <bool NOISE>
__device__ __forceinline__ WalkRoot walk_setup(const LaunchArgs &g, float4 *records, uint32_t *locals,
                                               uint32_t *root_words, int lane, uint32_t pick, bool valid,
                                               uint32_t P) {
    const AssetArgs &a = g.a;
    const FrameArgs &f = g.f;
    const ParamArgs &p = g.p;
    uint32_t local = __ldg(g.order + pick);
    if (local >= g.count) {
        local = 0u;
        valid = false;
    }
    const Root root = sample_root(a, f, p.seed, g.first_strand + local);
    if (g.roots) {
#pragma unroll
        for (int w = 0; w < 12; ++w) { root_words[lane * 12 + w] = root_word(root, w); }
    }
    if (valid) {  // generate.h:621-623
        if (g.root_uvs) { g.root_uvs[local] = make_float2(root.u, root.v); }
        if (g.point_counts) { g.point_counts[local] = P; }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) { records[q * 32 + lane] = make_float4(0.0f, 0.0f, 0.0f, 0.0f); }
    float *slot_words = reinterpret_cast<float *>(records);
    float wsum = 0.0f;
    float nearest_d2 = FLT_MAX;
    uint32_t nearest = kInvalid;
    uint32_t blended = 0u;
#pragma unroll 1
    for (uint32_t j = 0; j < kSlots; ++j) {
        const Slot s = eval_slot(a, f, p, root, j);
        if ((s.flags & kSlotEligible) && s.d2 < nearest_d2) {  // strict first minimum (generate.h:234)
            nearest_d2 = s.d2;
            nearest = s.guide;
        }
        if (s.flags & kSlotBlended) {
            float *dst = slot_words + ((blended >> 1) * 32u + lane) * 4u + (blended & 1u) * 2u;
            dst[0] = __uint_as_float(s.guide * P);
            dst[1] = s.w;
            ++blended;
            wsum = __fadd_rn(wsum, s.w);
        }
    }
    float inv = 0.0f;
    F3 normal_term = {0.0f, 0.0f, 0.0f};
    uint32_t nb = blended;
    if (wsum > 1.0e-12f) {
        inv = 1.0f / wsum;
    } else if (nearest != kInvalid) {
        records[lane] = make_float4(__uint_as_float(nearest * P), 1.0f, 0.0f, 0.0f);
        nb = 1u;
        inv = 1.0f;
    } else {
        nb = 0u;
        normal_term = root.normal;
    }
    records[4 * 32 + lane] = make_float4(root.position.x, root.position.y, root.position.z, inv);
    records[5 * 32 + lane] = make_float4(normal_term.x, normal_term.y, normal_term.z, __uint_as_float(nb));
    locals[lane] = local | (valid ? 0u : 0x80000000u);
    WalkRoot r;
    r.position = root.position;
    r.normal = root.normal;
    r.surface_u = F3{0.0f, 0.0f, 0.0f};
    r.domain = F3{0.0f, 0.0f, 0.0f};
    if constexpr (NOISE) {
        r.surface_u = root_surface_u(a, f, root);
        const float decorrelation = 1.0f - p.noise_correlation;
        const float domain_scale = 100.0f * decorrelation * decorrelation;
        r.domain = (rest_root_position(a, root) + F3{0.419276f, 0.184247f, 0.805721f}) * domain_scale;
    }
    return r;
}

// The staged RootSample words of the batch, twelve consecutive words per
// strand (lanes over words, so a warp store covers whole records).
__device__ __forceinline__ void walk_store_roots(const LaunchArgs &g, const uint32_t *root_words,
                                                 const uint32_t *locals, int lane, int in_batch) {
    for (int i = lane; i < in_batch * 12; i += 32) {
        const int s = i / 12;
        const uint32_t word = locals[s];
        if ((word >> 31) == 0u) { g.roots[static_cast<uint64_t>(word) * 12u + static_cast<uint32_t>(i - s * 12)] = root_words[i]; }
    }
}

// Strand of a flattened (strand, CV) item: floor((item + 0.5) / P), exact for
// item < 32 * 32 (the quotient is at least 0.5 / P from an integer).
__device__ __forceinline__ int walk_strand(int item, float inv_p) {
    return static_cast<int>((static_cast<float>(item) + 0.5f) * inv_p);
}

// Base step: item = s * P + c over the batch, 32 consecutive items per pass.
__device__ __forceinline__ void walk_base(const LaunchArgs &g, const float4 *records, float4 *stage,
                                          const float *tvals, const float *rvals, const float4 *offsets, int lane,
                                          int in_batch, int P, float inv_p) {
    const int items = in_batch * P;
    const float ls = g.p.length_scale;
#pragma unroll 2
    for (int item = lane; item < items; item += 32) {
        const int s = walk_strand(item, inv_p);
        const int c = item - s * P;
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
        const float t = tvals[c];
        const F3 off = acc * head.w + F3{tail.x, tail.y, tail.z} * t;
        const F3 base = F3{head.x, head.y, head.z} + off * ls;
        stage[s * kWalkStride + c] = make_float4(base.x, base.y, base.z, rvals[c]);
    }
}

// noise - 0.5 along one axis from the strand's lattice columns (the
// regrouped blend of lattice_noise).
__device__ __forceinline__ float walk_lattice_delta(const float2 *lat, int axis, int lo, int n, float x) {
    const float fx = floorf(x);
    const float w = x - fx;
    int k = static_cast<int>(fx) - lo;
    k = max(0, min(k, n - 2));
    const float2 c0 = lat[(axis * kWalkAxisColumns + k) * 32];
    const float2 c1 = lat[(axis * kWalkAxisColumns + k + 1) * 32];
    const float s = s_curve(w);
    const float v0 = c0.x * w + c0.y;
    const float v1 = c1.x * (w - 1.0f) + c1.y;
    return 0.5f * (v0 + s * (v1 - v0));
}

// Frame step for the strand whose staged row is `row` (this lane's strand):
// arc lengths into row[c].w, the lattice, then the cursor walk, leaving the
// noisy points (with radii) in the row.
__device__ __forceinline__ void walk_frame(const ParamArgs &p, const WalkRoot &wr, float4 *row, float2 *lat,
                                           const float *tvals, const float *rvals, const float4 *table, int P) {
    // Arc-length prefix of the base curve (generate.h:420-433, :465-468).
    float arc = 0.0f;
    {
        F3 prev = xyz(row[0]);
        reinterpret_cast<float *>(row)[3] = 0.0f;
        for (int c = 1; c < P; ++c) {
            const F3 cur = xyz(row[c]);
            const F3 d = cur - prev;
            arc += sqrtf(dot(d, d));
            reinterpret_cast<float *>(row + c)[3] = arc;
            prev = cur;
        }
    }
    const float original_length = arc;
    const float f_eff = original_length > 0.0f ? fmaxf(0.5f / original_length, p.noise_frequency)
                                               : p.noise_frequency;

    // Lattice columns (A, B) of the three noise axes (see lattice_noise):
    // columns lo .. floor(d0 + span) + 2 cover every CV's X and X + 1 with one
    // column of margin for rounding in the arc-length prefix.
    const F3 dom = wr.domain;
    const float span = original_length * f_eff;
    int lo[3], n[3];
    bool fits = true;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        const float d0 = component(dom, ax);
        lo[ax] = static_cast<int>(floorf(d0));
        n[ax] = static_cast<int>(floorf(d0 + span)) + 3 - lo[ax];
        fits = fits && n[ax] >= 2 && n[ax] <= kWalkAxisColumns;
    }
    if (fits) {
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
                const int X = lo[ax];
                const int cx = ax == 0 ? X : Yb + ob;
                const int cy = ax == 1 ? X : (ax == 0 ? Yb + ob : Zc + oc);
                const int cz = ax == 2 ? X : Zc + oc;
                seed[corner] = static_cast<uint32_t>(cx) * kLcgA2 + static_cast<uint32_t>(cy) * kLcgA +
                               static_cast<uint32_t>(cz) + kLcgK;
                wgt[corner] = (ob ? sb : 1.0f - sb) * (oc ? sc : 1.0f - sc);
                wdb[corner] = wgt[corner] * (wb - static_cast<float>(ob));
                wdc[corner] = wgt[corner] * (wc - static_cast<float>(oc));
            }
            for (int k = 0; k < n[ax]; ++k) {
                float A = 0.0f, B = 0.0f;
#pragma unroll
                for (int corner = 0; corner < 4; ++corner) {
                    const float4 gr = table[temper_index(seed[corner] + static_cast<uint32_t>(k) * step)];
                    A += wgt[corner] * component4(gr, ax);
                    B += component4(gr, ib) * wdb[corner] + component4(gr, ic) * wdc[corner];
                }
                lat[(ax * kWalkAxisColumns + k) * 32] = make_float2(A, B);
            }
        }
    }

    // The cursor walk (generate.h:465-502).  Tangent after CV c: the next
    // segment's direction, carried over zero-length segments and at the tip;
    // the transported normal rotates by rotate_by(axis, acos(cos)) with
    // cos(acos x) = x and sin(acos x) = sqrt(1 - x^2):
    //   M v = cos v + (1 - cos)(axis . v) axis + sin (axis x v).
    const float mscale = p.noise_mask * p.noise_amplitude;
    const bool preserve = p.noise_preserve_length > 0.001f;
    F3 tan = wr.normal;
    F3 v = wr.surface_u;
    float4 cur4 = row[0];
    F3 nxt = xyz(row[1]);
    F3 previous_point = xyz(cur4);
    float noisy = 0.0f;
    for (int c = 0; c < P; ++c) {
        const F3 cur = xyz(cur4);
        F3 ntan = tan;
        if (c + 1 < P) {
            const F3 seg = xsub(nxt, cur);
            if (xdot(seg, seg) > 0.0f) { ntan = normalize(seg); }
        }
        const F3 axis = xcross(tan, ntan);
        if (xdot(axis, axis) > 0.0f) {
            const float cs = fminf(fmaxf(dot(tan, ntan), -1.0f), 1.0f);
            const float sn = sqrtf(fmaf(-cs, cs, 1.0f));
            const float k = (1.0f - cs) * dot(axis, v);
            const F3 axv = cross(axis, v);
            v = normalize(F3{v.x * cs + axis.x * k + axv.x * sn, v.y * cs + axis.y * k + axv.y * sn,
                             v.z * cs + axis.z * k + axv.z * sn});
        }
        const F3 bn = cross(v, ntan);
        const F3 tt = cross(bn, v);
        F3 q = cur;
        if (c > 0) {
            const float distance = cur4.w * f_eff;
            const float magnitude = mscale * tvals[c];
            float gx, gy, gz;
            if (fits) {
                gx = walk_lattice_delta(lat, 0, lo[0], n[0], dom.x + distance);
                gy = walk_lattice_delta(lat, 1, lo[1], n[1], dom.y + distance);
                gz = walk_lattice_delta(lat, 2, lo[2], n[2], dom.z + distance);
            } else {
                gx = gradient_noise(table, dom.x + distance, dom.y, dom.z) - 0.5f;
                gy = gradient_noise(table, dom.x, dom.y + distance, dom.z) - 0.5f;
                gz = gradient_noise(table, dom.x, dom.y, dom.z + distance) - 0.5f;
            }
            q = q + v * (gx * magnitude) + bn * (gy * magnitude) + tt * (gz * magnitude);
        }
        row[c] = make_float4(q.x, q.y, q.z, rvals[c]);
        if (preserve) {
            const F3 d = q - previous_point;
            noisy += c > 0 ? sqrtf(dot(d, d)) : 0.0f;
            previous_point = q;
        }
        tan = ntan;
        if (c + 1 < P) { cur4 = row[c + 1]; }
        if (c + 2 < P) { nxt = xyz(row[c + 2]); }
    }

    // preserveLength (generate.h:553-563) from the noisy points of the walk,
    // scaling the strand about its root.
    if (preserve && noisy > 0.0f) {
        const float target = original_length * p.noise_preserve_length + noisy * (1.0f - p.noise_preserve_length);
        if (fabsf(noisy - target) >= 0.0001f) {
            const float scale = target / noisy;
            const F3 root = wr.position;
            for (int c = 0; c < P; ++c) {
                const F3 q = root + (xyz(row[c]) - root) * scale;
                row[c].x = q.x;
                row[c].y = q.y;
                row[c].z = q.z;
            }
        }
    }
}

// Store step: item = s * P + c; the Classic application (scale about the
// first point, width override, drop rule) as in emit_strand.
template <bool CLASSIC>
__device__ __forceinline__ void walk_store(const LaunchArgs &g, const float4 *stage, const uint32_t *locals, int lane,
                                           int in_batch, int P, float inv_p) {
    const ParamArgs &p = g.p;
    const int items = in_batch * P;
    for (int item = lane; item < items; item += 32) {
        const int s = walk_strand(item, inv_p);
        const int c = item - s * P;
        const uint32_t word = locals[s];
        if (word >> 31) { continue; }
        const float4 *row = stage + s * kWalkStride;
        float4 q = row[c];
        if constexpr (CLASSIC) {
            const float2 sc = __ldg(g.scalars + word);
            const F3 front = xyz(row[0]);
            const F3 back = xyz(row[P - 1]);
            const float scale = g.classic_length ? sc.x : 1.0f;
            const float raw_width = g.classic_width ? sc.y
                : (p.radius_scale > 0.0f ? __fdiv_rn(__fmul_rn(2.0f, strand_radius(p, 0.0f)), p.radius_scale) : 0.0f);
            bool keep = !(raw_width < 1.0e-4f);
            const F3 chord = back - front;
            if (keep && !(sqrtf(dot(chord, chord)) * scale > 1.01e-4f)) {
                keep = !(__fmul_rn(classic_spline_length(row, P), scale) < 1.0e-4f);
            }
            if (g.classic_length) {
                const F3 v = xadd(front, xmul(xsub(xyz(q), front), scale));
                q.x = v.x;
                q.y = v.y;
                q.z = v.z;
            }
            if (g.classic_width) {
                q.w = __fmul_rn(__fmul_rn(0.5f, raw_width < 0.0f ? 0.0f : raw_width), p.radius_scale);
            }
            if (!keep && c == 0 && g.point_counts != nullptr) { g.point_counts[word] = 0u; }
        }
        const uint64_t index = static_cast<uint64_t>(word) * static_cast<uint32_t>(P) + static_cast<uint32_t>(c);
        if (g.vec3_points) {
            // Vec3 positions, 3P consecutive floats per strand (device_contract.h:47-52)
            float *out3 = g.vec3_points + 3u * index;
            __stcs(out3, q.x);
            __stcs(out3 + 1, q.y);
            __stcs(out3 + 2, q.z);
        } else {
            __stcs(g.points + index, q);
        }
    }
}

} // namespace dev
} // namespace nxg
