// generator_core.cuh -- the two phases of the warp-parallel strand
// generator, shared by the single-description kernels (generate.cu) and the
// batched multi-description kernel (batched.cu).
//
// Phase A (setup_strand): one lane per strand sets up 32 strands of a warp --
// alias root sample, the eight stencil slots, the blend mode and the noise
// frame inputs -- into per-strand records in shared memory.
// Phase B (emit_strand): a group of L lanes per strand, each lane owning PPT
// consecutive CVs, evaluates the base curve from the guide-offset table, the
// transported frame and the gradient noise, and writes the strand.
#pragma once

#include "nxg_internal.h"
#include "nxg_classic.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

namespace nxg {
namespace dev {
struct LaunchArgs {
    AssetArgs a;
    FrameArgs f;
    ParamArgs p;
    uint32_t first_strand;   // global id of output record 0
    uint32_t count;          // strands in this launch
    uint32_t range_begin;    // lane-walk kernels: positions [range_begin, range_end) of the order
    uint32_t range_end;
    float4 *points;
    float *vec3_points;      // when set: sample-major Vec3 output instead of float4 (motion contract)
    uint32_t *roots;         // 12 words per strand, or nullptr
    float2 *root_uvs;
    uint32_t *point_counts;
    const uint32_t *order;   // permutation of [0, count), or nullptr for identity
    const float4 *guide_frames;  // 2 per guide (guide_frame_entry), or nullptr
    uint32_t zero_row;           // offset-table index of kWalkMaxCvs zero entries (unused lane-walk slots)
    const float2 *scalars;   // Classic per-root (length scale, width), or nullptr
    uint32_t classic_length; // scale each strand about its first point by scalars.x
    uint32_t classic_width;  // radius = 0.5 * max(scalars.y, 0) * radius_scale
};

constexpr int kTableFloat4 = NXG_NOISE_GRADIENT_COUNT;  // float4 entries of the staged table

__device__ __forceinline__ uint32_t root_word(const Root &r, int w) {
    switch (w) {
        case 0: return __float_as_uint(r.position.x);
        case 1: return __float_as_uint(r.position.y);
        case 2: return __float_as_uint(r.position.z);
        case 3: return __float_as_uint(r.normal.x);
        case 4: return __float_as_uint(r.normal.y);
        case 5: return __float_as_uint(r.normal.z);
        case 6: return __float_as_uint(r.u);
        case 7: return __float_as_uint(r.v);
        case 8: return r.triangle;
        case 9: return __float_as_uint(r.b1);
        case 10: return __float_as_uint(r.b2);
        default: return r.triangle;  // surface_face_id == triangle_index (generate.h:134)
    }
}

__device__ __forceinline__ float strand_radius(const ParamArgs &p, float t) {
    const float width = p.root_width * (1.0f - t) + p.tip_width * t;  // generate.h:577-581
    return 0.5f * width * p.radius_scale;
}

// ---------------------------------------------------------------------------
// Per-strand records a warp stages in shared memory between its two phases
// (one column per strand of the warp's 32-strand batch).
// ---------------------------------------------------------------------------
enum RecordField : int {
    kRecPx = 0, kRecPy, kRecPz,        // root position
    kRecNx, kRecNy, kRecNz,            // root normal
    kRecMode,                          // blended-slot count | mode << 8
    kRecInvW,                          // 1 / weight_sum (mode 0)
    kRecGuide0,                        // 8 blended guides, in slot order
    kRecWeight0 = kRecGuide0 + 8,      // their weights
    kRecNearest = kRecWeight0 + 8,     // nearest eligible guide (mode 1)
    kRecSUx, kRecSUy, kRecSUz,         // surface_u (noise)
    kRecDx, kRecDy, kRecDz,            // noise domain (noise)
    kRecLocal,                         // output record | invalid << 31
    kRecFields
};
enum : uint32_t { kModeBlend = 0u, kModeNearest = 1u, kModeNormal = 2u };

struct Records {
    uint32_t *base;  // kRecFields x 32 words
    __device__ __forceinline__ uint32_t &u(int field, int strand) const { return base[field * 32 + strand]; }
    __device__ __forceinline__ float f(int field, int strand) const { return __uint_as_float(base[field * 32 + strand]); }
    __device__ __forceinline__ void setf(int field, int strand, float v) const { base[field * 32 + strand] = __float_as_uint(v); }
    __device__ __forceinline__ F3 f3(int field, int strand) const { return {f(field, strand), f(field + 1, strand), f(field + 2, strand)}; }
};

// Phase A: lane i sets up strand i of the batch -- root sample, the eight
// stencil slots, the blend mode and (with noise) the surface frame inputs.
template <bool NOISE>
__device__ __forceinline__ void setup_strand(const LaunchArgs &g, const Records &rec, int lane, uint32_t pick,
                                             bool valid) {
    const AssetArgs &a = g.a;
    const FrameArgs &f = g.f;
    const ParamArgs &p = g.p;
    uint32_t local = __ldg(g.order + pick);
    if (local >= g.count) {
        local = 0u;
        valid = false;
    }
    const Root root = sample_root(a, f, p.seed, g.first_strand + local);
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
            rec.u(kRecGuide0 + blended, lane) = s.guide;
            rec.setf(kRecWeight0 + blended, lane, s.w);
            ++blended;
            wsum = __fadd_rn(wsum, s.w);
        }
    }
    const uint32_t mode = wsum > 1.0e-12f ? kModeBlend : (nearest != kInvalid ? kModeNearest : kModeNormal);
    rec.u(kRecMode, lane) = blended | (mode << 8);
    rec.setf(kRecInvW, lane, mode == kModeBlend ? 1.0f / wsum : 0.0f);
    rec.u(kRecNearest, lane) = nearest;
    rec.setf(kRecPx, lane, root.position.x);
    rec.setf(kRecPy, lane, root.position.y);
    rec.setf(kRecPz, lane, root.position.z);
    rec.setf(kRecNx, lane, root.normal.x);
    rec.setf(kRecNy, lane, root.normal.y);
    rec.setf(kRecNz, lane, root.normal.z);
    rec.u(kRecLocal, lane) = local | (valid ? 0u : 0x80000000u);
    if constexpr (NOISE) {
        const F3 su = root_surface_u(a, f, root);
        const float decorrelation = 1.0f - p.noise_correlation;
        const float domain_scale = 100.0f * decorrelation * decorrelation;
        const F3 dom = (rest_root_position(a, root) + F3{0.419276f, 0.184247f, 0.805721f}) * domain_scale;
        rec.setf(kRecSUx, lane, su.x);
        rec.setf(kRecSUy, lane, su.y);
        rec.setf(kRecSUz, lane, su.z);
        rec.setf(kRecDx, lane, dom.x);
        rec.setf(kRecDy, lane, dom.y);
        rec.setf(kRecDz, lane, dom.z);
    }
}

// generate.h:404-418 rotate_by for angle = acos(c), with cos(angle) = c and
// sin(angle) = sqrt(1 - c^2) evaluated as sqrt(fma(-c, c, 1)) (one rounding,
// accurate near |c| = 1).
__device__ __forceinline__ M3 rotation_cs(F3 axis, float c, float s) {
    const float omc = 1.0f - c;
    M3 r;
    r.m[0] = axis.x * axis.x * omc + c;
    r.m[1] = axis.x * axis.y * omc - axis.z * s;
    r.m[2] = axis.x * axis.z * omc + axis.y * s;
    r.m[3] = axis.x * axis.y * omc + axis.z * s;
    r.m[4] = axis.y * axis.y * omc + c;
    r.m[5] = axis.y * axis.z * omc - axis.x * s;
    r.m[6] = axis.x * axis.z * omc - axis.y * s;
    r.m[7] = axis.y * axis.z * omc + axis.x * s;
    r.m[8] = axis.z * axis.z * omc + c;
    return r;
}

__device__ __forceinline__ float component(F3 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }
__device__ __forceinline__ float component4(float4 v, int axis) { return axis == 0 ? v.x : (axis == 1 ? v.y : v.z); }

// Gradient noise along one axis of a strand (generate.h:370-402 evaluated at
// domain + distance * e_axis).  Only the `axis` coordinate moves along the
// strand, so the fade weights of the two fixed axes are constants and the
// eight-corner trilinear blend folds, per lattice column X of the moving
// axis, into A(X) = sum_corners w_b w_c g_axis and
// B(X) = sum_corners w_b w_c (g_b (f_b - o_b) + g_c (f_c - o_c)):
//   noise = 0.5 * ((1 - s(f)) (A(X) f + B(X)) + s(f) (A(X+1) (f - 1) + B(X+1))) + 0.5
// with X = floor(x), f = x - X.  The columns of a strand are filled once;
// each CV then needs two table entries instead of eight hashed corners.
struct Lattice {
    float2 *col[3];   // per axis: (A, B) for X = lo[axis] + k
    int lo[3];
    int n[3];
};

__device__ __forceinline__ float lattice_noise(const Lattice &lat, int axis, float x) {
    const float fx = floorf(x);
    const float w = x - fx;
    int k = static_cast<int>(fx) - lat.lo[axis];
    k = max(0, min(k, lat.n[axis] - 2));
    const float2 c0 = lat.col[axis][k];
    const float2 c1 = lat.col[axis][k + 1];
    const float s = s_curve(w);
    const float v0 = c0.x * w + c0.y;
    const float v1 = c1.x * (w - 1.0f) + c1.y;
    return 0.5f * ((1.0f - s) * v0 + s * v1) + 0.5f;
}

// Fill column k of `axis`: the four corners (o_b, o_c) of lattice column X.
__device__ __forceinline__ float2 lattice_column(const float4 *table, int axis, int X, F3 dom) {
    const int ib = axis == 0 ? 1 : 0;           // the fixed axes, ascending
    const int ic = axis == 2 ? 1 : 2;
    const float db = component(dom, ib), dc = component(dom, ic);
    const float fb = floorf(db), fc = floorf(dc);
    const float wb = db - fb, wc = dc - fc;
    const float sb = s_curve(wb), sc = s_curve(wc);
    const int Yb = static_cast<int>(fb), Zc = static_cast<int>(fc);
    float A = 0.0f, B = 0.0f;
#pragma unroll
    for (int corner = 0; corner < 4; ++corner) {
        const int ob = corner & 1, oc = corner >> 1;
        const int cx = axis == 0 ? X : Yb + ob;
        const int cy = axis == 1 ? X : (axis == 0 ? Yb + ob : Zc + oc);
        const int cz = axis == 2 ? X : Zc + oc;
        const uint32_t seed = static_cast<uint32_t>(cx) * kLcgA2 + static_cast<uint32_t>(cy) * kLcgA +
                              static_cast<uint32_t>(cz) + kLcgK;
        const float4 gr = table[temper_index(seed)];
        const float wgt = (ob ? sb : 1.0f - sb) * (oc ? sc : 1.0f - sc);
        A += wgt * component4(gr, axis);
        B += wgt * (component4(gr, ib) * (wb - static_cast<float>(ob)) + component4(gr, ic) * (wc - static_cast<float>(oc)));
    }
    return make_float2(A, B);
}

// ---------------------------------------------------------------------------
// Classic cLength (xgen_classic_runtime.cpp:591-662): the uniform cubic
// B-spline through the CVs, with mirrored phantom end CVs, sampled at
// 2P + 4 intervals whose first and last samples are the raw end CVs.  Every
// operation is rounded as the reference's, so a strand's measured length
// matches the CPU runtime's for the same points.
// ---------------------------------------------------------------------------
__device__ __forceinline__ F3 xyz(float4 v) { return {v.x, v.y, v.z}; }

// pt(i) returns CV i of the strand.
template <class Pts>
__device__ inline F3 classic_curve_eval_by(Pts pt, int P, float t) {
    if (t < 1.0e-7f) { return pt(0); }
    if (t > 1.0f - 1.0e-7f) { return pt(P - 1); }
    const float scaled = __fmul_rn(t, static_cast<float>(P - 1));
    const int span = static_cast<int>(static_cast<uint32_t>(scaled));
    const float f = __fsub_rn(scaled, static_cast<float>(span));
    const float f2 = __fmul_rn(f, f);
    const float f3 = __fmul_rn(f2, f);
    const float omf = __fsub_rn(1.0f, f);
    const float b0 = __fmul_rn(__fmul_rn(omf, omf), omf);
    const float b1 = __fadd_rn(__fsub_rn(__fmul_rn(3.0f, f3), __fmul_rn(6.0f, f2)), 4.0f);
    const float b2 =
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(-3.0f, f3), __fmul_rn(3.0f, f2)), __fmul_rn(3.0f, f)), 1.0f);
    const F3 p0 = span == 0 ? xsub(xmul(pt(0), 2.0f), pt(1)) : pt(span - 1);
    const F3 p1 = pt(span);
    const F3 p2 = pt(span + 1);
    const F3 p3 = span + 2 == P ? xsub(xmul(pt(P - 1), 2.0f), pt(P - 2)) : pt(span + 2);
    return xmul(xadd(xadd(xadd(xmul(p0, b0), xmul(p1, b1)), xmul(p2, b2)), xmul(p3, f3)), 1.0f / 6.0f);
}

template <class Pts>
__device__ inline float classic_spline_length_by(Pts pt, int P) {
    const int intervals = 2 * P + 4;
    const float step = __fdiv_rn(1.0f, static_cast<float>(intervals));
    F3 previous = pt(0);
    float length = 0.0f;
    for (int k = 1; k < intervals; ++k) {
        const F3 current = classic_curve_eval_by(pt, P, __fmul_rn(step, static_cast<float>(k)));
        const F3 d = xsub(current, previous);
        length = __fadd_rn(length, __fsqrt_rn(xdot(d, d)));
        previous = current;
    }
    const F3 d = xsub(pt(P - 1), previous);
    return __fadd_rn(length, __fsqrt_rn(xdot(d, d)));
}

__device__ inline float classic_spline_length(const float4 *pts, int P) {
    return classic_spline_length_by([pts](int i) { return xyz(pts[i]); }, P);
}

// Phase B: strand b of the batch on an L-lane group; lane gl owns the
// consecutive CVs gl*PPT .. gl*PPT+PPT-1.
template <int L, int PPT, bool NOISE, bool CLASSIC = false>
__device__ __forceinline__ void emit_strand(const LaunchArgs &g, const Records &rec, int b, int gl,
                                            const float4 *table, const float4 *offsets, const float *tvals,
                                            float4 *stage, float2 *lattice_area, int lattice_max) {
    const ParamArgs &p = g.p;
    const int P = static_cast<int>(p.cvs_per_strand);
    const uint32_t local_word = rec.u(kRecLocal, b);
    const bool active = (local_word >> 31) == 0u;
    const uint32_t local = local_word & 0x7fffffffu;
    const F3 root = rec.f3(kRecPx, b);
    const F3 rnormal = rec.f3(kRecNx, b);
    const uint32_t mode_word = rec.u(kRecMode, b);
    const uint32_t nb = mode_word & 0xffu;
    const uint32_t mode = mode_word >> 8;
    const int cv0 = gl * PPT;

    // Base curve (generate.h:246-267, :300-310) from the guide-offset table:
    // offsets[g*P + cv] = sample_guide(g, cv/(P-1)) - guide_root(g).
    float tcv[PPT];
    F3 base[PPT];
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        tcv[j] = tvals[min(cv0 + j, P - 1)];
        base[j] = F3{0.0f, 0.0f, 0.0f};
    }
    if (mode == kModeBlend) {
#pragma unroll
        for (uint32_t k = 0; k < kSlots; ++k) {
            if (k < nb) {
                const float4 *row = offsets + static_cast<uint64_t>(rec.u(kRecGuide0 + k, b)) * P;
                const float w = rec.f(kRecWeight0 + k, b);
#pragma unroll
                for (int j = 0; j < PPT; ++j) {
                    const float4 d = __ldg(row + min(cv0 + j, P - 1));
                    base[j] = base[j] + F3{d.x, d.y, d.z} * w;
                }
            }
        }
        const float inv = rec.f(kRecInvW, b);
#pragma unroll
        for (int j = 0; j < PPT; ++j) { base[j] = base[j] * inv; }
    } else if (mode == kModeNearest) {
        const float4 *row = offsets + static_cast<uint64_t>(rec.u(kRecNearest, b)) * P;
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            const float4 d = __ldg(row + min(cv0 + j, P - 1));
            base[j] = F3{d.x, d.y, d.z};
        }
    } else {
#pragma unroll
        for (int j = 0; j < PPT; ++j) { base[j] = rnormal * tcv[j]; }
    }
#pragma unroll
    for (int j = 0; j < PPT; ++j) { base[j] = root + base[j] * p.length_scale; }

    F3 point[PPT];
    if constexpr (!NOISE) {
#pragma unroll
        for (int j = 0; j < PPT; ++j) { point[j] = base[j]; }
    } else {
        const F3 surface_u = rec.f3(kRecSUx, b);
        const F3 domain = rec.f3(kRecDx, b);
        const F3 prev_lane_base = group_shfl_up<L>(base[PPT - 1], 1);
        const F3 next_lane_base = group_shfl_down<L>(base[0], 1);

        // Arc length: prefix of segment lengths (generate.h:420-433, :465-468).
        float arc[PPT];
        float run = 0.0f;
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            const int cv = cv0 + j;
            const F3 prev = j > 0 ? base[j > 0 ? j - 1 : 0] : prev_lane_base;
            const F3 d = base[j] - prev;
            run += (cv >= 1 && cv < P) ? sqrtf(dot(d, d)) : 0.0f;
            arc[j] = run;
        }
        const float lane_incl = group_scan_add<L>(run, gl);
        const float lane_excl = __shfl_up_sync(kFull, lane_incl, 1, L);
        const float offset_arc = gl > 0 ? lane_excl : 0.0f;
#pragma unroll
        for (int j = 0; j < PPT; ++j) { arc[j] += offset_arc; }
        const float original_length = __shfl_sync(kFull, lane_incl, L - 1, L);
        const float f_eff = original_length > 0.0f ? fmaxf(0.5f / original_length, p.noise_frequency)
                                                   : p.noise_frequency;

        // Tangent after CV k: the next segment's direction, carried forward over
        // zero-length segments and at the tip (generate.h:470-474).
        F3 cand[PPT];
        bool valid[PPT];
        int lane_last = -1;
        F3 lane_last_cand = {0.0f, 0.0f, 0.0f};
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            const int cv = cv0 + j;
            const F3 next = j + 1 < PPT ? base[j + 1 < PPT ? j + 1 : j] : next_lane_base;
            const F3 e = xsub(next, base[j]);
            valid[j] = (cv + 1 < P) && xdot(e, e) > 0.0f;
            cand[j] = valid[j] ? xnormalize(e) : F3{0.0f, 0.0f, 0.0f};
            if (valid[j]) {
                lane_last = cv;
                lane_last_cand = cand[j];
            }
        }
        const int incl_last = group_scan_max<L>(lane_last, gl);
        const int up_last = __shfl_up_sync(kFull, incl_last, 1, L);  // every lane shuffles
        const int excl_last = gl > 0 ? up_last : -1;
        const F3 from_lanes = group_shfl<L>(lane_last_cand, max(excl_last, 0) / PPT);
        F3 carry_t = excl_last >= 0 ? from_lanes : rnormal;
        F3 tan[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            if (valid[j]) { carry_t = cand[j]; }
            tan[j] = carry_t;
        }

        // Transported normal N_k = normalize(M_k ... M_0 surface_u) with M_k the
        // reference's rotate_by matrix (generate.h:475-481): a lane multiplies
        // its own matrices, an exclusive scan across lanes supplies the product
        // of all earlier CVs, and the lane then walks its CVs.
        M3 mats[PPT];
        M3 lane_prod = identity3();
        const F3 prev_lane_tan = group_shfl_up<L>(tan[PPT - 1], 1);
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            const int cv = cv0 + j;
            const F3 tp = j > 0 ? tan[j > 0 ? j - 1 : 0] : (gl > 0 ? prev_lane_tan : rnormal);
            const F3 axis = xcross(tp, tan[j]);
            mats[j] = identity3();
            if (cv < P && xdot(axis, axis) > 0.0f) {
                const float cs = fminf(fmaxf(dot(tp, tan[j]), -1.0f), 1.0f);
                mats[j] = rotation_cs(axis, cs, sqrtf(fmaf(-cs, cs, 1.0f)));
            }
            lane_prod = j == 0 ? mats[0] : mul3(mats[j], lane_prod);
        }
        const M3 incl_prod = group_scan_mat<L>(lane_prod, gl);
        M3 earlier;
#pragma unroll
        for (int i = 0; i < 9; ++i) { earlier.m[i] = __shfl_up_sync(kFull, incl_prod.m[i], 1, L); }
        F3 v = gl > 0 ? apply3(earlier, surface_u) : surface_u;
        F3 normal[PPT];
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            v = normalize(apply3(mats[j], v));
            normal[j] = v;
        }

        // Lattice columns of the three noise axes for this strand.
        Lattice lat;
        const float span = original_length * f_eff;
        bool fits = true;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            const float d0 = component(domain, ax);
            lat.lo[ax] = static_cast<int>(floorf(d0));
            // columns lo .. floor(d0 + span) + 2: every CV's X and X + 1, with one
            // column of margin for rounding in the arc-length prefix
            lat.n[ax] = static_cast<int>(floorf(d0 + span)) + 3 - lat.lo[ax];
            fits = fits && lat.n[ax] >= 2 && lat.n[ax] <= lattice_max;
            lat.col[ax] = lattice_area + ax * lattice_max;
        }
        const int total = fits ? lat.n[0] + lat.n[1] + lat.n[2] : 0;
        int rounds = (total + L - 1) / L;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) { rounds = max(rounds, __shfl_xor_sync(kFull, rounds, d)); }
        rounds = min(rounds, (3 * lattice_max + L - 1) / L);  // a group never has more columns
        for (int r = 0; r < rounds; ++r) {
            const int item = r * L + gl;
            if (item < total) {
                const int ax = item < lat.n[0] ? 0 : (item < lat.n[0] + lat.n[1] ? 1 : 2);
                const int k = item - (ax > 0 ? lat.n[0] : 0) - (ax > 1 ? lat.n[1] : 0);
                lat.col[ax][k] = lattice_column(table, ax, lat.lo[ax] + k, domain);
            }
        }
        __syncwarp();

        // Displacement in the transported frame (generate.h:482-502).
        const float magnitude_scale = p.noise_mask * p.noise_amplitude;
#pragma unroll
        for (int j = 0; j < PPT; ++j) {
            const int cv = cv0 + j;
            F3 q = base[j];
            if (cv > 0 && cv < P) {
                const F3 n = normal[j];
                const F3 bn = cross(n, tan[j]);
                const F3 t = cross(bn, n);
                const float distance = arc[j] * f_eff;
                const float magnitude = magnitude_scale * tcv[j];
                float gx, gy, gz;
                if (fits) {
                    gx = lattice_noise(lat, 0, domain.x + distance);
                    gy = lattice_noise(lat, 1, domain.y + distance);
                    gz = lattice_noise(lat, 2, domain.z + distance);
                } else {
                    gx = gradient_noise(table, domain.x + distance, domain.y, domain.z);
                    gy = gradient_noise(table, domain.x, domain.y + distance, domain.z);
                    gz = gradient_noise(table, domain.x, domain.y, domain.z + distance);
                }
                q = q + n * ((gx - 0.5f) * magnitude) + bn * ((gy - 0.5f) * magnitude) + t * ((gz - 0.5f) * magnitude);
            }
            point[j] = q;
        }

        // preserveLength (generate.h:553-563), from the noisy points already in
        // registers instead of a second cursor pass.
        if (p.noise_preserve_length > 0.001f) {
            const F3 prev_lane_point = group_shfl_up<L>(point[PPT - 1], 1);
            float partial = 0.0f;
#pragma unroll
            for (int j = 0; j < PPT; ++j) {
                const int cv = cv0 + j;
                const F3 prev = j > 0 ? point[j > 0 ? j - 1 : 0] : prev_lane_point;
                const F3 d = point[j] - prev;
                partial += (cv >= 1 && cv < P) ? sqrtf(dot(d, d)) : 0.0f;
            }
            const float noisy = group_sum<L>(partial);
            float scale = 1.0f;
            if (noisy > 0.0f) {
                const float target = original_length * p.noise_preserve_length +
                                     noisy * (1.0f - p.noise_preserve_length);
                if (fabsf(noisy - target) >= 0.0001f) { scale = target / noisy; }
            }
            if (scale != 1.0f) {
#pragma unroll
                for (int j = 0; j < PPT; ++j) { point[j] = root + (point[j] - root) * scale; }
            }
        }
    }

    // Classic length and width (xgen_classic_runtime.cpp:1650-1678,
    // :1827-1858) from the strand's per-root scalars: scale about the first
    // point, override the radius, and drop (point count 0) a strand whose
    // scaled cLength or width is below 1e-4.
    bool width_override = false;
    float override_radius = 0.0f;
    if constexpr (CLASSIC) {
        const float2 sc = __ldg(g.scalars + local);
        const F3 front = group_shfl<L>(point[0], 0);
        F3 last = point[0];
#pragma unroll
        for (int j = 1; j < PPT; ++j) {
            if (cv0 + j == P - 1) { last = point[j]; }
        }
        const F3 back = group_shfl<L>(last, (P - 1) / PPT);
        const float s = g.classic_length ? sc.x : 1.0f;
        const float raw_width = g.classic_width ? sc.y
            : (p.radius_scale > 0.0f ? __fdiv_rn(__fmul_rn(2.0f, strand_radius(p, 0.0f)), p.radius_scale) : 0.0f);
        bool keep = !(raw_width < 1.0e-4f);
        // cLength is at least the root-tip chord, so only strands near the
        // threshold measure the sampled spline (group-uniform branch).
        const F3 chord = back - front;
        if (keep && !(sqrtf(dot(chord, chord)) * s > 1.01e-4f)) {
            const int lane = static_cast<int>(threadIdx.x & 31u);
            const unsigned group_mask = L == 32 ? kFull : (((1u << L) - 1u) << (lane - gl));
#pragma unroll
            for (int j = 0; j < PPT; ++j) {
                if (cv0 + j < P) { stage[cv0 + j] = make_float4(point[j].x, point[j].y, point[j].z, 0.0f); }
            }
            __syncwarp(group_mask);
            float c_length = gl == 0 ? classic_spline_length(stage, P) : 0.0f;
            c_length = __shfl_sync(group_mask, c_length, 0, L);
            __syncwarp(group_mask);
            keep = !(__fmul_rn(c_length, s) < 1.0e-4f);
        }
        if (g.classic_length) {
#pragma unroll
            for (int j = 0; j < PPT; ++j) { point[j] = xadd(front, xmul(xsub(point[j], front), s)); }
        }
        if (g.classic_width) {
            width_override = true;
            override_radius = __fmul_rn(__fmul_rn(0.5f, raw_width < 0.0f ? 0.0f : raw_width), p.radius_scale);
        }
        if (!keep && active && gl == 0 && g.point_counts != nullptr) { g.point_counts[local] = 0u; }
    }

    // Stage the strand's float4s in shared memory, then write them with
    // consecutive lanes on consecutive CVs (coalesced streaming stores).
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
        const int cv = cv0 + j;
        if (cv < P) {
            stage[cv] = make_float4(point[j].x, point[j].y, point[j].z,
                                    width_override ? override_radius : strand_radius(p, tcv[j]));
        }
    }
    __syncwarp();
    if (active) {
        if (g.vec3_points) {
            // Vec3 positions, 3P consecutive floats per strand (device_contract.h:47-52)
            float *out3 = g.vec3_points + static_cast<uint64_t>(local) * static_cast<uint32_t>(3 * P);
            const float *st = reinterpret_cast<const float *>(stage);
            for (int i = gl; i < 3 * P; i += L) {
                const int cv = i / 3;
                __stcs(out3 + i, st[4 * cv + (i - 3 * cv)]);
            }
        } else {
            float4 *out = g.points + static_cast<uint64_t>(local) * static_cast<uint32_t>(P);
            for (int cv = gl; cv < P; cv += L) { __stcs(out + cv, stage[cv]); }
        }
    }
    __syncwarp();
}

// offsets[g*P + cv] = sample_guide(g, cv/(P-1)) - guide_root(g) for the frame,
// in the reference's exact (uncontracted) arithmetic (generate.h:137-205).
__device__ __forceinline__ float4 guide_offset_entry(const AssetArgs &a, const FrameArgs &f, uint32_t P, uint32_t gi,
                                                     uint32_t cv) {
    const uint32_t *rec = a.guides + 14u * static_cast<uint64_t>(gi);
    const uint32_t first = __ldg(rec + 0);
    if (first >= a.guide_cv_count) { return make_float4(0.0f, 0.0f, 0.0f, 0.0f); }
    const uint32_t count = min(__ldg(rec + 1) & 0xffffu, a.guide_cv_count - first);
    const uint32_t gtri = __ldg(rec + 2);
    const float gb1 = __uint_as_float(__ldg(rec + 4));
    const float gb2 = __uint_as_float(__ldg(rec + 5));
    const F3 rest_root = {__uint_as_float(__ldg(rec + 8)), __uint_as_float(__ldg(rec + 9)),
                          __uint_as_float(__ldg(rec + 10))};
    const bool bound = gtri < a.triangle_count;
    F3 groot = rest_root;
    if (f.deformed_guide_cvs) {
        groot = ld3(f.guide_cvs, first);
    } else if (f.deformed_positions && bound) {
        const uint3 t = load_triangle(a, gtri);
        const float gb0 = __fsub_rn(__fsub_rn(1.0f, gb1), gb2);
        groot = xbary(ld3(f.positions, t.x), ld3(f.positions, t.y), ld3(f.positions, t.z), gb0, gb1, gb2);
    }
    F3 v;
    if (count <= 1u) {
        v = ld3(f.guide_cvs, first);
    } else {
        const float t = __fdiv_rn(static_cast<float>(cv), static_cast<float>(P - 1u));
        const float x = __fmul_rn(fminf(fmaxf(t, 0.0f), 1.0f), static_cast<float>(count - 1u));
        uint32_t i = static_cast<uint32_t>(x);
        if (i >= count - 1u) { i = count - 2u; }
        const float fr = __fsub_rn(x, static_cast<float>(i));
        v = xadd(xmul(ld3(f.guide_cvs, first + i), __fsub_rn(1.0f, fr)), xmul(ld3(f.guide_cvs, first + i + 1u), fr));
    }
    if (!f.deformed_guide_cvs && f.deformed_positions && bound) { v = xsub(xadd(v, groot), rest_root); }
    const F3 d = xsub(v, groot);
    return make_float4(d.x, d.y, d.z, 0.0f);
}

} // namespace dev

// Host-side helpers defined in generate.cu.
dev::AssetArgs resolve_asset(const nxg_device_asset_desc &desc);
dev::FrameArgs resolve_frame(const dev::AssetArgs &a, const nxg_deformed_desc &d);
dev::ParamArgs resolve_params(const nxg_generation_params &p, float radius_scale);
uint32_t record_cuda(cudaError_t e);
int device_sm_count();
uint32_t validate_range_request(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                const nxg_generation_params *params, const nxg_packed_output_desc *output,
                                const nxg_launch_config *config, uint32_t first, uint32_t count);
uint32_t check_launch_inputs(const nxg_device_asset_desc &asset, const nxg_packed_output_desc *output);
uint32_t check_workspace(const nxg_device_asset_desc &asset, uint32_t count, uint32_t P, const void *workspace,
                         uint64_t bytes);
uint32_t launch_order(const nxg_device_asset_desc &asset, uint32_t seed, uint32_t first, uint32_t count,
                      uint32_t P, void *workspace, cudaStream_t stream);
uint32_t launch_generate(const nxg_device_asset_desc &asset, const nxg_deformed_desc &deformed,
                         const nxg_generation_params &params, const nxg_packed_output_desc &output,
                         const nxg_launch_config &config, uint32_t first, uint32_t count, void *workspace,
                         cudaStream_t stream, float *vec3_points, const nxg_classic_apply_desc *classic);

} // namespace nxg
