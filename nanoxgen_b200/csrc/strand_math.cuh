// strand_math.cuh -- device-side strand math for sm_100a.
//
// The functions here restate include/nanoxgen/generate.h for a CUDA warp
// layout in which a group of L lanes owns one strand and each lane owns the
// CVs cv = c*L + lane (chunk c).  Two arithmetic regimes are used:
//
//   * "exact" helpers (x-prefixed) use __f*_rn intrinsics, which nvcc never
//     contracts into FMA.  They reproduce the reference's IEEE-rounded
//     operations (it builds with -ffp-contract=off) bit for bit, and are used
//     for every value that feeds an index decision: the alias draw, the root
//     position/normal, guide roots/normals, d^2 and the normal-rejection dot
//     product.  Root triangle indices, stencil indices and nearest guides are
//     therefore identical to the CPU generator's.
//   * everything else (CV interpolation, noise, frame transport) is ordinary
//     CUDA float arithmetic and matches the CPU generator to the stated
//     position tolerance.
#pragma once

#include <cstdint>

#include "nxg.h"

namespace nxg {
namespace dev {

constexpr uint32_t kSlots = NXG_GUIDE_STENCIL_SIZE;
constexpr uint32_t kInvalid = NXG_INVALID_INDEX;
constexpr unsigned kFull = 0xffffffffu;

struct F3 {
    float x, y, z;
};

// ---------------------------------------------------------------------------
// Exact (non-contracted) arithmetic.
// ---------------------------------------------------------------------------
__device__ __forceinline__ F3 xadd(F3 a, F3 b) {
    return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)};
}
__device__ __forceinline__ F3 xsub(F3 a, F3 b) {
    return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)};
}
__device__ __forceinline__ F3 xmul(F3 a, float s) {
    return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)};
}
__device__ __forceinline__ F3 xdiv(F3 a, float s) {
    return {__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)};
}
__device__ __forceinline__ float xdot(F3 a, F3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ F3 xcross(F3 a, F3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
// generate.h:67-70
__device__ __forceinline__ F3 xnormalize(F3 v) {
    const float l2 = xdot(v, v);
    return l2 > 1.0e-20f ? xdiv(v, __fsqrt_rn(l2)) : F3{0.0f, 1.0f, 0.0f};
}
// (p0*b0 + p1*b1) + p2*b2, the reference's barycentric evaluation order.
__device__ __forceinline__ F3 xbary(F3 p0, F3 p1, F3 p2, float b0, float b1, float b2) {
    return xadd(xadd(xmul(p0, b0), xmul(p1, b1)), xmul(p2, b2));
}

// ---------------------------------------------------------------------------
// Ordinary arithmetic (FMA allowed).
// ---------------------------------------------------------------------------
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ F3 normalize(F3 v) {
    const float l2 = dot(v, v);
    return l2 > 1.0e-20f ? v * rsqrtf(l2) : F3{0.0f, 1.0f, 0.0f};
}

__device__ __forceinline__ F3 ld3(const float *p, uint32_t i) {
    const float *q = p + 3u * static_cast<uint64_t>(i);
    return {__ldg(q), __ldg(q + 1), __ldg(q + 2)};
}

// ---------------------------------------------------------------------------
// Kernel arguments: device pointers resolved on the host from the validated
// header mirror, so kernels never read counts or offsets from device memory.
// ---------------------------------------------------------------------------
struct AssetArgs {
    const float *positions;      // rest positions (V x 3)
    const float *normals;        // rest normals (V x 3)
    const float *texcoords;      // V x 2, or nullptr
    const uint32_t *triangles;   // T x 3
    const uint2 *alias;          // T x {probability bits, alias}
    const uint32_t *guides;      // G x 14 words (GuideRecord)
    const float *guide_cvs;      // rest guide CVs (GCV x 3)
    const uint32_t *stencil;     // T x 8
    const float *gradients;      // 256 x 3
    uint32_t vertex_count, triangle_count, guide_count, guide_cv_count, flags;
};

struct FrameArgs {            // generate.h:86-99 frame_* overlays
    const float *positions;   // deformed or rest
    const float *normals;     // deformed or rest
    const float *guide_cvs;   // deformed or rest
    uint32_t deformed_positions, deformed_normals, deformed_guide_cvs;
};

struct ParamArgs {
    uint32_t strand_count, cvs_per_strand, seed;
    float support_scale, weight_power, rejection_cos, length_scale;
    float root_width, tip_width, noise_amplitude, noise_frequency, noise_mask;
    float noise_correlation, noise_preserve_length, radius_scale;
    uint32_t noise;  // generate.h:291-293 noise_is_enabled
};

// ---------------------------------------------------------------------------
// Random identity: generate.h:72-84
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16u;
    x *= 0x7feb352du;
    x ^= x >> 15u;
    x *= 0x846ca68bu;
    x ^= x >> 16u;
    return x;
}
__device__ __forceinline__ float random01(uint32_t seed, uint32_t strand, uint32_t dim) {
    const uint32_t h = hash32(seed ^ hash32(strand + 0x9e3779b9u * (dim + 1u)));
    return __fmul_rn(__uint2float_rn(h >> 8u), 1.0f / 16777216.0f);
}

__device__ __forceinline__ uint3 load_triangle(const AssetArgs &a, uint32_t t) {
    const uint32_t *p = a.triangles + 3u * static_cast<uint64_t>(t);
    const uint32_t vmax = a.vertex_count - 1u;
    return make_uint3(min(__ldg(p), vmax), min(__ldg(p + 1), vmax), min(__ldg(p + 2), vmax));
}

// Alias draw of generate.h:107-112 (the triangle decision alone).
__device__ __forceinline__ uint32_t sample_triangle(const AssetArgs &a, uint32_t seed, uint32_t strand) {
    const float choose = __fmul_rn(random01(seed, strand, 0u), __uint2float_rn(a.triangle_count));
    uint32_t bucket = static_cast<uint32_t>(choose);
    if (bucket >= a.triangle_count) { bucket = a.triangle_count - 1u; }
    const uint2 entry = __ldg(a.alias + bucket);
    return random01(seed, strand, 1u) < __uint_as_float(entry.x)
        ? bucket : min(entry.y, a.triangle_count - 1u);
}

struct Root {
    F3 position, normal;
    float u, v;
    uint32_t triangle;
    float b1, b2;
};

// generate.h:101-135 sample_root
__device__ __forceinline__ Root sample_root(const AssetArgs &a, const FrameArgs &f,
                                            uint32_t seed, uint32_t strand) {
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
    r.position = xbary(p0, p1, p2, b0, r.b1, r.b2);
    if (a.flags & NXG_ASSET_HAS_NORMALS) {  // the face normal is replaced by the vertex normals' blend
        r.normal = xnormalize(xbary(ld3(f.normals, t.x), ld3(f.normals, t.y), ld3(f.normals, t.z),
                                    b0, r.b1, r.b2));
    } else {
        r.normal = xnormalize(xcross(xsub(p1, p0), xsub(p2, p0)));
    }
    r.u = 0.0f;
    r.v = 0.0f;
    if ((a.flags & NXG_ASSET_HAS_TEXCOORDS) && a.texcoords) {
        const float *t0 = a.texcoords + 2u * static_cast<uint64_t>(t.x);
        const float *t1 = a.texcoords + 2u * static_cast<uint64_t>(t.y);
        const float *t2 = a.texcoords + 2u * static_cast<uint64_t>(t.z);
        r.u = __fadd_rn(__fadd_rn(__fmul_rn(__ldg(t0), b0), __fmul_rn(__ldg(t1), r.b1)),
                        __fmul_rn(__ldg(t2), r.b2));
        r.v = __fadd_rn(__fadd_rn(__fmul_rn(__ldg(t0 + 1), b0), __fmul_rn(__ldg(t1 + 1), r.b1)),
                        __fmul_rn(__ldg(t2 + 1), r.b2));
    }
    return r;
}

// ---------------------------------------------------------------------------
// Guide stencil slot (generate.h:137-187 and the loop body of :214-244).
// ---------------------------------------------------------------------------
enum : uint32_t { kSlotEligible = 1u, kSlotBlended = 2u, kSlotFollow = 4u };

struct Slot {             // 48 bytes, staged in shared memory per strand
    float gx, gy, gz, w;  // current guide root, blend weight
    float rx, ry, rz, d2; // rest guide root (for the patch-follow case), distance^2
    uint32_t guide, first_cv, cv_count, flags;
};

// The frame's guide root (generate.h:137-151) and guide normal
// (generate.h:153-172) from the guide record's fields.
__device__ __forceinline__ void frame_guide(const AssetArgs &a, const FrameArgs &f, uint32_t first, uint32_t gtri,
                                            float gb1, float gb2, F3 rest_root, F3 rest_normal, F3 &groot,
                                            F3 &gnormal) {
    const bool bound = gtri < a.triangle_count;
    groot = rest_root;
    if (f.deformed_guide_cvs) {
        groot = ld3(f.guide_cvs, first);
    } else if (f.deformed_positions && bound) {
        const uint3 t = load_triangle(a, gtri);
        const float gb0 = __fsub_rn(__fsub_rn(1.0f, gb1), gb2);
        groot = xbary(ld3(f.positions, t.x), ld3(f.positions, t.y), ld3(f.positions, t.z), gb0, gb1, gb2);
    }
    gnormal = rest_normal;
    if (bound && (f.deformed_positions || f.deformed_normals)) {
        const uint3 t = load_triangle(a, gtri);
        const float gb0 = __fsub_rn(__fsub_rn(1.0f, gb1), gb2);
        if (f.deformed_normals) {
            gnormal = xnormalize(xbary(ld3(f.normals, t.x), ld3(f.normals, t.y), ld3(f.normals, t.z),
                                       gb0, gb1, gb2));
        } else {
            const F3 p0 = ld3(f.positions, t.x);
            gnormal = xnormalize(xcross(xsub(ld3(f.positions, t.y), p0), xsub(ld3(f.positions, t.z), p0)));
        }
    }
}

// Per-frame guide record for the lane-walk generator: (guide root, support
// radius * support_scale) and (guide normal, 1), or a zero second word for a
// corrupt record (first CV past the CV array).
__device__ __forceinline__ void guide_frame_entry(const AssetArgs &a, const FrameArgs &f, float support_scale,
                                                  uint32_t gi, float4 *out) {
    const uint32_t *g = a.guides + 14u * static_cast<uint64_t>(gi);
    const uint32_t first = __ldg(g + 0);
    if (first >= a.guide_cv_count) {
        out[0] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        out[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const float support = __uint_as_float(__ldg(g + 3));
    const F3 rest_root = {__uint_as_float(__ldg(g + 8)), __uint_as_float(__ldg(g + 9)),
                          __uint_as_float(__ldg(g + 10))};
    const F3 rest_normal = {__uint_as_float(__ldg(g + 11)), __uint_as_float(__ldg(g + 12)),
                            __uint_as_float(__ldg(g + 13))};
    F3 groot, gnormal;
    frame_guide(a, f, first, __ldg(g + 2), __uint_as_float(__ldg(g + 4)), __uint_as_float(__ldg(g + 5)), rest_root,
                rest_normal, groot, gnormal);
    out[0] = make_float4(groot.x, groot.y, groot.z, __fmul_rn(support, support_scale));
    out[1] = make_float4(gnormal.x, gnormal.y, gnormal.z, __uint_as_float(1u));
}

__device__ __forceinline__ Slot eval_slot(const AssetArgs &a, const FrameArgs &f, const ParamArgs &p,
                                          const Root &root, uint32_t j) {
    Slot s;
    s.gx = s.gy = s.gz = s.w = 0.0f;
    s.rx = s.ry = s.rz = s.d2 = 0.0f;
    s.guide = kInvalid;
    s.first_cv = 0u;
    s.cv_count = 0u;
    s.flags = 0u;
    const uint32_t gi = __ldg(a.stencil + static_cast<uint64_t>(root.triangle) * kSlots + j);
    if (gi == kInvalid || gi >= a.guide_count) { return s; }
    const uint32_t *g = a.guides + 14u * static_cast<uint64_t>(gi);
    const uint32_t first = __ldg(g + 0);
    uint32_t count = __ldg(g + 1) & 0xffffu;
    if (first >= a.guide_cv_count) { return s; }  // corrupt record: never read past the CVs
    count = min(count, a.guide_cv_count - first);
    const uint32_t gtri = __ldg(g + 2);
    const float support = __uint_as_float(__ldg(g + 3));
    const float gb1 = __uint_as_float(__ldg(g + 4));
    const float gb2 = __uint_as_float(__ldg(g + 5));
    const F3 rest_root = {__uint_as_float(__ldg(g + 8)), __uint_as_float(__ldg(g + 9)),
                          __uint_as_float(__ldg(g + 10))};
    const F3 rest_normal = {__uint_as_float(__ldg(g + 11)), __uint_as_float(__ldg(g + 12)),
                            __uint_as_float(__ldg(g + 13))};
    const bool bound = gtri < a.triangle_count;
    F3 groot, gnormal;
    frame_guide(a, f, first, gtri, gb1, gb2, rest_root, rest_normal, groot, gnormal);
    const F3 delta = xsub(root.position, groot);
    const float d2 = xdot(delta, delta);
    s.gx = groot.x;
    s.gy = groot.y;
    s.gz = groot.z;
    s.rx = rest_root.x;
    s.ry = rest_root.y;
    s.rz = rest_root.z;
    s.d2 = d2;
    s.guide = gi;
    s.first_cv = first;
    s.cv_count = count;
    if (!f.deformed_guide_cvs && f.deformed_positions && bound) { s.flags |= kSlotFollow; }
    if (xdot(root.normal, gnormal) < p.rejection_cos) {
        s.guide = kInvalid;
        return s;
    }
    s.flags |= kSlotEligible;
    const float radius = __fmul_rn(support, p.support_scale);
    if (radius <= 0.0f || d2 >= __fmul_rn(radius, radius)) { return s; }
    s.w = powf(__fsub_rn(1.0f, __fdiv_rn(__fsqrt_rn(d2), radius)), p.weight_power);
    s.flags |= kSlotBlended;
    return s;
}

// generate.h:189-205 sample_guide, minus the current guide root (the
// difference interpolate_offset accumulates).
__device__ __forceinline__ F3 guide_offset(const float *cvs, const Slot &s, float t) {
    F3 v;
    if (s.cv_count <= 1u) {
        v = ld3(cvs, s.first_cv);
    } else {
        const float x = fminf(fmaxf(t, 0.0f), 1.0f) * static_cast<float>(s.cv_count - 1u);
        uint32_t i = static_cast<uint32_t>(x);
        if (i >= s.cv_count - 1u) { i = s.cv_count - 2u; }
        const float fr = x - static_cast<float>(i);
        const F3 va = ld3(cvs, s.first_cv + i);
        const F3 vb = ld3(cvs, s.first_cv + i + 1u);
        v = va * (1.0f - fr) + vb * fr;
    }
    const F3 groot = {s.gx, s.gy, s.gz};
    if (s.flags & kSlotFollow) { v = (v + groot) - F3{s.rx, s.ry, s.rz}; }
    return v - groot;
}

// ---------------------------------------------------------------------------
// Surface frame and noise (generate.h:312-418).
// ---------------------------------------------------------------------------
__device__ __forceinline__ F3 fallback_surface_u(F3 n) {
    const F3 axis = (n.z > -0.999f && n.z < 0.999f) ? F3{0.0f, 0.0f, 1.0f} : F3{0.0f, 1.0f, 0.0f};
    return normalize(cross(n, axis));
}

__device__ __forceinline__ F3 root_surface_u(const AssetArgs &a, const FrameArgs &f, const Root &root) {
    F3 tangent = {0.0f, 0.0f, 0.0f};
    if ((a.flags & NXG_ASSET_HAS_TEXCOORDS) && a.texcoords) {
        const uint3 t = load_triangle(a, root.triangle);
        const F3 p0 = ld3(f.positions, t.x);
        const F3 e1 = ld3(f.positions, t.y) - p0;
        const F3 e2 = ld3(f.positions, t.z) - p0;
        const float *uv0 = a.texcoords + 2u * static_cast<uint64_t>(t.x);
        const float *uv1 = a.texcoords + 2u * static_cast<uint64_t>(t.y);
        const float *uv2 = a.texcoords + 2u * static_cast<uint64_t>(t.z);
        const float du1 = __ldg(uv1) - __ldg(uv0), dv1 = __ldg(uv1 + 1) - __ldg(uv0 + 1);
        const float du2 = __ldg(uv2) - __ldg(uv0), dv2 = __ldg(uv2 + 1) - __ldg(uv0 + 1);
        const float det = du1 * dv2 - dv1 * du2;
        if (fabsf(det) > 1.0e-12f) {
            tangent = (e1 * dv2 - e2 * dv1) * (1.0f / det);
            tangent = tangent - root.normal * dot(tangent, root.normal);
        }
    }
    return dot(tangent, tangent) > 1.0e-20f ? normalize(tangent) : fallback_surface_u(root.normal);
}

// generate.h:343-351, rest pose, with b0 recomputed from the stored pair.
__device__ __forceinline__ F3 rest_root_position(const AssetArgs &a, const Root &root) {
    const uint3 t = load_triangle(a, root.triangle);
    const float b0 = __fsub_rn(__fsub_rn(1.0f, root.b1), root.b2);
    return xbary(ld3(a.positions, t.x), ld3(a.positions, t.y), ld3(a.positions, t.z), b0, root.b1, root.b2);
}

// generate.h:353-364 noise_hash.  The LCG chain over (x, y, z) is linear
// modulo 2^32: seed = x*A^2 + y*A + z + C*(A^2 + A + 1), so the eight cube
// corners differ from the base seed by constants.  The final combine
// (((s & 0xff0000) >> 4) + (s & 0xff)) & 0xff keeps only the low byte.
constexpr uint32_t kLcgA = 1664525u;
constexpr uint32_t kLcgC = 1013904223u;
constexpr uint32_t kLcgA2 = kLcgA * kLcgA;
constexpr uint32_t kLcgK = kLcgC * kLcgA2 + kLcgC * kLcgA + kLcgC;

__device__ __forceinline__ uint32_t temper_index(uint32_t s) {
    s ^= s >> 11u;
    s ^= (s << 7u) & 0x9d2c5680u;
    s ^= (s << 15u) & 0xefc60000u;
    s ^= s >> 18u;
    return s & 0xffu;
}

__device__ __forceinline__ float s_curve(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }

// generate.h:370-402 gradient_noise over a shared-memory copy of the asset's
// gradient table (float4-padded).
__device__ __forceinline__ float gradient_noise(const float4 *table, float x, float y, float z) {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int32_t ix = static_cast<int32_t>(fx), iy = static_cast<int32_t>(fy), iz = static_cast<int32_t>(fz);
    const float wx = x - fx, wy = y - fy, wz = z - fz;
    const uint32_t base = static_cast<uint32_t>(ix) * kLcgA2 + static_cast<uint32_t>(iy) * kLcgA +
                          static_cast<uint32_t>(iz) + kLcgK;
    float v[8];
#pragma unroll
    for (uint32_t corner = 0u; corner < 8u; ++corner) {
        const uint32_t ox = corner & 1u, oy = (corner >> 1u) & 1u, oz = (corner >> 2u) & 1u;
        const uint32_t seed = base + (ox ? kLcgA2 : 0u) + (oy ? kLcgA : 0u) + oz;
        const float4 g = table[temper_index(seed)];
        v[corner] = g.x * (wx - static_cast<float>(ox)) + g.y * (wy - static_cast<float>(oy)) +
                    g.z * (wz - static_cast<float>(oz));
    }
    const float ax = s_curve(wx), ay = s_curve(wy), az = s_curve(wz);
    v[0] = (1.0f - ax) * v[0] + ax * v[1];
    v[2] = (1.0f - ax) * v[2] + ax * v[3];
    v[4] = (1.0f - ax) * v[4] + ax * v[5];
    v[6] = (1.0f - ax) * v[6] + ax * v[7];
    v[0] = (1.0f - ay) * v[0] + ay * v[2];
    v[4] = (1.0f - ay) * v[4] + ay * v[6];
    v[0] = (1.0f - az) * v[0] + az * v[4];
    return 0.5f * v[0] + 0.5f;
}

// 3x3 row-major matrix for the transported frame.
struct M3 {
    float m[9];
};

__device__ __forceinline__ M3 identity3() {
    M3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) { r.m[i] = (i % 4 == 0) ? 1.0f : 0.0f; }
    return r;
}

// generate.h:404-418 rotate_by as a matrix (axis is not normalised, exactly
// as the reference passes cross(t_prev, t_next)).
__device__ __forceinline__ M3 rotation3(F3 axis, float angle) {
    float s, c;
    sincosf(angle, &s, &c);
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

__device__ __forceinline__ M3 mul3(const M3 &a, const M3 &b) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            r.m[3 * i + j] = a.m[3 * i] * b.m[j] + a.m[3 * i + 1] * b.m[3 + j] + a.m[3 * i + 2] * b.m[6 + j];
        }
    }
    return r;
}

__device__ __forceinline__ F3 apply3(const M3 &a, F3 v) {
    return {a.m[0] * v.x + a.m[1] * v.y + a.m[2] * v.z, a.m[3] * v.x + a.m[4] * v.y + a.m[5] * v.z,
            a.m[6] * v.x + a.m[7] * v.y + a.m[8] * v.z};
}

// ---------------------------------------------------------------------------
// Group (L-lane) collectives.  Every lane of the warp executes them.
// ---------------------------------------------------------------------------
template <int L>
__device__ __forceinline__ float group_shfl(float v, int src) { return __shfl_sync(kFull, v, src, L); }
template <int L>
__device__ __forceinline__ F3 group_shfl(F3 v, int src) {
    return {__shfl_sync(kFull, v.x, src, L), __shfl_sync(kFull, v.y, src, L), __shfl_sync(kFull, v.z, src, L)};
}
template <int L>
__device__ __forceinline__ F3 group_shfl_up(F3 v, int d) {
    return {__shfl_up_sync(kFull, v.x, d, L), __shfl_up_sync(kFull, v.y, d, L), __shfl_up_sync(kFull, v.z, d, L)};
}
template <int L>
__device__ __forceinline__ F3 group_shfl_down(F3 v, int d) {
    return {__shfl_down_sync(kFull, v.x, d, L), __shfl_down_sync(kFull, v.y, d, L),
            __shfl_down_sync(kFull, v.z, d, L)};
}
template <int L>
__device__ __forceinline__ float group_scan_add(float v, int lane) {
#pragma unroll
    for (int d = 1; d < L; d <<= 1) {
        const float u = __shfl_up_sync(kFull, v, d, L);
        if (lane >= d) { v += u; }
    }
    return v;
}
template <int L>
__device__ __forceinline__ int group_scan_max(int v, int lane) {
#pragma unroll
    for (int d = 1; d < L; d <<= 1) {
        const int u = __shfl_up_sync(kFull, v, d, L);
        if (lane >= d) { v = max(v, u); }
    }
    return v;
}
template <int L>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int d = L / 2; d > 0; d >>= 1) { v += __shfl_xor_sync(kFull, v, d, L); }
    return v;
}
// Inclusive prefix product X_k = M_k * ... * M_0 (later factors on the left).
template <int L>
__device__ __forceinline__ M3 group_scan_mat(M3 x, int lane) {
#pragma unroll
    for (int d = 1; d < L; d <<= 1) {
        M3 y;
#pragma unroll
        for (int i = 0; i < 9; ++i) { y.m[i] = __shfl_up_sync(kFull, x.m[i], d, L); }
        if (lane >= d) { x = mul3(x, y); }
    }
    return x;
}
template <int L>
__device__ __forceinline__ M3 group_shfl(const M3 &x, int src) {
    M3 r;
#pragma unroll
    for (int i = 0; i < 9; ++i) { r.m[i] = __shfl_sync(kFull, x.m[i], src, L); }
    return r;
}

} // namespace dev
} // namespace nxg
