/*
 * nxg_oracle.c -- CPU restatement of NanoXGen's per-strand packed generator.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * generator in nanoxgen_b200/csrc.  Only tests/, __graft_entry__.smoke() and
 * the cpu_baseline / reference legs of bench.py may load it.  The product path
 * never calls it and must fail loudly instead of falling back to it.
 *
 * It restates, in plain C11, the arithmetic of the reference header
 * include/nanoxgen/generate.h (functions cited per definition) and the asset
 * validator of src/asset.cpp.  Every float expression keeps the reference's
 * evaluation order, and the file is compiled with -ffp-contract=off (the
 * reference's strict build, Makefile:13-17) so that, on the same libm, its
 * output is bitwise identical to the reference's generate_packed_cpu.  That
 * claim is pinned by tests/test_oracle.py against the reference compiled from
 * its own sources (oracle/_ref) and against committed golden vectors.
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

typedef struct { float x, y; } V2;
typedef struct { float x, y, z; } V3;
typedef struct { uint32_t x, y, z; } U3;
typedef struct { float probability; uint32_t alias; } AliasEntry;

/* include/nanoxgen/types.h:62-72 (56 bytes) */
typedef struct {
    uint32_t first_cv;
    uint16_t cv_count;
    uint16_t flags;
    uint32_t triangle_index;
    float support_radius;
    V2 barycentric;
    V2 root_uv;
    V3 root_position;
    V3 root_normal;
} Guide;

/* include/nanoxgen/types.h:81-101 (128 bytes, 64-byte aligned) */
typedef struct {
    uint64_t magic;
    uint16_t version_major, version_minor;
    uint32_t flags;
    uint64_t byte_size;
    uint64_t content_hash;
    uint32_t vertex_count, triangle_count, guide_count, guide_cv_count;
    uint32_t guide_stencil_size, noise_gradient_count;
    uint64_t positions_offset, normals_offset, texcoords_offset, triangles_offset;
    uint64_t alias_table_offset, guides_offset, guide_cvs_offset;
    uint64_t triangle_guides_offset, noise_gradients_offset;
} Header;

/* include/nanoxgen/types.h:108-124 */
typedef struct {
    uint32_t strand_count, cvs_per_strand, seed, reserved;
    float guide_support_scale, guide_weight_power, normal_rejection_cos;
    float length_scale, root_width, tip_width;
    float noise_amplitude, noise_frequency, noise_mask;
    float noise_correlation, noise_preserve_length;
} Params;

/* include/nanoxgen/types.h:126-136 (48 bytes) */
typedef struct {
    V3 position;
    V3 normal;
    V2 uv;
    uint32_t triangle_index;
    V2 barycentric;
    uint32_t surface_face_id;
} Root;

typedef struct { const V3 *positions, *normals, *guide_cvs; } Deformed;

/* Per-strand state exported for stencil/root parity checks
 * (generate.h:207-212 GuideBlendState, generate.h:281-289 StrandGenerationState). */
typedef struct {
    Root root;
    uint32_t indices[8];
    float weights[8];
    float weight_sum;
    uint32_t nearest;
    V3 surface_u;
    V3 noise_domain;
    float original_length;
    float effective_noise_frequency;
    float preserve_scale;
} StrandState;

_Static_assert(sizeof(Guide) == 56, "GuideRecord layout");
_Static_assert(sizeof(Header) == 128, "AssetHeader layout");
_Static_assert(sizeof(Root) == 48, "RootSample layout");
_Static_assert(sizeof(Params) == 60, "GenerationParams layout");

#define K_STENCIL 8u
#define INVALID 0xffffffffu
#define HAS_NORMALS 1u
#define HAS_TEXCOORDS 2u

/* ---- vector helpers: types.h:42-52, generate.h:51-70 ---- */
static inline V3 v3(float x, float y, float z) { V3 r = {x, y, z}; return r; }
static inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 mul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 dvs(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline V2 add2(V2 a, V2 b) { V2 r = {a.x + b.x, a.y + b.y}; return r; }
static inline V2 mul2(V2 a, float s) { V2 r = {a.x * s, a.y * s}; return r; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len2(V3 v) { return dot(v, v); }
static inline float fmax_(float a, float b) { return a > b ? a : b; }
static inline float fmin_(float a, float b) { return a < b ? a : b; }
static inline float clamp_(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
static inline float fabs_(float x) { return x < 0.0f ? -x : x; }
static inline V3 normalize(V3 v) {            /* generate.h:67-70 */
    const float l2 = len2(v);
    return l2 > 1.0e-20f ? dvs(v, sqrtf(l2)) : v3(0.0f, 1.0f, 0.0f);
}

/* ---- asset view: device_view.h:7-40 ---- */
typedef struct {
    const unsigned char *base;
    const Header *h;
} Asset;

static inline Asset asset_of(const void *bytes) {
    Asset a;
    a.base = (const unsigned char *)bytes;
    a.h = (const Header *)bytes;
    return a;
}
#define SECTION(a, T, off) ((const T *)((a).base + (a).h->off))

/* ---- random identity: generate.h:72-84 ---- */
static inline uint32_t hash32(uint32_t x) {
    x ^= x >> 16u;
    x *= 0x7feb352du;
    x ^= x >> 15u;
    x *= 0x846ca68bu;
    x ^= x >> 16u;
    return x;
}
static inline float random01(uint32_t seed, uint32_t strand, uint32_t dim) {
    const uint32_t h = hash32(seed ^ hash32(strand + 0x9e3779b9u * (dim + 1u)));
    return (float)(h >> 8u) * (1.0f / 16777216.0f);
}

static inline const V3 *frame_positions(Asset a, const Deformed *d) {  /* generate.h:86-89 */
    return d->positions ? d->positions : SECTION(a, V3, positions_offset);
}
static inline const V3 *frame_normals(Asset a, const Deformed *d) {    /* generate.h:91-94 */
    return d->normals ? d->normals : SECTION(a, V3, normals_offset);
}
static inline const V3 *frame_guide_cvs(Asset a, const Deformed *d) {  /* generate.h:96-99 */
    return d->guide_cvs ? d->guide_cvs : SECTION(a, V3, guide_cvs_offset);
}

/* generate.h:101-135 */
static Root sample_root(Asset a, const Deformed *d, const Params *p, uint32_t strand) {
    const Header *h = a.h;
    const float choose = random01(p->seed, strand, 0u) * (float)h->triangle_count;
    uint32_t bucket = (uint32_t)choose;
    if (bucket >= h->triangle_count) bucket = h->triangle_count - 1u;
    const AliasEntry entry = SECTION(a, AliasEntry, alias_table_offset)[bucket];
    const uint32_t tri_index =
        random01(p->seed, strand, 1u) < entry.probability ? bucket : entry.alias;
    const float r1 = random01(p->seed, strand, 2u);
    const float r2 = random01(p->seed, strand, 3u);
    const float s = sqrtf(r1);
    const float b0 = 1.0f - s;
    const float b1 = s * (1.0f - r2);
    const float b2 = s * r2;
    const U3 tri = SECTION(a, U3, triangles_offset)[tri_index];
    const V3 *pos = frame_positions(a, d);
    const V3 pp = add(add(mul(pos[tri.x], b0), mul(pos[tri.y], b1)), mul(pos[tri.z], b2));
    V3 n = normalize(cross(sub(pos[tri.y], pos[tri.x]), sub(pos[tri.z], pos[tri.x])));
    if ((h->flags & HAS_NORMALS) != 0u) {
        const V3 *nrm = frame_normals(a, d);
        n = normalize(add(add(mul(nrm[tri.x], b0), mul(nrm[tri.y], b1)), mul(nrm[tri.z], b2)));
    }
    V2 uv = {0.0f, 0.0f};
    if ((h->flags & HAS_TEXCOORDS) != 0u) {
        const V2 *tc = SECTION(a, V2, texcoords_offset);
        uv = add2(add2(mul2(tc[tri.x], b0), mul2(tc[tri.y], b1)), mul2(tc[tri.z], b2));
    }
    Root r;
    r.position = pp;
    r.normal = n;
    r.uv = uv;
    r.triangle_index = tri_index;
    r.barycentric.x = b1;
    r.barycentric.y = b2;
    r.surface_face_id = tri_index;
    return r;
}

/* generate.h:137-151 */
static V3 guide_root(Asset a, const Deformed *d, const Guide *g) {
    if (d->guide_cvs) return d->guide_cvs[g->first_cv];
    if (d->positions && g->triangle_index < a.h->triangle_count) {
        const U3 tri = SECTION(a, U3, triangles_offset)[g->triangle_index];
        const float b1 = g->barycentric.x;
        const float b2 = g->barycentric.y;
        const float b0 = 1.0f - b1 - b2;
        return add(add(mul(d->positions[tri.x], b0), mul(d->positions[tri.y], b1)),
                   mul(d->positions[tri.z], b2));
    }
    return g->root_position;
}

/* generate.h:153-172 */
static V3 guide_normal(Asset a, const Deformed *d, const Guide *g) {
    if (g->triangle_index >= a.h->triangle_count || (!d->positions && !d->normals)) {
        return g->root_normal;
    }
    const U3 tri = SECTION(a, U3, triangles_offset)[g->triangle_index];
    const float b1 = g->barycentric.x;
    const float b2 = g->barycentric.y;
    const float b0 = 1.0f - b1 - b2;
    if (d->normals) {
        return normalize(add(add(mul(d->normals[tri.x], b0), mul(d->normals[tri.y], b1)),
                             mul(d->normals[tri.z], b2)));
    }
    const V3 *pos = frame_positions(a, d);
    return normalize(cross(sub(pos[tri.y], pos[tri.x]), sub(pos[tri.z], pos[tri.x])));
}

/* generate.h:174-187 */
static V3 follow_deformed_guide_root(Asset a, const Deformed *d, const Guide *g, V3 point) {
    if (!d->guide_cvs && d->positions && g->triangle_index < a.h->triangle_count) {
        point = sub(add(point, guide_root(a, d, g)), g->root_position);
    }
    return point;
}

/* generate.h:189-205 */
static V3 sample_guide(Asset a, const Deformed *d, const Guide *g, float t) {
    const V3 *cvs = frame_guide_cvs(a, d);
    if (g->cv_count <= 1u) return follow_deformed_guide_root(a, d, g, cvs[g->first_cv]);
    const float x = clamp_(t, 0.0f, 1.0f) * (float)((uint32_t)g->cv_count - 1u);
    uint32_t i = (uint32_t)x;
    if (i >= (uint32_t)g->cv_count - 1u) i = (uint32_t)g->cv_count - 2u;
    const float f = x - (float)i;
    const V3 va = cvs[g->first_cv + i];
    const V3 vb = cvs[g->first_cv + i + 1u];
    return follow_deformed_guide_root(a, d, g, add(mul(va, 1.0f - f), mul(vb, f)));
}

typedef struct {
    uint32_t indices[8];
    float weights[8];
    float weight_sum;
    uint32_t nearest;
} Blend;

/* generate.h:214-244 */
static Blend make_guide_blend_state(Asset a, const Deformed *d, const Params *p, const Root *root) {
    Blend b;
    memset(&b, 0, sizeof b);
    b.nearest = INVALID;
    for (uint32_t j = 0; j < K_STENCIL; ++j) b.indices[j] = INVALID;
    const uint32_t *stencil = SECTION(a, uint32_t, triangle_guides_offset) +
                              (size_t)root->triangle_index * a.h->guide_stencil_size;
    const Guide *guides = SECTION(a, Guide, guides_offset);
    float nearest_d2 = 3.402823466e+38f;
    for (uint32_t j = 0; j < a.h->guide_stencil_size; ++j) {
        const uint32_t gi = stencil[j];
        if (gi == INVALID) continue;
        const Guide *g = &guides[gi];
        const V3 current_root = guide_root(a, d, g);
        const float d2 = len2(sub(root->position, current_root));
        if (dot(root->normal, guide_normal(a, d, g)) < p->normal_rejection_cos) continue;
        if (d2 < nearest_d2) { nearest_d2 = d2; b.nearest = gi; }
        const float radius = g->support_radius * p->guide_support_scale;
        if (radius <= 0.0f || d2 >= radius * radius) continue;
        const float w = powf(1.0f - sqrtf(d2) / radius, fmax_(p->guide_weight_power, 0.0f));
        b.indices[j] = gi;
        b.weights[j] = w;
        b.weight_sum += w;
    }
    return b;
}

/* generate.h:246-267 */
static V3 interpolate_offset(Asset a, const Deformed *d, const Root *root, const Blend *b, float t) {
    const Guide *guides = SECTION(a, Guide, guides_offset);
    V3 offset = v3(0.0f, 0.0f, 0.0f);
    for (uint32_t j = 0; j < K_STENCIL; ++j) {
        const uint32_t gi = b->indices[j];
        if (gi == INVALID) continue;
        const Guide *g = &guides[gi];
        offset = add(offset, mul(sub(sample_guide(a, d, g, t), guide_root(a, d, g)), b->weights[j]));
    }
    if (b->weight_sum > 1.0e-12f) return dvs(offset, b->weight_sum);
    if (b->nearest != INVALID) {
        const Guide *g = &guides[b->nearest];
        return sub(sample_guide(a, d, g, t), guide_root(a, d, g));
    }
    return mul(root->normal, t);
}

typedef struct {
    Root root;
    Blend blend;
    V3 surface_u;
    V3 noise_domain;
    float original_length;
    float effective_noise_frequency;
    float preserve_scale;
} State;

static inline int noise_is_enabled(const Params *p) {   /* generate.h:291-293 */
    return p->noise_amplitude != 0.0f && p->noise_mask != 0.0f;
}
static inline float strand_parameter(const Params *p, uint32_t cv) {  /* generate.h:295-298 */
    return (float)cv / (float)(p->cvs_per_strand - 1u);
}

/* generate.h:300-310 */
static V3 evaluate_base_strand_cv(Asset a, const Deformed *d, const Params *p, const State *s, uint32_t cv) {
    const float t = strand_parameter(p, cv);
    return add(s->root.position, mul(interpolate_offset(a, d, &s->root, &s->blend, t), p->length_scale));
}

/* generate.h:312-316 */
static V3 fallback_surface_u(V3 n) {
    const V3 axis = (n.z > -0.999f && n.z < 0.999f) ? v3(0.0f, 0.0f, 1.0f) : v3(0.0f, 1.0f, 0.0f);
    return normalize(cross(n, axis));
}

/* generate.h:318-341 */
static V3 root_surface_u(Asset a, const Deformed *d, const Root *root) {
    const U3 tri = SECTION(a, U3, triangles_offset)[root->triangle_index];
    const V3 *pos = frame_positions(a, d);
    V3 tangent = v3(0.0f, 0.0f, 0.0f);
    if ((a.h->flags & HAS_TEXCOORDS) != 0u) {
        const V2 *uvs = SECTION(a, V2, texcoords_offset);
        const V3 e1 = sub(pos[tri.y], pos[tri.x]);
        const V3 e2 = sub(pos[tri.z], pos[tri.x]);
        const V2 duv1 = {uvs[tri.y].x - uvs[tri.x].x, uvs[tri.y].y - uvs[tri.x].y};
        const V2 duv2 = {uvs[tri.z].x - uvs[tri.x].x, uvs[tri.z].y - uvs[tri.x].y};
        const float det = duv1.x * duv2.y - duv1.y * duv2.x;
        if (fabs_(det) > 1.0e-12f) {
            tangent = dvs(sub(mul(e1, duv2.y), mul(e2, duv1.y)), det);
            tangent = sub(tangent, mul(root->normal, dot(tangent, root->normal)));
        }
    }
    return len2(tangent) > 1.0e-20f ? normalize(tangent) : fallback_surface_u(root->normal);
}

/* generate.h:343-351 */
static V3 rest_root_position(Asset a, const Root *root) {
    const U3 tri = SECTION(a, U3, triangles_offset)[root->triangle_index];
    const V3 *pos = SECTION(a, V3, positions_offset);
    const float b1 = root->barycentric.x;
    const float b2 = root->barycentric.y;
    const float b0 = 1.0f - b1 - b2;
    return add(add(mul(pos[tri.x], b0), mul(pos[tri.y], b1)), mul(pos[tri.z], b2));
}

/* generate.h:353-364 */
static inline uint32_t noise_hash(int32_t x, int32_t y, int32_t z) {
    uint32_t seed = 0u;
    seed = seed * 1664525u + (uint32_t)x + 1013904223u;
    seed = seed * 1664525u + (uint32_t)y + 1013904223u;
    seed = seed * 1664525u + (uint32_t)z + 1013904223u;
    seed ^= seed >> 11u;
    seed ^= (seed << 7u) & 0x9d2c5680u;
    seed ^= (seed << 15u) & 0xefc60000u;
    seed ^= seed >> 18u;
    return (((seed & 0x00ff0000u) >> 4u) + (seed & 0xffu)) & 0xffu;
}

/* generate.h:366-368 */
static inline float noise_s_curve(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }

/* generate.h:370-402 */
static float gradient_noise(Asset a, V3 sample) {
    const V3 *grads = SECTION(a, V3, noise_gradients_offset);
    const float fx = floorf(sample.x);
    const float fy = floorf(sample.y);
    const float fz = floorf(sample.z);
    const int32_t ix = (int32_t)fx;
    const int32_t iy = (int32_t)fy;
    const int32_t iz = (int32_t)fz;
    const V3 w = v3(sample.x - fx, sample.y - fy, sample.z - fz);
    float values[8];
    for (uint32_t corner = 0u; corner < 8u; ++corner) {
        const int32_t ox = (int32_t)(corner & 1u);
        const int32_t oy = (int32_t)((corner >> 1u) & 1u);
        const int32_t oz = (int32_t)((corner >> 2u) & 1u);
        const V3 g = grads[noise_hash(ix + ox, iy + oy, iz + oz)];
        values[corner] = g.x * (w.x - (float)ox) + g.y * (w.y - (float)oy) + g.z * (w.z - (float)oz);
    }
    const float alphas[3] = {noise_s_curve(w.x), noise_s_curve(w.y), noise_s_curve(w.z)};
    for (int32_t dim = 2; dim >= 0; --dim) {
        const int32_t count = 1 << dim;
        for (int32_t value = 0; value < count; ++value) {
            const int32_t index = value * (1 << (3 - dim));
            const int32_t axis = 3 - dim - 1;
            const int32_t other = index + (1 << axis);
            values[index] = (1.0f - alphas[axis]) * values[index] + alphas[axis] * values[other];
        }
    }
    return 0.5f * values[0] + 0.5f;
}

/* generate.h:404-418 */
static V3 rotate_by(V3 value, V3 axis, float angle) {
    const float c = cosf(angle);
    const float s = sinf(angle);
    const float omc = 1.0f - c;
    return v3(dot(value, v3(axis.x * axis.x * omc + c, axis.x * axis.y * omc - axis.z * s,
                            axis.x * axis.z * omc + axis.y * s)),
              dot(value, v3(axis.x * axis.y * omc + axis.z * s, axis.y * axis.y * omc + c,
                            axis.y * axis.z * omc - axis.x * s)),
              dot(value, v3(axis.x * axis.z * omc - axis.y * s, axis.y * axis.z * omc + axis.x * s,
                            axis.z * axis.z * omc + c)));
}

/* generate.h:420-433 */
static float base_strand_length(Asset a, const Deformed *d, const Params *p, const State *s) {
    V3 prev = evaluate_base_strand_cv(a, d, p, s, 0u);
    float length = 0.0f;
    for (uint32_t cv = 1u; cv < p->cvs_per_strand; ++cv) {
        const V3 cur = evaluate_base_strand_cv(a, d, p, s, cv);
        length += sqrtf(len2(sub(cur, prev)));
        prev = cur;
    }
    return length;
}

/* generate.h:435-443 */
typedef struct {
    uint32_t cv;
    V3 previous_base, current_base, next_base, tangent, transported_normal;
    float arc_length;
} Cursor;

/* generate.h:445-457 */
static Cursor make_noise_cursor(Asset a, const Deformed *d, const Params *p, const State *s) {
    Cursor c;
    memset(&c, 0, sizeof c);
    c.current_base = evaluate_base_strand_cv(a, d, p, s, 0u);
    c.previous_base = c.current_base;
    c.next_base = evaluate_base_strand_cv(a, d, p, s, 1u);
    c.tangent = s->root.normal;
    c.transported_normal = s->surface_u;
    return c;
}

/* generate.h:459-515 */
static V3 evaluate_and_advance_noise_cursor(Asset a, const Deformed *d, const Params *p, const State *s, Cursor *c) {
    if (c->cv > 0u) c->arc_length += sqrtf(len2(sub(c->current_base, c->previous_base)));
    V3 next_tangent = c->tangent;
    if (c->cv + 1u < p->cvs_per_strand) {
        const V3 segment = sub(c->next_base, c->current_base);
        if (len2(segment) > 0.0f) next_tangent = normalize(segment);
    }
    const V3 axis = cross(c->tangent, next_tangent);
    if (len2(axis) > 0.0f) {
        const float angle = acosf(clamp_(dot(c->tangent, next_tangent), -1.0f, 1.0f));
        c->transported_normal = normalize(rotate_by(c->transported_normal, axis, angle));
    }
    const V3 normal = c->transported_normal;
    const V3 binormal = cross(normal, next_tangent);
    const V3 tangent = cross(binormal, normal);
    V3 point = c->current_base;
    if (c->cv > 0u) {
        const float distance = c->arc_length * s->effective_noise_frequency;
        const float magnitude = p->noise_mask * p->noise_amplitude * strand_parameter(p, c->cv);
        const V3 dom = s->noise_domain;
        const V3 local = v3(
            (gradient_noise(a, v3(dom.x + distance, dom.y, dom.z)) - 0.5f) * magnitude,
            (gradient_noise(a, v3(dom.x, dom.y + distance, dom.z)) - 0.5f) * magnitude,
            (gradient_noise(a, v3(dom.x, dom.y, dom.z + distance)) - 0.5f) * magnitude);
        point = add(add(add(point, mul(normal, local.x)), mul(binormal, local.y)), mul(tangent, local.z));
    }
    c->tangent = next_tangent;
    c->previous_base = c->current_base;
    if (c->cv + 1u < p->cvs_per_strand) {
        c->current_base = c->next_base;
        if (c->cv + 2u < p->cvs_per_strand) {
            c->next_base = evaluate_base_strand_cv(a, d, p, s, c->cv + 2u);
        }
    }
    ++c->cv;
    return point;
}

/* generate.h:517-532 */
static float noisy_strand_length(Asset a, const Deformed *d, const Params *p, const State *s) {
    Cursor c = make_noise_cursor(a, d, p, s);
    V3 prev = evaluate_and_advance_noise_cursor(a, d, p, s, &c);
    float length = 0.0f;
    for (uint32_t cv = 1u; cv < p->cvs_per_strand; ++cv) {
        const V3 cur = evaluate_and_advance_noise_cursor(a, d, p, s, &c);
        length += sqrtf(len2(sub(cur, prev)));
        prev = cur;
    }
    return length;
}

/* generate.h:534-566 */
static State make_state_from_root(Asset a, const Deformed *d, const Params *p, Root root) {
    State s;
    memset(&s, 0, sizeof s);
    s.preserve_scale = 1.0f;
    s.root = root;
    s.blend = make_guide_blend_state(a, d, p, &s.root);
    if (noise_is_enabled(p)) {
        s.surface_u = root_surface_u(a, d, &s.root);
        s.original_length = base_strand_length(a, d, p, &s);
        s.effective_noise_frequency = s.original_length > 0.0f
            ? fmax_(0.5f / s.original_length, p->noise_frequency) : p->noise_frequency;
        const float decorrelation = 1.0f - p->noise_correlation;
        const float domain_scale = 100.0f * decorrelation * decorrelation;
        s.noise_domain = mul(add(rest_root_position(a, &s.root), v3(0.419276f, 0.184247f, 0.805721f)),
                             domain_scale);
        if (p->noise_preserve_length > 0.001f) {
            const float noisy = noisy_strand_length(a, d, p, &s);
            if (noisy > 0.0f) {
                const float target = s.original_length * p->noise_preserve_length +
                                     noisy * (1.0f - p->noise_preserve_length);
                if (fabs_(noisy - target) >= 0.0001f) s.preserve_scale = target / noisy;
            }
        }
    }
    return s;
}

/* generate.h:577-581 */
static inline float evaluate_strand_width(const Params *p, uint32_t cv) {
    const float t = strand_parameter(p, cv);
    return p->root_width * (1.0f - t) + p->tip_width * t;
}

typedef struct { float x, y, z, radius; } Packed;

/* generate.h:612-642; `slot` is where this strand's records land in the outputs. */
static void generate_packed_strand(Asset a, const Params *p, uint32_t strand, uint64_t slot,
                                   Packed *points, Root *roots, V2 *root_uvs, uint32_t *counts,
                                   float radius_scale, const Deformed *d) {
    const State s = make_state_from_root(a, d, p, sample_root(a, d, p, strand));
    const int noise = noise_is_enabled(p);
    if (roots) roots[slot] = s.root;
    if (root_uvs) root_uvs[slot] = s.root.uv;
    if (counts) counts[slot] = p->cvs_per_strand;
    Cursor c;
    memset(&c, 0, sizeof c);
    if (noise) c = make_noise_cursor(a, d, p, &s);
    for (uint32_t cv = 0u; cv < p->cvs_per_strand; ++cv) {
        V3 point = noise ? evaluate_and_advance_noise_cursor(a, d, p, &s, &c)
                         : evaluate_base_strand_cv(a, d, p, &s, cv);
        if (s.preserve_scale != 1.0f) {
            point = add(s.root.position, mul(sub(point, s.root.position), s.preserve_scale));
        }
        const float width = evaluate_strand_width(p, cv);
        const uint64_t index = slot * p->cvs_per_strand + cv;
        Packed out = {point.x, point.y, point.z, 0.5f * width * radius_scale};
        points[index] = out;
    }
}

/* ------------------------------------------------------------------------ */
/* Exported C entry points (ctypes).                                         */
/* ------------------------------------------------------------------------ */

float orc_random01(uint32_t seed, uint32_t strand, uint32_t dim) { return random01(seed, strand, dim); }

float orc_gradient_noise(const void *asset, float x, float y, float z) {
    return gradient_noise(asset_of(asset), v3(x, y, z));
}

uint32_t orc_noise_hash(int32_t x, int32_t y, int32_t z) { return noise_hash(x, y, z); }

void orc_strand_state(const void *asset, const V3 *def_positions, const V3 *def_normals,
                      const V3 *def_guide_cvs, const Params *p, uint32_t strand, StrandState *out) {
    const Asset a = asset_of(asset);
    const Deformed d = {def_positions, def_normals, def_guide_cvs};
    const State s = make_state_from_root(a, &d, p, sample_root(a, &d, p, strand));
    out->root = s.root;
    memcpy(out->indices, s.blend.indices, sizeof out->indices);
    memcpy(out->weights, s.blend.weights, sizeof out->weights);
    out->weight_sum = s.blend.weight_sum;
    out->nearest = s.blend.nearest;
    out->surface_u = s.surface_u;
    out->noise_domain = s.noise_domain;
    out->original_length = s.original_length;
    out->effective_noise_frequency = s.effective_noise_frequency;
    out->preserve_scale = s.preserve_scale;
}

/* FNV-1a 64, src/asset.cpp:34-41 */
uint64_t orc_fnv1a(const void *bytes, uint64_t size) {
    const unsigned char *b = (const unsigned char *)bytes;
    uint64_t hash = 1469598103934665603ull;
    for (uint64_t i = 0; i < size; ++i) {
        hash ^= b[i];
        hash *= 1099511628211ull;
    }
    return hash;
}

static int section_fits(const Header *h, uint64_t offset, uint64_t count, uint64_t elem) {
    /* src/asset.cpp:152-158 */
    if (count == 0u) return offset == 0u;
    if (offset < sizeof(Header) || offset > h->byte_size) return 0;
    return count * elem <= h->byte_size - offset;
}

/* src/asset.cpp:295-338.  Returns 0 when valid, else writes the reference's message. */
int orc_validate_asset(const void *bytes, uint64_t size, char *msg, uint64_t cap) {
    const char *err = NULL;
    Header h;
    if (size < sizeof(Header)) { err = "blob is smaller than AssetHeader"; goto done; }
    if (((uintptr_t)bytes) % 64u != 0u) { err = "blob base is not 64-byte aligned"; goto done; }
    memcpy(&h, bytes, sizeof h);
    if (h.magic != 0x4e4547584f4e414eull) { err = "bad NanoXGen magic"; goto done; }
    if (h.version_major != 0u || h.version_minor != 2u) { err = "unsupported NanoXGen asset version"; goto done; }
    if (h.byte_size != size) { err = "header byte_size does not match file size"; goto done; }
    if (h.triangle_count == 0u || h.vertex_count == 0u || h.guide_count == 0u) { err = "required section is empty"; goto done; }
    if (h.guide_stencil_size != K_STENCIL) { err = "unsupported guide stencil size"; goto done; }
    if (h.noise_gradient_count != 256u) { err = "unsupported noise gradient table"; goto done; }
    if (!section_fits(&h, h.positions_offset, h.vertex_count, sizeof(V3)) ||
        !section_fits(&h, h.normals_offset, h.vertex_count, sizeof(V3)) ||
        !section_fits(&h, h.texcoords_offset, (h.flags & HAS_TEXCOORDS) ? h.vertex_count : 0u, sizeof(V2)) ||
        !section_fits(&h, h.triangles_offset, h.triangle_count, sizeof(U3)) ||
        !section_fits(&h, h.alias_table_offset, h.triangle_count, sizeof(AliasEntry)) ||
        !section_fits(&h, h.guides_offset, h.guide_count, sizeof(Guide)) ||
        !section_fits(&h, h.guide_cvs_offset, h.guide_cv_count, sizeof(V3)) ||
        !section_fits(&h, h.triangle_guides_offset, (uint64_t)h.triangle_count * h.guide_stencil_size,
                      sizeof(uint32_t)) ||
        !section_fits(&h, h.noise_gradients_offset, h.noise_gradient_count, sizeof(V3))) {
        err = "one or more sections are out of bounds";
        goto done;
    }
    if (orc_fnv1a((const unsigned char *)bytes + sizeof(Header), size - sizeof(Header)) != h.content_hash) {
        err = "content hash mismatch";
        goto done;
    }
    {
        const Asset a = asset_of(bytes);
        const U3 *tris = SECTION(a, U3, triangles_offset);
        for (uint32_t i = 0; i < h.triangle_count; ++i) {
            if (tris[i].x >= h.vertex_count || tris[i].y >= h.vertex_count || tris[i].z >= h.vertex_count) {
                err = "triangle index out of bounds";
                goto done;
            }
        }
        const Guide *guides = SECTION(a, Guide, guides_offset);
        for (uint32_t i = 0; i < h.guide_count; ++i) {
            const Guide *g = &guides[i];
            if (g->cv_count < 2u || g->first_cv > h.guide_cv_count ||
                g->cv_count > h.guide_cv_count - g->first_cv) {
                err = "guide CV range out of bounds";
                goto done;
            }
        }
    }
done:
    if (msg && cap) {
        snprintf(msg, (size_t)cap, "%s", err ? err : "");
    }
    return err ? 1 : 0;
}

/* Worker pool with atomically claimed strand tiles, the scheduling pattern of
 * src/asset.cpp:160-202 (results do not depend on the schedule). */
typedef struct {
    Asset a;
    const Params *p;
    const Deformed *d;
    const uint32_t *strands;   /* NULL: strands first..first+count-1 */
    uint32_t first, count, tile;
    Packed *points;
    Root *roots;
    V2 *root_uvs;
    uint32_t *counts;
    float radius_scale;
    atomic_uint next;
} Job;

static void *worker(void *arg) {
    Job *job = (Job *)arg;
    for (;;) {
        const uint32_t block = atomic_fetch_add_explicit(&job->next, 1u, memory_order_relaxed);
        const uint64_t begin = (uint64_t)block * job->tile;
        if (begin >= job->count) break;
        uint64_t end = begin + job->tile;
        if (end > job->count) end = job->count;
        for (uint64_t i = begin; i < end; ++i) {
            const uint32_t strand = job->strands ? job->strands[i] : job->first + (uint32_t)i;
            generate_packed_strand(job->a, job->p, strand, i, job->points, job->roots, job->root_uvs,
                                   job->counts, job->radius_scale, job->d);
        }
    }
    return NULL;
}

/* Generate `count` strands (the listed ids, or first..first+count-1) into
 * outputs indexed by list position.  Returns 0 on success. */
int orc_generate_packed(const void *asset, const Params *p, float radius_scale,
                        const V3 *def_positions, const V3 *def_normals, const V3 *def_guide_cvs,
                        const uint32_t *strands, uint32_t first, uint32_t count,
                        Packed *points, Root *roots, V2 *root_uvs, uint32_t *counts, int threads) {
    if (!asset || !p || !points || p->cvs_per_strand < 2u) return 1;
    Deformed d = {def_positions, def_normals, def_guide_cvs};
    Job job;
    job.a = asset_of(asset);
    job.p = p;
    job.d = &d;
    job.strands = strands;
    job.first = first;
    job.count = count;
    job.tile = 128u;
    job.points = points;
    job.roots = roots;
    job.root_uvs = root_uvs;
    job.counts = counts;
    job.radius_scale = radius_scale;
    atomic_init(&job.next, 0u);
    if (threads <= 1) {
        worker(&job);
        return 0;
    }
    if (threads > 256) threads = 256;
    pthread_t tids[256];
    int started = 0;
    for (int i = 0; i < threads; ++i) {
        if (pthread_create(&tids[i], NULL, worker, &job) != 0) break;
        ++started;
    }
    if (started == 0) worker(&job);
    for (int i = 0; i < started; ++i) pthread_join(tids[i], NULL);
    return 0;
}
