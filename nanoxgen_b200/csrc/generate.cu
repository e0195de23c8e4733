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
//                        so one CTA's strands read the same guide CVs from L1;
//   4. generate        : persistent CTAs walk contiguous ranges of the
//                        permutation; a group of L lanes owns one strand and
//                        each lane owns CVs c*L + lane.  Stencil slots are
//                        evaluated one per lane and staged in shared memory,
//                        the base curve, arc length, transported frame and
//                        gradient noise are computed lane-parallel (prefix
//                        scans over shuffles replace the reference's serial
//                        cursor), and float4 points leave as coalesced
//                        streaming stores.
// Strands longer than 128 CVs take a serial per-thread kernel that walks the
// reference's cursor directly.
#include "nxg_internal.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <algorithm>
#include <cstring>

namespace nxg {
namespace dev {

struct LaunchArgs {
    AssetArgs a;
    FrameArgs f;
    ParamArgs p;
    uint32_t first_strand;   // global id of output record 0
    uint32_t count;          // strands in this launch
    float4 *points;
    uint32_t *roots;         // 12 words per strand, or nullptr
    float2 *root_uvs;
    uint32_t *point_counts;
    const uint32_t *order;   // permutation of [0, count), or nullptr for identity
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

// One strand on an L-lane group; see the file comment for the layout.
template <int L, int PPT, bool NOISE>
__device__ __forceinline__ void process_strand(const LaunchArgs &g, uint32_t local, bool active, int gl,
                                               Slot *slots, const float4 *table) {
    const AssetArgs &a = g.a;
    const FrameArgs &f = g.f;
    const ParamArgs &p = g.p;
    const uint32_t P = p.cvs_per_strand;
    const uint32_t strand = g.first_strand + local;

    const Root root = sample_root(a, f, p.seed, strand);
    if (gl < static_cast<int>(kSlots)) { slots[gl] = eval_slot(a, f, p, root, static_cast<uint32_t>(gl)); }
    __syncwarp();

    // Blend state (generate.h:214-244): weight sum in slot order, nearest
    // eligible guide by strict first minimum.
    float wsum = 0.0f;
    float nearest_d2 = FLT_MAX;
    int nearest = -1;
    uint32_t blended = 0u;
#pragma unroll
    for (uint32_t j = 0; j < kSlots; ++j) {
        const uint32_t flags = slots[j].flags;
        const float d2 = slots[j].d2;
        if (flags & kSlotEligible) {
            if (d2 < nearest_d2) {
                nearest_d2 = d2;
                nearest = static_cast<int>(j);
            }
        }
        if (flags & kSlotBlended) {
            wsum = __fadd_rn(wsum, slots[j].w);
            blended |= 1u << j;
        }
    }

    // Base curve (generate.h:246-267, :300-310).
    float tcv[PPT];
    F3 base[PPT];
#pragma unroll
    for (int c = 0; c < PPT; ++c) {
        const uint32_t cv = static_cast<uint32_t>(c * L + gl);
        tcv[c] = cv < P ? __fdiv_rn(static_cast<float>(cv), static_cast<float>(P - 1u)) : 1.0f;
        base[c] = F3{0.0f, 0.0f, 0.0f};
    }
    if (wsum > 1.0e-12f) {
#pragma unroll
        for (uint32_t j = 0; j < kSlots; ++j) {
            if (blended & (1u << j)) {
                const Slot s = slots[j];
#pragma unroll
                for (int c = 0; c < PPT; ++c) { base[c] = base[c] + guide_offset(f.guide_cvs, s, tcv[c]) * s.w; }
            }
        }
        const float inv = 1.0f / wsum;
#pragma unroll
        for (int c = 0; c < PPT; ++c) { base[c] = base[c] * inv; }
    } else if (nearest >= 0) {
        const Slot s = slots[nearest];
#pragma unroll
        for (int c = 0; c < PPT; ++c) { base[c] = guide_offset(f.guide_cvs, s, tcv[c]); }
    } else {
#pragma unroll
        for (int c = 0; c < PPT; ++c) { base[c] = root.normal * tcv[c]; }
    }
#pragma unroll
    for (int c = 0; c < PPT; ++c) { base[c] = root.position + base[c] * p.length_scale; }

    float4 *out = g.points + static_cast<uint64_t>(local) * P;

    if constexpr (!NOISE) {
#pragma unroll
        for (int c = 0; c < PPT; ++c) {
            const uint32_t cv = static_cast<uint32_t>(c * L + gl);
            if (active && cv < P) {
                __stcs(out + cv, make_float4(base[c].x, base[c].y, base[c].z, strand_radius(p, tcv[c])));
            }
        }
    } else {
        const F3 surface_u = root_surface_u(a, f, root);
        // Arc length: inclusive prefix of segment lengths (generate.h:420-433, :465-468).
        float arc[PPT];
        float carry = 0.0f;
#pragma unroll
        for (int c = 0; c < PPT; ++c) {
            const uint32_t cv = static_cast<uint32_t>(c * L + gl);
            const F3 up = group_shfl_up<L>(base[c], 1);
            const F3 prev_chunk = c > 0 ? group_shfl<L>(base[c > 0 ? c - 1 : 0], L - 1) : base[c];
            const F3 pb = gl > 0 ? up : prev_chunk;
            const F3 d = base[c] - pb;
            const float seg = (cv >= 1u && cv < P) ? sqrtf(dot(d, d)) : 0.0f;
            const float inc = group_scan_add<L>(seg, gl) + carry;
            arc[c] = inc;
            carry = group_shfl<L>(inc, L - 1);
        }
        const float original_length = carry;
        const float f_eff = original_length > 0.0f ? fmaxf(0.5f / original_length, p.noise_frequency)
                                                   : p.noise_frequency;
        const float decorrelation = 1.0f - p.noise_correlation;
        const float domain_scale = 100.0f * decorrelation * decorrelation;
        const F3 domain = (rest_root_position(a, root) + F3{0.419276f, 0.184247f, 0.805721f}) * domain_scale;

        // Tangent after CV k: the next segment's direction, carried forward over
        // zero-length segments and at the tip (generate.h:470-474).
        F3 cand[PPT];
        F3 tan[PPT];
        int last_valid = -1;
#pragma unroll
        for (int c = 0; c < PPT; ++c) {
            const uint32_t cv = static_cast<uint32_t>(c * L + gl);
            const F3 dn = group_shfl_down<L>(base[c], 1);
            const F3 next_chunk = c + 1 < PPT ? group_shfl<L>(base[c + 1 < PPT ? c + 1 : c], 0) : base[c];
            const F3 nb = gl < L - 1 ? dn : next_chunk;
            const F3 e = xsub(nb, base[c]);
            const bool valid = (cv + 1u < P) && xdot(e, e) > 0.0f;
            cand[c] = valid ? xnormalize(e) : F3{0.0f, 0.0f, 0.0f};
            const int jv = valid ? static_cast<int>(cv) : -1;
            const int jm = max(group_scan_max<L>(jv, gl), last_valid);
            last_valid = __shfl_sync(kFull, jm, L - 1, L);
            F3 sel = root.normal;
#pragma unroll
            for (int c2 = 0; c2 <= c; ++c2) {
                const F3 v = group_shfl<L>(cand[c2], jm & (L - 1));
                if (jm >= 0 && jm / L == c2) { sel = v; }
            }
            tan[c] = sel;
        }

        // Transported normal: N_k = normalize(M_k ... M_0 surface_u), with M_k the
        // reference's rotate_by matrix (generate.h:475-481); the product of the
        // per-CV matrices is an inclusive scan across lanes and chunks.
        F3 normal[PPT];
        M3 carry_m = identity3();
#pragma unroll
        for (int c = 0; c < PPT; ++c) {
            const uint32_t cv = static_cast<uint32_t>(c * L + gl);
            const F3 up = group_shfl_up<L>(tan[c], 1);
            const F3 prev_chunk = c > 0 ? group_shfl<L>(tan[c > 0 ? c - 1 : 0], L - 1) : root.normal;
            const F3 tp = gl > 0 ? up : prev_chunk;
            const F3 axis = xcross(tp, tan[c]);
            M3 m = identity3();
            if (cv < P && xdot(axis, axis) > 0.0f) {
                const float angle = acosf(fminf(fmaxf(dot(tp, tan[c]), -1.0f), 1.0f));
                m = rotation3(axis, angle);
            }
            M3 q = group_scan_mat<L>(m, gl);
            q = mul3(q, carry_m);
            carry_m = group_shfl<L>(q, L - 1);
            normal[c] = normalize(apply3(q, surface_u));
        }

        // Displacement in the transported frame (generate.h:482-502).
        const float magnitude_scale = p.noise_mask * p.noise_amplitude;
        F3 point[PPT];
#pragma unroll
        for (int c = 0; c < PPT; ++c) {
            const uint32_t cv = static_cast<uint32_t>(c * L + gl);
            F3 q = base[c];
            if (cv > 0u && cv < P) {
                const F3 n = normal[c];
                const F3 b = cross(n, tan[c]);
                const F3 t = cross(b, n);
                const float distance = arc[c] * f_eff;
                const float magnitude = magnitude_scale * tcv[c];
                const float lx = (gradient_noise(table, domain.x + distance, domain.y, domain.z) - 0.5f) * magnitude;
                const float ly = (gradient_noise(table, domain.x, domain.y + distance, domain.z) - 0.5f) * magnitude;
                const float lz = (gradient_noise(table, domain.x, domain.y, domain.z + distance) - 0.5f) * magnitude;
                q = q + n * lx + b * ly + t * lz;
            }
            point[c] = q;
        }

        // preserveLength (generate.h:553-563), from the noisy points already in
        // registers instead of a second cursor pass.
        float scale = 1.0f;
        if (p.noise_preserve_length > 0.001f) {
            float partial = 0.0f;
#pragma unroll
            for (int c = 0; c < PPT; ++c) {
                const uint32_t cv = static_cast<uint32_t>(c * L + gl);
                const F3 up = group_shfl_up<L>(point[c], 1);
                const F3 prev_chunk = c > 0 ? group_shfl<L>(point[c > 0 ? c - 1 : 0], L - 1) : point[c];
                const F3 pb = gl > 0 ? up : prev_chunk;
                const F3 d = point[c] - pb;
                partial += (cv >= 1u && cv < P) ? sqrtf(dot(d, d)) : 0.0f;
            }
            const float noisy = group_sum<L>(partial);
            if (noisy > 0.0f) {
                const float target = original_length * p.noise_preserve_length +
                                     noisy * (1.0f - p.noise_preserve_length);
                if (fabsf(noisy - target) >= 0.0001f) { scale = target / noisy; }
            }
        }
#pragma unroll
        for (int c = 0; c < PPT; ++c) {
            const uint32_t cv = static_cast<uint32_t>(c * L + gl);
            F3 q = point[c];
            if (scale != 1.0f) { q = root.position + (q - root.position) * scale; }
            if (active && cv < P) { __stcs(out + cv, make_float4(q.x, q.y, q.z, strand_radius(p, tcv[c]))); }
        }
    }

    if (active) {
        if (g.roots && gl < 12) { g.roots[static_cast<uint64_t>(local) * 12u + gl] = root_word(root, gl); }
        if (gl == 0) {
            if (g.root_uvs) { g.root_uvs[local] = make_float2(root.u, root.v); }
            if (g.point_counts) { g.point_counts[local] = P; }
        }
    }
}

template <int L, int PPT, bool NOISE>
__global__ void generate_kernel(LaunchArgs g) {
    extern __shared__ float4 smem[];
    float4 *table = smem;
    Slot *all_slots = reinterpret_cast<Slot *>(smem + kTableFloat4);
    if constexpr (NOISE) {
        for (int i = threadIdx.x; i < kTableFloat4; i += blockDim.x) {
            table[i] = make_float4(__ldg(g.a.gradients + 3 * i), __ldg(g.a.gradients + 3 * i + 1),
                                   __ldg(g.a.gradients + 3 * i + 2), 0.0f);
        }
        __syncthreads();
    }
    constexpr int kGroups = 32 / L;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int warps = blockDim.x >> 5;
    const int group = lane / L;
    const int gl = lane % L;
    Slot *slots = all_slots + (warp * kGroups + group) * kSlots;
    const uint32_t begin = static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x) * g.count / gridDim.x);
    const uint32_t end = static_cast<uint32_t>(static_cast<uint64_t>(blockIdx.x + 1u) * g.count / gridDim.x);
    for (uint32_t base = begin + static_cast<uint32_t>(warp * kGroups); base < end;
         base += static_cast<uint32_t>(warps * kGroups)) {
        const uint32_t item = base + static_cast<uint32_t>(group);
        bool active = item < end;
        const uint32_t pick = active ? item : begin;
        uint32_t local = g.order ? __ldg(g.order + pick) : pick;
        if (local >= g.count) {
            local = 0u;
            active = false;
        }
        process_strand<L, PPT, NOISE>(g, local, active, gl, slots, table);
        __syncwarp();
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
        float4 *out = g.points + static_cast<uint64_t>(local) * P;
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
                out[cv] = make_float4(q.x, q.y, q.z, strand_radius(p, t));
            }
        } else {
            for (uint32_t cv = 0u; cv < P; ++cv) {
                const F3 q = serial_base_cv(g, root, slots, wsum, nearest, cv);
                const float t = __fdiv_rn(static_cast<float>(cv), static_cast<float>(P - 1u));
                out[cv] = make_float4(q.x, q.y, q.z, strand_radius(p, t));
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

} // namespace dev

namespace {

using dev::LaunchArgs;

constexpr uint64_t kWorkspaceAlign = 256u;
inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1u) / a * a; }

struct WorkspaceLayout {
    uint64_t keys, order, hist, total;
};

WorkspaceLayout workspace_layout(uint32_t guide_count, uint32_t count) {
    WorkspaceLayout w{};
    w.keys = 0u;
    w.order = align_up(uint64_t{count} * 4u, kWorkspaceAlign);
    w.hist = w.order + align_up(uint64_t{count} * 4u, kWorkspaceAlign);
    w.total = w.hist + align_up((uint64_t{guide_count} + 1u) * 4u, kWorkspaceAlign);
    return w;
}

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

using KernelFn = void (*)(LaunchArgs);

template <int L, int PPT>
KernelFn pick_noise(bool noise) {
    return noise ? dev::generate_kernel<L, PPT, true> : dev::generate_kernel<L, PPT, false>;
}

// Tile shape for P CVs: the narrowest power-of-two lane group that holds the
// strand in one chunk, else 32 lanes with up to 4 CVs per lane.
KernelFn pick_kernel(uint32_t P, bool noise, int *lanes) {
    if (P <= 8u) { *lanes = 8; return pick_noise<8, 1>(noise); }
    if (P <= 16u) { *lanes = 16; return pick_noise<16, 1>(noise); }
    *lanes = 32;
    if (P <= 32u) { return pick_noise<32, 1>(noise); }
    if (P <= 64u) { return pick_noise<32, 2>(noise); }
    if (P <= 96u) { return pick_noise<32, 3>(noise); }
    if (P <= 128u) { return pick_noise<32, 4>(noise); }
    return nullptr;
}

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

uint32_t check_workspace(const nxg_device_asset_desc &asset, uint32_t count, const void *workspace,
                         uint64_t workspace_bytes) {
    const WorkspaceLayout ws = workspace_layout(asset.header.guide_count, count);
    if (!workspace || workspace_bytes < ws.total) { return NXG_ERROR_WORKSPACE_TOO_SMALL; }
    if (reinterpret_cast<std::uintptr_t>(workspace) % kWorkspaceAlign != 0u) { return NXG_ERROR_MISALIGNED_OUTPUT; }
    return NXG_ERROR_NONE;
}

// Counting sort of strands [first, first + count) by their triangle's first
// stencil guide; leaves the permutation in the workspace's order section.
uint32_t launch_order(const nxg_device_asset_desc &asset, uint32_t seed, uint32_t first, uint32_t count,
                      void *workspace, cudaStream_t stream) {
    const WorkspaceLayout ws = workspace_layout(asset.header.guide_count, count);
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
    dev::scatter_order_kernel<<<blocks, threads, 0, stream>>>(keys, hist, count, bins, order);
    return record_cuda(cudaGetLastError());
}

// The generator over a strand order (the workspace's, or identity when
// `workspace` is null).
uint32_t launch_generate(const nxg_device_asset_desc &asset, const nxg_deformed_desc &deformed,
                         const nxg_generation_params &params, const nxg_packed_output_desc &output,
                         const nxg_launch_config &config, uint32_t first, uint32_t count, const void *workspace,
                         cudaStream_t stream) {
    set_last_cuda_error(0);
    LaunchArgs g{};
    g.a = resolve_asset(asset);
    g.f = resolve_frame(g.a, deformed);
    g.p = resolve_params(params, output.radius_scale);
    g.first_strand = first;
    g.count = count;
    g.points = reinterpret_cast<float4 *>(output.points);
    g.roots = reinterpret_cast<uint32_t *>(output.roots);
    g.root_uvs = reinterpret_cast<float2 *>(output.root_uvs);
    g.point_counts = output.point_counts;
    g.order = workspace ? reinterpret_cast<const uint32_t *>(static_cast<const unsigned char *>(workspace) +
                                                             workspace_layout(asset.header.guide_count, count).order)
                        : nullptr;
    const int sms = device_sm_count();
    uint32_t status = NXG_ERROR_NONE;
    const uint32_t block = std::max<uint32_t>(32u, (config.block_size + 31u) / 32u * 32u);
    int lanes = 32;
    KernelFn fn = pick_kernel(params.cvs_per_strand, g.p.noise != 0u, &lanes);
    if (!fn) {
        const uint32_t threads = 128u;
        const uint32_t blocks = static_cast<uint32_t>(std::min<uint64_t>((count + threads - 1u) / threads,
                                                                          static_cast<uint64_t>(sms) * 8u));
        dev::generate_serial_kernel<<<blocks, threads, 0, stream>>>(g);
        return record_cuda(cudaGetLastError());
    }
    const uint32_t warps = block / 32u;
    const uint32_t groups = warps * static_cast<uint32_t>(32 / lanes);
    const size_t shm = sizeof(float4) * dev::kTableFloat4 + sizeof(dev::Slot) * dev::kSlots * groups;
    if (shm > 48u * 1024u) {
        if ((status = record_cuda(cudaFuncSetAttribute(reinterpret_cast<const void *>(fn),
                                                       cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(shm))))) {
            return status;
        }
    }
    int per_sm = 0;
    if ((status = record_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
             &per_sm, reinterpret_cast<const void *>(fn), static_cast<int>(block), shm)))) {
        return status;
    }
    per_sm = std::max(per_sm, 1);
    const uint64_t needed = (uint64_t{count} + groups - 1u) / groups;
    const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(needed, static_cast<uint64_t>(sms) * per_sm));
    fn<<<grid, block, shm, stream>>>(g);
    return record_cuda(cudaGetLastError());
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

} // namespace
} // namespace nxg

extern "C" {

uint64_t nxg_packed_workspace_size(const nxg_device_asset_desc *asset, uint32_t strand_count) {
    if (!asset || strand_count == 0u) { return 0u; }
    return nxg::workspace_layout(asset->header.guide_count, strand_count).total;
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
    if ((error = nxg::check_workspace(*asset, strand_count, workspace, workspace_bytes)) != NXG_ERROR_NONE) {
        return error;
    }
    const auto s = static_cast<cudaStream_t>(stream);
    nxg::set_last_cuda_error(0);
    if ((error = nxg::launch_order(*asset, params->seed, first_strand, strand_count, workspace, s))) { return error; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    return nxg::launch_generate(*asset, deformed ? *deformed : none, *params, *output,
                                config ? *config : default_config, first_strand, strand_count, workspace, s);
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
    if ((error = nxg::check_workspace(*asset, strand_count, workspace, workspace_bytes)) != NXG_ERROR_NONE) {
        return error;
    }
    nxg::set_last_cuda_error(0);
    return nxg::launch_order(*asset, params->seed, first_strand, strand_count, workspace,
                             static_cast<cudaStream_t>(stream));
}

uint32_t nxg_generate_packed_ordered(const nxg_device_asset_desc *asset, const nxg_deformed_desc *deformed,
                                     const nxg_generation_params *params, const nxg_packed_output_desc *output,
                                     const nxg_launch_config *config, uint32_t first_strand,
                                     uint32_t strand_count, const void *workspace, uint64_t workspace_bytes,
                                     void *stream) {
    uint32_t error =
        nxg::validate_range_request(asset, deformed, params, output, config, first_strand, strand_count);
    if (error != NXG_ERROR_NONE) { return error; }
    if ((error = nxg::check_launch_inputs(*asset, output)) != NXG_ERROR_NONE) { return error; }
    if (strand_count == 0u) { return NXG_ERROR_NONE; }
    if (workspace &&
        (error = nxg::check_workspace(*asset, strand_count, workspace, workspace_bytes)) != NXG_ERROR_NONE) {
        return error;
    }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    return nxg::launch_generate(*asset, deformed ? *deformed : none, *params, *output,
                                config ? *config : default_config, first_strand, strand_count, workspace,
                                static_cast<cudaStream_t>(stream));
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

} // extern "C"
