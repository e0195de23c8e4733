// stencil.cu -- the per-triangle guide stencil search of build_asset on sm_100a.
//
// For every triangle the reference (src/asset.cpp:252-269) scores each guide
// by |centroid - root|^2, plus 1e20 when the face normal and the guide's root
// normal disagree (dot < -0.25), and keeps the 8 smallest (score, guide)
// pairs in ascending order.  That is triangles x guides candidates (8.2e8 for
// a 200,000-triangle mesh with 4,096 guides), the only super-linear step of
// the asset build.
//
// Layout: one thread per triangle, 128-thread CTAs; the guide roots (one
// plane per axis) and normals stream through shared memory in tiles of
// kStencilTile guides, read by every lane at the same address (broadcast).
// The eight best candidates live in registers.  Scores use the exact
// helpers of strand_math.cuh (__f*_rn, never contracted), so they equal the
// host build's bit for bit, and the insertion replays the host's procedure
// (host.cpp build_stencils), so the rows are identical even for ties and
// non-finite scores.
//
// Rejection: a candidate whose |centroid - root|^2 alone is above the
// current eighth score cannot enter (the penalty only adds).  The kernel
// tests four guides at a time with packed f32x2 arithmetic (about ten
// issued instructions per candidate instead of twenty-three) and scores the
// rare group that passes exactly.
//
// guide_nearest_kernel, one warp per guide, finds each guide's nearest
// other root for the automatic support radius (guide_count^2 distances).
#include "generator_core.cuh"
#include "nxg_internal.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <cstdint>

namespace nxg {
namespace dev {
namespace {

constexpr uint32_t kStencilThreads = 128u;
constexpr uint32_t kTrianglesPerThread = 1u;
constexpr uint32_t kStencilTile = 512u;  // guides per shared-memory tile (14 KB)

struct Candidate {
    float key;
    uint32_t guide;
};

// std::pair<float, uint32_t>::operator<, as host.cpp candidate_less.
__device__ __forceinline__ bool candidate_less(float ak, uint32_t ag, float bk, uint32_t bg) {
    return ak < bk || (!(bk < ak) && ag < bg);
}

// The host's insertion step: the hole is at `hole`; entries move up while the
// new candidate orders before them, and it lands where that first fails.
// Unrolled over fixed indices so the list stays in registers.
__device__ __forceinline__ void insert_candidate(Candidate (&best)[kSlots], Candidate c, uint32_t hole) {
    bool moving = true;
#pragma unroll
    for (int k = static_cast<int>(kSlots) - 1; k >= 1; --k) {
        if (static_cast<uint32_t>(k) <= hole && moving) {
            if (candidate_less(c.key, c.guide, best[k - 1].key, best[k - 1].guide)) {
                best[k] = best[k - 1];
            } else {
                best[k] = c;
                moving = false;
            }
        }
    }
    if (moving) { best[0] = c; }
}

// Packed pairs of floats (sm_100a f32x2 arithmetic), half the issued
// instructions of the scalar form.  On the GPU their |d|^2 did not equal the
// scalar __f*_rn result bit for bit (tied guides came out in the wrong
// order), so they only filter: a group of guides is skipped when its
// smallest packed |d|^2, shrunk by kFilterMargin, still exceeds the eighth
// score, and every guide of a group that passes is scored again with the
// exact scalar helpers.  Both are sums of the same three squares of the
// same differences, so they can differ by rounding only (a few ulps, about
// 2^-21 relative); the margin is 2^-16, so no guide the host keeps is ever
// skipped, and a packed value that is too small only lets a group through.
typedef unsigned long long f32x2;
constexpr float kFilterMargin = 0.9999847412109375f;  // 1 - 2^-16

__device__ __forceinline__ f32x2 pair(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ float2 unpair(f32x2 v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

struct GuideTile {
    float x[kStencilTile], y[kStencilTile], z[kStencilTile];  // roots, one plane per axis
    float4 normal[kStencilTile];
};

// One candidate, exactly as the host: skip when |d|^2 alone already loses
// (the score is |d|^2 + 0 or 1e20 >= |d|^2), else score with the penalty and
// insert.  `hole` is the fill position while the list is not yet full.
__device__ __forceinline__ void consider(Candidate (&best)[kSlots], float l2, uint32_t gi, uint32_t count,
                                         F3 face, float4 m) {
    if (gi >= count && best[kSlots - 1].key < l2) { return; }
    const float penalty = xdot(face, F3{m.x, m.y, m.z}) < -0.25f ? 1.0e20f : 0.0f;
    const Candidate c{__fadd_rn(l2, penalty), gi};
    uint32_t hole = gi;
    if (gi >= count) {
        if (!candidate_less(c.key, c.guide, best[kSlots - 1].key, best[kSlots - 1].guide)) { return; }
        hole = kSlots - 1;
    }
    insert_candidate(best, c, hole);
}

__device__ __forceinline__ float root_distance2(F3 centroid, const GuideTile &t, uint32_t j) {
    const F3 d = xsub(centroid, F3{t.x[j], t.y[j], t.z[j]});
    return xdot(d, d);
}

// One triangle's search state, all in registers.
struct TriangleSearch {
    F3 centroid, face;
    f32x2 cx, cy, cz;  // the centroid's coordinates, each in both halves
    bool live;
    Candidate best[kSlots];
};

__device__ __forceinline__ void begin_triangle(TriangleSearch &t, uint32_t ti, const nxg_vec3 *__restrict__ positions,
                                               uint32_t vertex_count, const nxg_uint3 *__restrict__ triangles,
                                               uint32_t triangle_count, uint32_t *__restrict__ stencil) {
    t.live = ti < triangle_count;
    t.centroid = F3{0.0f, 0.0f, 0.0f};
    t.face = F3{0.0f, 1.0f, 0.0f};
    if (t.live) {
        const nxg_uint3 tri = triangles[ti];
        if (tri.x < vertex_count && tri.y < vertex_count && tri.z < vertex_count) {
            const nxg_vec3 a = positions[tri.x], b = positions[tri.y], c = positions[tri.z];
            const F3 p0{a.x, a.y, a.z}, p1{b.x, b.y, b.z}, p2{c.x, c.y, c.z};
            t.centroid = xdiv(xadd(xadd(p0, p1), p2), 3.0f);
            t.face = xnormalize(xcross(xsub(p1, p0), xsub(p2, p0)));
        } else {
            t.live = false;  // an out-of-range triangle keeps an all-invalid row
            uint4 *row = reinterpret_cast<uint4 *>(stencil + static_cast<size_t>(ti) * kSlots);
            row[0] = make_uint4(kInvalid, kInvalid, kInvalid, kInvalid);
            row[1] = make_uint4(kInvalid, kInvalid, kInvalid, kInvalid);
        }
    }
    t.cx = pair(t.centroid.x, t.centroid.x);
    t.cy = pair(t.centroid.y, t.centroid.y);
    t.cz = pair(t.centroid.z, t.centroid.z);
#pragma unroll
    for (uint32_t k = 0; k < kSlots; ++k) { t.best[k] = {0.0f, kInvalid}; }
}

// Guides j..j+3 of the tile for one triangle: packed |d|^2 of all four, and
// the group skipped when even its smallest one (less the margin) loses.  A
// NaN |d|^2 past the fill can never enter (its guide index is larger than
// every listed one), so fminf dropping it is exact.
__device__ __forceinline__ void consider_group(TriangleSearch &t, const GuideTile &tile, uint32_t j, uint32_t gi,
                                               uint32_t count, ulonglong2 gx, ulonglong2 gy, ulonglong2 gz) {
    const f32x2 dx0 = sub2(t.cx, gx.x), dx1 = sub2(t.cx, gx.y);
    const f32x2 dy0 = sub2(t.cy, gy.x), dy1 = sub2(t.cy, gy.y);
    const f32x2 dz0 = sub2(t.cz, gz.x), dz1 = sub2(t.cz, gz.y);
    const float2 a = unpair(add2(add2(mul2(dx0, dx0), mul2(dy0, dy0)), mul2(dz0, dz0)));
    const float2 b = unpair(add2(add2(mul2(dx1, dx1), mul2(dy1, dy1)), mul2(dz1, dz1)));
    const float low = fminf(fminf(a.x, a.y), fminf(b.x, b.y));
    if (t.best[kSlots - 1].key < low * kFilterMargin) { return; }
    // The group passed: each guide is checked on its own packed value before
    // its exact score (a warp runs a guide's exact path only when one of its
    // lanes needs it).
    const float packed[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
    for (uint32_t k = 0; k < 4u; ++k) {
        if (t.best[kSlots - 1].key < packed[k] * kFilterMargin) { continue; }
        consider(t.best, root_distance2(t.centroid, tile, j + k), gi + k, count, t.face, tile.normal[j + k]);
    }
}

__device__ __forceinline__ void end_triangle(const TriangleSearch &t, uint32_t ti, uint32_t keep,
                                             uint32_t *__restrict__ stencil) {
    if (!t.live) { return; }
    uint32_t out[kSlots];
#pragma unroll
    for (uint32_t k = 0; k < kSlots; ++k) { out[k] = k < keep ? t.best[k].guide : kInvalid; }
    uint4 *row = reinterpret_cast<uint4 *>(stencil + static_cast<size_t>(ti) * kSlots);
    row[0] = make_uint4(out[0], out[1], out[2], out[3]);
    row[1] = make_uint4(out[4], out[5], out[6], out[7]);
}

// One triangle per thread, 128-thread CTAs (56 registers, 9 CTAs per SM).
// Measured slower: two triangles per thread sharing each guide load (fewer
// warps per SM to hide the dependency chains), and a 40-register cap that
// fits a 200,000-triangle mesh in one wave (spills).
__global__ void __launch_bounds__(kStencilThreads)
stencil_kernel(const nxg_vec3 *__restrict__ positions, uint32_t vertex_count, const nxg_uint3 *__restrict__ triangles,
               uint32_t triangle_count, const nxg_vec3 *__restrict__ guide_roots,
               const nxg_vec3 *__restrict__ guide_normals, uint32_t guide_count, uint32_t keep,
               uint32_t *__restrict__ stencil) {
    __shared__ __align__(16) GuideTile tile;
    const uint32_t first = blockIdx.x * (kStencilThreads * kTrianglesPerThread) + threadIdx.x;
    TriangleSearch tri[kTrianglesPerThread];
#pragma unroll
    for (uint32_t q = 0; q < kTrianglesPerThread; ++q) {
        begin_triangle(tri[q], first + q * kStencilThreads, positions, vertex_count, triangles, triangle_count,
                       stencil);
    }
    bool any = false;
#pragma unroll
    for (uint32_t q = 0; q < kTrianglesPerThread; ++q) { any = any || tri[q].live; }
    const uint32_t count = guide_count < kSlots ? guide_count : kSlots;

    for (uint32_t base = 0; base < guide_count; base += kStencilTile) {
        const uint32_t n = guide_count - base < kStencilTile ? guide_count - base : kStencilTile;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n; i += kStencilThreads) {
            const nxg_vec3 r = guide_roots[base + i], m = guide_normals[base + i];
            tile.x[i] = r.x;
            tile.y[i] = r.y;
            tile.z[i] = r.z;
            tile.normal[i] = make_float4(m.x, m.y, m.z, 0.0f);
        }
        __syncthreads();
        if (!any) { continue; }
        // The first `count` guides fill the lists (tile 0 only; count <= 8).
        uint32_t j = base == 0u ? count : 0u;
        for (uint32_t f = 0; f < j; ++f) {
#pragma unroll
            for (uint32_t q = 0; q < kTrianglesPerThread; ++q) {
                if (tri[q].live) {
                    consider(tri[q].best, root_distance2(tri[q].centroid, tile, f), f, count, tri[q].face,
                             tile.normal[f]);
                }
            }
        }
        for (; j + 4u <= n; j += 4u) {
            const ulonglong2 gx = *reinterpret_cast<const ulonglong2 *>(&tile.x[j]);
            const ulonglong2 gy = *reinterpret_cast<const ulonglong2 *>(&tile.y[j]);
            const ulonglong2 gz = *reinterpret_cast<const ulonglong2 *>(&tile.z[j]);
#pragma unroll
            for (uint32_t q = 0; q < kTrianglesPerThread; ++q) {
                if (tri[q].live) { consider_group(tri[q], tile, j, base + j, count, gx, gy, gz); }
            }
        }
        for (; j < n; ++j) {
#pragma unroll
            for (uint32_t q = 0; q < kTrianglesPerThread; ++q) {
                if (tri[q].live) {
                    consider(tri[q].best, root_distance2(tri[q].centroid, tile, j), base + j, count, tri[q].face,
                             tile.normal[j]);
                }
            }
        }
    }
#pragma unroll
    for (uint32_t q = 0; q < kTrianglesPerThread; ++q) { end_triangle(tri[q], first + q * kStencilThreads, keep, stencil); }
}

// Distance from every guide root to its nearest other root (the automatic
// support radius, src/asset.cpp automatic_support_radius): |root_i - root_j|
// with IEEE sqrt, minimum over j != i with a CV count > 0.  One warp per
// guide, lanes striding over j, then a warp minimum: every distance is >= +0,
// a NaN one never replaces a lane's running value (which starts at FLT_MAX,
// as the host's), so the minimum is the host's whatever the order.
__global__ void __launch_bounds__(kStencilThreads)
guide_nearest_kernel(const nxg_vec3 *__restrict__ roots, const uint32_t *__restrict__ cv_counts, uint32_t guide_count,
                     float *__restrict__ nearest) {
    const uint32_t gi = (blockIdx.x * kStencilThreads + threadIdx.x) >> 5, lane = threadIdx.x & 31u;
    if (gi >= guide_count) { return; }  // whole warps
    const nxg_vec3 r = roots[gi];
    const F3 root{r.x, r.y, r.z};
    float best = 3.402823466e38f;  // FLT_MAX
    for (uint32_t j = lane; j < guide_count; j += 32u) {
        if (j == gi || cv_counts[j] == 0u) { continue; }
        const nxg_vec3 o = roots[j];
        const F3 d = xsub(root, F3{o.x, o.y, o.z});
        const float dist = __fsqrt_rn(xdot(d, d));
        best = dist < best ? dist : best;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) { best = fminf(best, __shfl_xor_sync(kFull, best, o)); }
    if (lane == 0u) { nearest[gi] = best; }
}

uint32_t slots_kept(uint32_t guide_count, uint32_t stencil_slots) {
    const uint32_t count = guide_count < kSlots ? guide_count : kSlots;
    return stencil_slots == 0u || stencil_slots > count ? count : stencil_slots;
}

cudaError_t launch_stencils(const nxg_vec3 *positions, uint32_t vertex_count, const nxg_uint3 *triangles,
                         uint32_t triangle_count, const nxg_vec3 *guide_roots, const nxg_vec3 *guide_normals,
                         uint32_t guide_count, uint32_t stencil_slots, uint32_t *stencil, cudaStream_t stream) {
    const uint32_t per_block = kStencilThreads * kTrianglesPerThread;
    const uint32_t blocks = (triangle_count + per_block - 1u) / per_block;
    stencil_kernel<<<blocks, kStencilThreads, 0, stream>>>(positions, vertex_count, triangles, triangle_count,
                                                           guide_roots, guide_normals, guide_count,
                                                           slots_kept(guide_count, stencil_slots), stencil);
    return cudaGetLastError();
}

size_t align256(size_t n) { return (n + 255u) & ~size_t{255u}; }

} // namespace
} // namespace dev

int device_guide_search(const nxg_vec3 *positions, uint32_t vertex_count, const nxg_uint3 *triangles,
                        uint32_t triangle_count, const nxg_vec3 *guide_roots, const nxg_vec3 *guide_normals,
                        const uint32_t *guide_cv_counts, uint32_t guide_count, uint32_t stencil_slots,
                        uint32_t *stencil, float *nearest, void *stream, const char **what) noexcept {
    using dev::align256;
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t vb = size_t{vertex_count} * sizeof(nxg_vec3), tb = size_t{triangle_count} * sizeof(nxg_uint3);
    const size_t gb = size_t{guide_count} * sizeof(nxg_vec3), sb = size_t{triangle_count} * NXG_GUIDE_STENCIL_SIZE * 4u;
    const size_t o_tri = align256(vb), o_root = o_tri + align256(tb), o_normal = o_root + align256(gb);
    const size_t cb = size_t{guide_count} * 4u, o_counts = o_normal + align256(gb);
    const size_t o_nearest = o_counts + align256(cb), o_stencil = o_nearest + align256(cb);
    const size_t total = o_stencil + align256(sb);
    char *base = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&base), total, s);
    if (e != cudaSuccess) {
        *what = cudaGetErrorString(e);
        set_last_cuda_error(static_cast<int32_t>(e));
        return static_cast<int>(e);
    }
    auto *d_pos = reinterpret_cast<nxg_vec3 *>(base);
    auto *d_tri = reinterpret_cast<nxg_uint3 *>(base + o_tri);
    auto *d_root = reinterpret_cast<nxg_vec3 *>(base + o_root);
    auto *d_normal = reinterpret_cast<nxg_vec3 *>(base + o_normal);
    auto *d_counts = reinterpret_cast<uint32_t *>(base + o_counts);
    auto *d_nearest = reinterpret_cast<float *>(base + o_nearest);
    auto *d_stencil = reinterpret_cast<uint32_t *>(base + o_stencil);
    if ((e = cudaMemcpyAsync(d_pos, positions, vb, cudaMemcpyHostToDevice, s)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d_tri, triangles, tb, cudaMemcpyHostToDevice, s)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d_root, guide_roots, gb, cudaMemcpyHostToDevice, s)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d_normal, guide_normals, gb, cudaMemcpyHostToDevice, s)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d_counts, guide_cv_counts, cb, cudaMemcpyHostToDevice, s)) == cudaSuccess) {
        const uint64_t threads = uint64_t{guide_count} * 32u;
        const uint32_t blocks = static_cast<uint32_t>((threads + dev::kStencilThreads - 1u) / dev::kStencilThreads);
        dev::guide_nearest_kernel<<<blocks, dev::kStencilThreads, 0, s>>>(d_root, d_counts, guide_count, d_nearest);
        if ((e = cudaGetLastError()) == cudaSuccess &&
            (e = dev::launch_stencils(d_pos, vertex_count, d_tri, triangle_count, d_root, d_normal, guide_count,
                                      stencil_slots, d_stencil, s)) == cudaSuccess &&
            (e = cudaMemcpyAsync(nearest, d_nearest, cb, cudaMemcpyDeviceToHost, s)) == cudaSuccess) {
            e = cudaMemcpyAsync(stencil, d_stencil, sb, cudaMemcpyDeviceToHost, s);
        }
    }
    const cudaError_t freed = cudaFreeAsync(base, s);
    const cudaError_t synced = cudaStreamSynchronize(s);
    if (e == cudaSuccess) { e = freed != cudaSuccess ? freed : synced; }
    if (e != cudaSuccess) {
        *what = cudaGetErrorString(e);
        set_last_cuda_error(static_cast<int32_t>(e));
        return static_cast<int>(e);
    }
    return 0;
}

} // namespace nxg

extern "C" uint32_t nxg_build_stencils_device(const nxg_vec3 *positions, uint32_t vertex_count,
                                              const nxg_uint3 *triangles, uint32_t triangle_count,
                                              const nxg_vec3 *guide_roots, const nxg_vec3 *guide_normals,
                                              uint32_t guide_count, uint32_t stencil_slots, uint32_t *stencil,
                                              void *stream) {
    if (!positions || !triangles || !guide_roots || !guide_normals || !stencil || vertex_count == 0u ||
        triangle_count == 0u || guide_count == 0u || stencil_slots > NXG_GUIDE_STENCIL_SIZE) {
        return NXG_ERROR_INVALID_ARGUMENT;
    }
    if (reinterpret_cast<uintptr_t>(stencil) % 16u != 0u) { return NXG_ERROR_MISALIGNED_OUTPUT; }
    nxg::set_last_cuda_error(0);
    return nxg::record_cuda(nxg::dev::launch_stencils(positions, vertex_count, triangles, triangle_count, guide_roots,
                                                      guide_normals, guide_count, stencil_slots, stencil,
                                                      static_cast<cudaStream_t>(stream)));
}
