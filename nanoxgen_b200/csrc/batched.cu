// batched.cu -- many descriptions in one persistent generate launch.
//
// A frame of several descriptions (each its own .nxg asset, strand count,
// CV count, stencil and noise settings) is generated by:
//   batched_clear      zero the per-description bins and the work counter;
//   batched_prepare    one pass over every strand of every description:
//                      root triangle, sort key (first stencil guide) with its
//                      histogram, and for lane-group descriptions the
//                      RootSample / root UV / point count outputs (lane-walk
//                      items write theirs in batched_generate);
//   batched_scan       one CTA per description: bin offsets;
//   batched_scatter    per-description strand-locality orders (ranks in
//                      shared memory, one global atomic per block and bin);
//   batched_offsets    every description's guide-offset table and guide
//                      frame records;
//   batched_generate   one launch per class of work item -- noisy
//                      lane-walk items, noise-free items, noisy lane-group
//                      items -- each with the CTA shape, shared memory and
//                      register budget of its variants; persistent warps pull
//                      (description, 32-strand batch) items of their class
//                      from an atomic counter -- items of the costliest
//                      descriptions first -- and run each item with its
//                      description's tile (lanes per strand x CVs per lane,
//                      or the lane walk for strands of up to 32 CVs).
// Six to eight launches per frame whatever the description count, all
// enqueue-only and capturable in one CUDA graph.
#include "generator_core.cuh"
#include "walk.cuh"
#include "nxg_classic.h"
#include "nxg_internal.h"
#include "strand_math.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <vector>

namespace nxg {
namespace dev {

constexpr int kMaxBatch = NXG_MAX_BATCH;

struct BatchDesc {
    LaunchArgs g;              // asset, frame, params, count, outputs, order
    const float4 *offsets;     // guide-offset table (G x P)
    uint32_t *keys;            // count
    uint32_t *bins;            // guide_count + 1
    uint32_t lanes;            // tile: lanes per strand
    uint32_t ppt;              // tile: CVs per lane (2 or 4)
    uint32_t noise;
    uint32_t want_roots;       // any of roots / root_uvs / point_counts
    uint32_t strand_begin;     // prefix of strand counts (flat strand index)
    uint32_t item_begin;       // first work item (32 strands each)
    uint64_t offset_begin;     // prefix of guide_count * P (flat table index)
};

struct BatchArgs {
    uint32_t count;
    uint32_t warp_bytes[3];    // shared memory per warp of each class's generate launch (after the CTA's head)
    uint32_t total_strands;
    // Work-item classes, each its own generate launch: 0 = noisy
    // descriptions on lane-walk items, 1 = noise-free descriptions, 2 = noisy
    // descriptions on lane-group items.  Descriptions d[k] of class c are k
    // in [desc_first[c], desc_end[c]).
    uint32_t total_items[3];
    uint32_t desc_first[3], desc_end[3];
    uint32_t *item_counter;    // one counter per class
    uint64_t total_offsets;
    BatchDesc d[kMaxBatch];
};

__device__ __forceinline__ int desc_of_strand(const BatchArgs &b, uint32_t i) {
    int d = 0;
    while (d + 1 < static_cast<int>(b.count) && b.d[d + 1].strand_begin <= i) { ++d; }
    return d;
}

__global__ void batched_clear_kernel(const __grid_constant__ BatchArgs b) {
    if (blockIdx.x == 0 && threadIdx.x < 3) { b.item_counter[threadIdx.x] = 0u; }
    for (uint32_t d = 0; d < b.count; ++d) {
        const uint32_t bins = b.d[d].g.a.guide_count + 1u;
        for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < bins; i += gridDim.x * blockDim.x) {
            b.d[d].bins[i] = 0u;
        }
    }
}

// One CTA (1024 threads) per description: exclusive scan of its bins.
__global__ void __launch_bounds__(1024) batched_scan_kernel(const __grid_constant__ BatchArgs b) {
    __shared__ uint32_t warp_sums[32];
    const BatchDesc &d = b.d[blockIdx.x];
    uint32_t *data = d.bins;
    const uint32_t n = d.g.a.guide_count + 1u;
    const uint32_t tid = threadIdx.x;
    const uint32_t per = (n + blockDim.x - 1u) / blockDim.x;
    const uint32_t lo = min(n, tid * per), hi = min(n, lo + per);
    uint32_t sum = 0u;
    for (uint32_t i = lo; i < hi; ++i) { sum += data[i]; }
    uint32_t incl = sum;
    const int lane = tid & 31;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
        const uint32_t u = __shfl_up_sync(kFull, incl, k);
        if (lane >= k) { incl += u; }
    }
    if (lane == 31) { warp_sums[tid >> 5] = incl; }
    __syncthreads();
    if (tid < 32) {
        uint32_t w = tid < (blockDim.x >> 5) ? warp_sums[tid] : 0u;
#pragma unroll
        for (int k = 1; k < 32; k <<= 1) {
            const uint32_t u = __shfl_up_sync(kFull, w, k);
            if (lane >= k) { w += u; }
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

// Block-aggregated scatter (see scatter_order_blocked_kernel): a block whose
// flat range lies in one description with up to kBatchScatterBins bins
// ranks its strands in shared memory and takes one global atomic per
// non-empty bin; a block straddling descriptions takes one per strand.
constexpr uint32_t kBatchScatterBins = 8192u;

__global__ void __launch_bounds__(1024) batched_scatter_blocked_kernel(const __grid_constant__ BatchArgs b,
                                                                       uint32_t chunk) {
    extern __shared__ uint32_t slots[];
    const uint32_t begin = blockIdx.x * chunk;
    const uint32_t end = min(b.total_strands, begin + chunk);
    if (begin >= end) { return; }
    const int home = desc_of_strand(b, begin);
    const BatchDesc &d = b.d[home];
    const uint32_t bins = d.g.a.guide_count + 1u;
    uint32_t *order = const_cast<uint32_t *>(d.g.order);
    if (desc_of_strand(b, end - 1u) != home || bins > kBatchScatterBins) {
        for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
            const BatchDesc &e = b.d[desc_of_strand(b, i)];
            const uint32_t local = i - e.strand_begin;
            const uint32_t pos = atomicAdd(&e.bins[min(e.keys[local], e.g.a.guide_count)], 1u);
            if (pos < e.g.count) { const_cast<uint32_t *>(e.g.order)[pos] = local; }
        }
        return;
    }
    const uint32_t lo = begin - d.strand_begin, hi = end - d.strand_begin;
    for (uint32_t k = threadIdx.x; k < bins; k += blockDim.x) { slots[k] = 0u; }
    __syncthreads();
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) { atomicAdd(&slots[min(d.keys[i], bins - 1u)], 1u); }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < bins; k += blockDim.x) {
        const uint32_t n = slots[k];
        slots[k] = n ? atomicAdd(&d.bins[k], n) : 0u;
    }
    __syncthreads();
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t pos = atomicAdd(&slots[min(d.keys[i], bins - 1u)], 1u);
        if (pos < d.g.count) { order[pos] = i; }
    }
}

__global__ void batched_offsets_kernel(const __grid_constant__ BatchArgs b) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < b.total_offsets;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        int di = 0;
        while (di + 1 < static_cast<int>(b.count) && b.d[di + 1].offset_begin <= i) { ++di; }
        const BatchDesc &d = b.d[di];
        const uint64_t local = i - d.offset_begin;
        const uint32_t P = d.g.p.cvs_per_strand;
        const uint64_t table = static_cast<uint64_t>(d.g.a.guide_count) * P;
        if (local < table) {
            const_cast<float4 *>(d.offsets)[local] = guide_offset_entry(d.g.a, d.g.f, P,
                                                                        static_cast<uint32_t>(local / P),
                                                                        static_cast<uint32_t>(local % P));
        } else if (local < table + d.g.a.guide_count) {
            const uint64_t gi = local - table;
            guide_frame_entry(d.g.a, d.g.f, d.g.p.support_scale, static_cast<uint32_t>(gi),
                              const_cast<float4 *>(d.offsets) + table + 2u * gi);
        } else {  // the zero row after the frame records
            const_cast<float4 *>(d.offsets)[d.g.zero_row + (local - table - d.g.a.guide_count)] =
                make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
    }
}

// Per flat strand: the root triangle, its sort key (first stencil guide)
// with the description's key histogram, and -- for descriptions on
// lane-group tiles -- the full root sample and the RootSample / root UV /
// point count outputs.  Block b owns the contiguous flat range
// [b*chunk, (b+1)*chunk), so its strands are mostly one description's and
// that description's histogram is kept in shared memory.  Roots of a warp
// whose 32 strands share a description are written as consecutive words.
constexpr uint32_t kBatchPrivateBins = 4096u;

__global__ void __launch_bounds__(256) batched_prepare_kernel(const __grid_constant__ BatchArgs b, uint32_t chunk) {
    __shared__ uint32_t staged[8][32 * 12 + 1];
    __shared__ uint32_t hist[kBatchPrivateBins];
    const uint32_t begin = blockIdx.x * chunk;
    const uint32_t end = min(begin + chunk, b.total_strands);
    if (begin >= end) { return; }
    const int home = desc_of_strand(b, begin);
    const uint32_t home_bins = b.d[home].g.a.guide_count + 1u;
    const bool priv = home_bins <= kBatchPrivateBins;
    if (priv) {
        for (uint32_t i = threadIdx.x; i < home_bins; i += blockDim.x) { hist[i] = 0u; }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    for (uint32_t base = begin + static_cast<uint32_t>(warp) * 32u; base < end; base += (blockDim.x >> 5) * 32u) {
        const uint32_t i = base + static_cast<uint32_t>(lane);
        const bool valid = i < end;
        const uint32_t fi = valid ? i : base;
        const int di = desc_of_strand(b, fi);
        const BatchDesc &d = b.d[di];
        const uint32_t local = fi - d.strand_begin;
        // Lane-walk descriptions write their root outputs in the generate
        // kernel; here they need only the root triangle.
        const bool outputs = d.lanes != 1u;
        uint32_t *rec = staged[warp] + lane * 12;
        uint32_t triangle;
        Root r{};
        if (outputs) {
            r = sample_root(d.g.a, d.g.f, d.g.p.seed, d.g.first_strand + local);
            for (int w = 0; w < 12; ++w) { rec[w] = root_word(r, w); }
            triangle = r.triangle;
        } else {
            triangle = sample_triangle(d.g.a, d.g.p.seed, d.g.first_strand + local);
        }
        if (valid) {
            const uint32_t gi = __ldg(d.g.a.stencil + static_cast<uint64_t>(triangle) * kSlots);
            const uint32_t key = gi < d.g.a.guide_count ? gi : d.g.a.guide_count;
            d.keys[local] = key;
            if (priv && di == home) {
                atomicAdd(&hist[key], 1u);
            } else {
                atomicAdd(&d.bins[key], 1u);
            }
            if (outputs && d.g.root_uvs) { d.g.root_uvs[local] = make_float2(r.u, r.v); }
            if (outputs && d.g.point_counts) { d.g.point_counts[local] = d.g.p.cvs_per_strand; }
        }
        __syncwarp();
        const int d0 = __shfl_sync(kFull, di, 0);
        if (__all_sync(kFull, di == d0)) {
            const BatchDesc &dd = b.d[d0];
            if (dd.g.roots && dd.lanes != 1u) {
                const uint32_t local0 = __shfl_sync(kFull, local, 0);
                const uint32_t n = min(32u, end - base);
                uint32_t *dst = dd.g.roots + static_cast<uint64_t>(local0) * 12u;
                for (uint32_t w = lane; w < n * 12u; w += 32u) { dst[w] = staged[warp][w]; }
            }
        } else if (valid && outputs && d.g.roots) {  // the warp straddles two descriptions
            for (int w = 0; w < 12; ++w) { d.g.roots[static_cast<uint64_t>(local) * 12u + w] = rec[w]; }
        }
        __syncwarp();
    }
    __syncthreads();
    if (priv) {
        for (uint32_t k = threadIdx.x; k < home_bins; k += blockDim.x) {
            if (hist[k]) { atomicAdd(&b.d[home].bins[k], hist[k]); }
        }
    }
}

// Per-warp shared memory of the batched kernel.
// Shared memory of batched_generate: a head per CTA (the current
// description's gradient table, t values and, for 2..32 CVs, radii -- every
// warp of a CTA works on the same description), then one region per warp.
constexpr size_t kBatchTableBytes = sizeof(float4) * kTableFloat4;              // 4096
constexpr size_t kBatchTvalBytes = sizeof(float) * 128u;                        // P <= 128
constexpr size_t kBatchHeadBytes = kBatchTableBytes + kBatchTvalBytes;
constexpr size_t kBatchRecordBytes = sizeof(uint32_t) * kRecFields * 32u;       // 4480
constexpr size_t kBatchStageBytes = sizeof(float4) * 32u * 4u;                  // 32 lanes x 4 CVs
constexpr size_t kBatchLatticeBytes = sizeof(float2) * 384u;
constexpr size_t kBatchWarpBytes = kBatchRecordBytes + kBatchStageBytes + kBatchLatticeBytes;
// 32-strand batches per warp in one work item of each class: four for the
// noisy classes (fewer CTA-wide claims between long batches), one for the
// noise-free class (its descriptions are small; finer items balance better).
__host__ __device__ constexpr uint32_t batches_per_warp(int cls) { return cls == 1 ? 1u : 4u; }

static_assert(kBatchRecordBytes >= kWalkRecordBytes, "lane-walk records fit the record area");
static_assert(kBatchStageBytes >= sizeof(float4) * kWalkMaxCvs, "spline scratch fits the stage area");
static_assert(kBatchStageBytes >= kWalkRootWordBytes, "RootSample words fit the stage area");
static_assert(kBatchLatticeBytes >= kWalkLocalBytes, "output words fit the lattice area");

// Per-warp shared memory of the noisy lane-walk class in a CTA of `warps`
// warps: stage | records aliased by the lattice (walk_lattice_columns) |
// output words.
__host__ __device__ constexpr size_t batch_walk_warp_bytes(int warps) {
    return kWalkStageBytes + walk_lattice_bytes(walk_lattice_columns(warps)) + kWalkLocalBytes;
}
static_assert(walk_lattice_bytes(walk_lattice_columns(11)) >= kWalkRecordBytes, "records fit the lattice area");

// A noisy description on the lane-walk tile (2..32 CVs): setup (with the
// root outputs), base into the stage, the frame walk and the store step
// (walk.cuh), with the Classic application when the description has scalars.
template <bool CLASSIC>
__device__ __noinline__ void batched_noise_walk_item(const BatchDesc &d, uint32_t batch, uint32_t end, int lane,
                                                     unsigned char *mine, const float4 *table, const float *tvals,
                                                     int columns) {
    const float *rvals = tvals + 2 * kWalkMaxCvs;
    float *stage = reinterpret_cast<float *>(mine);
    unsigned char *after_stage = mine + kWalkStageBytes;
    float4 *records = reinterpret_cast<float4 *>(after_stage);
    float2 *lattice = reinterpret_cast<float2 *>(after_stage);
    uint32_t *locals = reinterpret_cast<uint32_t *>(after_stage + walk_lattice_bytes(columns));
    const int P = static_cast<int>(d.g.p.cvs_per_strand);
    const uint32_t item = batch + static_cast<uint32_t>(lane);
    const bool valid = item < end;
    const int in_batch = static_cast<int>(end - batch);
    const WalkRoot wr = walk_setup<true>(d.g, records, locals, lane, valid ? item : batch, valid,
                                         static_cast<uint32_t>(P));
    __syncwarp();
    walk_base_direct<false, true>(d.g, records, locals, tvals, rvals, d.offsets, lane, in_batch, P, stage);
    __syncwarp();
    walk_frame(d.g.p, wr, lane < in_batch, stage + lane * kWalkRowFloats, lattice + lane, tvals, table, P,
               columns);
    __syncwarp();
    if (CLASSIC && d.g.scalars != nullptr) {
        walk_classic_strand(d.g, records, stage, locals, lane, in_batch, P);
        __syncwarp();
        walk_store8_classic(d.g, records, stage, locals, rvals, lane, in_batch, P);
    } else {
        walk_store8(d.g, stage, locals, rvals, lane, in_batch, P);
    }
    __syncwarp();
}

// A noise-free description on the lane-walk tile (2..32 CVs): setup and the
// lane-parallel base step writing the output directly (walk.cuh), with the
// Classic application when the description has scalars; setup writes the
// root outputs.
template <bool CLASSIC>
__device__ __noinline__ void batched_walk_item(const BatchDesc &d, uint32_t batch, uint32_t end, int lane,
                                               unsigned char *mine, const float *tvals) {
    const float *rvals = tvals + 2 * kWalkMaxCvs;
    float4 *records = reinterpret_cast<float4 *>(mine);
    float4 *scratch = reinterpret_cast<float4 *>(mine + kBatchRecordBytes);
    uint32_t *locals = reinterpret_cast<uint32_t *>(mine + kBatchRecordBytes + kBatchStageBytes);
    const int P = static_cast<int>(d.g.p.cvs_per_strand);
    const uint32_t item = batch + static_cast<uint32_t>(lane);
    const bool valid = item < end;
    const int in_batch = static_cast<int>(end - batch);
    walk_setup<false>(d.g, records, locals, lane, valid ? item : batch, valid, static_cast<uint32_t>(P));
    __syncwarp();
    if (CLASSIC && d.g.scalars != nullptr) {
        walk_classic_setup(d.g, records, lane, valid, locals[lane] & 0x7fffffffu, tvals, d.offsets, scratch, P);
        __syncwarp();
        walk_base_direct<true>(d.g, records, locals, tvals, rvals, d.offsets, lane, in_batch, P);
    } else {
        walk_base_direct<false>(d.g, records, locals, tvals, rvals, d.offsets, lane, in_batch, P);
    }
    __syncwarp();
}

template <int L, int PPT, bool NOISE, bool CLASSIC>
__device__ __noinline__ void batched_item(const BatchDesc &d, uint32_t batch, uint32_t end, int lane,
                                             unsigned char *mine, const float4 *table, const float *tvals) {
    const Records rec{reinterpret_cast<uint32_t *>(mine)};
    float4 *stage_base = reinterpret_cast<float4 *>(mine + kBatchRecordBytes);
    float2 *lattice_base = reinterpret_cast<float2 *>(mine + kBatchRecordBytes + kBatchStageBytes);
    constexpr int kGroups = 32 / L;
    const int group = lane / L;
    const int gl = lane % L;
    const uint32_t item = batch + static_cast<uint32_t>(lane);
    const bool valid = item < end;
    setup_strand<NOISE>(d.g, rec, lane, valid ? item : batch, valid);
    __syncwarp();
    const uint32_t in_batch = end - batch;
#pragma unroll 1
    for (uint32_t r = 0; r < in_batch; r += kGroups) {
        emit_strand<L, PPT, NOISE, CLASSIC>(d.g, rec, static_cast<int>(r) + group, gl, table, d.offsets, tvals,
                                   stage_base + group * (L * PPT), lattice_base + group * (384 / kGroups),
                                   384 / 3 / kGroups);
    }
    __syncwarp();
}

template <int PPT, bool NOISE, bool CLASSIC>
__device__ __forceinline__ void batched_dispatch_lanes(const BatchDesc &d, uint32_t batch, uint32_t end, int lane,
                                                       unsigned char *mine, const float4 *table, const float *tvals) {
    switch (d.lanes) {
        case 2: batched_item<2, PPT, NOISE, CLASSIC>(d, batch, end, lane, mine, table, tvals); break;
        case 4: batched_item<4, PPT, NOISE, CLASSIC>(d, batch, end, lane, mine, table, tvals); break;
        case 8: batched_item<8, PPT, NOISE, CLASSIC>(d, batch, end, lane, mine, table, tvals); break;
        case 16: batched_item<16, PPT, NOISE, CLASSIC>(d, batch, end, lane, mine, table, tvals); break;
        default: batched_item<32, PPT, NOISE, CLASSIC>(d, batch, end, lane, mine, table, tvals); break;
    }
}

// CLASSIC: some description applies Classic per-root scalars; descriptions
// without scalars still take the plain item.  CLS: the work-item class this
// launch runs (0: noisy lane-walk items, 1: noise-free items, 2: noisy
// lane-group items), so each launch holds only its variants' code and runs
// at their register and shared-memory footprint.
template <int PPT, bool CLASSIC, int CLS>
__global__ void __launch_bounds__(CLS == 1 ? 256 : 352, CLS == 1 ? 3 : 1)
    batched_generate_kernel(const __grid_constant__ BatchArgs b) {
    extern __shared__ float4 smem[];
    __shared__ uint32_t claimed;
    __shared__ uint32_t next_batch;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const uint32_t warps = blockDim.x >> 5;
    const uint32_t per_item = warps * batches_per_warp(CLS);
    // The next class's launch reads nothing this one writes (its own
    // descriptions' outputs; the strand order and offset tables were done
    // before this launch began), so it may start as soon as this launch's
    // CTAs leave SMs free.
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    float4 *table = smem;
    float *tvals = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(smem) + kBatchTableBytes);
    unsigned char *mine = reinterpret_cast<unsigned char *>(smem) + kBatchHeadBytes + b.warp_bytes[CLS] * warp;
    const uint32_t total = b.total_items[CLS];
    const int first = static_cast<int>(b.desc_first[CLS]);
    const int last = static_cast<int>(b.desc_end[CLS]) - 1;
    int current = -1;
    // A work item is a contiguous slice of one description's strand order,
    // batches_per_warp(CLS) 32-strand batches per warp of the CTA, so the CTA's
    // strands share guide-offset rows in L1; its warps take the item's
    // batches from a shared counter, so a slow batch holds up only its own
    // warp until the item ends.  Each pass of the loop consumes one item.
    for (uint32_t guard = 0; guard <= total; ++guard) {
        if (threadIdx.x == 0) {
            claimed = atomicAdd(b.item_counter + CLS, 1u);
            next_batch = 0u;
        }
        __syncthreads();
        const uint32_t item = claimed;
        __syncthreads();
        if (item >= total) { break; }
        int di = first;
        while (di < last && b.d[di + 1].item_begin <= item) { ++di; }
        const BatchDesc &d = b.d[di];
        if (di != current) {  // the whole CTA: every warp works on the item's description
            const int P = static_cast<int>(d.g.p.cvs_per_strand);
            if (d.noise) {
                for (int i = threadIdx.x; i < kTableFloat4; i += blockDim.x) {
                    table[i] = make_float4(__ldg(d.g.a.gradients + 3 * i), __ldg(d.g.a.gradients + 3 * i + 1),
                                           __ldg(d.g.a.gradients + 3 * i + 2), 0.0f);
                }
            }
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                tvals[i] = __fdiv_rn(static_cast<float>(i), static_cast<float>(P - 1));
                if (P <= kWalkMaxCvs) { tvals[2 * kWalkMaxCvs + i] = strand_radius(d.g.p, tvals[i]); }
            }
            __syncthreads();
            current = di;
        }
        for (;;) {
        uint32_t k = 0u;
        if (lane == 0) { k = atomicAdd(&next_batch, 1u); }
        k = __shfl_sync(kFull, k, 0);
        if (k >= per_item) { break; }
        const uint32_t batch = ((item - d.item_begin) * per_item + k) * 32u;
        if (batch >= d.g.count) { break; }
        const uint32_t end = min(batch + 32u, d.g.count);
        if constexpr (CLS == 0) {
            batched_noise_walk_item<CLASSIC>(d, batch, end, lane, mine, table, tvals,
                                             walk_lattice_columns(static_cast<int>(warps)));
        } else if constexpr (CLS == 1) {
            if (d.lanes == 1u) {
                batched_walk_item<CLASSIC>(d, batch, end, lane, mine, tvals);
            } else if (CLASSIC && d.g.scalars != nullptr) {
                batched_dispatch_lanes<PPT, false, CLASSIC>(d, batch, end, lane, mine, table, tvals);
            } else {
                batched_dispatch_lanes<PPT, false, false>(d, batch, end, lane, mine, table, tvals);
            }
        } else if (CLASSIC && d.g.scalars != nullptr) {
            batched_dispatch_lanes<PPT, true, CLASSIC>(d, batch, end, lane, mine, table, tvals);
        } else {
            batched_dispatch_lanes<PPT, true, false>(d, batch, end, lane, mine, table, tvals);
        }
        }
        __syncthreads();  // the item's batches are done before the next claim resets the counter
    }
}

} // namespace dev

namespace {

constexpr uint64_t kAlign = 256u;
inline uint64_t up(uint64_t v) { return (v + kAlign - 1u) / kAlign * kAlign; }

struct BatchLayout {
    uint64_t counter;
    std::vector<uint64_t> keys, order, bins, offsets;
    uint64_t total;
};

BatchLayout batch_layout(const nxg_device_asset_desc *assets, const nxg_generation_params *params, uint32_t count) {
    BatchLayout l{};
    l.counter = 0u;
    uint64_t at = kAlign;
    for (uint32_t d = 0; d < count; ++d) {
        const uint64_t S = params[d].strand_count, P = params[d].cvs_per_strand, G = assets[d].header.guide_count;
        l.keys.push_back(at);
        at += up(S * 4u);
        l.order.push_back(at);
        at += up(S * 4u);
        l.bins.push_back(at);
        at += up((G + 1u) * 4u);
        l.offsets.push_back(at);
        at += up((G * (P + 2u) + dev::kWalkMaxCvs) * 16u);  // offset table, 2 guide frame records per guide, zero row
    }
    l.total = at;
    return l;
}

// Lanes per strand of a description in a batched launch whose CVs per lane
// are `ppt`: 1 (lane-walk items) for a description on the lane-walk tile; the registered tile's lanes when it uses the same CVs per
// lane; else the narrowest power-of-two group holding the strand.
uint32_t batch_lanes(uint32_t P, bool noise, uint32_t ppt) {
    nxg_tile t{};
    nxg_get_tile(P, noise ? 1u : 0u, &t);
    if (t.lanes_per_strand == 1u && P <= static_cast<uint32_t>(dev::kWalkMaxCvs)) { return 1u; }
    if (t.cvs_per_lane == ppt && t.lanes_per_strand * ppt >= P) { return t.lanes_per_strand; }
    uint32_t l = 2u;
    while (l * ppt < P) { l *= 2u; }
    return l;
}

int sm_count() {
    int device = 0, sms = 148;
    if (cudaGetDevice(&device) == cudaSuccess) { cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device); }
    return sms > 0 ? sms : 148;
}

} // namespace
} // namespace nxg

extern "C" uint64_t nxg_batched_workspace_size(const nxg_device_asset_desc *assets,
                                               const nxg_generation_params *params, uint32_t count) {
    if (!assets || !params || count == 0u || count > NXG_MAX_BATCH) { return 0u; }
    return nxg::batch_layout(assets, params, count).total;
}

namespace nxg {
namespace {

uint32_t generate_batched(const nxg_device_asset_desc *assets, const nxg_deformed_desc *deformed,
                          const nxg_generation_params *params, const nxg_packed_output_desc *outputs,
                          const nxg_classic_apply_desc *classic, uint32_t count, const nxg_launch_config *config,
                          void *workspace, uint64_t workspace_bytes, void *stream) {
    if (!assets || !params || !outputs || count == 0u || count > NXG_MAX_BATCH) { return NXG_ERROR_INVALID_ARGUMENT; }
    bool any_classic = false;
    if (classic) {
        for (uint32_t d = 0; d < count; ++d) {
            if (classic[d].root_scalars == nullptr) { continue; }
            if (reinterpret_cast<std::uintptr_t>(classic[d].root_scalars) % 8u != 0u) {
                return NXG_ERROR_MISALIGNED_OUTPUT;
            }
            any_classic = true;
        }
    }
    const nxg_launch_config cfg = config ? *config : nxg_launch_config{128u};
    for (uint32_t d = 0; d < count; ++d) {
        const uint32_t error = nxg_validate_packed_request(&assets[d], deformed ? &deformed[d] : nullptr, &params[d],
                                                           &outputs[d], &cfg);
        if (error != NXG_ERROR_NONE) { return error; }
        if (!sections_in_bounds(assets[d].header)) { return NXG_ERROR_INVALID_ASSET_METADATA; }
        if (reinterpret_cast<std::uintptr_t>(outputs[d].points) % 16u != 0u ||
            reinterpret_cast<std::uintptr_t>(outputs[d].roots) % 4u != 0u ||
            reinterpret_cast<std::uintptr_t>(outputs[d].root_uvs) % 8u != 0u ||
            reinterpret_cast<std::uintptr_t>(outputs[d].point_counts) % 4u != 0u) {
            return NXG_ERROR_MISALIGNED_OUTPUT;
        }
        if (params[d].cvs_per_strand > 128u ||
            uint64_t{assets[d].header.guide_count} * params[d].cvs_per_strand * 16u > (uint64_t{1} << 30)) {
            return NXG_ERROR_INVALID_ARGUMENT;  // long strands take nxg_generate_packed's serial kernel
        }
    }
    const BatchLayout layout = batch_layout(assets, params, count);
    if (!workspace || workspace_bytes < layout.total) { return NXG_ERROR_WORKSPACE_TOO_SMALL; }
    if (reinterpret_cast<std::uintptr_t>(workspace) % kAlign != 0u) { return NXG_ERROR_MISALIGNED_OUTPUT; }

    // Tile family of the launch: two CVs per lane when every strand fits 32 x 2.
    uint32_t max_cvs = 0u;
    for (uint32_t d = 0; d < count; ++d) { max_cvs = std::max(max_cvs, params[d].cvs_per_strand); }
    const uint32_t ppt = max_cvs <= 64u ? 2u : 4u;
    // Work-item class of each description, one generate launch per class at
    // its own occupancy: 0 for noisy descriptions on the lane-walk tile, whose
    // warps need the walk's stage and lattice (eleven-warp CTAs fill the SM's
    // shared memory); 1 for noise-free descriptions; 2 for noisy descriptions
    // on lane-group tiles.
    constexpr uint32_t kClasses = 3u;
    std::vector<uint32_t> cls(count);
    for (uint32_t d = 0; d < count; ++d) {
        const bool noise = params[d].noise_amplitude != 0.0f && params[d].noise_mask != 0.0f;
        cls[d] = !noise ? 1u : (batch_lanes(params[d].cvs_per_strand, true, ppt) == 1u ? 0u : 2u);
    }
    const auto kernel = [&](uint32_t c) -> const void * {
        if (c == 0u) {
            return any_classic ? reinterpret_cast<const void *>(dev::batched_generate_kernel<2, true, 0>)
                               : reinterpret_cast<const void *>(dev::batched_generate_kernel<2, false, 0>);
        }
        if (c == 1u) {
            if (any_classic) {
                return ppt == 2u ? reinterpret_cast<const void *>(dev::batched_generate_kernel<2, true, 1>)
                                 : reinterpret_cast<const void *>(dev::batched_generate_kernel<4, true, 1>);
            }
            return ppt == 2u ? reinterpret_cast<const void *>(dev::batched_generate_kernel<2, false, 1>)
                             : reinterpret_cast<const void *>(dev::batched_generate_kernel<4, false, 1>);
        }
        if (any_classic) {
            return ppt == 2u ? reinterpret_cast<const void *>(dev::batched_generate_kernel<2, true, 2>)
                             : reinterpret_cast<const void *>(dev::batched_generate_kernel<4, true, 2>);
        }
        return ppt == 2u ? reinterpret_cast<const void *>(dev::batched_generate_kernel<2, false, 2>)
                         : reinterpret_cast<const void *>(dev::batched_generate_kernel<4, false, 2>);
    };
    uint32_t status = NXG_ERROR_NONE;
    int device = 0, smem_optin = 48 * 1024;
    if (cudaGetDevice(&device) == cudaSuccess) {
        cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    }
    // CTA size per class (work items are one 32-strand batch per warp).
    auto warp_bytes_of = [](uint32_t c, uint32_t warps) {
        return c == 0u ? dev::batch_walk_warp_bytes(static_cast<int>(warps)) : dev::kBatchWarpBytes;
    };
    size_t class_warp_bytes[kClasses] = {0u, 0u, 0u};
    uint32_t class_block[kClasses] = {0u, 0u, 0u};
    for (uint32_t c = 0; c < kClasses; ++c) {
        cudaFuncAttributes attr{};
        if ((status = record_cuda(cudaFuncGetAttributes(&attr, kernel(c))))) { return status; }
        uint32_t block = std::min(static_cast<uint32_t>(attr.maxThreadsPerBlock) / 32u * 32u,
                                  c == 0u ? 352u : std::max<uint32_t>(32u, (cfg.block_size + 31u) / 32u * 32u));
        while (block > 32u && dev::kBatchHeadBytes + warp_bytes_of(c, block / 32u) * (block / 32u) + 64u >
                                  static_cast<size_t>(smem_optin)) {
            block -= 32u;
        }
        class_block[c] = block;
        class_warp_bytes[c] = warp_bytes_of(c, block / 32u);
    }

    auto *w = static_cast<unsigned char *>(workspace);
    dev::BatchArgs b{};
    b.count = count;
    for (uint32_t c = 0; c < kClasses; ++c) { b.warp_bytes[c] = static_cast<uint32_t>(class_warp_bytes[c]); }
    b.item_counter = reinterpret_cast<uint32_t *>(w + layout.counter);
    // Costliest descriptions first (CVs per strand, tripled with noise), so the
    // longest work items start early and the tail is made of cheap ones.
    std::vector<uint32_t> rank(count);
    std::iota(rank.begin(), rank.end(), 0u);
    auto cost = [&](uint32_t d) {
        const bool noise = params[d].noise_amplitude != 0.0f && params[d].noise_mask != 0.0f;
        return uint64_t{params[d].cvs_per_strand} * (noise ? 3u : 1u);
    };
    std::stable_sort(rank.begin(), rank.end(), [&](uint32_t x, uint32_t y) {
        return cls[x] != cls[y] ? cls[x] < cls[y] : cost(x) > cost(y);
    });
    uint32_t strands = 0u, items[kClasses] = {0u, 0u, 0u};
    for (uint32_t c = 0; c < kClasses; ++c) { b.desc_first[c] = b.desc_end[c] = count; }
    uint64_t offsets = 0u;
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t d = rank[k];
        dev::BatchDesc &bd = b.d[k];
        const nxg_deformed_desc none{};
        bd.g.a = resolve_asset(assets[d]);
        bd.g.f = resolve_frame(bd.g.a, deformed ? deformed[d] : none);
        bd.g.p = resolve_params(params[d], outputs[d].radius_scale);
        bd.g.first_strand = 0u;
        bd.g.count = params[d].strand_count;
        bd.g.points = reinterpret_cast<float4 *>(outputs[d].points);
        bd.g.vec3_points = nullptr;
        bd.g.roots = reinterpret_cast<uint32_t *>(outputs[d].roots);
        bd.g.root_uvs = reinterpret_cast<float2 *>(outputs[d].root_uvs);
        bd.g.point_counts = outputs[d].point_counts;
        bd.g.order = reinterpret_cast<const uint32_t *>(w + layout.order[d]);
        if (classic && classic[d].root_scalars) {
            bd.g.scalars = reinterpret_cast<const float2 *>(classic[d].root_scalars);
            bd.g.classic_length = classic[d].apply_length != 0u;
            bd.g.classic_width = classic[d].apply_width != 0u;
        }
        bd.offsets = reinterpret_cast<const float4 *>(w + layout.offsets[d]);
        bd.g.guide_frames = bd.offsets + uint64_t{assets[d].header.guide_count} * params[d].cvs_per_strand;
        bd.g.zero_row = assets[d].header.guide_count * (params[d].cvs_per_strand + 2u);
        bd.keys = reinterpret_cast<uint32_t *>(w + layout.keys[d]);
        bd.bins = reinterpret_cast<uint32_t *>(w + layout.bins[d]);
        bd.noise = bd.g.p.noise;
        bd.want_roots = (outputs[d].roots || outputs[d].root_uvs || outputs[d].point_counts) ? 1u : 0u;
        bd.strand_begin = strands;
        const uint32_t c = cls[d];
        if (b.desc_first[c] == count) { b.desc_first[c] = k; }
        b.desc_end[c] = k + 1u;
        bd.item_begin = items[c];
        bd.offset_begin = offsets;
        strands += params[d].strand_count;
        const uint32_t per_item = 32u * (class_block[c] / 32u) * dev::batches_per_warp(static_cast<int>(c));
        items[c] += (params[d].strand_count + per_item - 1u) / per_item;
        offsets += uint64_t{assets[d].header.guide_count} * (params[d].cvs_per_strand + 1u) + dev::kWalkMaxCvs;
    }
    b.total_strands = strands;
    for (uint32_t c = 0; c < kClasses; ++c) { b.total_items[c] = items[c]; }
    b.total_offsets = offsets;
    // One CVs-per-lane value per launch keeps the kernel's register footprint
    // that of a single tile family: two when every strand fits 32 lanes x 2.
    for (uint32_t k = 0; k < count; ++k) {
        b.d[k].ppt = ppt;
        b.d[k].lanes = batch_lanes(b.d[k].g.p.cvs_per_strand, b.d[k].noise != 0u, ppt);
    }

    const auto s = static_cast<cudaStream_t>(stream);
    const int sms = sm_count();
    set_last_cuda_error(0);
    dev::batched_clear_kernel<<<std::max(1, sms), 256, 0, s>>>(b);
    if ((status = record_cuda(cudaGetLastError()))) { return status; }
    {
        const uint32_t prepare_blocks = static_cast<uint32_t>(std::min<uint64_t>((strands + 255u) / 256u,
                                                                                 uint64_t(sms) * 8u));
        const uint32_t chunk = ((strands + prepare_blocks - 1u) / prepare_blocks + 31u) / 32u * 32u;
        dev::batched_prepare_kernel<<<std::max(1u, prepare_blocks), 256, 0, s>>>(b, chunk);
        if ((status = record_cuda(cudaGetLastError()))) { return status; }
    }
    dev::batched_scan_kernel<<<count, 1024, 0, s>>>(b);
    if ((status = record_cuda(cudaGetLastError()))) { return status; }
    {
        const uint32_t scatter_blocks = static_cast<uint32_t>(std::max(1, sms));
        const uint32_t chunk = (strands + scatter_blocks - 1u) / scatter_blocks;
        dev::batched_scatter_blocked_kernel<<<(strands + chunk - 1u) / chunk, 1024,
                                              dev::kBatchScatterBins * sizeof(uint32_t), s>>>(b, chunk);
    }
    if ((status = record_cuda(cudaGetLastError()))) { return status; }
    const uint32_t offset_blocks = static_cast<uint32_t>(std::min<uint64_t>((offsets + 255u) / 256u, uint64_t(sms) * 16u));
    dev::batched_offsets_kernel<<<std::max(1u, offset_blocks), 256, 0, s>>>(b);
    if ((status = record_cuda(cudaGetLastError()))) { return status; }

    // One generate launch per class with work, in stream order; each runs
    // persistent CTAs at its own occupancy.
    bool launched = false;
    for (uint32_t c = 0; c < kClasses; ++c) {
        if (items[c] == 0u) { continue; }
        const void *fn = kernel(c);
        const uint32_t block = class_block[c];
        const size_t shm = dev::kBatchHeadBytes + class_warp_bytes[c] * (block / 32u);
        if ((status = record_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                       static_cast<int>(shm))))) {
            return status;
        }
        int per_sm = 0;
        if ((status = record_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, static_cast<int>(block),
                                                                                shm)))) {
            return status;
        }
        const uint32_t grid = static_cast<uint32_t>(
            std::min<uint64_t>(items[c], static_cast<uint64_t>(std::max(1, sms * std::max(per_sm, 1)))));
        void *args[] = {&b};
        // Every class launch after the first of the frame is a programmatic
        // dependent of the one before: its CTAs take the SMs that the earlier
        // class's tail leaves idle.  That is safe because the classes share
        // no output, and the strand order and offset tables they read were
        // complete before the first class started.
        cudaLaunchConfig_t lc{};
        lc.gridDim = dim3(grid);
        lc.blockDim = dim3(block);
        lc.dynamicSmemBytes = shm;
        lc.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = launched ? 1 : 0;
        lc.attrs = attr;
        lc.numAttrs = 1;
        if ((status = record_cuda(cudaLaunchKernelExC(&lc, fn, args)))) { return status; }
        launched = true;
    }
    return record_cuda(cudaGetLastError());
}

} // namespace
} // namespace nxg

extern "C" uint32_t nxg_generate_batched(const nxg_device_asset_desc *assets, const nxg_deformed_desc *deformed,
                                         const nxg_generation_params *params,
                                         const nxg_packed_output_desc *outputs, uint32_t count,
                                         const nxg_launch_config *config, void *workspace,
                                         uint64_t workspace_bytes, void *stream) {
    return nxg::generate_batched(assets, deformed, params, outputs, nullptr, count, config, workspace,
                                 workspace_bytes, stream);
}

extern "C" uint32_t nxg_generate_batched_classic(const nxg_device_asset_desc *assets,
                                                 const nxg_deformed_desc *deformed,
                                                 const nxg_generation_params *params,
                                                 const nxg_packed_output_desc *outputs,
                                                 const nxg_classic_apply_desc *classic, uint32_t count,
                                                 const nxg_launch_config *config, void *workspace,
                                                 uint64_t workspace_bytes, void *stream) {
    if (!classic) { return NXG_ERROR_INVALID_ARGUMENT; }
    return nxg::generate_batched(assets, deformed, params, outputs, classic, count, config, workspace,
                                 workspace_bytes, stream);
}
