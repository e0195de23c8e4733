// host.cpp -- host half of libnxg_b200.so: error strings, the checked
// request validators, asset validation and the asset builder.
//
// Compiled with -ffp-contract=off: the asset builder must reproduce the
// reference's float arithmetic (src/asset.cpp:43-293) bit for bit so that a
// blob built here is byte-identical to one built by the reference.
#include "nxg_internal.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace {

thread_local int32_t g_last_cuda_error = 0;

constexpr float kFloatMax = 3.402823466e+38f;

// ---- small vector helpers (types.h:42-52, generate.h:67-70) ----
inline nxg_vec3 add(nxg_vec3 a, nxg_vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline nxg_vec3 sub(nxg_vec3 a, nxg_vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline nxg_vec3 divs(nxg_vec3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline float dot(nxg_vec3 a, nxg_vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline nxg_vec3 cross(nxg_vec3 a, nxg_vec3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float len2(nxg_vec3 v) { return dot(v, v); }
inline nxg_vec3 normalize(nxg_vec3 v) {
    const float l2 = len2(v);
    return l2 > 1.0e-20f ? divs(v, std::sqrt(l2)) : nxg_vec3{0.0f, 1.0f, 0.0f};
}

void copy_message(const char *text, char *out, uint64_t cap) {
    if (!out || cap == 0u) { return; }
    const std::size_t n = std::min<std::size_t>(std::strlen(text), static_cast<std::size_t>(cap - 1u));
    std::memcpy(out, text, n);
    out[n] = '\0';
}

// FNV-1a 64 (asset.cpp:34-41).
uint64_t fnv1a(const unsigned char *bytes, uint64_t size) {
    uint64_t hash = 1469598103934665603ull;
    for (uint64_t i = 0; i < size; ++i) {
        hash ^= bytes[i];
        hash *= 1099511628211ull;
    }
    return hash;
}

// asset.cpp:152-158
bool section_fits(const nxg_asset_header &h, uint64_t offset, uint64_t count, uint64_t elem) {
    if (count == 0u) { return offset == 0u; }
    if (offset < sizeof(nxg_asset_header) || offset > h.byte_size) { return false; }
    if (count > std::numeric_limits<uint64_t>::max() / elem) { return false; }
    return count * elem <= h.byte_size - offset;
}

bool all_sections_fit(const nxg_asset_header &h) {
    return section_fits(h, h.positions_offset, h.vertex_count, sizeof(nxg_vec3)) &&
        section_fits(h, h.normals_offset, h.vertex_count, sizeof(nxg_vec3)) &&
        section_fits(h, h.texcoords_offset,
                     (h.flags & NXG_ASSET_HAS_TEXCOORDS) ? h.vertex_count : 0u, sizeof(nxg_vec2)) &&
        section_fits(h, h.triangles_offset, h.triangle_count, sizeof(nxg_uint3)) &&
        section_fits(h, h.alias_table_offset, h.triangle_count, sizeof(nxg_alias_entry)) &&
        section_fits(h, h.guides_offset, h.guide_count, sizeof(nxg_guide_record)) &&
        section_fits(h, h.guide_cvs_offset, h.guide_cv_count, sizeof(nxg_vec3)) &&
        section_fits(h, h.triangle_guides_offset,
                     static_cast<uint64_t>(h.triangle_count) * h.guide_stencil_size,
                     sizeof(uint32_t)) &&
        section_fits(h, h.noise_gradients_offset, h.noise_gradient_count, sizeof(nxg_vec3));
}

// asset.cpp:295-338, plus the stencil/alias index checks documented in nxg.h.
const char *validate_blob(const void *bytes, uint64_t size) {
    if (!bytes || size < sizeof(nxg_asset_header)) { return "blob is smaller than AssetHeader"; }
    if (reinterpret_cast<std::uintptr_t>(bytes) % 64u != 0u) { return "blob base is not 64-byte aligned"; }
    nxg_asset_header h{};
    std::memcpy(&h, bytes, sizeof h);
    if (h.magic != NXG_MAGIC) { return "bad NanoXGen magic"; }
    if (h.version_major != NXG_VERSION_MAJOR || h.version_minor != NXG_VERSION_MINOR) {
        return "unsupported NanoXGen asset version";
    }
    if (h.byte_size != size) { return "header byte_size does not match file size"; }
    if (h.triangle_count == 0u || h.vertex_count == 0u || h.guide_count == 0u) {
        return "required section is empty";
    }
    if (h.guide_stencil_size != NXG_GUIDE_STENCIL_SIZE) { return "unsupported guide stencil size"; }
    if (h.noise_gradient_count != NXG_NOISE_GRADIENT_COUNT) { return "unsupported noise gradient table"; }
    if (!all_sections_fit(h)) { return "one or more sections are out of bounds"; }
    const auto *base = static_cast<const unsigned char *>(bytes);
    if (fnv1a(base + sizeof h, size - sizeof h) != h.content_hash) { return "content hash mismatch"; }
    const auto *tris = reinterpret_cast<const nxg_uint3 *>(base + h.triangles_offset);
    for (uint32_t i = 0; i < h.triangle_count; ++i) {
        if (tris[i].x >= h.vertex_count || tris[i].y >= h.vertex_count || tris[i].z >= h.vertex_count) {
            return "triangle index out of bounds";
        }
    }
    const auto *guides = reinterpret_cast<const nxg_guide_record *>(base + h.guides_offset);
    for (uint32_t i = 0; i < h.guide_count; ++i) {
        const nxg_guide_record &g = guides[i];
        if (g.cv_count < 2u || g.first_cv > h.guide_cv_count ||
            g.cv_count > h.guide_cv_count - g.first_cv) {
            return "guide CV range out of bounds";
        }
    }
    // Additions: indices a device kernel would otherwise follow out of bounds.
    const auto *stencil = reinterpret_cast<const uint32_t *>(base + h.triangle_guides_offset);
    const uint64_t slots = static_cast<uint64_t>(h.triangle_count) * h.guide_stencil_size;
    for (uint64_t i = 0; i < slots; ++i) {
        if (stencil[i] != NXG_INVALID_INDEX && stencil[i] >= h.guide_count) {
            return "guide stencil index out of bounds";
        }
    }
    const auto *alias = reinterpret_cast<const nxg_alias_entry *>(base + h.alias_table_offset);
    for (uint32_t i = 0; i < h.triangle_count; ++i) {
        if (alias[i].alias >= h.triangle_count) { return "alias table index out of bounds"; }
    }
    return nullptr;
}

// device_contract.h:120-135
bool valid_generation_parameters(const nxg_generation_params &p) {
    using std::isfinite;
    return p.strand_count != 0u && p.cvs_per_strand >= 2u &&
        isfinite(p.guide_support_scale) && p.guide_support_scale >= 0.0f &&
        isfinite(p.guide_weight_power) && p.guide_weight_power >= 0.0f &&
        isfinite(p.normal_rejection_cos) && p.normal_rejection_cos >= -1.0f &&
        p.normal_rejection_cos <= 1.0f && isfinite(p.length_scale) && p.length_scale >= 0.0f &&
        isfinite(p.root_width) && p.root_width >= 0.0f && isfinite(p.tip_width) &&
        p.tip_width >= 0.0f && isfinite(p.noise_amplitude) && p.noise_amplitude >= 0.0f &&
        isfinite(p.noise_frequency) && p.noise_frequency >= 0.0f && isfinite(p.noise_mask) &&
        p.noise_mask >= 0.0f && p.noise_mask <= 1.0f && isfinite(p.noise_correlation) &&
        p.noise_correlation >= 0.0f && p.noise_correlation <= 1.0f &&
        isfinite(p.noise_preserve_length) && p.noise_preserve_length >= 0.0f &&
        p.noise_preserve_length <= 1.0f;
}

// device_contract.h:183-186
bool optional_capacity_valid(const void *pointer, uint64_t capacity, uint64_t required) {
    return pointer ? capacity >= required : capacity == 0u;
}

// ---- asset builder (asset.cpp:19-293) ----

struct BuildError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

float triangle_area(nxg_vec3 a, nxg_vec3 b, nxg_vec3 c) {  // asset.cpp:43-45
    return 0.5f * std::sqrt(len2(cross(sub(b, a), sub(c, a))));
}

// Walker alias table over rest-pose triangle areas (asset.cpp:47-73).  The
// small/large work lists are stacks, exactly as in the reference, because the
// pairing order decides the table contents.
std::vector<nxg_alias_entry> make_alias_table(const nxg_asset_build_input &in) {
    const std::size_t n = in.triangle_count;
    std::vector<double> scaled(n);
    double area_sum = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        const nxg_uint3 t = in.triangles[i];
        scaled[i] = triangle_area(in.positions[t.x], in.positions[t.y], in.positions[t.z]);
        area_sum += scaled[i];
    }
    if (!(area_sum > 0.0)) { throw BuildError("mesh has zero total area"); }
    for (double &p : scaled) { p = p * static_cast<double>(n) / area_sum; }
    std::vector<std::size_t> small, large;
    for (std::size_t i = 0; i < n; ++i) { (scaled[i] < 1.0 ? small : large).push_back(i); }
    std::vector<nxg_alias_entry> table(n);
    while (!small.empty() && !large.empty()) {
        const std::size_t s = small.back();
        small.pop_back();
        const std::size_t l = large.back();
        large.pop_back();
        table[s] = {static_cast<float>(scaled[s]), static_cast<uint32_t>(l)};
        scaled[l] = scaled[l] + scaled[s] - 1.0;
        (scaled[l] < 1.0 ? small : large).push_back(l);
    }
    for (const std::size_t i : large) { table[i] = {1.0f, static_cast<uint32_t>(i)}; }
    for (const std::size_t i : small) { table[i] = {1.0f, static_cast<uint32_t>(i)}; }
    return table;
}

// asset.cpp:75-86: caller normals verbatim, else accumulated face normals.
std::vector<nxg_vec3> make_normals(const nxg_asset_build_input &in) {
    if (in.normals) { return {in.normals, in.normals + in.vertex_count}; }
    std::vector<nxg_vec3> normals(in.vertex_count, nxg_vec3{0.0f, 0.0f, 0.0f});
    for (uint32_t i = 0; i < in.triangle_count; ++i) {
        const nxg_uint3 t = in.triangles[i];
        const nxg_vec3 n = cross(sub(in.positions[t.y], in.positions[t.x]),
                                 sub(in.positions[t.z], in.positions[t.x]));
        normals[t.x] = add(normals[t.x], n);
        normals[t.y] = add(normals[t.y], n);
        normals[t.z] = add(normals[t.z], n);
    }
    for (nxg_vec3 &n : normals) { n = normalize(n); }
    return normals;
}

// asset.cpp:88-97 (std::min keeps the first argument unless the second is smaller).
float radius_from_nearest(float nearest) {
    return std::isfinite(nearest) ? std::max(nearest * 1.75f, 1.0e-4f) : 1.0f;
}

float automatic_support_radius(const nxg_asset_build_input &in, const std::vector<uint64_t> &first,
                               uint32_t index) {
    if (in.guide_support_radii[index] > 0.0f) { return in.guide_support_radii[index]; }
    const nxg_vec3 root = in.guide_cvs[first[index]];
    float nearest = std::numeric_limits<float>::max();
    for (uint32_t j = 0; j < in.guide_count; ++j) {
        if (j == index || in.guide_cv_counts[j] == 0u) { continue; }
        const float d = std::sqrt(len2(sub(root, in.guide_cvs[first[j]])));
        nearest = (d < nearest) ? d : nearest;
    }
    return radius_from_nearest(nearest);
}

// asset.cpp:99-150 (the Classic-metadata checks have no fields in this input).
void check_input(const nxg_asset_build_input &in) {
    if (in.vertex_count == 0u || !in.positions) { throw BuildError("asset needs vertices"); }
    if (in.triangle_count == 0u || !in.triangles) { throw BuildError("asset needs triangles"); }
    if (in.guide_count == 0u) { throw BuildError("asset needs at least one guide"); }
    if (!in.guide_cv_counts || !in.guide_cvs || !in.guide_root_normals || !in.guide_root_uvs ||
        !in.guide_triangles || !in.guide_barycentrics || !in.guide_support_radii) {
        throw BuildError("guide arrays are required");
    }
    for (uint32_t i = 0; i < in.triangle_count; ++i) {
        const nxg_uint3 t = in.triangles[i];
        if (t.x >= in.vertex_count || t.y >= in.vertex_count || t.z >= in.vertex_count) {
            throw BuildError("triangle index out of bounds");
        }
    }
    for (uint32_t g = 0; g < in.guide_count; ++g) {
        if (in.guide_cv_counts[g] < 2u || in.guide_cv_counts[g] > 65535u) {
            throw BuildError("each guide needs 2..65535 CVs");
        }
    }
    if (in.stencil_slots > NXG_GUIDE_STENCIL_SIZE) { throw BuildError("stencil_slots must be 0..8"); }
}

struct Candidate {
    float key;
    uint32_t guide;
};
// std::pair<float, uint32_t>::operator< (the reference sorts pairs).
inline bool candidate_less(const Candidate &a, const Candidate &b) {
    return a.key < b.key || (!(b.key < a.key) && a.guide < b.guide);
}

// Per-triangle guide stencil (asset.cpp:252-269): the `count` smallest
// (distance^2 + normal penalty, guide) pairs in ascending order, i.e. the
// first `count` elements std::partial_sort leaves in place.  A bounded
// insertion list gives the same set and order in O(G) per triangle.
void build_stencils(const nxg_asset_build_input &in, const std::vector<nxg_guide_record> &guides,
                    std::vector<uint32_t> &stencil) {
    const uint32_t guide_count = in.guide_count;
    const uint32_t count = std::min<uint32_t>(NXG_GUIDE_STENCIL_SIZE, guide_count);
    const uint32_t keep = in.stencil_slots == 0u ? count : std::min(count, in.stencil_slots);
    unsigned workers = in.worker_count ? in.worker_count : std::max(1u, std::thread::hardware_concurrency());
    workers = std::min<unsigned>(workers, std::max<uint32_t>(1u, in.triangle_count / 256u));
    std::atomic<uint32_t> next{0u};
    constexpr uint32_t kChunk = 256u;
    auto work = [&] {
        Candidate best[NXG_GUIDE_STENCIL_SIZE];
        for (;;) {
            const uint32_t begin = next.fetch_add(kChunk);
            if (begin >= in.triangle_count) { return; }
            const uint32_t end = std::min(in.triangle_count, begin + kChunk);
            for (uint32_t ti = begin; ti < end; ++ti) {
                const nxg_uint3 t = in.triangles[ti];
                const nxg_vec3 p0 = in.positions[t.x], p1 = in.positions[t.y], p2 = in.positions[t.z];
                const nxg_vec3 centroid = divs(add(add(p0, p1), p2), 3.0f);
                const nxg_vec3 face_normal = normalize(cross(sub(p1, p0), sub(p2, p0)));
                uint32_t filled = 0u;
                for (uint32_t gi = 0; gi < guide_count; ++gi) {
                    const float penalty = dot(face_normal, guides[gi].root_normal) < -0.25f ? 1.0e20f : 0.0f;
                    const nxg_vec3 d = sub(centroid, guides[gi].root_position);
                    const Candidate c{len2(d) + penalty, gi};
                    if (filled < count) {
                        uint32_t k = filled++;
                        while (k > 0u && candidate_less(c, best[k - 1u])) { best[k] = best[k - 1u]; --k; }
                        best[k] = c;
                    } else if (candidate_less(c, best[count - 1u])) {
                        uint32_t k = count - 1u;
                        while (k > 0u && candidate_less(c, best[k - 1u])) { best[k] = best[k - 1u]; --k; }
                        best[k] = c;
                    }
                }
                uint32_t *row = stencil.data() + static_cast<std::size_t>(ti) * NXG_GUIDE_STENCIL_SIZE;
                for (uint32_t j = 0; j < keep; ++j) { row[j] = best[j].guide; }
            }
        }
    };
    if (workers <= 1u) {
        work();
        return;
    }
    std::vector<std::thread> pool;
    pool.reserve(workers);
    for (unsigned i = 0; i < workers; ++i) { pool.emplace_back(work); }
    for (auto &th : pool) { th.join(); }
}

struct Blob {
    unsigned char *data = nullptr;
    uint64_t size = 0;
    uint64_t capacity = 0;
    ~Blob() { std::free(data); }
    void resize(uint64_t n) {
        if (n > capacity) {
            uint64_t cap = std::max<uint64_t>(n, capacity * 2u);
            cap = (cap + 63u) & ~uint64_t{63u};
            auto *p = static_cast<unsigned char *>(std::aligned_alloc(64u, cap));
            if (!p) { throw std::bad_alloc(); }
            if (data) { std::memcpy(p, data, size); }
            std::free(data);
            data = p;
            capacity = cap;
        }
        if (n > size) { std::memset(data + size, 0, n - size); }
        size = n;
    }
    // asset.cpp:25-32: 16-byte (or stronger) aligned section, offset 0 if empty.
    uint64_t append(const void *values, uint64_t bytes, uint64_t alignment) {
        if (bytes == 0u) { return 0u; }
        const uint64_t align = std::max<uint64_t>(16u, alignment);
        const uint64_t offset = (size + align - 1u) & ~(align - 1u);
        resize(offset + bytes);
        std::memcpy(data + offset, values, bytes);
        return offset;
    }
};

const nxg_vec3 kGradients[NXG_NOISE_GRADIENT_COUNT] = {
#include "seexpr_gradients.inc"
};

} // namespace

namespace nxg {

void set_last_cuda_error(int32_t code) noexcept { g_last_cuda_error = code; }

uint32_t validate_common(const nxg_device_asset_desc &asset, const nxg_deformed_desc &deformed,
                         const nxg_generation_params &params, const nxg_launch_config &config) noexcept {
    if (!asset.asset) { return NXG_ERROR_NULL_ASSET; }
    if (reinterpret_cast<std::uintptr_t>(asset.asset) % alignof(nxg_asset_header) != 0u) {
        return NXG_ERROR_MISALIGNED_ASSET;
    }
    const nxg_asset_header &h = asset.header;
    if (h.magic != NXG_MAGIC || h.version_major != NXG_VERSION_MAJOR ||
        h.version_minor != NXG_VERSION_MINOR || h.byte_size < sizeof(nxg_asset_header) ||
        h.vertex_count == 0u || h.triangle_count == 0u || h.guide_count == 0u ||
        h.guide_cv_count == 0u || h.guide_stencil_size != NXG_GUIDE_STENCIL_SIZE ||
        h.noise_gradient_count != NXG_NOISE_GRADIENT_COUNT ||
        h.noise_gradients_offset < sizeof(nxg_asset_header) ||
        h.noise_gradients_offset > h.byte_size ||
        static_cast<uint64_t>(h.noise_gradient_count) * sizeof(nxg_vec3) >
            h.byte_size - h.noise_gradients_offset) {
        return NXG_ERROR_INVALID_ASSET_METADATA;
    }
    if (asset.byte_capacity < h.byte_size) { return NXG_ERROR_ASSET_CAPACITY_TOO_SMALL; }
    if (!valid_generation_parameters(params)) { return NXG_ERROR_INVALID_GENERATION_PARAMETERS; }
    if (config.block_size == 0u || config.block_size > 1024u) { return NXG_ERROR_INVALID_BLOCK_SIZE; }
    if ((deformed.positions == nullptr) != (deformed.position_count == 0u) ||
        (deformed.positions && deformed.position_count != h.vertex_count)) {
        return NXG_ERROR_DEFORMED_POSITION_COUNT_MISMATCH;
    }
    if ((deformed.normals == nullptr) != (deformed.normal_count == 0u) ||
        (deformed.normals && deformed.normal_count != h.vertex_count)) {
        return NXG_ERROR_DEFORMED_NORMAL_COUNT_MISMATCH;
    }
    if ((deformed.guide_cvs == nullptr) != (deformed.guide_cv_count == 0u) ||
        (deformed.guide_cvs && deformed.guide_cv_count != h.guide_cv_count)) {
        return NXG_ERROR_DEFORMED_GUIDE_CV_COUNT_MISMATCH;
    }
    return NXG_ERROR_NONE;
}

bool sections_in_bounds(const nxg_asset_header &header) noexcept {
    return header.byte_size >= sizeof(nxg_asset_header) && all_sections_fit(header);
}

} // namespace nxg

extern "C" {

const char *nxg_error_message(uint32_t code) {
    switch (code) {
        case NXG_ERROR_NONE: return "";
        case NXG_ERROR_NULL_ASSET: return "device asset pointer is null";
        case NXG_ERROR_MISALIGNED_ASSET: return "device asset pointer is not 64-byte aligned";
        case NXG_ERROR_INVALID_ASSET_METADATA: return "device asset metadata is invalid";
        case NXG_ERROR_ASSET_CAPACITY_TOO_SMALL: return "device asset allocation is too small";
        case NXG_ERROR_INVALID_GENERATION_PARAMETERS: return "generation parameters are invalid";
        case NXG_ERROR_INVALID_BLOCK_SIZE: return "GPU block size must be in [1, 1024]";
        case NXG_ERROR_DEFORMED_POSITION_COUNT_MISMATCH:
            return "deformed position count does not match the asset";
        case NXG_ERROR_DEFORMED_NORMAL_COUNT_MISMATCH:
            return "deformed normal count does not match the asset";
        case NXG_ERROR_DEFORMED_GUIDE_CV_COUNT_MISMATCH:
            return "deformed guide-CV count does not match the asset";
        case NXG_ERROR_MISSING_OUTPUT: return "no device output was supplied";
        case NXG_ERROR_POINT_CAPACITY_TOO_SMALL: return "device point output is too small";
        case NXG_ERROR_WIDTH_CAPACITY_TOO_SMALL: return "device width output is too small";
        case NXG_ERROR_ROOT_CAPACITY_TOO_SMALL: return "device root output is too small";
        case NXG_ERROR_ROOT_UV_CAPACITY_TOO_SMALL: return "device root-UV output is too small";
        case NXG_ERROR_POINT_COUNT_CAPACITY_TOO_SMALL: return "device point-count output is too small";
        case NXG_ERROR_INVALID_RADIUS_SCALE:
            return "device curve radius scale must be finite and non-negative";
        case NXG_ERROR_MISSING_MOTION_SAMPLES: return "no motion samples were supplied";
        case NXG_ERROR_INVALID_MOTION_TIMES:
            return "motion sample times must be finite and strictly increasing";
        case NXG_ERROR_MOTION_POINT_CAPACITY_TOO_SMALL: return "device motion-point output is too small";
        case NXG_ERROR_OUTPUT_SIZE_OVERFLOW: return "device output size overflows uint64";
        case NXG_ERROR_INVALID_ARGUMENT: return "a required descriptor pointer is null";
        case NXG_ERROR_INVALID_STRAND_RANGE: return "strand range exceeds the description's strand count";
        case NXG_ERROR_WORKSPACE_TOO_SMALL: return "device workspace is missing or too small";
        case NXG_ERROR_MISALIGNED_OUTPUT:
            return "device point output must be 16-byte aligned and workspace 256-byte aligned";
        case NXG_ERROR_STATIC_SCRATCH_LIMIT:
            return "request needs more scratch than the library's static scratch holds (NXG_STATIC_SCRATCH_BYTES)";
        case NXG_ERROR_EXPRESSION_SYNTAX: return "scalar expression did not compile";
        case NXG_ERROR_EXPRESSION_LIMIT: return "scalar expression exceeds the device program limits";
        case NXG_ERROR_EXPRESSION_INPUT: return "scalar expression uses a variable the runtime cannot bind";
        case NXG_ERROR_EXPRESSION_DOMAIN:
            return "scalar expression produced a non-finite value or a negative length";
        case NXG_ERROR_SURROGATE: return "surrogate model is missing, untrained or misconfigured";
        case NXG_ERROR_CUDA: return "a CUDA runtime call failed";
        default: return "unknown device generation error";
    }
}

uint32_t nxg_abi_version(void) { return NXG_ABI_VERSION; }

int32_t nxg_last_cuda_error(void) { return g_last_cuda_error; }

uint64_t nxg_fnv1a(const void *bytes, uint64_t size) {
    return bytes ? fnv1a(static_cast<const unsigned char *>(bytes), size) : 1469598103934665603ull;
}

int nxg_validate_asset(const void *bytes, uint64_t size, char *message, uint64_t message_capacity) {
    const char *error = validate_blob(bytes, size);
    copy_message(error ? error : "", message, message_capacity);
    return error ? 1 : 0;
}

uint32_t nxg_make_device_asset_descriptor(const void *host_bytes, uint64_t host_size,
                                          const void *device_data, uint64_t device_capacity,
                                          nxg_device_asset_desc *out, char *message,
                                          uint64_t message_capacity) {
    if (!out) { return NXG_ERROR_INVALID_ARGUMENT; }
    const char *error = validate_blob(host_bytes, host_size);
    if (error) {
        copy_message(error, message, message_capacity);
        return NXG_ERROR_INVALID_ASSET_METADATA;
    }
    if (!device_data) {
        copy_message("device asset pointer is null", message, message_capacity);
        return NXG_ERROR_NULL_ASSET;
    }
    if (reinterpret_cast<std::uintptr_t>(device_data) % 64u != 0u) {
        copy_message("device asset pointer is not 64-byte aligned", message, message_capacity);
        return NXG_ERROR_MISALIGNED_ASSET;
    }
    if (device_capacity < host_size) {
        copy_message("device asset allocation is smaller than the asset", message, message_capacity);
        return NXG_ERROR_ASSET_CAPACITY_TOO_SMALL;
    }
    std::memset(out, 0, sizeof *out);
    out->asset = device_data;
    std::memcpy(&out->header, host_bytes, sizeof out->header);
    out->byte_capacity = device_capacity;
    copy_message("", message, message_capacity);
    return NXG_ERROR_NONE;
}

namespace {

// asset.cpp:229-293 build_asset; `device` runs the stencil search on the
// current CUDA device (stencil.cu) instead of the host threads.
int build_asset_blob(const nxg_asset_build_input *input, bool device, void *stream, void **out_bytes,
                     uint64_t *out_size, char *message, uint64_t message_capacity) {
    if (!input || !out_bytes || !out_size) {
        copy_message("null argument", message, message_capacity);
        return 1;
    }
    try {
        const nxg_asset_build_input &in = *input;
        check_input(in);
        const std::vector<nxg_vec3> normals = make_normals(in);
        const std::vector<nxg_alias_entry> alias = make_alias_table(in);
        std::vector<uint64_t> first(in.guide_count);
        uint64_t total_cvs = 0u;
        for (uint32_t g = 0; g < in.guide_count; ++g) {
            first[g] = total_cvs;
            total_cvs += in.guide_cv_counts[g];
        }
        if (total_cvs > std::numeric_limits<uint32_t>::max()) { throw BuildError("too many guide CVs"); }
        // asset.cpp:234-250
        std::vector<nxg_guide_record> guides(in.guide_count);
        for (uint32_t g = 0; g < in.guide_count; ++g) {
            nxg_guide_record r{};
            r.first_cv = static_cast<uint32_t>(first[g]);
            r.cv_count = static_cast<uint16_t>(in.guide_cv_counts[g]);
            r.flags = 0u;
            r.triangle_index = in.guide_triangles[g];
            // The device build finds the nearest roots on the GPU below.
            r.support_radius = device ? in.guide_support_radii[g] : automatic_support_radius(in, first, g);
            r.barycentric = in.guide_barycentrics[g];
            r.root_uv = in.guide_root_uvs[g];
            r.root_position = in.guide_cvs[first[g]];
            r.root_normal = normalize(in.guide_root_normals[g]);
            guides[g] = r;
        }
        std::vector<uint32_t> stencil(static_cast<std::size_t>(in.triangle_count) * NXG_GUIDE_STENCIL_SIZE,
                                      NXG_INVALID_INDEX);
        if (device) {
            std::vector<nxg_vec3> roots(in.guide_count), root_normals(in.guide_count);
            for (uint32_t g = 0; g < in.guide_count; ++g) {
                roots[g] = guides[g].root_position;
                root_normals[g] = guides[g].root_normal;
            }
            std::vector<float> nearest(in.guide_count);
            const char *what = "";
            if (nxg::device_guide_search(in.positions, in.vertex_count, in.triangles, in.triangle_count,
                                         roots.data(), root_normals.data(), in.guide_cv_counts, in.guide_count,
                                         in.stencil_slots, stencil.data(), nearest.data(), stream, &what) != 0) {
                throw BuildError(std::string("device stencil search: ") + what);
            }
            for (uint32_t g = 0; g < in.guide_count; ++g) {
                if (!(in.guide_support_radii[g] > 0.0f)) { guides[g].support_radius = radius_from_nearest(nearest[g]); }
            }
        } else {
            build_stencils(in, guides, stencil);
        }
        // asset.cpp:271-291
        Blob blob;
        blob.resize(sizeof(nxg_asset_header));
        nxg_asset_header h{};
        h.magic = NXG_MAGIC;
        h.version_major = NXG_VERSION_MAJOR;
        h.version_minor = NXG_VERSION_MINOR;
        h.flags = NXG_ASSET_HAS_NORMALS | (in.texcoords ? NXG_ASSET_HAS_TEXCOORDS : 0u);
        h.vertex_count = in.vertex_count;
        h.triangle_count = in.triangle_count;
        h.guide_count = in.guide_count;
        h.guide_cv_count = static_cast<uint32_t>(total_cvs);
        h.guide_stencil_size = NXG_GUIDE_STENCIL_SIZE;
        h.noise_gradient_count = NXG_NOISE_GRADIENT_COUNT;
        h.positions_offset = blob.append(in.positions, uint64_t{in.vertex_count} * sizeof(nxg_vec3), 4u);
        h.normals_offset = blob.append(normals.data(), normals.size() * sizeof(nxg_vec3), 4u);
        h.texcoords_offset = in.texcoords
            ? blob.append(in.texcoords, uint64_t{in.vertex_count} * sizeof(nxg_vec2), 4u) : 0u;
        h.triangles_offset = blob.append(in.triangles, uint64_t{in.triangle_count} * sizeof(nxg_uint3), 4u);
        h.alias_table_offset = blob.append(alias.data(), alias.size() * sizeof(nxg_alias_entry), 4u);
        h.guides_offset = blob.append(guides.data(), guides.size() * sizeof(nxg_guide_record), 4u);
        h.guide_cvs_offset = blob.append(in.guide_cvs, total_cvs * sizeof(nxg_vec3), 4u);
        h.triangle_guides_offset = blob.append(stencil.data(), stencil.size() * sizeof(uint32_t), 4u);
        h.noise_gradients_offset = blob.append(kGradients, sizeof kGradients, 4u);
        h.byte_size = blob.size;
        h.content_hash = fnv1a(blob.data + sizeof h, blob.size - sizeof h);
        std::memcpy(blob.data, &h, sizeof h);
        *out_bytes = blob.data;
        *out_size = blob.size;
        blob.data = nullptr;
        copy_message("", message, message_capacity);
        return 0;
    } catch (const std::exception &error) {
        copy_message(error.what(), message, message_capacity);
        return 1;
    }
}

} // namespace

int nxg_build_asset(const nxg_asset_build_input *input, void **out_bytes, uint64_t *out_size,
                    char *message, uint64_t message_capacity) {
    return build_asset_blob(input, false, nullptr, out_bytes, out_size, message, message_capacity);
}

int nxg_build_asset_device(const nxg_asset_build_input *input, void *stream, void **out_bytes,
                           uint64_t *out_size, char *message, uint64_t message_capacity) {
    return build_asset_blob(input, true, stream, out_bytes, out_size, message, message_capacity);
}

void nxg_free(void *pointer) { std::free(pointer); }

uint32_t nxg_validate_generation_request(const nxg_device_asset_desc *asset,
                                         const nxg_deformed_desc *deformed,
                                         const nxg_generation_params *params,
                                         const nxg_generated_output_desc *output,
                                         const nxg_launch_config *config) {
    if (!asset || !params || !output) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    const uint32_t error = nxg::validate_common(*asset, deformed ? *deformed : none, *params,
                                                config ? *config : default_config);
    if (error != NXG_ERROR_NONE) { return error; }
    if (!output->points && !output->widths && !output->roots) { return NXG_ERROR_MISSING_OUTPUT; }
    const uint64_t point_count = uint64_t{params->strand_count} * params->cvs_per_strand;
    if (!optional_capacity_valid(output->points, output->point_capacity, point_count)) {
        return NXG_ERROR_POINT_CAPACITY_TOO_SMALL;
    }
    if (!optional_capacity_valid(output->widths, output->width_capacity, point_count)) {
        return NXG_ERROR_WIDTH_CAPACITY_TOO_SMALL;
    }
    if (!optional_capacity_valid(output->roots, output->root_capacity, params->strand_count)) {
        return NXG_ERROR_ROOT_CAPACITY_TOO_SMALL;
    }
    return NXG_ERROR_NONE;
}

uint32_t nxg_validate_packed_request(const nxg_device_asset_desc *asset,
                                     const nxg_deformed_desc *deformed,
                                     const nxg_generation_params *params,
                                     const nxg_packed_output_desc *output,
                                     const nxg_launch_config *config) {
    if (!asset || !params || !output) { return NXG_ERROR_INVALID_ARGUMENT; }
    const nxg_deformed_desc none{};
    const nxg_launch_config default_config{128u};
    const uint32_t error = nxg::validate_common(*asset, deformed ? *deformed : none, *params,
                                                config ? *config : default_config);
    if (error != NXG_ERROR_NONE) { return error; }
    if (!output->points) { return NXG_ERROR_MISSING_OUTPUT; }
    if (!std::isfinite(output->radius_scale) || output->radius_scale < 0.0f) {
        return NXG_ERROR_INVALID_RADIUS_SCALE;
    }
    const uint64_t point_count = uint64_t{params->strand_count} * params->cvs_per_strand;
    if (output->point_capacity < point_count) { return NXG_ERROR_POINT_CAPACITY_TOO_SMALL; }
    if (!optional_capacity_valid(output->roots, output->root_capacity, params->strand_count)) {
        return NXG_ERROR_ROOT_CAPACITY_TOO_SMALL;
    }
    if (!optional_capacity_valid(output->root_uvs, output->root_uv_capacity, params->strand_count)) {
        return NXG_ERROR_ROOT_UV_CAPACITY_TOO_SMALL;
    }
    if (!optional_capacity_valid(output->point_counts, output->point_count_capacity,
                                 params->strand_count)) {
        return NXG_ERROR_POINT_COUNT_CAPACITY_TOO_SMALL;
    }
    return NXG_ERROR_NONE;
}

uint32_t nxg_validate_motion_request(const nxg_device_asset_desc *asset,
                                     const nxg_motion_sample_desc *samples,
                                     uint32_t sample_count,
                                     const nxg_generation_params *params,
                                     const nxg_motion_output_desc *output,
                                     const nxg_launch_config *config) {
    if (!asset || !params || !output) { return NXG_ERROR_INVALID_ARGUMENT; }
    if (!samples || sample_count == 0u) { return NXG_ERROR_MISSING_MOTION_SAMPLES; }
    const nxg_launch_config default_config{128u};
    float previous = -std::numeric_limits<float>::infinity();
    for (uint32_t i = 0; i < sample_count; ++i) {
        if (!std::isfinite(samples[i].time) || samples[i].time <= previous) {
            return NXG_ERROR_INVALID_MOTION_TIMES;
        }
        previous = samples[i].time;
        const uint32_t error = nxg::validate_common(*asset, samples[i].deformation, *params,
                                                    config ? *config : default_config);
        if (error != NXG_ERROR_NONE) { return error; }
    }
    const uint64_t per_sample = uint64_t{params->strand_count} * params->cvs_per_strand;
    if (per_sample > std::numeric_limits<uint64_t>::max() / sample_count) {
        return NXG_ERROR_OUTPUT_SIZE_OVERFLOW;
    }
    if (!output->points || output->point_capacity < per_sample * sample_count) {
        return NXG_ERROR_MOTION_POINT_CAPACITY_TOO_SMALL;
    }
    return NXG_ERROR_NONE;
}

} // extern "C"
