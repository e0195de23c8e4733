"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No production grooming assets are available, so these generators stand in
for them: UV spheres (optionally displaced), guides rooted at seeded
area-weighted surface points with CVs along the surface normal, and the
generation parameters each configuration names.  Everything is derived from
fixed seeds with numpy's PCG64, so a workload is reproducible on any host.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional

import numpy as np

from ._abi import INVALID_INDEX, GenerationParams
from .asset import AssetBuildInput, GuideSet


def sphere_mesh(n_lon: int, n_rings: int,
                radius: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None):
    """UV sphere: `n_rings` vertex rings pole to pole (n_rings-1 bands), `n_lon`
    segments, a duplicated seam column for continuous UVs, 2*n_lon*(n_rings-1)
    triangles wound outward.  Returns (positions, texcoords, triangles)."""
    j = np.arange(n_rings, dtype=np.float64)
    i = np.arange(n_lon + 1, dtype=np.float64)
    theta = (math.pi * j / (n_rings - 1))[:, None] * np.ones((1, n_lon + 1))
    phi = np.ones((n_rings, 1)) * (2.0 * math.pi * i / n_lon)[None, :]
    r = np.ones_like(theta) if radius is None else radius(theta, phi)
    pos = np.stack([r * np.sin(theta) * np.cos(phi), r * np.cos(theta), r * np.sin(theta) * np.sin(phi)], -1)
    uv = np.stack([np.broadcast_to(i[None, :] / n_lon, theta.shape), np.broadcast_to(j[:, None] / (n_rings - 1), theta.shape)], -1)
    cols = n_lon + 1
    jj, ii = np.meshgrid(np.arange(n_rings - 1), np.arange(n_lon), indexing="ij")
    v00 = jj * cols + ii
    v01 = v00 + 1
    v10 = v00 + cols
    v11 = v10 + 1
    tris = np.stack([np.stack([v00, v01, v11], -1), np.stack([v00, v11, v10], -1)], axis=2).reshape(-1, 3)
    return (pos.reshape(-1, 3).astype(np.float32), uv.reshape(-1, 2).astype(np.float32),
            tris.astype(np.uint32))


def vertex_normals(positions: np.ndarray, triangles: np.ndarray) -> np.ndarray:
    p = positions.astype(np.float64)
    t = triangles.astype(np.int64)
    n = np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]])
    acc = np.zeros_like(p)
    for k in range(3):
        np.add.at(acc, t[:, k], n)
    length = np.linalg.norm(acc, axis=1, keepdims=True)
    acc = np.where(length > 1e-30, acc / np.maximum(length, 1e-30), np.array([0.0, 1.0, 0.0]))
    return acc.astype(np.float32)


def triangle_areas(positions: np.ndarray, triangles: np.ndarray) -> np.ndarray:
    p = positions.astype(np.float64)
    t = triangles.astype(np.int64)
    return 0.5 * np.linalg.norm(np.cross(p[t[:, 1]] - p[t[:, 0]], p[t[:, 2]] - p[t[:, 0]]), axis=1)


def surface_guides(positions, triangles, count, cvs, rng, length=(0.3, 0.6), jitter=0.02,
                   texcoords=None) -> GuideSet:
    """`count` guides rooted at area-weighted random surface points, each with
    `cvs` CVs running along the interpolated vertex normal for a length drawn
    from U(length), plus N(0, jitter) per-component jitter on CVs 1.."""
    areas = triangle_areas(positions, triangles)
    tri = rng.choice(triangles.shape[0], size=count, p=areas / areas.sum()).astype(np.int64)
    r1 = rng.random(count)
    r2 = rng.random(count)
    s = np.sqrt(r1)
    b = np.stack([1.0 - s, s * (1.0 - r2), s * r2], 1)
    t = triangles[tri].astype(np.int64)
    p = positions.astype(np.float64)
    root = (p[t[:, 0]] * b[:, :1] + p[t[:, 1]] * b[:, 1:2] + p[t[:, 2]] * b[:, 2:3])
    vn = vertex_normals(positions, triangles).astype(np.float64)
    nrm = vn[t[:, 0]] * b[:, :1] + vn[t[:, 1]] * b[:, 1:2] + vn[t[:, 2]] * b[:, 2:3]
    nrm /= np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
    lengths = rng.uniform(length[0], length[1], size=count)
    steps = np.linspace(0.0, 1.0, cvs)
    curve = root[:, None, :] + nrm[:, None, :] * (lengths[:, None, None] * steps[None, :, None])
    noise = rng.normal(0.0, jitter, size=curve.shape)
    noise[:, 0, :] = 0.0
    curve = (curve + noise).astype(np.float32)
    curve[:, 0, :] = root.astype(np.float32)
    uv = np.zeros((count, 2), np.float32)
    if texcoords is not None:
        tc = texcoords.astype(np.float64)
        uv = (tc[t[:, 0]] * b[:, :1] + tc[t[:, 1]] * b[:, 1:2] + tc[t[:, 2]] * b[:, 2:3]).astype(np.float32)
    return GuideSet(cv_counts=np.full(count, cvs, np.uint32), cvs=curve.reshape(-1, 3),
                    root_normals=nrm.astype(np.float32), root_uvs=uv, triangles=tri.astype(np.uint32),
                    barycentrics=b[:, 1:].astype(np.float32), support_radii=np.zeros(count, np.float32))


@dataclasses.dataclass
class Workload:
    name: str
    build_input: AssetBuildInput
    stencil_slots: int
    params: GenerationParams
    radius_scale: float = 1.0
    note: str = ""

    @property
    def points(self) -> int:
        return int(self.params.strand_count) * int(self.params.cvs_per_strand)


def plain_sphere(strands: int = 10_000, cvs: int = 16, seed: int = 2024) -> Workload:
    """Plain method, CPU-runnable size: unit UV sphere with 2,048 triangles
    (32 segments x 33 rings), 64 guides of 16 CVs, 4-guide stencils,
    10,000 strands x 16 points, taper 0.01 -> 0.001, noise 0.1 at frequency 8."""
    rng = np.random.default_rng(seed)
    pos, uv, tris = sphere_mesh(32, 33)
    guides = surface_guides(pos, tris, 64, 16, rng, texcoords=uv)
    params = GenerationParams(strand_count=strands, cvs_per_strand=cvs, seed=7, root_width=0.01,
                              tip_width=0.001, noise_amplitude=0.1, noise_frequency=8.0)
    return Workload("uv-sphere-2k-tris/64-guides/k4/10k-strands-x16", AssetBuildInput(pos, tris, guides, None, uv),
                    4, params)


# Per-CV guide jitter of the 32-CV guides: a tenth of the mean CV spacing
# (0.45 / 31).  Jitter comparable to the spacing folds guides back on
# themselves (consecutive tangents turning by close to 180 degrees), where the
# reference's transported frame (generate.h:475-481) is ill-conditioned: a
# one-ulp change of a base CV then moves noisy points by up to 1e-3.
GUIDE_JITTER_32 = 0.1 * 0.45 / 31


def displaced_sphere_radius(theta, phi):
    return 1.0 + 0.05 * np.sin(7.0 * theta) * np.sin(5.0 * phi)


def large_sphere(strands: int = 1_000_000, cvs: int = 32, guides: int = 4096, seed: int = 2025,
                 n_lon: int = 400, n_rings: int = 251, jitter: float = GUIDE_JITTER_32) -> Workload:
    """Single large description: displaced sphere (200,000 triangles, radial
    displacement 0.05 sin(7 theta) sin(5 phi)), 4,096 guides of 32 CVs,
    8-guide stencils, 1,000,000 strands x 32 points, taper 0.02 -> 0.002,
    noise 0.2 at frequency 12 (output 32M float4 = 512 MiB).  `jitter` is the
    guides' per-CV N(0, jitter) (the plain sphere's 0.02 is 1.4 CV spacings
    here; the default is a tenth of one)."""
    rng = np.random.default_rng(seed)
    pos, uv, tris = sphere_mesh(n_lon, n_rings, displaced_sphere_radius)
    gs = surface_guides(pos, tris, guides, 32, rng, texcoords=uv, jitter=jitter)
    params = GenerationParams(strand_count=strands, cvs_per_strand=cvs, seed=11, root_width=0.02,
                              tip_width=0.002, noise_amplitude=0.2, noise_frequency=12.0)
    name = "displaced-sphere-%dk-tris/%d-guides/k8/%d-strands-x%d" % (tris.shape[0] // 1000, guides, strands, cvs)
    return Workload(name, AssetBuildInput(pos, tris, gs, None, uv), 8, params)


# The Classic per-root expressions of the surrogate workload (SplinePrimitive
# length and width; $v is the root's v texture coordinate).
CLASSIC_LENGTH = "0.5*(1+0.4*noise($Prefg*6))*clamp(1-$v,0.2,1)"
CLASSIC_WIDTH = "0.01*(1+0.3*noise($Prefg*20))"


def classic_sphere(strands: int = 4_000_000, cvs: int = 24) -> Workload:
    """Learned-expression workload: the large displaced sphere (200,000
    triangles, 4,096 guides of 32 CVs, 8-guide stencils), 4,000,000 strands x
    24 points, generator noise off (the reference's default), per-root length
    and width from CLASSIC_LENGTH / CLASSIC_WIDTH."""
    w = large_sphere(strands=strands, cvs=cvs)
    params = w.params.copy(noise_amplitude=0.0)
    name = "displaced-sphere-200k-tris/4096-guides/k8/%d-strands-x%d/classic-length-width" % (strands, cvs)
    return Workload(name, w.build_input, w.stencil_slots, params)


def reference_unit_fixture() -> AssetBuildInput:
    """The one-triangle, one-guide asset the reference's unit tests use
    (tests/test_main.cpp:39-53)."""
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    nrm = np.array([[0, 1, 0]] * 3, np.float32)
    uv = np.array([[0, 0], [1, 0], [0, 1]], np.float32)
    tris = np.array([[0, 1, 2]], np.uint32)
    guides = GuideSet(cv_counts=np.array([3], np.uint32),
                      cvs=np.array([[0.25, 0.0, 0.25], [0.25, 0.5, 0.25], [0.5, 1.0, 0.25]], np.float32),
                      root_normals=np.array([[0, 1, 0]], np.float32), root_uvs=np.zeros((1, 2), np.float32),
                      triangles=np.array([0], np.uint32), barycentrics=np.array([[0.25, 0.25]], np.float32),
                      support_radii=np.array([10.0], np.float32))
    return AssetBuildInput(pos, tris, guides, nrm, uv)


def reference_area_fixture() -> AssetBuildInput:
    """Two triangles with areas 1.0 and 0.5 and one guide
    (tests/test_main.cpp:309-321)."""
    pos = np.array([[0, 0, 0], [2, 0, 0], [0, 0, 1], [10, 0, 0], [11, 0, 0], [10, 0, 1]], np.float32)
    nrm = np.array([[0, 1, 0]] * 6, np.float32)
    tris = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    guides = GuideSet(cv_counts=np.array([2], np.uint32), cvs=np.array([[0, 0, 0], [0, 1, 0]], np.float32),
                      root_normals=np.array([[0, 1, 0]], np.float32), root_uvs=np.zeros((1, 2), np.float32),
                      triangles=np.array([INVALID_INDEX], np.uint32), barycentrics=np.zeros((1, 2), np.float32),
                      support_radii=np.array([100.0], np.float32))
    return AssetBuildInput(pos, tris, guides, nrm, None)


def reference_benchmark_fixture() -> AssetBuildInput:
    """The reference benchmark's 10x10 quad with four 8-CV guides
    (tools/benchmark.cpp:22-41)."""
    pos = np.array([[-5, 0, -5], [5, 0, -5], [5, 0, 5], [-5, 0, 5]], np.float32)
    nrm = np.array([[0, 1, 0]] * 4, np.float32)
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    tris = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    roots = np.array([[-4, 0, -4], [4, 0, -4], [4, 0, 4], [-4, 0, 4]], np.float32)
    t = (np.arange(8, dtype=np.float32) / np.float32(7.0)).astype(np.float32)
    cvs = []
    for root in roots:
        for tv in t:
            cvs.append(root + np.array([np.float32(0.15) * tv * tv, np.float32(1.0) * tv,
                                        np.float32(0.08) * tv * tv], np.float32))
    guides = GuideSet(cv_counts=np.full(4, 8, np.uint32), cvs=np.array(cvs, np.float32),
                      root_normals=np.array([[0, 1, 0]] * 4, np.float32), root_uvs=np.zeros((4, 2), np.float32),
                      triangles=np.full(4, INVALID_INDEX, np.uint32), barycentrics=np.zeros((4, 2), np.float32),
                      support_radii=np.full(4, 12.0, np.float32))
    return AssetBuildInput(pos, tris, guides, nrm, uv)


@dataclasses.dataclass
class MotionFrames:
    """Deformed geometry of one description at several shutter times."""
    times: np.ndarray                 # (n,) float32, strictly increasing
    positions: list                   # n x (V, 3) float32
    normals: list                     # n x (V, 3) float32
    guide_cvs: list                   # n x (GCV, 3) float32


def motion_frames(build_input: AssetBuildInput, samples: int = 5, amplitude: float = 0.03,
                  seed: int = 4242) -> MotionFrames:
    """Seeded per-vertex sinusoidal displacement over `samples` shutter times:
    v(t) = v + amplitude * sin(2 pi t + phase_v) * dir_v, normals recomputed
    per sample, every guide translated with the displacement of its root's
    triangle (the same transform as its patch), topology and root identities
    shared."""
    rng = np.random.default_rng(seed)
    pos = build_input.positions.astype(np.float64)
    tris = build_input.triangles.astype(np.int64)
    V = pos.shape[0]
    phase = rng.uniform(0.0, 2.0 * math.pi, V)
    direction = rng.normal(size=(V, 3))
    direction /= np.linalg.norm(direction, axis=1, keepdims=True)
    g = build_input.guides
    counts = np.asarray(g.cv_counts, np.int64)
    owner = np.repeat(np.arange(counts.size), counts)
    gtri = np.asarray(g.triangles, np.int64)
    bound = gtri < tris.shape[0]
    bary = np.asarray(g.barycentrics, np.float64)
    b0 = 1.0 - bary[:, 0] - bary[:, 1]
    times = np.linspace(0.0, 1.0, samples).astype(np.float32)
    frames = MotionFrames(times, [], [], [])
    cvs = np.asarray(g.cvs, np.float64)
    for t in times:
        disp = amplitude * np.sin(2.0 * math.pi * float(t) + phase)[:, None] * direction
        moved = pos + disp
        frames.positions.append(moved.astype(np.float32))
        frames.normals.append(vertex_normals(moved.astype(np.float32), build_input.triangles))
        gd = np.zeros((counts.size, 3))
        t3 = tris[np.where(bound, gtri, 0)]
        gd[bound] = (disp[t3[bound, 0]] * b0[bound, None] + disp[t3[bound, 1]] * bary[bound, 0:1] +
                     disp[t3[bound, 2]] * bary[bound, 1:2])
        frames.guide_cvs.append((cvs + gd[owner]).astype(np.float32))
    return frames


@dataclasses.dataclass
class Batch:
    """Several descriptions on one mesh, each with its own guides and settings."""
    name: str
    workloads: list   # of Workload

    @property
    def points(self) -> int:
        return sum(w.points for w in self.workloads)

    @property
    def strands(self) -> int:
        return sum(int(w.params.strand_count) for w in self.workloads)


BATCH_CVS = (8, 12, 16, 24, 32, 48, 64)


def batched_descriptions(count: int = 9, n_lon: int = 1000, n_rings: int = 251, strands=(20_000, 1_000_000),
                         guides=(512, 2048), seed: int = 2026, size_seed: int = 2590) -> Batch:
    """Multi-description frame: `count` descriptions on one displaced sphere
    (1000 x 251 -> 500,000 triangles), each with its own seeded guides
    (count drawn from `guides`), stencil size 4 or 8, strand count
    log-uniform in `strands`, CVs per strand from {8,12,16,24,32,48,64}, and
    its own taper and noise (two in three descriptions noisy).  Strand and CV
    counts come from their own stream (`size_seed`; the default gives
    2,493,172 strands and 46,200,484 points for nine descriptions)."""
    sizes = np.random.default_rng(size_seed)
    lo, hi = math.log(strands[0]), math.log(strands[1])
    counts = [int(round(math.exp(sizes.uniform(lo, hi)))) for _ in range(count)]
    cv_counts = [int(sizes.choice(BATCH_CVS)) for _ in range(count)]
    rng = np.random.default_rng(seed)
    pos, uv, tris = sphere_mesh(n_lon, n_rings, displaced_sphere_radius)
    out = []
    for d in range(count):
        cvs, S = cv_counts[d], counts[d]
        g = int(rng.integers(guides[0], guides[1] + 1))
        gcv = max(cvs, 8)
        gs = surface_guides(pos, tris, g, gcv, rng, texcoords=uv, jitter=0.1 * 0.45 / (gcv - 1))
        noisy = rng.random() < 2.0 / 3.0
        params = GenerationParams(strand_count=S, cvs_per_strand=cvs, seed=100 + d,
                                  root_width=float(rng.uniform(0.005, 0.03)), tip_width=0.001,
                                  noise_amplitude=float(rng.uniform(0.05, 0.2)) if noisy else 0.0,
                                  noise_frequency=float(rng.uniform(4.0, 12.0)))
        k = int(rng.choice([4, 8]))
        out.append(Workload("desc%d/%d-guides/k%d/%d-strands-x%d%s" % (d, g, k, S, cvs, "/noise" if noisy else ""),
                            AssetBuildInput(pos, tris, gs, None, uv), k, params))
    total_tris = tris.shape[0]
    return Batch("%d-descriptions-on-%dk-tris" % (count, total_tris // 1000), out)
