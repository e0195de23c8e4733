"""Device-side generation API over libnxg_b200.so.

This is the Python face of the C ABI in include/nxg.h: ``DeviceAsset`` is
the uploaded blob plus its checked descriptor (asset.cpp:364-378
make_device_asset_descriptor), ``generate_packed`` is the device form of
``generate_packed_cpu`` / ``generate_packed_deformed_cpu`` (asset.cpp:412-449)
and returns the reference's renderer layout (float4(position, radius) per CV,
point counts, roots, root UVs) in CUDA tensors.  torch provides device memory
and streams only; every kernel is the library's.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Sequence

import numpy as np
import torch

from . import _abi
from ._abi import (DeformedDesc, DeviceAssetDesc, GenerationParams, LaunchConfig, PackedOutputDesc,
                   check, lib)
from .asset import Asset, aligned_struct


def _stream_handle(stream: Optional[torch.cuda.Stream]) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else int(t.data_ptr())


def build_stencils(positions: torch.Tensor, triangles: torch.Tensor, guide_roots: torch.Tensor,
                   guide_normals: torch.Tensor, stencil_slots: int = 8,
                   out: Optional[torch.Tensor] = None, stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """The stencil search of build_asset (asset.cpp:252-269) on CUDA tensors:
    positions [V, 3] float32, triangles [T, 3] int32 (vertex indices),
    guide_roots / guide_normals [G, 3] float32 (first CVs, normalized root
    normals).  Returns `out` or a new [T, 8] int32 tensor whose bits are the
    uint32 guide indices (INVALID_INDEX reads as -1)."""
    for t in (positions, triangles, guide_roots, guide_normals):
        if not t.is_cuda or not t.is_contiguous() or t.dim() != 2 or t.shape[1] != 3:
            raise ValueError("expected contiguous [n, 3] CUDA tensors")
    if positions.dtype != torch.float32 or guide_roots.dtype != torch.float32 or \
            guide_normals.dtype != torch.float32 or triangles.dtype != torch.int32:
        raise ValueError("positions, guide_roots, guide_normals float32; triangles int32")
    if guide_roots.shape != guide_normals.shape:
        raise ValueError("guide_roots and guide_normals differ in shape")
    tris = triangles.shape[0]
    if out is None:
        out = torch.empty((tris, 8), dtype=torch.int32, device=positions.device)
    check(lib().nxg_build_stencils_device(positions.data_ptr(), positions.shape[0], triangles.data_ptr(), tris,
                                          guide_roots.data_ptr(), guide_normals.data_ptr(), guide_roots.shape[0],
                                          stencil_slots, out.data_ptr(), _stream_handle(stream)),
          "build_stencils_device")
    return out


class DeviceAsset:
    """A validated asset copied to device memory, with its checked descriptor."""

    def __init__(self, asset: Asset, device: str | torch.device = "cuda",
                 stream: Optional[torch.cuda.Stream] = None):
        self.asset = asset
        self.device = torch.device(device)
        self.tensor = torch.empty(asset.nbytes, dtype=torch.uint8, device=self.device)
        host = torch.from_numpy(asset.buffer)
        with torch.cuda.stream(stream) if stream is not None else _nullcontext():
            self.tensor.copy_(host, non_blocking=False)
        self.desc = aligned_struct(DeviceAssetDesc)
        msg = ctypes.create_string_buffer(256)
        code = lib().nxg_make_device_asset_descriptor(asset.buffer.ctypes.data, asset.nbytes,
                                                      self.tensor.data_ptr(), asset.nbytes,
                                                      ctypes.byref(self.desc), msg, 256)
        if code:
            raise _abi.NxgError(code, "make_device_asset_descriptor " + msg.value.decode())
        self._workspaces: dict[tuple, torch.Tensor] = {}

    @property
    def header(self):
        return self.desc.header

    def workspace(self, params: GenerationParams, strand_count: int) -> torch.Tensor:
        """A cached device workspace for `strand_count` strands of `params`
        (256-byte aligned; reused by every call with the same sizes)."""
        need = int(lib().nxg_packed_workspace_size(ctypes.byref(self.desc), ctypes.byref(params), strand_count))
        key = (strand_count, int(params.cvs_per_strand))
        ws = self._workspaces.get(key)
        if ws is None or ws.numel() < need:
            ws = torch.empty(max(need, 256), dtype=torch.uint8, device=self.device)
            assert ws.data_ptr() % 256 == 0
            self._workspaces[key] = ws
        return ws


class _nullcontext:
    def __enter__(self):
        return None

    def __exit__(self, *exc):
        return False


@dataclasses.dataclass
class DeformedGeometry:
    """Frame-local overlays (types.h:152-160); None selects the rest array."""
    positions: Optional[torch.Tensor] = None   # (V, 3) float32 on device
    normals: Optional[torch.Tensor] = None     # (V, 3)
    guide_cvs: Optional[torch.Tensor] = None   # (GCV, 3)

    def descriptor(self) -> DeformedDesc:
        d = DeformedDesc()
        for name, count in (("positions", "position_count"), ("normals", "normal_count"),
                            ("guide_cvs", "guide_cv_count")):
            t = getattr(self, name)
            if t is not None:
                if t.dtype != torch.float32 or not t.is_contiguous():
                    raise ValueError(name + " must be a contiguous float32 tensor")
                setattr(d, name, t.data_ptr())
                setattr(d, count, t.numel() // 3)
        return d


@dataclasses.dataclass
class PackedCurves:
    """Renderer output (asset.h:74-81 PackedGeneratedCurves) in device tensors."""
    strand_count: int
    cvs_per_strand: int
    points: torch.Tensor                     # (S*P, 4) float32
    point_counts: Optional[torch.Tensor]     # (S,) int32 (uint32 bits)
    roots: Optional[torch.Tensor]            # (S, 12) int32 words of RootSample
    root_uvs: Optional[torch.Tensor]         # (S, 2) float32

    def roots_numpy(self) -> np.ndarray:
        return self.roots.cpu().numpy().view(_abi.ROOT_DTYPE).reshape(-1)


def packed_output_descriptor(points: torch.Tensor, roots=None, root_uvs=None, point_counts=None,
                             radius_scale: float = 1.0) -> PackedOutputDesc:
    out = PackedOutputDesc()
    out.points = points.data_ptr()
    out.point_capacity = points.numel() // 4
    out.radius_scale = radius_scale
    if roots is not None:
        out.roots = roots.data_ptr()
        out.root_capacity = roots.numel() // 12
    if root_uvs is not None:
        out.root_uvs = root_uvs.data_ptr()
        out.root_uv_capacity = root_uvs.numel() // 2
    if point_counts is not None:
        out.point_counts = point_counts.data_ptr()
        out.point_count_capacity = point_counts.numel()
    return out


def allocate_outputs(strands: int, cvs: int, device, roots: bool = True, root_uvs: bool = True,
                     point_counts: bool = True):
    points = torch.empty((strands * cvs, 4), dtype=torch.float32, device=device)
    r = torch.empty((strands, 12), dtype=torch.int32, device=device) if roots else None
    uv = torch.empty((strands, 2), dtype=torch.float32, device=device) if root_uvs else None
    pc = torch.empty((strands,), dtype=torch.int32, device=device) if point_counts else None
    return points, r, uv, pc


def generate_packed(dasset: DeviceAsset, params: GenerationParams, radius_scale: float = 1.0,
                    deformed: Optional[DeformedGeometry] = None, *, first_strand: int = 0,
                    count: Optional[int] = None, points: Optional[torch.Tensor] = None,
                    roots: Optional[torch.Tensor] = None, root_uvs: Optional[torch.Tensor] = None,
                    point_counts: Optional[torch.Tensor] = None, want_roots: bool = True,
                    block_size: int = 128, stream: Optional[torch.cuda.Stream] = None) -> PackedCurves:
    """Enqueue generation of strands [first_strand, first_strand + count) on
    `stream` (default: torch's current stream).  Output buffers are allocated
    when not supplied.  Raises NxgError with the reference's error message
    on any contract violation."""
    n = int(params.strand_count) - first_strand if count is None else int(count)
    cvs = int(params.cvs_per_strand)
    if points is None:
        points, r, uv, pc = allocate_outputs(n, cvs, dasset.device, want_roots, want_roots, want_roots)
        roots = roots if roots is not None else r
        root_uvs = root_uvs if root_uvs is not None else uv
        point_counts = point_counts if point_counts is not None else pc
    out = packed_output_descriptor(points, roots, root_uvs, point_counts, radius_scale)
    ddesc = deformed.descriptor() if deformed is not None else DeformedDesc()
    cfg = LaunchConfig(block_size)
    ws = dasset.workspace(params, max(n, 1))
    handle = _stream_handle(stream)
    if first_strand == 0 and n == int(params.strand_count):
        code = lib().nxg_generate_packed(ctypes.byref(dasset.desc), ctypes.byref(ddesc), ctypes.byref(params),
                                         ctypes.byref(out), ctypes.byref(cfg), ws.data_ptr(), ws.numel(), handle)
    else:
        code = lib().nxg_generate_packed_range(ctypes.byref(dasset.desc), ctypes.byref(ddesc),
                                               ctypes.byref(params), ctypes.byref(out), ctypes.byref(cfg),
                                               first_strand, n, ws.data_ptr(), ws.numel(), handle)
    check(code, "nxg_generate_packed")
    return PackedCurves(n, cvs, points, point_counts, roots, root_uvs)


def query_strand_states(dasset: DeviceAsset, params: GenerationParams, strands: Sequence[int] | np.ndarray,
                        deformed: Optional[DeformedGeometry] = None,
                        stream: Optional[torch.cuda.Stream] = None) -> np.ndarray:
    """Per-strand root and stencil blend state (nxg_strand_state records),
    evaluated by the generator's device functions; synchronises."""
    ids = torch.as_tensor(np.asarray(strands, dtype=np.uint32).view(np.int32), device=dasset.device)
    out = torch.empty((ids.numel(), _abi.STATE_DTYPE.itemsize // 4), dtype=torch.int32, device=dasset.device)
    ddesc = deformed.descriptor() if deformed is not None else DeformedDesc()
    code = lib().nxg_query_strand_states(ctypes.byref(dasset.desc), ctypes.byref(ddesc), ctypes.byref(params),
                                         ids.data_ptr(), ids.numel(), out.data_ptr(), _stream_handle(stream))
    check(code, "nxg_query_strand_states")
    torch.cuda.synchronize(dasset.device)
    return out.cpu().numpy().view(_abi.STATE_DTYPE).reshape(-1)


def query_walk_states(dasset: DeviceAsset, params: GenerationParams, strands: Sequence[int] | np.ndarray,
                      deformed: Optional[DeformedGeometry] = None,
                      stream: Optional[torch.cuda.Stream] = None) -> np.ndarray:
    """The lane-walk generator's own stencil decisions per strand
    (nxg_walk_state records: blend mode, nearest guide, the weight sum the
    mode was decided on, the weighted slots), for global strand ids."""
    ids = torch.as_tensor(np.asarray(strands, np.uint32).view(np.int32), device=dasset.device)
    out = torch.empty((ids.numel(), _abi.WALK_STATE_DTYPE.itemsize // 4), dtype=torch.int32, device=dasset.device)
    ddesc = deformed.descriptor() if deformed is not None else DeformedDesc()
    ws = dasset.workspace(params, max(1, ids.numel()))
    code = lib().nxg_query_walk_states(ctypes.byref(dasset.desc), ctypes.byref(ddesc), ctypes.byref(params),
                                       ids.data_ptr(), ids.numel(), out.data_ptr(), ws.data_ptr(),
                                       ws.numel() * ws.element_size(), _stream_handle(stream))
    check(code, "nxg_query_walk_states")
    torch.cuda.synchronize(dasset.device)
    return out.cpu().numpy().view(_abi.WALK_STATE_DTYPE).reshape(-1)


def validate_packed_request(dasset_desc: DeviceAssetDesc, params: GenerationParams, output: PackedOutputDesc,
                            deformed: Optional[DeformedDesc] = None, block_size: int = 128) -> int:
    """nxg_validate_packed_request (device_contract.h:221-254); pure host."""
    cfg = LaunchConfig(block_size)
    return int(lib().nxg_validate_packed_request(ctypes.byref(dasset_desc),
                                                 ctypes.byref(deformed) if deformed is not None else None,
                                                 ctypes.byref(params), ctypes.byref(output), ctypes.byref(cfg)))


def prepare_strand_order(dasset: DeviceAsset, params: GenerationParams, first_strand: int = 0,
                         count: Optional[int] = None, stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """Phase 1 (nxg_prepare_strand_order): sort the strand range into the
    asset's cached workspace, which is returned for phase 2."""
    n = int(params.strand_count) - first_strand if count is None else int(count)
    ws = dasset.workspace(params, max(n, 1))
    check(lib().nxg_prepare_strand_order(ctypes.byref(dasset.desc), ctypes.byref(params), first_strand, n,
                                         ws.data_ptr(), ws.numel(), _stream_handle(stream)),
          "nxg_prepare_strand_order")
    return ws


def generate_packed_ordered(dasset: DeviceAsset, params: GenerationParams, points: torch.Tensor,
                            roots=None, root_uvs=None, point_counts=None, radius_scale: float = 1.0,
                            deformed: Optional[DeformedGeometry] = None, first_strand: int = 0,
                            count: Optional[int] = None, workspace: Optional[torch.Tensor] = None,
                            block_size: int = 128, stream: Optional[torch.cuda.Stream] = None) -> None:
    """Phase 2 (nxg_generate_packed_ordered) over a workspace prepared by
    prepare_strand_order for the same range."""
    n = int(params.strand_count) - first_strand if count is None else int(count)
    if workspace is None:
        workspace = dasset.workspace(params, max(n, 1))
    out = packed_output_descriptor(points, roots, root_uvs, point_counts, radius_scale)
    ddesc = deformed.descriptor() if deformed is not None else DeformedDesc()
    cfg = LaunchConfig(block_size)
    check(lib().nxg_generate_packed_ordered(
        ctypes.byref(dasset.desc), ctypes.byref(ddesc), ctypes.byref(params), ctypes.byref(out),
        ctypes.byref(cfg), first_strand, n, workspace.data_ptr(), workspace.numel(), _stream_handle(stream)),
        "nxg_generate_packed_ordered")


class HostPipeline:
    """The reference API's contract -- host asset in, host arrays out
    (generate_packed_cpu, asset.cpp:412-419) -- served by the GPU.

    Each run() uploads the asset from pinned memory on an upload stream,
    generates the strands in `chunks` ranges on a compute stream and copies
    every finished range to pinned host arrays on a copy stream.  Readback
    overlaps generation, and a run's upload and generation overlap the
    previous run's readback: a range is regenerated once its previous
    readback is done, and the asset is replaced once the previous run's
    generation no longer reads it.  The readback (device to host) and the
    upload (host to device) use the two directions of the link."""

    def __init__(self, asset: Asset, params: GenerationParams, radius_scale: float = 1.0, chunks: int = 8,
                 device: str | torch.device = "cuda", first_strand: int = 0, count: Optional[int] = None):
        self.params = params
        self.radius_scale = radius_scale
        self.first = first_strand
        self.count = int(params.strand_count) - first_strand if count is None else int(count)
        self.dasset = DeviceAsset(asset, device)
        self.pinned_asset = torch.from_numpy(asset.buffer).pin_memory()
        P = int(params.cvs_per_strand)
        self.points, self.roots, self.root_uvs, self.point_counts = allocate_outputs(self.count, P, device)
        self.host_points = torch.empty(self.points.shape, dtype=torch.float32, pin_memory=True)
        self.host_roots = torch.empty(self.roots.shape, dtype=torch.int32, pin_memory=True)
        self.host_uvs = torch.empty(self.root_uvs.shape, dtype=torch.float32, pin_memory=True)
        self.host_counts = torch.empty(self.point_counts.shape, dtype=torch.int32, pin_memory=True)
        self.compute = torch.cuda.Stream(device)
        self.copy = torch.cuda.Stream(device)
        self.upload = torch.cuda.Stream(device)
        bounds = np.linspace(0, self.count, max(1, chunks) + 1).astype(np.int64)
        self.ranges = [(int(a), int(b)) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]
        self.events = [torch.cuda.Event() for _ in self.ranges]      # range generated
        self.read_back = [None for _ in self.ranges]                 # range copied out (previous run)
        for a, b in self.ranges:
            self.dasset.workspace(params, b - a)

    @property
    def h2d_bytes(self) -> int:
        return int(self.pinned_asset.numel())

    @property
    def d2h_bytes(self) -> int:
        return sum(int(t.numel()) * 4 for t in (self.points, self.roots, self.root_uvs, self.point_counts))

    def run(self) -> None:
        """Enqueue one full upload -> generate -> readback; returns without
        synchronising (wait on `self.copy`)."""
        P = int(self.params.cvs_per_strand)
        with torch.cuda.stream(self.upload):
            self.upload.wait_stream(self.compute)  # the previous run's generation is done with the asset
            self.dasset.tensor.copy_(self.pinned_asset, non_blocking=True)
        with torch.cuda.stream(self.compute):
            self.compute.wait_stream(self.upload)
            for i, ((a, b), ev) in enumerate(zip(self.ranges, self.events)):
                if self.read_back[i] is not None:
                    self.compute.wait_event(self.read_back[i])  # previous readback done with this range
                n = b - a
                generate_packed(self.dasset, self.params, self.radius_scale, first_strand=self.first + a,
                                count=n, points=self.points[a * P:b * P], roots=self.roots[a:b],
                                root_uvs=self.root_uvs[a:b], point_counts=self.point_counts[a:b],
                                stream=self.compute)
                ev.record(self.compute)
        with torch.cuda.stream(self.copy):
            for i, ((a, b), ev) in enumerate(zip(self.ranges, self.events)):
                self.copy.wait_event(ev)
                self.host_points[a * P:b * P].copy_(self.points[a * P:b * P], non_blocking=True)
                self.host_roots[a:b].copy_(self.roots[a:b], non_blocking=True)
                self.host_uvs[a:b].copy_(self.root_uvs[a:b], non_blocking=True)
                self.host_counts[a:b].copy_(self.point_counts[a:b], non_blocking=True)
                done = torch.cuda.Event()
                done.record(self.copy)
                self.read_back[i] = done


def set_tile(cvs_per_strand: int, noise: bool, lanes: int = 0, cvs_per_lane: int = 0, block_size: int = 0) -> None:
    """nxg_set_tile; lanes == 0 restores the built-in tile."""
    tile = _abi.Tile(lanes, cvs_per_lane, block_size) if lanes else None
    check(lib().nxg_set_tile(cvs_per_strand, 1 if noise else 0, ctypes.byref(tile) if tile else None),
          "nxg_set_tile")


def get_tile(cvs_per_strand: int, noise: bool) -> tuple[int, int, int]:
    tile = _abi.Tile()
    check(lib().nxg_get_tile(cvs_per_strand, 1 if noise else 0, ctypes.byref(tile)), "nxg_get_tile")
    return tile.lanes_per_strand, tile.cvs_per_lane, tile.block_size


def autotune(dasset: DeviceAsset, params: GenerationParams, points: torch.Tensor, *, first_strand: int = 0,
             count: Optional[int] = None, repeats: int = 3, stream: Optional[torch.cuda.Stream] = None):
    """nxg_autotune_packed over `points` (overwritten): returns
    ((lanes, cvs_per_lane, block_size), ms) and registers the winner."""
    n = int(params.strand_count) - first_strand if count is None else int(count)
    out = packed_output_descriptor(points)
    ws = dasset.workspace(params, max(n, 1))
    tile = _abi.Tile()
    ms = ctypes.c_float()
    check(lib().nxg_autotune_packed(ctypes.byref(dasset.desc), ctypes.byref(DeformedDesc()), ctypes.byref(params),
                                    ctypes.byref(out), first_strand, n, ws.data_ptr(), ws.numel(), repeats,
                                    _stream_handle(stream), ctypes.byref(tile), ctypes.byref(ms)),
          "nxg_autotune_packed")
    return (tile.lanes_per_strand, tile.cvs_per_lane, tile.block_size), float(ms.value)


def _motion_samples(frames, times) -> "ctypes.Array":
    samples = (_abi.MotionSampleDesc * len(frames))()
    for s, f, t in zip(samples, frames, times):
        s.deformation = f.descriptor()
        s.time = float(t)
    return samples


def generate_motion_packed(dasset: DeviceAsset, params: GenerationParams, frames: Sequence[DeformedGeometry],
                           times: Sequence[float], radius_scale: float = 1.0, outputs=None,
                           block_size: int = 128, stream: Optional[torch.cuda.Stream] = None) -> list:
    """nxg_generate_motion_packed: one packed output per shutter sample."""
    S, P = int(params.strand_count), int(params.cvs_per_strand)
    if outputs is None:
        outputs = [allocate_outputs(S, P, dasset.device) for _ in frames]
    descs = (PackedOutputDesc * len(frames))(*[packed_output_descriptor(o[0], o[1], o[2], o[3], radius_scale)
                                               for o in outputs])
    samples = _motion_samples(frames, times)
    ws = dasset.workspace(params, S)
    check(lib().nxg_generate_motion_packed(ctypes.byref(dasset.desc), samples, len(frames), ctypes.byref(params),
                                           descs, ctypes.byref(LaunchConfig(block_size)), ws.data_ptr(),
                                           ws.numel(), _stream_handle(stream)), "nxg_generate_motion_packed")
    return [PackedCurves(S, P, *o[:1], o[3], o[1], o[2]) for o in outputs]


def generate_motion(dasset: DeviceAsset, params: GenerationParams, frames: Sequence[DeformedGeometry],
                    times: Sequence[float], points: Optional[torch.Tensor] = None, block_size: int = 128,
                    stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
    """nxg_generate_motion (device_contract.h:42-53): sample-major absolute
    Vec3 positions, shape (samples, strands * cvs, 3)."""
    S, P = int(params.strand_count), int(params.cvs_per_strand)
    if points is None:
        points = torch.empty((len(frames), S * P, 3), dtype=torch.float32, device=dasset.device)
    out = _abi.MotionOutputDesc(points=points.data_ptr(), point_capacity=points.numel() // 3)
    samples = _motion_samples(frames, times)
    ws = dasset.workspace(params, S)
    check(lib().nxg_generate_motion(ctypes.byref(dasset.desc), samples, len(frames), ctypes.byref(params),
                                    ctypes.byref(out), ctypes.byref(LaunchConfig(block_size)), ws.data_ptr(),
                                    ws.numel(), _stream_handle(stream)), "nxg_generate_motion")
    return points


class BatchRunner:
    """nxg_generate_batched over several uploaded descriptions, with the
    output buffers and the workspace allocated once."""

    def __init__(self, dassets: Sequence[DeviceAsset], params: Sequence[GenerationParams],
                 radius_scale: float = 1.0, with_roots: bool = True):
        self.dassets = list(dassets)
        self.params = list(params)
        device = self.dassets[0].device
        n = len(self.dassets)
        self._assets = (DeviceAssetDesc * n)()
        for i, d in enumerate(self.dassets):
            ctypes.memmove(ctypes.byref(self._assets[i]), ctypes.byref(d.desc), ctypes.sizeof(DeviceAssetDesc))
        self._params = (GenerationParams * n)(*self.params)
        self.outputs = [allocate_outputs(int(p.strand_count), int(p.cvs_per_strand), device, with_roots, with_roots,
                                         with_roots) for p in self.params]
        self._outs = (PackedOutputDesc * n)(*[packed_output_descriptor(o[0], o[1], o[2], o[3], radius_scale)
                                              for o in self.outputs])
        need = int(lib().nxg_batched_workspace_size(self._assets, self._params, n))
        if need == 0:
            raise ValueError("batch of %d descriptions is empty or exceeds NXG_MAX_BATCH" % n)
        self.workspace = torch.empty(need, dtype=torch.uint8, device=device)

    @property
    def points(self) -> int:
        return sum(int(p.strand_count) * int(p.cvs_per_strand) for p in self.params)

    def run(self, block_size: int = 128, stream: Optional[torch.cuda.Stream] = None,
            scalars: Optional[Sequence[Optional[torch.Tensor]]] = None, apply_length: bool = True,
            apply_width: bool = True) -> None:
        """One batched frame; with `scalars` (per description an (n, 2) Classic
        (length scale, width) tensor or None) the Classic application is fused
        into generation (nxg_generate_batched_classic)."""
        cfg = ctypes.byref(LaunchConfig(block_size))
        if scalars is None:
            check(lib().nxg_generate_batched(self._assets, None, self._params, self._outs, len(self.dassets), cfg,
                                             self.workspace.data_ptr(), self.workspace.numel(),
                                             _stream_handle(stream)), "nxg_generate_batched")
            return
        classic = (_abi.ClassicApplyDesc * len(self.dassets))()
        for i, t in enumerate(scalars):
            if t is not None:
                classic[i] = _abi.ClassicApplyDesc(t.data_ptr(), int(apply_length), int(apply_width))
        check(lib().nxg_generate_batched_classic(self._assets, None, self._params, self._outs, classic,
                                                 len(self.dassets), cfg, self.workspace.data_ptr(),
                                                 self.workspace.numel(), _stream_handle(stream)),
              "nxg_generate_batched_classic")

    def curves(self) -> list:
        return [PackedCurves(int(p.strand_count), int(p.cvs_per_strand), o[0], o[3], o[1], o[2])
                for p, o in zip(self.params, self.outputs)]
