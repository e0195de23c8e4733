"""Host side of the .nxg asset: build, validate, save and load.

Mirrors the reference's asset API (include/nanoxgen/asset.h:14-128,
src/asset.cpp:229-378) over the C ABI of libnxg_b200.so.  An ``Asset`` owns
its blob in a 64-byte aligned host buffer, as the reference's
AlignedByteVector does (blob_storage.h:11-63).
"""
from __future__ import annotations

import ctypes
import dataclasses
import os
from typing import Optional

import numpy as np

from . import _abi
from ._abi import AssetBuildInput as _CBuildInput
from ._abi import AssetHeader, lib


def aligned_empty(nbytes: int, alignment: int = 64) -> np.ndarray:
    """A uint8 array of `nbytes` whose data pointer is `alignment`-aligned."""
    raw = np.empty(nbytes + alignment, dtype=np.uint8)
    offset = (-raw.ctypes.data) % alignment
    return raw[offset:offset + nbytes]


def aligned_struct(cls):
    """A ctypes structure instance placed at a 64-byte aligned address."""
    buf = aligned_empty(ctypes.sizeof(cls))
    buf[:] = 0
    inst = cls.from_buffer(buf)
    inst._keepalive = buf
    return inst


@dataclasses.dataclass
class GuideSet:
    """Guide curves of an AssetBuildInput (asset.h:14-32), as flat arrays."""
    cv_counts: np.ndarray        # (G,) uint32, each in [2, 65535]
    cvs: np.ndarray              # (sum(cv_counts), 3) float32; CV 0 is the root
    root_normals: np.ndarray     # (G, 3) float32
    root_uvs: np.ndarray         # (G, 2) float32
    triangles: np.ndarray        # (G,) uint32, INVALID_INDEX when unbound
    barycentrics: np.ndarray     # (G, 2) float32
    support_radii: np.ndarray    # (G,) float32, 0 selects the automatic radius


@dataclasses.dataclass
class AssetBuildInput:
    """asset.h:34-44 AssetBuildInput."""
    positions: np.ndarray               # (V, 3) float32
    triangles: np.ndarray               # (T, 3) uint32
    guides: GuideSet
    normals: Optional[np.ndarray] = None    # (V, 3) float32, None = computed
    texcoords: Optional[np.ndarray] = None  # (V, 2) float32


def _c(array: np.ndarray, dtype) -> np.ndarray:
    return np.ascontiguousarray(array, dtype=dtype)


class Asset:
    """A validated, relocatable .nxg blob in aligned host memory."""

    def __init__(self, data: bytes | np.ndarray, validate: bool = True):
        raw = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
        self._buf = aligned_empty(raw.size)
        self._buf[:] = raw.view(np.uint8).reshape(-1)
        if validate:
            error = validate_asset(self._buf)
            if error:
                raise ValueError("invalid NanoXGen asset: " + error)

    @property
    def buffer(self) -> np.ndarray:
        return self._buf

    @property
    def nbytes(self) -> int:
        return int(self._buf.size)

    def bytes(self) -> bytes:
        return self._buf.tobytes()

    @property
    def header(self) -> AssetHeader:
        return AssetHeader.from_buffer_copy(self._buf[:_abi.HEADER_SIZE].tobytes())

    def section(self, name: str, dtype, count: int, width: int = 1) -> np.ndarray:
        """A read-only numpy view of one section (device_view.h:19-29)."""
        offset = getattr(self.header, name + "_offset")
        if offset == 0:
            return np.zeros((0, width) if width > 1 else (0,), dtype=dtype)
        n = count * width
        view = self._buf[offset:offset + n * np.dtype(dtype).itemsize].view(dtype)
        return view.reshape(count, width) if width > 1 else view

    def positions(self) -> np.ndarray:
        return self.section("positions", np.float32, self.header.vertex_count, 3)

    def normals(self) -> np.ndarray:
        return self.section("normals", np.float32, self.header.vertex_count, 3)

    def guide_cvs(self) -> np.ndarray:
        return self.section("guide_cvs", np.float32, self.header.guide_cv_count, 3)

    def triangles(self) -> np.ndarray:
        return self.section("triangles", np.uint32, self.header.triangle_count, 3)

    def stencil(self) -> np.ndarray:
        return self.section("triangle_guides", np.uint32, self.header.triangle_count, 8)

    def guides(self) -> np.ndarray:
        h = self.header
        return self._buf[h.guides_offset:h.guides_offset + 56 * h.guide_count].view(_abi.GUIDE_DTYPE)

    def bbox_diagonal(self) -> float:
        p = self.positions().astype(np.float64)
        return float(np.linalg.norm(p.max(axis=0) - p.min(axis=0)))

    def save(self, path: str) -> None:
        """asset.cpp:340-348 save_asset."""
        error = validate_asset(self._buf)
        if error:
            raise RuntimeError("refusing to save invalid asset: " + error)
        with open(path, "wb") as handle:
            handle.write(self._buf.tobytes())


def validate_asset(data: np.ndarray | bytes) -> str:
    """asset.cpp:295-338 validate_asset: '' when valid, else the message."""
    if not isinstance(data, np.ndarray) or data.ctypes.data % 64 != 0:
        raw = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
        buf = aligned_empty(raw.size)
        buf[:] = raw.view(np.uint8).reshape(-1)
        data = buf
    msg = ctypes.create_string_buffer(256)
    lib().nxg_validate_asset(data.ctypes.data, data.size, msg, 256)
    return msg.value.decode()


def load_asset(path: str) -> Asset:
    """asset.cpp:350-362 load_asset."""
    with open(path, "rb") as handle:
        return Asset(handle.read())


def build_asset(source: AssetBuildInput, stencil_slots: int = 8, workers: int = 0) -> Asset:
    """asset.cpp:229-293 build_asset.  `stencil_slots` < 8 writes the slots
    beyond it as INVALID_INDEX (a K-guide stencil in the 8-slot format)."""
    return _build(source, stencil_slots, workers, None)


def build_asset_device(source: AssetBuildInput, stencil_slots: int = 8, stream=None) -> Asset:
    """build_asset with its all-pairs searches on the current CUDA device:
    the per-triangle stencil (asset.cpp:252-269, triangles x guides
    candidates) and the automatic support radius's nearest roots
    (asset.cpp:88-97); the blob is byte-identical to build_asset's.  `stream` is a torch.cuda.Stream, a raw
    cudaStream_t handle or None (the legacy default stream)."""
    handle = getattr(stream, "cuda_stream", stream) or 0
    return _build(source, stencil_slots, 0, int(handle))


def _build(source: AssetBuildInput, stencil_slots: int, workers: int, stream: Optional[int]) -> Asset:
    g = source.guides
    keep = []

    def ptr(array, dtype, shape_tail=None):
        if array is None:
            return None
        a = _c(array, dtype)
        if shape_tail is not None:
            a = a.reshape((-1,) + shape_tail)
        keep.append(a)
        return a.ctypes.data

    positions = _c(source.positions, np.float32).reshape(-1, 3)
    triangles = _c(source.triangles, np.uint32).reshape(-1, 3)
    cin = _CBuildInput()
    cin.positions = ptr(positions, np.float32)
    cin.vertex_count = positions.shape[0]
    cin.normals = ptr(source.normals, np.float32, (3,))
    cin.texcoords = ptr(source.texcoords, np.float32, (2,))
    cin.triangles = ptr(triangles, np.uint32)
    cin.triangle_count = triangles.shape[0]
    cin.guide_count = int(np.asarray(g.cv_counts).size)
    cin.guide_cv_counts = ptr(g.cv_counts, np.uint32)
    cin.guide_cvs = ptr(g.cvs, np.float32, (3,))
    cin.guide_root_normals = ptr(g.root_normals, np.float32, (3,))
    cin.guide_root_uvs = ptr(g.root_uvs, np.float32, (2,))
    cin.guide_triangles = ptr(g.triangles, np.uint32)
    cin.guide_barycentrics = ptr(g.barycentrics, np.float32, (2,))
    cin.guide_support_radii = ptr(g.support_radii, np.float32)
    cin.stencil_slots = stencil_slots
    cin.worker_count = workers
    out = ctypes.c_void_p()
    size = ctypes.c_uint64()
    msg = ctypes.create_string_buffer(256)
    if stream is None:
        failed = lib().nxg_build_asset(ctypes.byref(cin), ctypes.byref(out), ctypes.byref(size), msg, 256)
    else:
        failed = lib().nxg_build_asset_device(ctypes.byref(cin), stream or None, ctypes.byref(out),
                                              ctypes.byref(size), msg, 256)
    if failed:
        raise ValueError(msg.value.decode())
    try:
        blob = np.ctypeslib.as_array(ctypes.cast(out, ctypes.POINTER(ctypes.c_uint8)), shape=(size.value,))
        # The builder wrote the header and content hash itself; validating
        # would hash the whole blob a second time.
        return Asset(blob.copy(), validate=False)
    finally:
        lib().nxg_free(out)


def fnv1a(data: np.ndarray | bytes) -> int:
    buf = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    return int(lib().nxg_fnv1a(buf.ctypes.data, buf.size))


def recompute_hash(blob: np.ndarray) -> None:
    """Rewrite content_hash after editing a blob in place (asset.cpp:290)."""
    digest = fnv1a(blob[_abi.HEADER_SIZE:])
    blob[24:32] = np.frombuffer(np.uint64(digest).tobytes(), dtype=np.uint8)


def file_size(path: str) -> int:
    return os.path.getsize(path)
