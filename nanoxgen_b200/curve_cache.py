"""The renderer curve cache (.nxc, src/curve_cache.cpp) through
libnxg_b200.so: blobs built and validated on the host exactly as the
reference does, and validated again after upload by one pass of a device
kernel (every element check of validate_curve_cache, a point-count sum and a
bit checksum of the points; the serial content hash stays on the host)."""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _abi
from ._abi import CurveCacheCheck, CurveCacheHeader, CurveCacheInput, check, lib
from .asset import aligned_empty
from .generator import _stream_handle


def _array(a, dtype, width: int = 1):
    if a is None:
        return None, 0
    a = np.ascontiguousarray(a, dtype)
    return a, a.size // width


def build_curve_cache(point_counts, points, texcoords=None, patch_uvs=None, face_uvs=None, face_ids=None,
                      motion_times=None, motion_points=None) -> np.ndarray:
    """build_curve_cache: a 64-byte aligned uint8 blob.  points is [N, 4]
    (position, radius); texcoords [N, 2]; patch/face uvs [S, 2]; face ids
    [S]; motion times [K] with motion points [K * N, 3] (sample-major).
    Raises ValueError with the reference's message."""
    keep = []
    fields = []
    for value, dtype, width in ((point_counts, np.uint32, 1), (points, np.float32, 4), (texcoords, np.float32, 2),
                                (patch_uvs, np.float32, 2), (face_uvs, np.float32, 2), (face_ids, np.uint32, 1),
                                (motion_times, np.float32, 1), (motion_points, np.float32, 3)):
        a, n = _array(value, dtype, width)
        keep.append(a)
        fields += [None if a is None else a.ctypes.data, n]
    desc = CurveCacheInput(*fields)
    blob = ctypes.c_void_p()
    size = ctypes.c_uint64()
    msg = ctypes.create_string_buffer(256)
    code = lib().nxg_curve_cache_build(ctypes.byref(desc), ctypes.byref(blob), ctypes.byref(size), msg, 256)
    if code != 0:
        raise ValueError(msg.value.decode())
    try:
        out = aligned_empty(size.value)
        ctypes.memmove(out.ctypes.data, blob.value, size.value)
    finally:
        lib().nxg_free(blob)
    return out


def error_message(code: int) -> str:
    return lib().nxg_curve_cache_error_message(code).decode()


def validate_curve_cache(blob: np.ndarray) -> str:
    """validate_curve_cache on the host: "" when valid, else the reference's
    message."""
    return error_message(lib().nxg_curve_cache_validate(blob.ctypes.data, blob.size))


def header(blob: np.ndarray) -> CurveCacheHeader:
    return CurveCacheHeader.from_buffer_copy(bytes(blob[:ctypes.sizeof(CurveCacheHeader)]))


def content_hash(data: np.ndarray) -> int:
    return int(lib().nxg_curve_cache_content_hash(data.ctypes.data, data.size))


def point_checksum(blob: np.ndarray) -> int:
    return int(lib().nxg_curve_cache_point_checksum(blob.ctypes.data, blob.size))


class DeviceCurveCache:
    """A blob uploaded to the device, with its header kept on the host."""

    def __init__(self, blob: np.ndarray, device="cuda", stream: Optional[torch.cuda.Stream] = None):
        if blob.size < ctypes.sizeof(CurveCacheHeader):
            raise ValueError(error_message(1))
        self.header = header(blob)
        self.size = int(blob.size)
        self.blob = torch.empty(self.size, dtype=torch.uint8, device=device)
        self.blob.copy_(torch.from_numpy(np.asarray(blob)), non_blocking=False)
        self.result = torch.zeros(ctypes.sizeof(CurveCacheCheck), dtype=torch.uint8, device=device)

    def validate(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Enqueues the device check; raises ValueError when the header alone
        fails."""
        header_error = ctypes.c_uint32()
        code = lib().nxg_curve_cache_validate_device(ctypes.byref(self.header), self.blob.data_ptr(), self.size,
                                                     self.result.data_ptr(), ctypes.byref(header_error),
                                                     _stream_handle(stream))
        if code == _abi.ERRORS["InvalidArgument"] and header_error.value:
            raise ValueError(error_message(header_error.value))
        check(code, "nxg_curve_cache_validate_device")

    def outcome(self) -> tuple[str, int, int]:
        """(message, point-count sum, bit checksum) of the last check
        (synchronises)."""
        r = CurveCacheCheck.from_buffer_copy(bytes(self.result.cpu().numpy()))
        return error_message(r.error), int(r.point_sum), int(r.checksum)
