"""Renderer payload batches (build_curve_batches, src/curve_payload.cpp)
on the device through libnxg_b200.so: every batch in one pass, concatenated
in batch order, with the batch boundaries alongside."""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional, Sequence

import numpy as np
import torch

from . import _abi
from ._abi import CurveSet, MotionSet, PayloadOptions, PayloadOutput, check, lib
from .generator import _stream_handle

IDENTITY = (1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.0)


@dataclasses.dataclass
class Curves:
    """A curve set on the device (the reference's CurveSetView): points
    [N, 3]; per-strand point counts [S] or a fixed CV count; optional
    per-point widths (full diameters) else a constant width; optional root
    uvs [S, 2] or RootSample words [S, 12]."""
    points: torch.Tensor
    strand_count: int
    fixed_cvs_per_strand: int = 0
    point_counts: Optional[torch.Tensor] = None
    widths: Optional[torch.Tensor] = None
    root_uvs: Optional[torch.Tensor] = None
    roots: Optional[torch.Tensor] = None
    constant_width: float = 0.0

    def descriptor(self) -> CurveSet:
        ptr = lambda t: None if t is None else t.data_ptr()
        return CurveSet(self.strand_count, self.fixed_cvs_per_strand, ptr(self.point_counts), self.points.data_ptr(),
                        self.points.numel() // 3, ptr(self.widths), ptr(self.root_uvs), ptr(self.roots),
                        self.constant_width, 0)


@dataclasses.dataclass
class Batches:
    point_counts: torch.Tensor
    points: torch.Tensor
    root_uvs: Optional[torch.Tensor]
    motion_points: Optional[torch.Tensor]
    batch_first_point: torch.Tensor
    status: torch.Tensor

    def error(self) -> str:
        """The device checks' message ("" when they passed; synchronises)."""
        return lib().nxg_payload_error_message(int(self.status[0].item())).decode()


def build_curve_batches(base: Curves, samples: Sequence[tuple[float, Curves]] = (), max_strands_per_batch=65536,
                        resample_cv_count: int = 0, radius_scale: float = 1.0, transform=IDENTITY,
                        stream: Optional[torch.cuda.Stream] = None) -> Batches:
    """Enqueues build_curve_batches; raises ValueError with the reference's
    message when a host-side check fails."""
    device = base.points.device
    options = PayloadOptions(max_strands_per_batch, resample_cv_count, radius_scale, (ctypes.c_float * 12)(*transform))
    desc = base.descriptor()
    motion = (MotionSet * max(1, len(samples)))(*(MotionSet(t, 0, c.descriptor()) for t, c in samples))
    total = int(lib().nxg_payload_point_count(ctypes.byref(desc), ctypes.byref(options)))
    batches = int(lib().nxg_payload_batch_count(ctypes.byref(desc), ctypes.byref(options)))
    S = base.strand_count
    counts = torch.empty(max(S, 1), dtype=torch.int32, device=device)
    points = torch.empty((max(total, 1), 4), dtype=torch.float32, device=device)
    has_uvs = base.root_uvs is not None or base.roots is not None
    uvs = torch.empty((max(S, 1), 2), dtype=torch.float32, device=device) if has_uvs else None
    motion_points = (torch.empty((len(samples) * max(total, 1), 3), dtype=torch.float32, device=device)
                     if samples else None)
    first = torch.empty(batches + 1, dtype=torch.int64, device=device)
    status = torch.zeros(2, dtype=torch.int32, device=device)
    ws_bytes = int(lib().nxg_payload_workspace_size(ctypes.byref(desc), motion, len(samples)))
    workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=device)
    ptr = lambda t: None if t is None else t.data_ptr()
    out = PayloadOutput(counts.data_ptr(), points.data_ptr(), ptr(uvs), ptr(motion_points), first.data_ptr())
    host_error = ctypes.c_uint32()
    code = lib().nxg_build_curve_batches(ctypes.byref(desc), motion, len(samples), ctypes.byref(options),
                                         ctypes.byref(out), workspace.data_ptr(), ws_bytes, status.data_ptr(),
                                         ctypes.byref(host_error), _stream_handle(stream))
    if code == _abi.ERRORS["InvalidArgument"] and host_error.value:
        raise ValueError(lib().nxg_payload_error_message(host_error.value).decode())
    check(code, "nxg_build_curve_batches")
    result = Batches(counts, points, uvs, motion_points, first, status)
    result._keep = (workspace, motion, desc)
    return result
