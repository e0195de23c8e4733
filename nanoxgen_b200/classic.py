"""Classic-expression per-root scalars (include/nxg_classic.h).

``Expression`` compiles an XGen scalar expression with the library's host
compiler (the reference's compile_xgen_scalar_expression +
make_xgen_float_expression_program, src/xgen_expression.cpp:771-818, and the
Classic noise($Prefg*k) rewrite, src/xgen_classic_runtime.cpp:237-347).
``root_scalars`` evaluates a description's length / width expressions for
every root on the device, and ``generate_packed_classic`` generates strands
with the scalars applied inside the generator (the reference applies them
afterwards on the host in apply_xgen_classic_float_runtime_plan_cpu,
src/xgen_classic_runtime.cpp:1650-1678 and :1827-1858).
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional

import numpy as np
import torch

from . import _abi
from ._abi import (ClassicApplyDesc, ClassicScalarPlan, DeformedDesc, ExpressionInfo, ExpressionInstruction,
                   ExpressionRampPoint, GenerationParams, LaunchConfig, check, lib)
from .generator import (DeformedGeometry, DeviceAsset, PackedCurves, _stream_handle, allocate_outputs,
                        packed_output_descriptor)


class ExpressionError(ValueError):
    """The compiler rejected the source; the message is the reference's text."""


class Expression:
    """A compiled scalar expression (host handle of nxg_expression)."""

    def __init__(self, source: str, name: str = "", object_type: str = "", classic: bool = False):
        handle = ctypes.c_void_p()
        msg = ctypes.create_string_buffer(512)
        code = lib().nxg_expression_compile(source.encode(), name.encode(), object_type.encode(),
                                            _abi.EXPRESSION_CLASSIC if classic else 0, ctypes.byref(handle), msg,
                                            512)
        if code == _abi.ERRORS["ExpressionSyntax"]:
            raise ExpressionError(msg.value.decode())
        check(code, "nxg_expression_compile")
        self.handle = handle
        self.source = source

    @classmethod
    def classic(cls, source: str, attribute: str, object_type: str = "SplinePrimitive") -> "Expression":
        """An attribute of a Classic object, as the Classic runtime compiles
        it (seed from attribute name + object type, noise($Prefg*k) bound)."""
        return cls(source, attribute, object_type, classic=True)

    def close(self) -> None:
        if getattr(self, "handle", None) and self.handle.value:
            lib().nxg_expression_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> ExpressionInfo:
        out = ExpressionInfo()
        check(lib().nxg_expression_get_info(self.handle, ctypes.byref(out)), "nxg_expression_get_info")
        return out

    @property
    def inputs(self) -> list[str]:
        n = self.info().input_count
        return [lib().nxg_expression_input_name(self.handle, i).decode() for i in range(n)]

    def describe(self) -> dict:
        """Every field of the float program as plain Python values (floats as
        their bit patterns), laid out like the reference's program."""
        info = self.info()
        ins = []
        for i in range(info.instruction_count):
            x = ExpressionInstruction()
            check(lib().nxg_expression_get_instruction(self.handle, i, ctypes.byref(x)), "get_instruction")
            ins.append((x.op, x.operand_offset, x.operand_count, x.auxiliary,
                        np.float32(x.immediate).view(np.uint32).item()))
        ops = []
        for i in range(info.operand_count):
            v = ctypes.c_uint32()
            check(lib().nxg_expression_get_operand(self.handle, i, ctypes.byref(v)), "get_operand")
            ops.append(int(v.value))
        pts = []
        for i in range(info.ramp_point_count):
            p = ExpressionRampPoint()
            check(lib().nxg_expression_get_ramp_point(self.handle, i, ctypes.byref(p)), "get_ramp_point")
            pts.append((np.float32(p.position).view(np.uint32).item(), np.float32(p.value).view(np.uint32).item(),
                        p.interpolation))
        return dict(instructions=ins, operands=ops, inputs=self.inputs, ramp_points=pts, ramp_count=info.ramp_count,
                    result=info.result, expression_seed=info.expression_seed,
                    random_call_count=info.random_call_count)

    @property
    def pref_noise_frequencies(self) -> np.ndarray:
        info = self.info()
        return np.array(info.pref_noise_frequencies[:info.pref_noise_count], np.float32)


@dataclasses.dataclass
class ScalarPlan:
    """A description's SplinePrimitive length / width expressions."""
    length: Optional[Expression] = None
    width: Optional[Expression] = None
    description_id: int = 0
    patch_name: str = ""

    def descriptor(self) -> ClassicScalarPlan:
        d = ClassicScalarPlan()
        d.length = self.length.handle.value if self.length is not None else None
        d.width = self.width.handle.value if self.width is not None else None
        d.description_id = self.description_id
        self._patch = self.patch_name.encode()
        d.patch_name = self._patch
        return d


def root_scalars(dasset: DeviceAsset, params: GenerationParams, plan: ScalarPlan, *, first_strand: int = 0,
                 count: Optional[int] = None, out: Optional[torch.Tensor] = None,
                 status: Optional[torch.Tensor] = None,
                 stream: Optional[torch.cuda.Stream] = None) -> tuple[torch.Tensor, torch.Tensor]:
    """Exact per-root (length scale, width) as an (n, 2) float32 tensor, and
    the 2-word device status (error code, failing strands).  Enqueue only."""
    n = int(params.strand_count) - first_strand if count is None else int(count)
    if out is None:
        out = torch.empty((max(n, 1), 2), dtype=torch.float32, device=dasset.device)
    if status is None:
        status = torch.zeros(2, dtype=torch.int32, device=dasset.device)
    desc = plan.descriptor()
    check(lib().nxg_classic_root_scalars(ctypes.byref(dasset.desc), ctypes.byref(params), ctypes.byref(desc),
                                         first_strand, n, out.data_ptr(), status.data_ptr(), _stream_handle(stream)),
          "nxg_classic_root_scalars")
    return out, status


def check_status(status: torch.Tensor) -> None:
    """Raises NxgError if a root_scalars launch reported a domain error."""
    code, failing = (int(v) for v in status.cpu().tolist())
    if code:
        raise _abi.NxgError(code, "root scalars (%d strands)" % failing)


def generate_packed_classic(dasset: DeviceAsset, params: GenerationParams, scalars: torch.Tensor,
                            apply_length: bool = True, apply_width: bool = True, radius_scale: float = 1.0,
                            deformed: Optional[DeformedGeometry] = None, *, first_strand: int = 0,
                            count: Optional[int] = None, points: Optional[torch.Tensor] = None,
                            roots: Optional[torch.Tensor] = None, root_uvs: Optional[torch.Tensor] = None,
                            point_counts: Optional[torch.Tensor] = None, want_roots: bool = True,
                            block_size: int = 128, stream: Optional[torch.cuda.Stream] = None) -> PackedCurves:
    """Generation with the Classic length / width application fused in; a
    dropped strand keeps its points and gets point count 0."""
    n = int(params.strand_count) - first_strand if count is None else int(count)
    cvs = int(params.cvs_per_strand)
    if points is None:
        points, r, uv, pc = allocate_outputs(n, cvs, dasset.device, want_roots, want_roots, True)
        roots = roots if roots is not None else r
        root_uvs = root_uvs if root_uvs is not None else uv
        point_counts = point_counts if point_counts is not None else pc
    out = packed_output_descriptor(points, roots, root_uvs, point_counts, radius_scale)
    ddesc = deformed.descriptor() if deformed is not None else DeformedDesc()
    apply = ClassicApplyDesc(scalars.data_ptr(), int(apply_length), int(apply_width))
    cfg = LaunchConfig(block_size)
    ws = dasset.workspace(params, max(n, 1))
    check(lib().nxg_generate_packed_classic(ctypes.byref(dasset.desc), ctypes.byref(ddesc), ctypes.byref(params),
                                            ctypes.byref(out), ctypes.byref(apply), ctypes.byref(cfg), first_strand,
                                            n, ws.data_ptr(), ws.numel(), _stream_handle(stream)),
          "nxg_generate_packed_classic")
    return PackedCurves(n, cvs, points, point_counts, roots, root_uvs)


# ------------------------------------------------------------- FX passes

NOISE_FX_ATTRIBUTES = ("mask", "magnitude", "magnitudeScale", "frequency", "correlation", "preserveLength")
CLUMP_FX_ATTRIBUTES = ("mask", "clump", "clumpScale", "noise", "noiseScale", "noiseFrequency", "noiseCorrelation")


class FxPlan:
    """A description's Classic runtime plan for nxg_classic_fx_apply: the
    SplinePrimitive length, width, taper, taperStart and widthRamp
    expressions (each optional) and its FX modules in order, each
    ``("noise", {mask, magnitude, magnitudeScale, frequency, correlation,
    preserveLength})``, ``("cut", {"amount": ...})`` or ``("clump", {mask,
    clump, clumpScale, noise, noiseScale, noiseFrequency,
    noiseCorrelation})``; every attribute is compiled as the Classic runtime
    compiles it (its own name and object type).  ``upload`` packs the plan
    into a device buffer once."""

    def __init__(self, primitive: dict, effects=(), description_id: int = 0, description_name: str = ""):
        keys = ("length", "width", "taper", "taperStart", "widthRamp")
        unknown = set(primitive) - set(keys)
        if unknown:
            raise ValueError("unknown SplinePrimitive attributes: %s" % sorted(unknown))
        if len(effects) > _abi.CLASSIC_MAX_FX:
            raise ValueError("at most %d FX modules" % _abi.CLASSIC_MAX_FX)
        self.primitive = {k: Expression.classic(v, k) for k, v in primitive.items() if v is not None}
        self.effects = []
        for kind, values in effects:
            if kind == "noise":
                self.effects.append((kind, {n: Expression.classic(values[n], n, "NoiseFXModule")
                                            for n in NOISE_FX_ATTRIBUTES}))
            elif kind == "cut":
                self.effects.append((kind, {"amount": Expression.classic(values["amount"], "amount", "CutFXModule")}))
            elif kind == "clump":
                self.effects.append((kind, {n: Expression.classic(values[n], n, "ClumpingFXModule")
                                            for n in CLUMP_FX_ATTRIBUTES}))
            else:
                raise ValueError("FX module %r is not supported (NoiseFX, CutFX and ClumpingFX are)" % (kind,))
        self.description_id = int(description_id)
        self.description_name = description_name.encode()
        self.device: Optional[torch.Tensor] = None

    @property
    def has_noise(self) -> bool:
        return any(kind == "noise" for kind, _ in self.effects)

    @property
    def clump_count(self) -> int:
        return sum(kind == "clump" for kind, _ in self.effects)

    @property
    def uses_random(self) -> bool:
        exprs = list(self.primitive.values()) + [e for _, v in self.effects for e in v.values()]
        return any(e.info().random_call_count != 0 for e in exprs)

    def descriptor(self) -> _abi.ClassicFxPlan:
        h = lambda e: e.handle.value if e is not None else None
        fx = (_abi.ClassicFx * max(1, len(self.effects)))()
        for i, (kind, values) in enumerate(self.effects):
            if kind == "noise":
                fx[i] = _abi.ClassicFx(_abi.CLASSIC_FX_NOISE, 0, *(h(values[n]) for n in NOISE_FX_ATTRIBUTES), None)
            elif kind == "cut":
                fx[i] = _abi.ClassicFx(_abi.CLASSIC_FX_CUT, 0, None, None, None, None, None, None,
                                       h(values["amount"]))
            else:
                mask, *rest = (h(values[n]) for n in CLUMP_FX_ATTRIBUTES)
                fx[i] = _abi.ClassicFx(_abi.CLASSIC_FX_CLUMP, 0, mask, None, None, None, None, None, None, *rest)
        self._fx = fx
        p = self.primitive
        return _abi.ClassicFxPlan(h(p.get("length")), h(p.get("width")), h(p.get("taper")), h(p.get("taperStart")),
                                  h(p.get("widthRamp")), fx, len(self.effects), self.description_id,
                                  self.description_name)

    def upload(self, device="cuda", stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
        """Packs the plan into a device buffer (kept as ``self.device``)."""
        nbytes = int(lib().nxg_classic_fx_plan_bytes())
        buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        assert buf.data_ptr() % 256 == 0
        desc = self.descriptor()
        check(lib().nxg_classic_fx_plan_upload(ctypes.byref(desc), buf.data_ptr(), nbytes, _stream_handle(stream)),
              "nxg_classic_fx_plan_upload")
        self.device = buf
        return buf


class ClumpGuides:
    """One ClumpingFX module's guides on the device (ClassicClumpRuntimeData,
    xgen_classic_runtime.h:59-88, world space): guide CVs [G, P, 3] (before
    the rebuild), normals and tangents [G, 3], uvs [G, 2], SeExpr prefixes
    [G], the guide of every strand [S] (NXG_INVALID_INDEX = none) and,
    optionally, the guide-noise domain positions [G, 3].  The render axes and
    spline lengths are prepared on the device (nxg_classic_clump_prepare);
    a [G, P, 4] scratch table lets the apply compute the guide noise once
    per guide where the module's programs allow it."""

    def __init__(self, axes, normals, tangents, uvs, random_prefixes, strand_guides, reference_positions=None,
                 device="cuda", stream: Optional[torch.cuda.Stream] = None, noise_table: bool = True):
        f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).to(device)
        u32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.uint32).view(np.int32)).to(device)
        self.axes = f32(axes)
        if self.axes.dim() != 3 or self.axes.shape[2] != 3:
            raise ValueError("guide axes are [guides, cvs, 3]")
        G, P = int(self.axes.shape[0]), int(self.axes.shape[1])
        self.normals, self.tangents, self.uvs = f32(normals), f32(tangents), f32(uvs)
        self.random_prefixes, self.strand_guides = u32(random_prefixes), u32(strand_guides)
        self.reference_positions = None if reference_positions is None else f32(reference_positions)
        self.render_axes = torch.empty_like(self.axes)
        self.noise_table = (torch.empty((G, P, 4), dtype=torch.float32, device=self.axes.device)
                            if noise_table else None)
        self.spline_lengths = torch.empty(G, dtype=torch.float32, device=self.axes.device)
        check(lib().nxg_classic_clump_prepare(self.axes.data_ptr(), G, P, self.render_axes.data_ptr(),
                                              self.spline_lengths.data_ptr(), _stream_handle(stream)),
              "nxg_classic_clump_prepare")
        self.guide_count = G

    def descriptor(self) -> _abi.ClassicClumpGuides:
        ptr = lambda t: None if t is None else t.data_ptr()
        return _abi.ClassicClumpGuides(self.axes.data_ptr(), self.render_axes.data_ptr(),
                                       self.spline_lengths.data_ptr(), self.normals.data_ptr(),
                                       self.tangents.data_ptr(), ptr(self.reference_positions), self.uvs.data_ptr(),
                                       self.random_prefixes.data_ptr(), self.strand_guides.data_ptr(),
                                       ptr(self.noise_table), self.guide_count, 0)


def classic_fx_apply(plan: FxPlan, curves: PackedCurves, surface_tangents: Optional[torch.Tensor] = None,
                     radius_scale: float = 1.0, first_id: int = 0, noise_domains: Optional[torch.Tensor] = None,
                     status: Optional[torch.Tensor] = None, stream: Optional[torch.cuda.Stream] = None,
                     random_prefixes: Optional[torch.Tensor] = None, clumps=()) -> torch.Tensor:
    """Applies the uploaded `plan` to generated curves in place (points,
    point counts; dropped strands get count 0).  `random_prefixes` (one
    SeExpr prefix per strand) is required when a program calls rand();
    `clumps` holds one ClumpGuides per ClumpingFX module, in plan order.
    Returns the 2-word device status (error code, failing strands).
    Enqueue only."""
    if plan.device is None:
        plan.upload(curves.points.device, stream)
    S, P = int(curves.strand_count), int(curves.cvs_per_strand)
    if status is None:
        status = torch.zeros(2, dtype=torch.int32, device=curves.points.device)
    ptr = lambda t: None if t is None else t.data_ptr()
    guides = (_abi.ClassicClumpGuides * max(1, len(clumps)))(*(c.descriptor() for c in clumps))
    desc = _abi.ClassicFxCurves(curves.points.data_ptr(), curves.point_counts.data_ptr(), curves.roots.data_ptr(),
                                ptr(surface_tangents), ptr(noise_domains), S, P, first_id, radius_scale,
                                ptr(random_prefixes), guides, len(clumps), 0)
    check(lib().nxg_classic_fx_apply(plan.device.data_ptr(), ctypes.byref(desc), status.data_ptr(),
                                     _stream_handle(stream)), "nxg_classic_fx_apply")
    return status
