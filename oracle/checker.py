"""Python access to the test-only checkers.

TEST INFRASTRUCTURE ONLY.  Loads oracle/liboracle.so (the C restatement in
nxg_oracle.c) and, where it was built, oracle/_ref/libnxg_ref.so (the
reference's own src/asset.cpp behind ref_shim.cpp).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU legs may import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libnxg_ref.so")

ROOT_DTYPE = np.dtype([("position", "<f4", 3), ("normal", "<f4", 3), ("uv", "<f4", 2),
                       ("triangle_index", "<u4"), ("barycentric", "<f4", 2), ("surface_face_id", "<u4")])
# StrandState of nxg_oracle.c / RefStrandState of ref_shim.cpp (156 bytes).
STATE_DTYPE = np.dtype([("root", ROOT_DTYPE), ("indices", "<u4", 8), ("weights", "<f4", 8),
                        ("weight_sum", "<f4"), ("nearest", "<u4"), ("surface_u", "<f4", 3),
                        ("noise_domain", "<f4", 3), ("original_length", "<f4"),
                        ("effective_noise_frequency", "<f4"), ("preserve_scale", "<f4")])
assert ROOT_DTYPE.itemsize == 48 and STATE_DTYPE.itemsize == 156

_P = ctypes.c_void_p


def _ensure_built(path: str, target: str) -> None:
    if not os.path.exists(path):
        subprocess.check_call(["make", "-s", "-C", HERE, target])


def _aligned(nbytes: int) -> np.ndarray:
    raw = np.empty(nbytes + 64, np.uint8)
    off = (-raw.ctypes.data) % 64
    return raw[off:off + nbytes]


def as_aligned_blob(data) -> np.ndarray:
    src = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else data.view(np.uint8)
    if src.ctypes.data % 64 == 0:
        return src
    buf = _aligned(src.size)
    buf[:] = src
    return buf


def _vec_ptr(a: Optional[np.ndarray]):
    return None if a is None else np.ascontiguousarray(a, np.float32).ctypes.data


class Oracle:
    """The C restatement of generate.h / asset.cpp (nxg_oracle.c)."""

    def __init__(self):
        _ensure_built(ORACLE_PATH, "oracle")
        lib = ctypes.CDLL(ORACLE_PATH)
        lib.orc_random01.restype = ctypes.c_float
        lib.orc_random01.argtypes = [ctypes.c_uint32] * 3
        lib.orc_gradient_noise.restype = ctypes.c_float
        lib.orc_gradient_noise.argtypes = [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        lib.orc_noise_hash.restype = ctypes.c_uint32
        lib.orc_noise_hash.argtypes = [ctypes.c_int32] * 3
        lib.orc_strand_state.restype = None
        lib.orc_strand_state.argtypes = [_P, _P, _P, _P, _P, ctypes.c_uint32, _P]
        lib.orc_fnv1a.restype = ctypes.c_uint64
        lib.orc_fnv1a.argtypes = [_P, ctypes.c_uint64]
        lib.orc_validate_asset.restype = ctypes.c_int
        lib.orc_validate_asset.argtypes = [_P, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64]
        lib.orc_generate_packed.restype = ctypes.c_int
        lib.orc_generate_packed.argtypes = [_P, _P, ctypes.c_float, _P, _P, _P, _P, ctypes.c_uint32,
                                            ctypes.c_uint32, _P, _P, _P, _P, ctypes.c_int]
        self.lib = lib

    def generate(self, blob, params, radius_scale: float = 1.0, positions=None, normals=None, guide_cvs=None,
                 strands=None, first: int = 0, count: Optional[int] = None, threads: int = 1):
        """Packed generation of the listed strands (or first..first+count-1)."""
        blob = as_aligned_blob(blob)
        P = int(params.cvs_per_strand)
        if strands is not None:
            ids = np.ascontiguousarray(strands, np.uint32)
            n = ids.size
        else:
            ids = None
            n = int(params.strand_count) - first if count is None else int(count)
        points = np.zeros((n * P, 4), np.float32)
        roots = np.zeros(n, ROOT_DTYPE)
        uvs = np.zeros((n, 2), np.float32)
        counts = np.zeros(n, np.uint32)
        keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (positions, normals, guide_cvs)]
        rc = self.lib.orc_generate_packed(
            blob.ctypes.data, ctypes.byref(params), radius_scale,
            *(k.ctypes.data if k is not None else None for k in keep),
            ids.ctypes.data if ids is not None else None, first, n,
            points.ctypes.data, roots.ctypes.data, uvs.ctypes.data, counts.ctypes.data, threads)
        assert rc == 0
        return points, roots, uvs, counts

    def strand_state(self, blob, params, strand: int, positions=None, normals=None, guide_cvs=None) -> np.ndarray:
        blob = as_aligned_blob(blob)
        out = np.zeros(1, STATE_DTYPE)
        keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (positions, normals, guide_cvs)]
        self.lib.orc_strand_state(blob.ctypes.data, *(k.ctypes.data if k is not None else None for k in keep),
                                  ctypes.byref(params), strand, out.ctypes.data)
        return out[0]

    def gradient_noise(self, blob, x: float, y: float, z: float) -> float:
        blob = as_aligned_blob(blob)
        return float(self.lib.orc_gradient_noise(blob.ctypes.data, x, y, z))

    def noise_hash(self, x: int, y: int, z: int) -> int:
        return int(self.lib.orc_noise_hash(x, y, z))

    def random01(self, seed: int, strand: int, dim: int) -> float:
        return float(self.lib.orc_random01(seed, strand, dim))

    def validate_asset(self, blob) -> str:
        blob = as_aligned_blob(blob)
        msg = ctypes.create_string_buffer(256)
        self.lib.orc_validate_asset(blob.ctypes.data, blob.size, msg, 256)
        return msg.value.decode()


def reference_available() -> bool:
    if os.path.exists(REF_PATH):
        return True
    ref = os.environ.get("NXG_REFERENCE_ROOT", os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
    if os.path.isfile(os.path.join(ref, "src", "asset.cpp")):
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", "REF=" + ref])
        return os.path.exists(REF_PATH)
    return False


class Reference:
    """The reference's own CPU implementation (oracle/_ref/libnxg_ref.so)."""

    def __init__(self):
        if not reference_available():
            raise FileNotFoundError("oracle/_ref/libnxg_ref.so is not built and the reference checkout is absent")
        lib = ctypes.CDLL(REF_PATH)
        lib.ref_build_asset.restype = ctypes.c_int
        lib.ref_build_asset.argtypes = [_P, ctypes.c_uint32, _P, _P, _P, ctypes.c_uint32, ctypes.c_uint32,
                                        _P, _P, _P, _P, _P, _P, _P, ctypes.POINTER(ctypes.c_void_p),
                                        ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p, ctypes.c_uint64]
        lib.ref_free.argtypes = [_P]
        lib.ref_validate_asset.restype = ctypes.c_int
        lib.ref_validate_asset.argtypes = [_P, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64]
        lib.ref_asset_create.restype = _P
        lib.ref_asset_create.argtypes = [_P, ctypes.c_uint64]
        lib.ref_asset_destroy.argtypes = [_P]
        lib.ref_generate_packed.restype = ctypes.c_int
        lib.ref_generate_packed.argtypes = [_P, _P, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32,
                                            _P, ctypes.c_uint64, _P, ctypes.c_uint64, _P, ctypes.c_uint64,
                                            _P, _P, _P, _P, ctypes.POINTER(ctypes.c_double), ctypes.c_char_p,
                                            ctypes.c_uint64]
        lib.ref_strand_state.argtypes = [_P, _P, _P, _P, _P, ctypes.c_uint32, _P]
        lib.ref_gradient_noise.restype = ctypes.c_float
        lib.ref_gradient_noise.argtypes = [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float]
        lib.ref_validate_packed_request.restype = ctypes.c_uint32
        lib.ref_validate_packed_request.argtypes = [_P, _P, ctypes.c_uint64, _P, ctypes.c_uint64, _P,
                                                    ctypes.c_uint64, _P, ctypes.c_uint64, _P, _P, _P, _P,
                                                    ctypes.c_float, _P, ctypes.c_uint64, ctypes.c_uint64,
                                                    ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32]
        lib.ref_validate_motion_request.restype = ctypes.c_uint32
        lib.ref_validate_motion_request.argtypes = [_P, _P, ctypes.c_uint64, _P, ctypes.c_uint32, _P, _P,
                                                    ctypes.c_uint64, ctypes.c_uint32]
        lib.ref_error_message.restype = ctypes.c_char_p
        lib.ref_error_message.argtypes = [ctypes.c_uint32]
        self.lib = lib

    def build_asset(self, src) -> np.ndarray:
        """asset.h:119 build_asset on an nanoxgen_b200.asset.AssetBuildInput."""
        g = src.guides
        arrs = dict(
            positions=np.ascontiguousarray(src.positions, np.float32),
            normals=None if src.normals is None else np.ascontiguousarray(src.normals, np.float32),
            texcoords=None if src.texcoords is None else np.ascontiguousarray(src.texcoords, np.float32),
            triangles=np.ascontiguousarray(src.triangles, np.uint32),
            counts=np.ascontiguousarray(g.cv_counts, np.uint32), cvs=np.ascontiguousarray(g.cvs, np.float32),
            rn=np.ascontiguousarray(g.root_normals, np.float32), ruv=np.ascontiguousarray(g.root_uvs, np.float32),
            gt=np.ascontiguousarray(g.triangles, np.uint32), gb=np.ascontiguousarray(g.barycentrics, np.float32),
            gr=np.ascontiguousarray(g.support_radii, np.float32))
        out = ctypes.c_void_p()
        size = ctypes.c_uint64()
        msg = ctypes.create_string_buffer(256)
        p = lambda a: None if a is None else a.ctypes.data
        rc = self.lib.ref_build_asset(p(arrs["positions"]), arrs["positions"].shape[0], p(arrs["normals"]),
                                      p(arrs["texcoords"]), p(arrs["triangles"]), arrs["triangles"].shape[0],
                                      arrs["counts"].size, p(arrs["counts"]), p(arrs["cvs"]), p(arrs["rn"]),
                                      p(arrs["ruv"]), p(arrs["gt"]), p(arrs["gb"]), p(arrs["gr"]),
                                      ctypes.byref(out), ctypes.byref(size), msg, 256)
        if rc != 0:
            raise ValueError(msg.value.decode())
        data = ctypes.string_at(out, size.value)
        self.lib.ref_free(out)
        return as_aligned_blob(data)

    def validate_asset(self, blob) -> str:
        blob = as_aligned_blob(blob)
        msg = ctypes.create_string_buffer(256)
        self.lib.ref_validate_asset(blob.ctypes.data, blob.size, msg, 256)
        return msg.value.decode()

    class Handle:
        def __init__(self, ref, blob):
            self.ref = ref
            blob = as_aligned_blob(blob)
            self.ptr = ref.lib.ref_asset_create(blob.ctypes.data, blob.size)

        def __del__(self):
            if getattr(self, "ptr", None):
                self.ref.lib.ref_asset_destroy(self.ptr)
                self.ptr = None

    def handle(self, blob) -> "Reference.Handle":
        return Reference.Handle(self, blob)

    def generate(self, handle, params, radius_scale: float = 1.0, workers: int = 1, tile: int = 128,
                 positions=None, normals=None, guide_cvs=None, want_output: bool = True):
        """generate_packed_deformed_cpu; returns (points, roots, uvs, counts, ms)."""
        S, P = int(params.strand_count), int(params.cvs_per_strand)
        points = np.zeros((S * P, 4), np.float32) if want_output else None
        roots = np.zeros(S, ROOT_DTYPE) if want_output else None
        uvs = np.zeros((S, 2), np.float32) if want_output else None
        counts = np.zeros(S, np.uint32) if want_output else None
        keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (positions, normals, guide_cvs)]
        n = [0 if k is None else k.size // 3 for k in keep]
        ms = ctypes.c_double()
        msg = ctypes.create_string_buffer(256)
        p = lambda a: None if a is None else a.ctypes.data
        rc = self.lib.ref_generate_packed(handle.ptr, ctypes.byref(params), radius_scale, workers, tile,
                                          p(keep[0]), n[0], p(keep[1]), n[1], p(keep[2]), n[2],
                                          p(points), p(roots), p(uvs), p(counts), ctypes.byref(ms), msg, 256)
        if rc != 0:
            raise ValueError(msg.value.decode())
        return points, roots, uvs, counts, ms.value

    def strand_state(self, handle, params, strand: int, positions=None, normals=None, guide_cvs=None):
        out = np.zeros(1, STATE_DTYPE)
        keep = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (positions, normals, guide_cvs)]
        self.lib.ref_strand_state(handle.ptr, *(k.ctypes.data if k is not None else None for k in keep),
                                  ctypes.byref(params), strand, out.ctypes.data)
        return out[0]

    def gradient_noise(self, handle, x, y, z) -> float:
        return float(self.lib.ref_gradient_noise(handle.ptr, x, y, z))

    # ------------------------------------------------ scalar expressions
    # (ref_classic_shim.cpp over src/xgen_expression.cpp and
    # src/xgen_classic_runtime.cpp)

    def _expression_prototypes(self):
        lib = self.lib
        if getattr(self, "_expr_ready", False):
            return lib
        u32, f32, c_p = ctypes.c_uint32, ctypes.c_float, ctypes.c_char_p
        lib.ref_expr_compile.restype = _P
        lib.ref_expr_compile.argtypes = [c_p, c_p, c_p, c_p, ctypes.c_uint64]
        lib.ref_expr_free.argtypes = [_P]
        lib.ref_expr_info.argtypes = [_P, _P]
        lib.ref_expr_instruction.argtypes = [_P, u32, _P, ctypes.POINTER(f32)]
        lib.ref_expr_operand.restype = u32
        lib.ref_expr_operand.argtypes = [_P, u32]
        lib.ref_expr_ramp_point.argtypes = [_P, u32, ctypes.POINTER(f32), ctypes.POINTER(f32), ctypes.POINTER(u32)]
        lib.ref_expr_input.restype = c_p
        lib.ref_expr_input.argtypes = [_P, u32]
        lib.ref_expr_eval_batch.argtypes = [_P, _P, u32, ctypes.c_uint64, _P, _P, _P, f32, _P, _P, _P]
        lib.ref_seexpr_hash_finish.restype = u32
        lib.ref_seexpr_hash_finish.argtypes = [u32]
        lib.ref_runtime_hash_component.restype = u32
        lib.ref_runtime_hash_component.argtypes = [f32]
        lib.ref_runtime_hash.restype = f32
        lib.ref_runtime_hash.argtypes = [_P, u32]
        lib.ref_runtime_face_seed.restype = f32
        lib.ref_runtime_face_seed.argtypes = [u32, c_p, u32]
        lib.ref_string_seed.restype = u32
        lib.ref_string_seed.argtypes = [c_p]
        lib.ref_classic_noise_batch.argtypes = [_P, ctypes.c_uint64, f32, _P]
        lib.ref_classic_plan.restype = _P
        lib.ref_classic_plan.argtypes = [c_p, c_p, u32, c_p, c_p, ctypes.c_uint64]
        lib.ref_classic_plan_free.argtypes = [_P]
        lib.ref_classic_plan_info.argtypes = [_P, _P, _P]
        lib.ref_classic_plan_program.restype = _P
        lib.ref_classic_plan_program.argtypes = [_P, u32]
        lib.ref_classic_apply.restype = u32
        lib.ref_classic_apply.argtypes = [_P, _P, _P, _P, _P, u32, u32, f32, _P, ctypes.c_uint64, u32, _P, c_p,
                                          ctypes.c_uint64]
        self._expr_ready = True
        return lib

    class Program:
        """A reference XgenFloatExpressionProgram."""

        def __init__(self, ref, ptr, owned=True):
            self.ref, self.ptr, self.owned = ref, ptr, owned

        def __del__(self):
            if getattr(self, "owned", False) and self.ptr:
                self.ref.lib.ref_expr_free(self.ptr)
                self.ptr = None

        def describe(self) -> dict:
            """Every field of the program, as plain Python values."""
            lib = self.ref.lib
            info = np.zeros(8, np.uint32)
            lib.ref_expr_info(self.ptr, info.ctypes.data)
            n_ins, n_ops, n_in, n_ramps, n_pts, result, seed, calls = (int(v) for v in info)
            ins = []
            for i in range(n_ins):
                w = np.zeros(4, np.uint32)
                imm = ctypes.c_float()
                lib.ref_expr_instruction(self.ptr, i, w.ctypes.data, ctypes.byref(imm))
                ins.append((int(w[0]), int(w[1]), int(w[2]), int(w[3]), np.float32(imm.value).view(np.uint32).item()))
            pts = []
            for i in range(n_pts):
                a, b, c = ctypes.c_float(), ctypes.c_float(), ctypes.c_uint32()
                lib.ref_expr_ramp_point(self.ptr, i, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
                pts.append((np.float32(a.value).view(np.uint32).item(), np.float32(b.value).view(np.uint32).item(),
                            int(c.value)))
            return dict(instructions=ins, operands=[int(lib.ref_expr_operand(self.ptr, i)) for i in range(n_ops)],
                        inputs=[lib.ref_expr_input(self.ptr, i).decode() for i in range(n_in)],
                        ramp_points=pts, ramp_count=n_ramps, result=result, expression_seed=seed,
                        random_call_count=calls)

        def evaluate(self, inputs, u=None, v=None, face_seed=None, t=0.0):
            """evaluate_xgen_scalar_expression_float per row; (values, ok)."""
            inputs = np.ascontiguousarray(inputs, np.float32)
            count = inputs.shape[0]
            cols = inputs.shape[1] if inputs.ndim == 2 else 0
            out = np.zeros(count, np.float32)
            ok = np.zeros(count, np.uint8)
            keep = [None if a is None else np.ascontiguousarray(a, np.float32) for a in (u, v, face_seed)]
            p = lambda a: None if a is None else a.ctypes.data
            self.ref.lib.ref_expr_eval_batch(self.ptr, inputs.ctypes.data, cols, count, p(keep[0]), p(keep[1]),
                                             p(keep[2]), t, None, out.ctypes.data, ok.ctypes.data)
            return out, ok.astype(bool)

    def compile_expression(self, source: str, name: str = "", object_type: str = ""):
        """compile + make_float_program; returns (Program or None, message)."""
        lib = self._expression_prototypes()
        msg = ctypes.create_string_buffer(512)
        ptr = lib.ref_expr_compile(source.encode(), name.encode(), object_type.encode(), msg, 512)
        return (Reference.Program(self, ptr) if ptr else None), msg.value.decode()

    def classic_noise(self, points, frequency: float) -> np.ndarray:
        """xgen_classic_noise_float(p * frequency) per point."""
        lib = self._expression_prototypes()
        pts = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros(pts.shape[0], np.float32)
        lib.ref_classic_noise_batch(pts.ctypes.data, pts.shape[0], frequency, out.ctypes.data)
        return out

    def runtime_face_seed(self, description_id: int, patch: str, face: int) -> float:
        return float(self._expression_prototypes().ref_runtime_face_seed(description_id, patch.encode(), face))

    class Plan:
        def __init__(self, ref, ptr, reasons):
            self.ref, self.ptr, self.fallback_reasons = ref, ptr, reasons

        def __del__(self):
            if getattr(self, "ptr", None):
                self.ref.lib.ref_classic_plan_free(self.ptr)
                self.ptr = None

        def info(self) -> dict:
            out = np.zeros(4, np.uint32)
            freqs = np.zeros(64, np.float32)
            self.ref.lib.ref_classic_plan_info(self.ptr, out.ctypes.data, freqs.ctypes.data)
            return dict(has_length=bool(out[0]), has_width=bool(out[1]), ptex=int(out[2]),
                        pref_noise=freqs[:int(out[3])].copy())

        def program(self, which: str):
            ptr = self.ref.lib.ref_classic_plan_program(self.ptr, 0 if which == "length" else 1)
            return Reference.Program(self.ref, ptr, owned=False) if ptr else None

    def classic_plan(self, length=None, width=None, description_id: int = 0, name: str = "description"):
        """compile_xgen_classic_float_runtime_plan for one SplinePrimitive."""
        lib = self._expression_prototypes()
        msg = ctypes.create_string_buffer(2048)
        enc = lambda s: None if s is None else s.encode()
        ptr = lib.ref_classic_plan(enc(length), enc(width), description_id, name.encode(), msg, 2048)
        if not ptr:
            raise ValueError(msg.value.decode())
        return Reference.Plan(self, ptr, [r for r in msg.value.decode().split("\n") if r])

    def classic_apply(self, plan, points, counts, roots, uvs, cvs: int, radius_scale: float,
                      runtime_inputs=None, workers: int = 1):
        """apply_xgen_classic_float_runtime_plan_cpu; returns the compacted
        (points, counts, roots, uvs)."""
        lib = self._expression_prototypes()
        points = np.ascontiguousarray(points, np.float32).copy()
        counts = np.ascontiguousarray(counts, np.uint32).copy()
        roots = np.ascontiguousarray(roots).copy()
        uvs = np.ascontiguousarray(uvs, np.float32).copy()
        S = counts.size
        inputs = None if runtime_inputs is None else np.ascontiguousarray(runtime_inputs, np.float32)
        kept = ctypes.c_uint32()
        msg = ctypes.create_string_buffer(512)
        rc = lib.ref_classic_apply(plan.ptr, points.ctypes.data, counts.ctypes.data, roots.ctypes.data,
                                   uvs.ctypes.data, S, cvs, radius_scale,
                                   None if inputs is None else inputs.ctypes.data,
                                   0 if inputs is None else inputs.size, workers, ctypes.byref(kept), msg, 512)
        if rc != 0:
            raise ValueError(msg.value.decode())
        k = kept.value
        return points[:k * cvs], counts[:k], roots[:k], uvs[:k]

    # ------------------------------------------------ Classic FX passes

    def classic_plan_fx(self, primitive: dict, effects: list, description_id: int = 0, name: str = "description"):
        """compile_xgen_classic_float_runtime_plan for a description with the
        SplinePrimitive attributes in `primitive` (length, width, taper,
        taperStart, widthRamp) and FX modules `effects`, each ("noise", {mask,
        magnitude, magnitudeScale, frequency, correlation, preserveLength}) or
        ("cut", {amount}) or ("clump", {mask, clump, clumpScale, noise,
        noiseScale, noiseFrequency, noiseCorrelation}), in order."""
        lib = self._expression_prototypes()
        if not getattr(self, "_fx_ready", False):
            lib.ref_classic_plan_fx.restype = _P
            lib.ref_classic_plan_fx.argtypes = [_P, ctypes.c_uint32, _P, _P, ctypes.c_uint32, ctypes.c_char_p,
                                                ctypes.c_char_p, ctypes.c_uint64]
            lib.ref_classic_plan_effects.argtypes = [_P, _P]
            lib.ref_classic_apply_fx.restype = ctypes.c_uint32
            lib.ref_classic_apply_fx.argtypes = [_P, _P, _P, _P, _P, ctypes.c_uint32, ctypes.c_uint32,
                                                 ctypes.c_float, _P, ctypes.c_uint64, _P, _P, ctypes.c_uint32, _P,
                                                 _P, _P, _P, _P, _P, _P, _P, ctypes.c_uint32, _P,
                                                 ctypes.c_char_p, ctypes.c_uint64]
            lib.ref_classic_clump_prepare.restype = ctypes.c_uint32
            lib.ref_classic_clump_prepare.argtypes = [_P, ctypes.c_uint32, ctypes.c_uint32, _P, _P,
                                                      ctypes.c_char_p, ctypes.c_uint64]
            self._fx_ready = True
        keep = []

        def text(v):
            if v is None:
                return None
            b = ctypes.c_char_p(v.encode())
            keep.append(b)
            return b
        prim = (ctypes.c_char_p * 5)(*[text(primitive.get(k)) for k in
                                       ("length", "width", "taper", "taperStart", "widthRamp")])
        kinds = {"noise": 0, "cut": 1, "clump": 2}
        types = np.array([kinds[kind] for kind, _ in effects] or [0], np.uint32)
        names = {"noise": ("mask", "magnitude", "magnitudeScale", "frequency", "correlation", "preserveLength"),
                 "cut": ("amount",),
                 "clump": ("mask", "clump", "clumpScale", "noise", "noiseScale", "noiseFrequency",
                           "noiseCorrelation")}
        attrs = []
        for kind, values in effects:
            row = [text(values.get(n)) for n in names[kind]]
            attrs += row + [None] * (7 - len(row))
        arr = (ctypes.c_char_p * max(1, len(attrs)))(*attrs)
        msg = ctypes.create_string_buffer(4096)
        ptr = lib.ref_classic_plan_fx(ctypes.cast(prim, _P), len(effects), types.ctypes.data, ctypes.cast(arr, _P),
                                      description_id, name.encode(), msg, 4096)
        if not ptr:
            raise ValueError(msg.value.decode())
        plan = Reference.Plan(self, ptr, [r for r in msg.value.decode().split("\n") if r])
        counts = np.zeros(4, np.uint32)
        lib.ref_classic_plan_effects(ptr, counts.ctypes.data)
        plan.effect_counts = tuple(int(c) for c in counts)
        return plan

    def curve_cache_build(self, point_counts, points, texcoords=None, patch_uvs=None, face_uvs=None,
                          face_ids=None, motion_times=None, motion_points=None) -> np.ndarray:
        """build_curve_cache: the blob as uint8 (raises ValueError with the
        reference's message)."""
        lib = self.lib
        if not getattr(self, "_cache_ready", False):
            lib.ref_curve_cache_build.restype = ctypes.c_uint64
            lib.ref_curve_cache_build.argtypes = [_P, ctypes.c_uint64] * 8 + [_P, ctypes.c_uint64, ctypes.c_char_p,
                                                                             ctypes.c_uint64]
            lib.ref_curve_cache_validate.argtypes = [_P, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64]
            self._cache_ready = True
        keep, args = [], []
        for value, dtype, width in ((point_counts, np.uint32, 1), (points, np.float32, 4), (texcoords, np.float32, 2),
                                    (patch_uvs, np.float32, 2), (face_uvs, np.float32, 2), (face_ids, np.uint32, 1),
                                    (motion_times, np.float32, 1), (motion_points, np.float32, 3)):
            if value is None:
                args += [None, 0]
                continue
            a = np.ascontiguousarray(value, dtype)
            keep.append(a)
            args += [a.ctypes.data, a.size // width]
        msg = ctypes.create_string_buffer(512)
        size = lib.ref_curve_cache_build(*args, None, 0, msg, 512)
        if size == 0:
            raise ValueError(msg.value.decode())
        out = np.zeros(size, np.uint8)
        lib.ref_curve_cache_build(*args, out.ctypes.data, size, msg, 512)
        return out

    def curve_cache_validate(self, blob: np.ndarray) -> str:
        """validate_curve_cache's message ("" when valid); `blob` must be
        64-byte aligned for the reference's alignment check to pass."""
        self.curve_cache_build([2], [[0, 0, 0, 0.1], [0, 1, 0, 0.1]])  # sets the prototypes
        msg = ctypes.create_string_buffer(512)
        self.lib.ref_curve_cache_validate(blob.ctypes.data, blob.size, msg, 512)
        return msg.value.decode()

    class _RefCurveSet(ctypes.Structure):
        _fields_ = [("strands", ctypes.c_uint32), ("fixed", ctypes.c_uint32), ("counts", ctypes.c_void_p),
                    ("points", ctypes.c_void_p), ("point_count", ctypes.c_uint64), ("widths", ctypes.c_void_p),
                    ("root_uvs", ctypes.c_void_p), ("roots", ctypes.c_void_p), ("constant_width", ctypes.c_float)]

    def build_curve_batches(self, base: dict, samples=(), per_batch: int = 65536, resample: int = 0,
                            radius_scale: float = 1.0, transform=(1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0)):
        """build_curve_batches with the batches concatenated.  A curve set is
        a dict: points [N, 3], strands, and optionally counts [S], fixed,
        widths [N], root_uvs [S, 2], roots (RootSample records),
        constant_width; samples are (time, set) pairs.  Returns point counts,
        points [total, 4], root uvs (or None), motion points and batch first
        points; raises ValueError with the reference's message."""
        lib = self.lib
        if not getattr(self, "_payload_ready", False):
            lib.ref_build_curve_batches.restype = ctypes.c_uint64
            lib.ref_build_curve_batches.argtypes = [_P, _P, _P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                                    ctypes.c_float, _P, _P, _P, _P, _P, _P, _P, ctypes.c_uint64,
                                                    ctypes.c_char_p, ctypes.c_uint64]
            self._payload_ready = True
        keep = []

        def arr(a, dtype):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            return a.ctypes.data

        def make(d):
            pts = np.ascontiguousarray(d["points"], np.float32).reshape(-1, 3)
            keep.append(pts)
            return Reference._RefCurveSet(d["strands"], d.get("fixed", 0), arr(d.get("counts"), np.uint32),
                                          pts.ctypes.data, pts.shape[0], arr(d.get("widths"), np.float32),
                                          arr(d.get("root_uvs"), np.float32),
                                          None if d.get("roots") is None else arr(d["roots"], np.uint8),
                                          d.get("constant_width", 0.0))
        b = make(base)
        sets = (Reference._RefCurveSet * max(1, len(samples)))(*[make(c) for _, c in samples])
        times = np.array([t for t, _ in samples] or [0.0], np.float32)
        n_points = np.asarray(base["points"]).size // 3
        S = int(base["strands"])
        cap = max(1, S * resample if resample else n_points)
        counts = np.zeros(max(S, 1), np.uint32)
        points = np.zeros((cap, 4), np.float32)
        uvs = np.zeros((max(S, 1), 2), np.float32)
        has = ctypes.c_uint32()
        motion = np.zeros((max(1, len(samples)) * cap, 3), np.float32)
        first = np.zeros(max(S, 1) + 2, np.uint64)
        tr = np.asarray(transform, np.float32)
        msg = ctypes.create_string_buffer(512)
        total = lib.ref_build_curve_batches(ctypes.byref(b), sets, times.ctypes.data, len(samples), per_batch,
                                            resample, radius_scale, tr.ctypes.data, counts.ctypes.data,
                                            points.ctypes.data, uvs.ctypes.data, ctypes.byref(has), motion.ctypes.data,
                                            first.ctypes.data, cap, msg, 512)
        if total == 0 and msg.value:
            raise ValueError(msg.value.decode())
        batches = (S + per_batch - 1) // per_batch
        return dict(point_counts=counts[:S], points=points[:total], root_uvs=uvs[:S] if has.value else None,
                    motion_points=motion[:len(samples) * total], batch_first_point=first[:batches + 1])

    def classic_clump_prepare(self, axes):
        """prepare_xgen_classic_clump_runtime_data of world-space guide axes
        [G, P, 3]: (render axes [G, P, 3], spline lengths [G])."""
        self.classic_plan_fx({}, [])  # sets the prototypes
        axes = np.ascontiguousarray(axes, np.float32)
        G, P = axes.shape[0], axes.shape[1]
        render = np.zeros_like(axes)
        lengths = np.zeros(G, np.float32)
        msg = ctypes.create_string_buffer(512)
        if self.lib.ref_classic_clump_prepare(axes.ctypes.data, G, P, render.ctypes.data, lengths.ctypes.data,
                                              msg, 512):
            raise ValueError(msg.value.decode())
        return render, lengths

    def classic_apply_fx(self, plan, points, counts, roots, uvs, cvs: int, radius_scale: float, runtime_inputs=None,
                         surface_tangents=None, workers: int = 1, random_prefixes=None, clumps=()):
        """apply_xgen_classic_float_runtime_plan_cpu with surface tangents,
        per-strand SeExpr prefixes and ClumpingFX guides (each a dict of
        axes [G, P, 3], normals, tangents [G, 3], uvs [G, 2], prefixes [G],
        strand_guides [S] and optionally reference_positions [G, 3]);
        returns the compacted (points, counts, roots, uvs)."""
        lib = self.lib
        points = np.ascontiguousarray(points, np.float32).copy()
        counts = np.ascontiguousarray(counts, np.uint32).copy()
        roots = np.ascontiguousarray(roots).copy()
        uvs = np.ascontiguousarray(uvs, np.float32).copy()
        S = counts.size
        inputs = None if runtime_inputs is None else np.ascontiguousarray(runtime_inputs, np.float32)
        tang = None if surface_tangents is None else np.ascontiguousarray(surface_tangents, np.float32)
        prefixes = None if random_prefixes is None else np.ascontiguousarray(random_prefixes, np.uint32)
        keep = []

        def arr(a, dtype):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype)
            keep.append(a)
            return a.ctypes.data
        n = max(1, len(clumps))
        tables = {k: (_P * n)(*[arr(c.get(k), np.uint32 if k in ("prefixes", "strand_guides") else np.float32)
                                 for c in clumps])
                  for k in ("axes", "normals", "tangents", "uvs", "prefixes", "reference_positions",
                            "strand_guides")}
        guide_counts = np.array([np.asarray(c["axes"]).shape[0] for c in clumps] or [0], np.uint32)
        kept = ctypes.c_uint32()
        msg = ctypes.create_string_buffer(512)
        rc = lib.ref_classic_apply_fx(plan.ptr, points.ctypes.data, counts.ctypes.data, roots.ctypes.data,
                                      uvs.ctypes.data, S, cvs, radius_scale,
                                      None if inputs is None else inputs.ctypes.data,
                                      0 if inputs is None else inputs.size,
                                      None if tang is None else tang.ctypes.data,
                                      None if prefixes is None else prefixes.ctypes.data, len(clumps),
                                      guide_counts.ctypes.data,
                                      *(ctypes.cast(tables[k], _P) for k in ("axes", "normals", "tangents", "uvs",
                                                                              "prefixes", "reference_positions",
                                                                              "strand_guides")),
                                      workers, ctypes.byref(kept), msg, 512)
        if rc != 0:
            raise ValueError(msg.value.decode())
        k = kept.value
        return points[:k * cvs], counts[:k], roots[:k], uvs[:k]
