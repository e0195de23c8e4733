"""ctypes mirror of include/nxg.h and the loader of libnxg_b200.so.

The library is built in-tree (``python -m nanoxgen_b200.build``).  There is
no fallback: importing this module without the built library raises, so a
missing CUDA build can never be mistaken for a working one.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(PKG, "libnxg_b200.so")

# Format constants (types.h:18-23).
MAGIC = 0x4E4547584F4E414E
GUIDE_STENCIL_SIZE = 8
NOISE_GRADIENT_COUNT = 256
INVALID_INDEX = 0xFFFFFFFF
HAS_NORMALS = 1
HAS_TEXCOORDS = 2
HEADER_SIZE = 128

c_float_p = ctypes.POINTER(ctypes.c_float)
c_u32_p = ctypes.POINTER(ctypes.c_uint32)


class Vec2(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float)]


class Vec3(ctypes.Structure):
    _fields_ = [("x", ctypes.c_float), ("y", ctypes.c_float), ("z", ctypes.c_float)]


class AssetHeader(ctypes.Structure):
    """nxg_asset_header / AssetHeader (types.h:76-101), 128 bytes."""
    _fields_ = [
        ("magic", ctypes.c_uint64), ("version_major", ctypes.c_uint16),
        ("version_minor", ctypes.c_uint16), ("flags", ctypes.c_uint32),
        ("byte_size", ctypes.c_uint64), ("content_hash", ctypes.c_uint64),
        ("vertex_count", ctypes.c_uint32), ("triangle_count", ctypes.c_uint32),
        ("guide_count", ctypes.c_uint32), ("guide_cv_count", ctypes.c_uint32),
        ("guide_stencil_size", ctypes.c_uint32), ("noise_gradient_count", ctypes.c_uint32),
        ("positions_offset", ctypes.c_uint64), ("normals_offset", ctypes.c_uint64),
        ("texcoords_offset", ctypes.c_uint64), ("triangles_offset", ctypes.c_uint64),
        ("alias_table_offset", ctypes.c_uint64), ("guides_offset", ctypes.c_uint64),
        ("guide_cvs_offset", ctypes.c_uint64), ("triangle_guides_offset", ctypes.c_uint64),
        ("noise_gradients_offset", ctypes.c_uint64),
    ]


class GenerationParams(ctypes.Structure):
    """nxg_generation_params / GenerationParams (types.h:108-124), with the
    reference's defaults."""
    _fields_ = [
        ("strand_count", ctypes.c_uint32), ("cvs_per_strand", ctypes.c_uint32),
        ("seed", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
        ("guide_support_scale", ctypes.c_float), ("guide_weight_power", ctypes.c_float),
        ("normal_rejection_cos", ctypes.c_float), ("length_scale", ctypes.c_float),
        ("root_width", ctypes.c_float), ("tip_width", ctypes.c_float),
        ("noise_amplitude", ctypes.c_float), ("noise_frequency", ctypes.c_float),
        ("noise_mask", ctypes.c_float), ("noise_correlation", ctypes.c_float),
        ("noise_preserve_length", ctypes.c_float),
    ]

    DEFAULTS = dict(strand_count=1024, cvs_per_strand=8, seed=1, reserved=0,
                    guide_support_scale=1.0, guide_weight_power=2.0,
                    normal_rejection_cos=-0.25, length_scale=1.0, root_width=0.01,
                    tip_width=0.001, noise_amplitude=0.0, noise_frequency=2.0,
                    noise_mask=1.0, noise_correlation=0.0, noise_preserve_length=0.0)

    def __init__(self, **kwargs):
        values = dict(self.DEFAULTS)
        unknown = set(kwargs) - set(values)
        if unknown:
            raise TypeError("unknown GenerationParams fields: %s" % sorted(unknown))
        values.update(kwargs)
        super().__init__(**values)

    def copy(self, **changes) -> "GenerationParams":
        values = {name: getattr(self, name) for name, _ in self._fields_}
        values.update(changes)
        return GenerationParams(**values)

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class DeviceAssetDesc(ctypes.Structure):
    """nxg_device_asset_desc / DeviceAssetDescriptor (device_contract.h:14-18)."""
    _fields_ = [("asset", ctypes.c_void_p), ("_pad", ctypes.c_uint8 * 56),
                ("header", AssetHeader), ("byte_capacity", ctypes.c_uint64),
                ("_tail", ctypes.c_uint8 * 56)]


class DeformedDesc(ctypes.Structure):
    """nxg_deformed_desc (device_contract.h:20-25)."""
    _fields_ = [("positions", ctypes.c_void_p), ("normals", ctypes.c_void_p),
                ("guide_cvs", ctypes.c_void_p), ("position_count", ctypes.c_uint64),
                ("normal_count", ctypes.c_uint64), ("guide_cv_count", ctypes.c_uint64)]


class GeneratedOutputDesc(ctypes.Structure):
    """nxg_generated_output_desc (device_contract.h:27-32)."""
    _fields_ = [("points", ctypes.c_void_p), ("widths", ctypes.c_void_p),
                ("roots", ctypes.c_void_p), ("point_capacity", ctypes.c_uint64),
                ("width_capacity", ctypes.c_uint64), ("root_capacity", ctypes.c_uint64)]


class PackedOutputDesc(ctypes.Structure):
    """nxg_packed_output_desc (device_contract.h:34-40, types.h:164-170)."""
    _fields_ = [("points", ctypes.c_void_p), ("roots", ctypes.c_void_p),
                ("root_uvs", ctypes.c_void_p), ("radius_scale", ctypes.c_float),
                ("point_counts", ctypes.c_void_p), ("point_capacity", ctypes.c_uint64),
                ("root_capacity", ctypes.c_uint64), ("root_uv_capacity", ctypes.c_uint64),
                ("point_count_capacity", ctypes.c_uint64)]


class MotionSampleDesc(ctypes.Structure):
    """nxg_motion_sample_desc (device_contract.h:42-45)."""
    _fields_ = [("deformation", DeformedDesc), ("time", ctypes.c_float)]


class MotionOutputDesc(ctypes.Structure):
    """nxg_motion_output_desc (device_contract.h:47-52)."""
    _fields_ = [("points", ctypes.c_void_p), ("point_capacity", ctypes.c_uint64)]


class LaunchConfig(ctypes.Structure):
    """nxg_launch_config (device_contract.h:54-56)."""
    _fields_ = [("block_size", ctypes.c_uint32)]


class Tile(ctypes.Structure):
    """nxg_tile: lanes per strand x CVs per lane, CTA size."""
    _fields_ = [("lanes_per_strand", ctypes.c_uint32), ("cvs_per_lane", ctypes.c_uint32),
                ("block_size", ctypes.c_uint32)]


EXPRESSION_CLASSIC = 1
EXPRESSION_MAX_INPUTS = 16

# XgenScalarOp order (xgen_expression.h:12-40).
EXPRESSION_OPS = ["constant", "input", "negate", "logical_not", "add", "subtract", "multiply", "divide",
                  "less", "less_equal", "greater", "greater_equal", "equal", "not_equal", "logical_and",
                  "logical_or", "select", "hash", "random", "minimum", "maximum", "clamp", "fit", "gamma",
                  "contrast", "smoothstep", "ramp"]


class ExpressionInfo(ctypes.Structure):
    """nxg_expression_info (nxg_classic.h)."""
    _fields_ = [("instruction_count", ctypes.c_uint32), ("operand_count", ctypes.c_uint32),
                ("input_count", ctypes.c_uint32), ("ramp_count", ctypes.c_uint32),
                ("ramp_point_count", ctypes.c_uint32), ("result", ctypes.c_uint32),
                ("expression_seed", ctypes.c_uint32), ("random_call_count", ctypes.c_uint32),
                ("pref_noise_count", ctypes.c_uint32),
                ("pref_noise_frequencies", ctypes.c_float * EXPRESSION_MAX_INPUTS)]


class ExpressionInstruction(ctypes.Structure):
    _fields_ = [("op", ctypes.c_uint32), ("operand_offset", ctypes.c_uint32), ("operand_count", ctypes.c_uint32),
                ("auxiliary", ctypes.c_uint32), ("immediate", ctypes.c_float)]


class ExpressionRampPoint(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float), ("value", ctypes.c_float), ("interpolation", ctypes.c_uint32)]


class ClassicScalarPlan(ctypes.Structure):
    """nxg_classic_scalar_plan (nxg_classic.h)."""
    _fields_ = [("length", ctypes.c_void_p), ("width", ctypes.c_void_p), ("description_id", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("patch_name", ctypes.c_char_p)]


class ClassicApplyDesc(ctypes.Structure):
    """nxg_classic_apply_desc (nxg_classic.h)."""
    _fields_ = [("root_scalars", ctypes.c_void_p), ("apply_length", ctypes.c_uint32),
                ("apply_width", ctypes.c_uint32)]


class ClassicFx(ctypes.Structure):
    """nxg_classic_fx (nxg_classic.h): one NoiseFX, CutFX or ClumpingFX module."""
    _fields_ = [("type", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("mask", ctypes.c_void_p),
                ("magnitude", ctypes.c_void_p), ("magnitude_scale", ctypes.c_void_p), ("frequency", ctypes.c_void_p),
                ("correlation", ctypes.c_void_p), ("preserve_length", ctypes.c_void_p), ("amount", ctypes.c_void_p),
                ("clump", ctypes.c_void_p), ("clump_scale", ctypes.c_void_p), ("noise", ctypes.c_void_p),
                ("noise_scale", ctypes.c_void_p), ("noise_frequency", ctypes.c_void_p),
                ("noise_correlation", ctypes.c_void_p)]


class ClassicClumpGuides(ctypes.Structure):
    """nxg_classic_clump_guides (nxg_classic.h): one ClumpingFX module's guides (device arrays)."""
    _fields_ = [("axes", ctypes.c_void_p), ("render_axes", ctypes.c_void_p), ("spline_lengths", ctypes.c_void_p),
                ("normals", ctypes.c_void_p), ("tangents", ctypes.c_void_p),
                ("reference_positions", ctypes.c_void_p), ("uvs", ctypes.c_void_p),
                ("random_prefixes", ctypes.c_void_p), ("strand_guides", ctypes.c_void_p),
                ("noise_table", ctypes.c_void_p), ("guide_count", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class ClassicFxPlan(ctypes.Structure):
    """nxg_classic_fx_plan (nxg_classic.h)."""
    _fields_ = [("length", ctypes.c_void_p), ("width", ctypes.c_void_p), ("taper", ctypes.c_void_p),
                ("taper_start", ctypes.c_void_p), ("width_ramp", ctypes.c_void_p),
                ("effects", ctypes.POINTER(ClassicFx)), ("effect_count", ctypes.c_uint32),
                ("description_id", ctypes.c_uint32), ("description_name", ctypes.c_char_p)]


class ClassicFxCurves(ctypes.Structure):
    """nxg_classic_fx_curves (nxg_classic.h)."""
    _fields_ = [("points", ctypes.c_void_p), ("point_counts", ctypes.c_void_p), ("roots", ctypes.c_void_p),
                ("surface_tangents", ctypes.c_void_p), ("noise_domains", ctypes.c_void_p),
                ("strand_count", ctypes.c_uint32), ("cvs_per_strand", ctypes.c_uint32),
                ("first_id", ctypes.c_uint32), ("radius_scale", ctypes.c_float),
                ("random_prefixes", ctypes.c_void_p), ("clumps", ctypes.POINTER(ClassicClumpGuides)),
                ("clump_count", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


class CurveCacheInput(ctypes.Structure):
    """nxg_curve_cache_input (nxg_cache.h)."""
    _fields_ = [(name, t) for pair in (("point_counts", "strand_count"), ("points", "point_count"),
                                        ("texcoords", "texcoord_count"), ("patch_uvs", "patch_uv_count"),
                                        ("face_uvs", "face_uv_count"), ("face_ids", "face_id_count"),
                                        ("motion_times", "motion_sample_count"),
                                        ("motion_points", "motion_point_count"))
                for name, t in ((pair[0], ctypes.c_void_p), (pair[1], ctypes.c_uint64))]


class CurveCacheHeader(ctypes.Structure):
    """nxg_curve_cache_header (nxg_cache.h): CurveCacheHeader, 128 bytes."""
    _fields_ = [("magic", ctypes.c_uint64), ("version_major", ctypes.c_uint16), ("version_minor", ctypes.c_uint16),
                ("flags", ctypes.c_uint32), ("byte_size", ctypes.c_uint64), ("content_hash", ctypes.c_uint64),
                ("strand_count", ctypes.c_uint32), ("point_count", ctypes.c_uint32),
                ("motion_sample_count", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("point_counts_offset", ctypes.c_uint64), ("points_offset", ctypes.c_uint64),
                ("motion_times_offset", ctypes.c_uint64), ("motion_points_offset", ctypes.c_uint64),
                ("texcoords_offset", ctypes.c_uint64), ("patch_uvs_offset", ctypes.c_uint64),
                ("face_uvs_offset", ctypes.c_uint64), ("face_ids_offset", ctypes.c_uint64),
                ("padding", ctypes.c_uint8 * 16)]


class CurveCacheCheck(ctypes.Structure):
    """nxg_curve_cache_check (nxg_cache.h)."""
    _fields_ = [("error", ctypes.c_uint32), ("reserved", ctypes.c_uint32), ("point_sum", ctypes.c_uint64),
                ("checksum", ctypes.c_uint64), ("first_bad", ctypes.c_uint64 * 8)]


class CurveSet(ctypes.Structure):
    """nxg_curve_set (nxg_payload.h): the reference's CurveSetView on the device."""
    _fields_ = [("strand_count", ctypes.c_uint32), ("fixed_cvs_per_strand", ctypes.c_uint32),
                ("point_counts", ctypes.c_void_p), ("points", ctypes.c_void_p), ("point_count", ctypes.c_uint64),
                ("widths", ctypes.c_void_p), ("root_uvs", ctypes.c_void_p), ("roots", ctypes.c_void_p),
                ("constant_width", ctypes.c_float), ("reserved", ctypes.c_uint32)]


class MotionSet(ctypes.Structure):
    """nxg_motion_set (nxg_payload.h)."""
    _fields_ = [("time", ctypes.c_float), ("reserved", ctypes.c_uint32), ("curves", CurveSet)]


class PayloadOptions(ctypes.Structure):
    """nxg_payload_options (nxg_payload.h)."""
    _fields_ = [("max_strands_per_batch", ctypes.c_uint32), ("resample_cv_count", ctypes.c_uint32),
                ("radius_scale", ctypes.c_float), ("transform", ctypes.c_float * 12)]


class PayloadOutput(ctypes.Structure):
    """nxg_payload_output (nxg_payload.h)."""
    _fields_ = [("point_counts", ctypes.c_void_p), ("points", ctypes.c_void_p), ("root_uvs", ctypes.c_void_p),
                ("motion_points", ctypes.c_void_p), ("batch_first_point", ctypes.c_void_p)]


PAYLOAD_MAX_SAMPLES = 32

CLASSIC_FX_NOISE = 0
CLASSIC_FX_CUT = 1
CLASSIC_FX_CLUMP = 2
CLASSIC_MAX_FX = 8
CLASSIC_MAX_FX_CVS = 64

SURROGATE_INPUTS = 8
SURROGATE_PARAMETERS = 12544


class SurrogateConfig(ctypes.Structure):
    """nxg_surrogate_config (nxg_classic.h)."""
    _fields_ = [("input_offset", ctypes.c_float * SURROGATE_INPUTS),
                ("input_scale", ctypes.c_float * SURROGATE_INPUTS), ("seed", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class SurrogateTrainConfig(ctypes.Structure):
    """nxg_surrogate_train_config (nxg_classic.h)."""
    _fields_ = [("epochs", ctypes.c_uint32), ("batch", ctypes.c_uint32), ("learning_rate", ctypes.c_float),
                ("lr_decay", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("epsilon", ctypes.c_float), ("seed", ctypes.c_uint32)]


class SurrogateCheck(ctypes.Structure):
    """nxg_surrogate_check (nxg_classic.h)."""
    _fields_ = [("length_tolerance", ctypes.c_float), ("width_tolerance", ctypes.c_float),
                ("checks_per_batch", ctypes.c_uint32), ("mode", ctypes.c_uint32)]


class AssetBuildInput(ctypes.Structure):
    """nxg_asset_build_input: the flattened AssetBuildInput of asset.h:14-44."""
    _fields_ = [
        ("positions", ctypes.c_void_p), ("vertex_count", ctypes.c_uint32),
        ("normals", ctypes.c_void_p), ("texcoords", ctypes.c_void_p),
        ("triangles", ctypes.c_void_p), ("triangle_count", ctypes.c_uint32),
        ("guide_count", ctypes.c_uint32), ("guide_cv_counts", ctypes.c_void_p),
        ("guide_cvs", ctypes.c_void_p), ("guide_root_normals", ctypes.c_void_p),
        ("guide_root_uvs", ctypes.c_void_p), ("guide_triangles", ctypes.c_void_p),
        ("guide_barycentrics", ctypes.c_void_p), ("guide_support_radii", ctypes.c_void_p),
        ("stencil_slots", ctypes.c_uint32), ("worker_count", ctypes.c_uint32),
    ]


assert ctypes.sizeof(AssetHeader) == 128
assert ctypes.sizeof(GenerationParams) == 60
assert ctypes.sizeof(DeviceAssetDesc) == 256
assert DeviceAssetDesc.header.offset == 64
assert ctypes.sizeof(PackedOutputDesc) == 72

# Record dtypes for numpy views of device/host arrays.
ROOT_DTYPE = np.dtype([("position", "<f4", 3), ("normal", "<f4", 3), ("uv", "<f4", 2),
                       ("triangle_index", "<u4"), ("barycentric", "<f4", 2),
                       ("surface_face_id", "<u4")])
STATE_DTYPE = np.dtype([("root", ROOT_DTYPE), ("indices", "<u4", 8), ("weights", "<f4", 8),
                        ("weight_sum", "<f4"), ("nearest", "<u4"), ("surface_u", "<f4", 3),
                        ("noise_domain", "<f4", 3)])
GUIDE_DTYPE = np.dtype([("first_cv", "<u4"), ("cv_count", "<u2"), ("flags", "<u2"),
                        ("triangle_index", "<u4"), ("support_radius", "<f4"),
                        ("barycentric", "<f4", 2), ("root_uv", "<f4", 2),
                        ("root_position", "<f4", 3), ("root_normal", "<f4", 3)])
assert ROOT_DTYPE.itemsize == 48 and STATE_DTYPE.itemsize == 144 and GUIDE_DTYPE.itemsize == 56
# nxg_walk_state: the lane walk's own stencil decisions (80 bytes).
WALK_STATE_DTYPE = np.dtype([("mode", "<u4"), ("nearest", "<u4"), ("weight_sum", "<f4"), ("slot_count", "<u4"),
                             ("guides", "<u4", 8), ("weights", "<f4", 8)])
assert WALK_STATE_DTYPE.itemsize == 80

# nxg_error (device_contract.h:58-80 plus additions).
ERROR_NAMES = [
    "None", "NullAsset", "MisalignedAsset", "InvalidAssetMetadata", "AssetCapacityTooSmall",
    "InvalidGenerationParameters", "InvalidBlockSize", "DeformedPositionCountMismatch",
    "DeformedNormalCountMismatch", "DeformedGuideCvCountMismatch", "MissingOutput",
    "PointCapacityTooSmall", "WidthCapacityTooSmall", "RootCapacityTooSmall",
    "RootUvCapacityTooSmall", "PointCountCapacityTooSmall", "InvalidRadiusScale",
    "MissingMotionSamples", "InvalidMotionTimes", "MotionPointCapacityTooSmall",
    "OutputSizeOverflow",
]
ERRORS = {name: code for code, name in enumerate(ERROR_NAMES)}
ERRORS.update(InvalidArgument=64, InvalidStrandRange=65, WorkspaceTooSmall=66,
              MisalignedOutput=67, StaticScratchLimit=68, ExpressionSyntax=69, ExpressionLimit=70,
              ExpressionInput=71, ExpressionDomain=72, Surrogate=73, Cuda=96)
STATIC_SCRATCH_BYTES = 4 << 20  # NXG_STATIC_SCRATCH_BYTES
ERROR_BY_CODE = {code: name for name, code in ERRORS.items()}

# Every entry point include/nxg.h declares: name -> (restype, argtypes).
_P = ctypes.c_void_p
_SIGNATURES = {
    "nxg_error_message": (ctypes.c_char_p, [ctypes.c_uint32]),
    "nxg_abi_version": (ctypes.c_uint32, []),
    "nxg_last_cuda_error": (ctypes.c_int32, []),
    "nxg_validate_asset": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_char_p, ctypes.c_uint64]),
    "nxg_make_device_asset_descriptor": (ctypes.c_uint32, [_P, ctypes.c_uint64, _P, ctypes.c_uint64,
                                                           ctypes.POINTER(DeviceAssetDesc),
                                                           ctypes.c_char_p, ctypes.c_uint64]),
    "nxg_build_asset": (ctypes.c_int, [ctypes.POINTER(AssetBuildInput), ctypes.POINTER(ctypes.c_void_p),
                                       ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p,
                                       ctypes.c_uint64]),
    "nxg_build_asset_device": (ctypes.c_int, [ctypes.POINTER(AssetBuildInput), _P, ctypes.POINTER(ctypes.c_void_p),
                                              ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p, ctypes.c_uint64]),
    "nxg_build_stencils_device": (ctypes.c_uint32, [_P, ctypes.c_uint32, _P, ctypes.c_uint32, _P, _P,
                                                    ctypes.c_uint32, ctypes.c_uint32, _P, _P]),
    "nxg_free": (None, [_P]),
    "nxg_fnv1a": (ctypes.c_uint64, [_P, ctypes.c_uint64]),
    "nxg_validate_generation_request": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                          ctypes.POINTER(DeformedDesc),
                                                          ctypes.POINTER(GenerationParams),
                                                          ctypes.POINTER(GeneratedOutputDesc),
                                                          ctypes.POINTER(LaunchConfig)]),
    "nxg_validate_packed_request": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                      ctypes.POINTER(DeformedDesc),
                                                      ctypes.POINTER(GenerationParams),
                                                      ctypes.POINTER(PackedOutputDesc),
                                                      ctypes.POINTER(LaunchConfig)]),
    "nxg_validate_motion_request": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                      ctypes.POINTER(MotionSampleDesc), ctypes.c_uint32,
                                                      ctypes.POINTER(GenerationParams),
                                                      ctypes.POINTER(MotionOutputDesc),
                                                      ctypes.POINTER(LaunchConfig)]),
    "nxg_packed_workspace_size": (ctypes.c_uint64, [ctypes.POINTER(DeviceAssetDesc),
                                                    ctypes.POINTER(GenerationParams), ctypes.c_uint32]),
    "nxg_generate_packed": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(DeformedDesc),
                                              ctypes.POINTER(GenerationParams),
                                              ctypes.POINTER(PackedOutputDesc),
                                              ctypes.POINTER(LaunchConfig), _P, ctypes.c_uint64, _P]),
    "nxg_generate_packed_range": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                    ctypes.POINTER(DeformedDesc),
                                                    ctypes.POINTER(GenerationParams),
                                                    ctypes.POINTER(PackedOutputDesc),
                                                    ctypes.POINTER(LaunchConfig), ctypes.c_uint32,
                                                    ctypes.c_uint32, _P, ctypes.c_uint64, _P]),
    "nxg_prepare_strand_order": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                   ctypes.POINTER(GenerationParams), ctypes.c_uint32,
                                                   ctypes.c_uint32, _P, ctypes.c_uint64, _P]),
    "nxg_generate_packed_ordered": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                      ctypes.POINTER(DeformedDesc),
                                                      ctypes.POINTER(GenerationParams),
                                                      ctypes.POINTER(PackedOutputDesc),
                                                      ctypes.POINTER(LaunchConfig), ctypes.c_uint32,
                                                      ctypes.c_uint32, _P, ctypes.c_uint64, _P]),
    "nxg_set_tile": (ctypes.c_uint32, [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(Tile)]),
    "nxg_get_tile": (ctypes.c_uint32, [ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(Tile)]),
    "nxg_autotune_packed": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(DeformedDesc),
                                              ctypes.POINTER(GenerationParams), ctypes.POINTER(PackedOutputDesc),
                                              ctypes.c_uint32, ctypes.c_uint32, _P, ctypes.c_uint64,
                                              ctypes.c_uint32, _P, ctypes.POINTER(Tile),
                                              ctypes.POINTER(ctypes.c_float)]),
    "nxg_generate_packed_static_scratch": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                             ctypes.POINTER(DeformedDesc),
                                                             ctypes.POINTER(GenerationParams),
                                                             ctypes.POINTER(PackedOutputDesc),
                                                             ctypes.POINTER(LaunchConfig), _P]),
    "nxg_generate_motion_packed": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(MotionSampleDesc),
                                                     ctypes.c_uint32, ctypes.POINTER(GenerationParams),
                                                     ctypes.POINTER(PackedOutputDesc), ctypes.POINTER(LaunchConfig),
                                                     _P, ctypes.c_uint64, _P]),
    "nxg_generate_motion": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(MotionSampleDesc),
                                              ctypes.c_uint32, ctypes.POINTER(GenerationParams),
                                              ctypes.POINTER(MotionOutputDesc), ctypes.POINTER(LaunchConfig), _P,
                                              ctypes.c_uint64, _P]),
    "nxg_batched_workspace_size": (ctypes.c_uint64, [_P, _P, ctypes.c_uint32]),
    "nxg_generate_batched": (ctypes.c_uint32, [_P, _P, _P, _P, ctypes.c_uint32, ctypes.POINTER(LaunchConfig), _P,
                                               ctypes.c_uint64, _P]),
    "nxg_query_strand_states": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc),
                                                  ctypes.POINTER(DeformedDesc),
                                                  ctypes.POINTER(GenerationParams), _P, ctypes.c_uint32,
                                                  _P, _P]),
    "nxg_query_walk_states": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(DeformedDesc),
                                                ctypes.POINTER(GenerationParams), _P, ctypes.c_uint32, _P, _P,
                                                ctypes.c_uint64, _P]),
    # nxg_classic.h
    "nxg_expression_compile": (ctypes.c_uint32, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_uint32,
                                                 ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_size_t]),
    "nxg_expression_destroy": (None, [_P]),
    "nxg_expression_get_info": (ctypes.c_uint32, [_P, ctypes.POINTER(ExpressionInfo)]),
    "nxg_expression_get_instruction": (ctypes.c_uint32, [_P, ctypes.c_uint32, ctypes.POINTER(ExpressionInstruction)]),
    "nxg_expression_get_operand": (ctypes.c_uint32, [_P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)]),
    "nxg_expression_get_ramp_point": (ctypes.c_uint32, [_P, ctypes.c_uint32, ctypes.POINTER(ExpressionRampPoint)]),
    "nxg_expression_input_name": (ctypes.c_char_p, [_P, ctypes.c_uint32]),
    "nxg_xgen_string_seed": (ctypes.c_uint32, [ctypes.c_char_p]),
    "nxg_classic_fx_plan_bytes": (ctypes.c_uint64, []),
    "nxg_classic_fx_plan_upload": (ctypes.c_uint32, [ctypes.POINTER(ClassicFxPlan), _P, ctypes.c_uint64, _P]),
    "nxg_classic_fx_apply": (ctypes.c_uint32, [_P, ctypes.POINTER(ClassicFxCurves), _P, _P]),
    "nxg_classic_clump_prepare": (ctypes.c_uint32, [_P, ctypes.c_uint32, ctypes.c_uint32, _P, _P, _P]),
    "nxg_curve_cache_error_message": (ctypes.c_char_p, [ctypes.c_uint32]),
    "nxg_payload_error_message": (ctypes.c_char_p, [ctypes.c_uint32]),
    "nxg_payload_point_count": (ctypes.c_uint64, [ctypes.POINTER(CurveSet), ctypes.POINTER(PayloadOptions)]),
    "nxg_payload_batch_count": (ctypes.c_uint32, [ctypes.POINTER(CurveSet), ctypes.POINTER(PayloadOptions)]),
    "nxg_payload_workspace_size": (ctypes.c_uint64, [ctypes.POINTER(CurveSet), _P, ctypes.c_uint32]),
    "nxg_build_curve_batches": (ctypes.c_uint32, [ctypes.POINTER(CurveSet), _P, ctypes.c_uint32,
                                                  ctypes.POINTER(PayloadOptions), ctypes.POINTER(PayloadOutput),
                                                  _P, ctypes.c_uint64, _P, ctypes.POINTER(ctypes.c_uint32), _P]),
    "nxg_curve_cache_build": (ctypes.c_uint32, [ctypes.POINTER(CurveCacheInput), ctypes.POINTER(ctypes.c_void_p),
                                                ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p, ctypes.c_uint64]),
    "nxg_curve_cache_validate": (ctypes.c_uint32, [_P, ctypes.c_uint64]),
    "nxg_curve_cache_content_hash": (ctypes.c_uint64, [_P, ctypes.c_uint64]),
    "nxg_curve_cache_point_checksum": (ctypes.c_uint64, [_P, ctypes.c_uint64]),
    "nxg_curve_cache_validate_device": (ctypes.c_uint32, [_P, _P, ctypes.c_uint64, _P,
                                                          ctypes.POINTER(ctypes.c_uint32), _P]),
    "nxg_classic_root_scalars": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(GenerationParams),
                                                   ctypes.POINTER(ClassicScalarPlan), ctypes.c_uint32,
                                                   ctypes.c_uint32, _P, _P, _P]),
    "nxg_generate_packed_classic": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(DeformedDesc),
                                                      ctypes.POINTER(GenerationParams),
                                                      ctypes.POINTER(PackedOutputDesc),
                                                      ctypes.POINTER(ClassicApplyDesc), ctypes.POINTER(LaunchConfig),
                                                      ctypes.c_uint32, ctypes.c_uint32, _P, ctypes.c_uint64, _P]),
    "nxg_generate_batched_classic": (ctypes.c_uint32, [_P, _P, _P, _P, _P, ctypes.c_uint32,
                                                       ctypes.POINTER(LaunchConfig), _P, ctypes.c_uint64, _P]),
    "nxg_surrogate_model_bytes": (ctypes.c_uint64, []),
    "nxg_surrogate_workspace_bytes": (ctypes.c_uint64, []),
    "nxg_surrogate_init": (ctypes.c_uint32, [_P, ctypes.POINTER(SurrogateConfig), _P]),
    "nxg_surrogate_features": (ctypes.c_uint32, [ctypes.POINTER(DeviceAssetDesc), ctypes.POINTER(GenerationParams),
                                                 ctypes.c_uint32, ctypes.c_uint32, _P, _P]),
    "nxg_surrogate_fit_outputs": (ctypes.c_uint32, [_P, _P, ctypes.c_uint32, _P]),
    "nxg_surrogate_train": (ctypes.c_uint32, [_P, _P, _P, ctypes.c_uint32, ctypes.POINTER(SurrogateTrainConfig), _P,
                                              ctypes.c_uint64, _P, _P]),
    "nxg_surrogate_gradients": (ctypes.c_uint32, [_P, _P, _P, ctypes.c_uint32, _P, _P, _P]),
    "nxg_surrogate_forward": (ctypes.c_uint32, [_P, _P, ctypes.c_uint32, _P, _P]),
    "nxg_surrogate_root_scalars": (ctypes.c_uint32, [_P, ctypes.POINTER(DeviceAssetDesc),
                                                     ctypes.POINTER(GenerationParams),
                                                     ctypes.POINTER(ClassicScalarPlan), ctypes.POINTER(SurrogateCheck),
                                                     ctypes.c_uint32, ctypes.c_uint32, _P, _P, _P]),
    "nxg_surrogate_parameters": (ctypes.c_uint32, [_P, ctypes.POINTER(ctypes.c_void_p)]),
}


class NxgError(RuntimeError):
    """A non-zero nxg_error status, with the library's message."""

    def __init__(self, code: int, where: str = ""):
        self.code = int(code)
        self.name = ERROR_BY_CODE.get(self.code, "Unknown")
        message = lib().nxg_error_message(self.code).decode()
        if self.code == ERRORS["Cuda"]:
            message += " (cudaError %d)" % lib().nxg_last_cuda_error()
        super().__init__("%s%s: %s" % (where + ": " if where else "", self.name, message))


_LIB = None


def lib() -> ctypes.CDLL:
    """The loaded libnxg_b200.so with typed prototypes (raises if unbuilt)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError("libnxg_b200.so is not built (run `python -m nanoxgen_b200.build`); "
                              "this package has no CPU fallback")
        handle = ctypes.CDLL(LIBRARY_PATH)
        for name, (restype, argtypes) in _SIGNATURES.items():
            if not hasattr(handle, name):
                raise ImportError("libnxg_b200.so lacks %s; rebuild it" % name)
            fn = getattr(handle, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _LIB = handle
    return _LIB


def declared_symbols() -> list[str]:
    return sorted(_SIGNATURES)


def check(code: int, where: str = "") -> None:
    if code != 0:
        raise NxgError(code, where)
