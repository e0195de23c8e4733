"""Shared helpers of the test suite (no product code)."""
import numpy as np

from nanoxgen_b200.asset import recompute_hash


def patch_stencil(blob: np.ndarray, slots: int) -> np.ndarray:
    """Invalidate stencil slots >= `slots` of every triangle and re-hash: the
    K-guide stencil of the benchmark configurations in the reference's
    fixed 8-slot format (types.h:20, generate.h:229 skips invalid slots)."""
    blob = blob.copy()
    tri_count = int(blob[36:40].view(np.uint32)[0])
    off = int(blob[112:120].view(np.uint64)[0])  # AssetHeader::triangle_guides_offset
    st = blob[off:off + tri_count * 32].view(np.uint32).reshape(tri_count, 8)
    st[:, slots:] = 0xFFFFFFFF
    recompute_hash(blob)
    return blob


def max_position_error(a: np.ndarray, b: np.ndarray) -> float:
    """Largest Euclidean distance between matching float4 positions."""
    d = a[:, :3].astype(np.float64) - b[:, :3].astype(np.float64)
    return float(np.sqrt((d * d).sum(-1)).max()) if d.size else 0.0
