"""The learned per-root scalar surrogate (include/nxg_classic.h, third part).

``Surrogate`` owns the model's device buffer and drives the library's
kernels: feature extraction from an asset's roots, output normalisation,
tensor-core training with Adam, forward evaluation, full-batch gradients
(for checking against the CPU oracle) and the judged per-root scalars that
replace nxg_classic_root_scalars in a generation pass.  torch supplies the
device memory and the stream only.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Optional

import numpy as np
import torch

from . import _abi
from ._abi import SurrogateCheck, SurrogateConfig, SurrogateTrainConfig, check, lib
from .classic import ScalarPlan
from .generator import DeviceAsset, _stream_handle

PARAMETERS = _abi.SURROGATE_PARAMETERS


def asset_input_normalisation(asset) -> tuple[np.ndarray, np.ndarray]:
    """Offsets and scales that map an asset's rest positions to [-1, 1]
    (normals and uv pass through as [-1, 1] and [0, 1] values)."""
    pos = asset.positions().reshape(-1, 3).astype(np.float64)
    lo, hi = pos.min(0), pos.max(0)
    centre = 0.5 * (lo + hi)
    half = np.maximum(0.5 * (hi - lo), 1e-12)
    offset = np.concatenate([centre, np.zeros(3), [0.5, 0.5]]).astype(np.float32)
    scale = np.concatenate([1.0 / half, np.ones(3), [2.0, 2.0]]).astype(np.float32)
    return offset, scale


@dataclasses.dataclass
class TrainResult:
    epoch_losses: np.ndarray   # mean training loss per epoch (normalised outputs)
    steps: int


class Surrogate:
    """A 3 x 64 BF16 MLP over (rest position, normal, uv) on one device."""

    def __init__(self, device: str | torch.device = "cuda", input_offset=None, input_scale=None, seed: int = 1):
        self.device = torch.device(device)
        self.model = torch.zeros(int(lib().nxg_surrogate_model_bytes()), dtype=torch.uint8, device=self.device)
        assert self.model.data_ptr() % 256 == 0
        self.workspace = torch.zeros(int(lib().nxg_surrogate_workspace_bytes()), dtype=torch.uint8,
                                     device=self.device)
        cfg = SurrogateConfig()
        off = np.zeros(8, np.float32) if input_offset is None else np.asarray(input_offset, np.float32)
        sc = np.ones(8, np.float32) if input_scale is None else np.asarray(input_scale, np.float32)
        for j in range(8):
            cfg.input_offset[j] = float(off[j])
            cfg.input_scale[j] = float(sc[j])
        cfg.seed = seed
        self.input_offset, self.input_scale = off, sc
        check(lib().nxg_surrogate_init(self.model.data_ptr(), ctypes.byref(cfg), _stream_handle(None)),
              "nxg_surrogate_init")

    # -- data ----------------------------------------------------------------
    @staticmethod
    def features(dasset: DeviceAsset, params, first_strand: int = 0, count: Optional[int] = None,
                 stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
        """Raw features (count, 8) of the roots of strands [first, first+count)."""
        n = int(params.strand_count) - first_strand if count is None else int(count)
        out = torch.empty((max(n, 1), 8), dtype=torch.float32, device=dasset.device)
        check(lib().nxg_surrogate_features(ctypes.byref(dasset.desc), ctypes.byref(params), first_strand, n,
                                           out.data_ptr(), _stream_handle(stream)), "nxg_surrogate_features")
        return out[:n]

    def fit_outputs(self, targets: torch.Tensor) -> None:
        check(lib().nxg_surrogate_fit_outputs(self.model.data_ptr(), targets.data_ptr(), targets.shape[0],
                                              _stream_handle(None)), "nxg_surrogate_fit_outputs")

    # -- learning ------------------------------------------------------------
    def train(self, features: torch.Tensor, targets: torch.Tensor, epochs: int = 10, batch: int = 16384,
              learning_rate: float = 2e-3, lr_decay: float = 0.8, seed: int = 7) -> TrainResult:
        cfg = SurrogateTrainConfig(epochs, batch, learning_rate, lr_decay, 0.9, 0.999, 1e-8, seed)
        history = torch.zeros(epochs, dtype=torch.float32, device=self.device)
        code = lib().nxg_surrogate_train(self.model.data_ptr(), features.data_ptr(), targets.data_ptr(),
                                         features.shape[0], ctypes.byref(cfg), self.workspace.data_ptr(),
                                         self.workspace.numel(), history.data_ptr(), _stream_handle(None))
        check(code, "nxg_surrogate_train")
        steps = (features.shape[0] + batch - 1) // batch
        return TrainResult(history.cpu().numpy() / steps, steps * epochs)

    def gradients(self, features: torch.Tensor, targets: torch.Tensor) -> tuple[float, np.ndarray]:
        grad = torch.empty(PARAMETERS, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        check(lib().nxg_surrogate_gradients(self.model.data_ptr(), features.data_ptr(), targets.data_ptr(),
                                            features.shape[0], grad.data_ptr(), loss.data_ptr(),
                                            _stream_handle(None)), "nxg_surrogate_gradients")
        torch.cuda.synchronize(self.device)
        return float(loss.item()), grad.cpu().numpy()

    # -- inference -----------------------------------------------------------
    def forward(self, features: torch.Tensor) -> torch.Tensor:
        out = torch.empty((features.shape[0], 2), dtype=torch.float32, device=self.device)
        check(lib().nxg_surrogate_forward(self.model.data_ptr(), features.data_ptr(), features.shape[0],
                                          out.data_ptr(), _stream_handle(None)), "nxg_surrogate_forward")
        return out

    def root_scalars(self, dasset: DeviceAsset, params, plan: ScalarPlan, *, length_tolerance: float = 1e-3,
                     width_tolerance: float = 1e-3, checks_per_batch: int = 4, mode: int = 0,
                     first_strand: int = 0, count: Optional[int] = None, out: Optional[torch.Tensor] = None,
                     status: Optional[torch.Tensor] = None,
                     stream: Optional[torch.cuda.Stream] = None) -> tuple[torch.Tensor, torch.Tensor]:
        """(scalars (n, 2), status (4,): error, failing roots, batches re-run
        exactly, batches checked).  Enqueue only."""
        n = int(params.strand_count) - first_strand if count is None else int(count)
        if out is None:
            out = torch.empty((max(n, 1), 2), dtype=torch.float32, device=dasset.device)
        if status is None:
            status = torch.zeros(4, dtype=torch.int32, device=dasset.device)
        chk = SurrogateCheck(length_tolerance, width_tolerance, checks_per_batch, mode)
        desc = plan.descriptor()
        check(lib().nxg_surrogate_root_scalars(self.model.data_ptr(), ctypes.byref(dasset.desc),
                                               ctypes.byref(params), ctypes.byref(desc), ctypes.byref(chk),
                                               first_strand, n, out.data_ptr(), status.data_ptr(),
                                               _stream_handle(stream)), "nxg_surrogate_root_scalars")
        return out, status

    # -- state ---------------------------------------------------------------
    def parameters(self) -> np.ndarray:
        ptr = ctypes.c_void_p()
        check(lib().nxg_surrogate_parameters(self.model.data_ptr(), ctypes.byref(ptr)), "nxg_surrogate_parameters")
        offset = ptr.value - self.model.data_ptr()
        return self.model[offset:offset + 4 * PARAMETERS].view(torch.float32).cpu().numpy().copy()

    def header(self) -> dict:
        raw = self.model[:256].cpu().numpy()
        f = raw.view(np.float32)
        u = raw.view(np.uint32)
        return dict(step=int(u[3]), input_offset=f[4:12].copy(), input_scale=f[12:20].copy(),
                    output_offset=f[20:22].copy(), output_scale=f[22:24].copy(), trained=int(u[25]))
