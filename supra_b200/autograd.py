"""Autograd entry points of the differentiable receive path (extension without a reference
counterpart): DAS with per-element apodisation and a speed-of-sound parameter, and the Hilbert FIR
envelope. `das_apod` / `envelope` run the libtorch autograd Functions (torch_ext/autograd_ops.cpp,
torch.ops.supra_b200.*); `das_apod_py` / `envelope_py` are the same operators as Python
torch.autograd.Functions. Forward and backward run the library's CUDA kernels (sb_das_forward_apod /
sb_das_adjoint, sb_hilbert_env_run / sb_hilbert_env_adjoint); aperture tiles are recomputed in the
backward pass, only the forward output is kept.
"""
from __future__ import annotations

import os
from typing import Optional

import torch

from .api import HilbertFirEnvelope, RxBeamformer


class DasApodFunction(torch.autograd.Function):
    """s = DAS(rf; apod, c). rf [frames][num_tx][num_channels][num_samples] FP32, apod [num_elements],
    c: 0-dim tensor, speed of sound in mm/s."""

    @staticmethod
    def forward(ctx, rf, apod, c, beamformer: RxBeamformer, f_number: float, window_type: int, window_parameter: float):
        c_val = float(c.detach().item()) if torch.is_tensor(c) else float(c)
        out = beamformer.forward_apod(rf.contiguous(), None if apod is None else apod.contiguous(), c_val, f_number,
                                      window_type, window_parameter)
        ctx.save_for_backward(rf, apod, out)
        ctx.cfg = (beamformer, c_val, f_number, window_type, window_parameter, torch.is_tensor(c))
        ctx.c_dtype = c.dtype if torch.is_tensor(c) else None
        ctx.c_device = c.device if torch.is_tensor(c) else None
        return out

    @staticmethod
    def backward(ctx, grad_out):
        rf, apod, out = ctx.saved_tensors
        beamformer, c_val, f_number, window_type, window_parameter, c_is_tensor = ctx.cfg
        need_rf, need_apod, need_c = ctx.needs_input_grad[0], ctx.needs_input_grad[1], ctx.needs_input_grad[2]
        g_rf, g_ap, g_c = beamformer.adjoint(rf.contiguous(), None if apod is None else apod.contiguous(),
                                             grad_out.contiguous(), c_val, out, f_number, window_type,
                                             window_parameter, need_rf, need_apod and apod is not None,
                                             need_c and c_is_tensor)
        if g_c is not None:
            g_c = g_c.reshape(()).to(device=ctx.c_device, dtype=ctx.c_dtype)
        return g_rf, g_ap, g_c, None, None, None, None


class EnvelopeFunction(torch.autograd.Function):
    """Hilbert FIR envelope of [num_samples][num_scanlines] (or a batch of them) FP32 images."""

    @staticmethod
    def forward(ctx, img, hilbert: HilbertFirEnvelope):
        img = img.contiguous()
        if img.dim() == 2:
            out = hilbert.demodulate(img)
        else:
            out = torch.stack([hilbert.demodulate(x) for x in img])
        ctx.save_for_backward(img)
        ctx.hilbert = hilbert
        return out

    @staticmethod
    def backward(ctx, grad_env):
        (img,) = ctx.saved_tensors
        h = ctx.hilbert
        grad_env = grad_env.contiguous()
        if img.dim() == 2:
            return h.adjoint(img, grad_env), None
        return torch.stack([h.adjoint(x, g) for x, g in zip(img, grad_env)]), None


_OPS_LOADED = False


def load_torch_ops() -> None:
    """Loads the libtorch autograd operators (torch.ops.supra_b200.das_apod / .envelope), built in-tree
    by `python -m supra_b200.build --torch-ops`. Raises if they are not built."""
    global _OPS_LOADED
    if _OPS_LOADED:
        return
    so = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "supra_b200_torch_ops.so")
    if not os.path.exists(so):
        raise OSError(f"libtorch operators not built: {so} (python -m supra_b200.build --torch-ops)")
    torch.ops.load_library(so)
    _OPS_LOADED = True


def das_apod(beamformer: RxBeamformer, rf: torch.Tensor, apod: Optional[torch.Tensor], c_mm_s: torch.Tensor,
             f_number=1.0, window_type=1, window_parameter=0.0) -> torch.Tensor:
    """Differentiable DAS through the libtorch autograd Function (DasApodFn in torch_ext/autograd_ops.cpp).
    rf [frames][num_tx][num_channels][num_samples] (or without the frame axis), c_mm_s a 0-dim tensor."""
    load_torch_ops()
    g = beamformer.geometry
    squeeze = rf.dim() == 3
    x = rf.unsqueeze(0) if squeeze else rf
    if not torch.is_tensor(c_mm_s):
        c_mm_s = torch.tensor(float(c_mm_s), dtype=torch.float64)
    out = torch.ops.supra_b200.das_apod(x, apod, c_mm_s, beamformer.handle.value, g.num_depths, g.num_rx,
                                        float(f_number), int(window_type), float(window_parameter))
    return out[0] if squeeze else out


def envelope(img: torch.Tensor, hilbert: HilbertFirEnvelope) -> torch.Tensor:
    """Hilbert FIR envelope through the libtorch autograd Function (EnvelopeFn)."""
    load_torch_ops()
    return torch.ops.supra_b200.envelope(img, hilbert.handle.value)


def das_apod_py(beamformer: RxBeamformer, rf: torch.Tensor, apod: Optional[torch.Tensor], c_mm_s, f_number=1.0,
                window_type=1, window_parameter=0.0) -> torch.Tensor:
    """The same operator as a Python torch.autograd.Function (same kernels)."""
    return DasApodFunction.apply(rf, apod, c_mm_s, beamformer, f_number, window_type, window_parameter)


def envelope_py(img: torch.Tensor, hilbert: HilbertFirEnvelope) -> torch.Tensor:
    return EnvelopeFunction.apply(img, hilbert)
