"""Python binding of the C ABI over torch device tensors.

Mirrors the reference's algorithm classes (RxBeamformerCuda, RawDelay, HilbertFirEnvelope,
LogCompressor, IQDemodulator, ScanConverter, RxBeamformerMV): the same constructor arguments and
per-call parameters, device buffers in and out, launched on the current torch stream. Every call
goes through libsupra_b200.so; there is no other implementation behind these classes.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np
import torch

from . import abi
from .abi import (SB_COMPLEX64, SB_FLOAT32, SB_INT16, SB_UINT8, SB_UINT16, check, load_library, sb_geometry,
                  sb_mv_stats)

_DT = {torch.int16: SB_INT16, torch.float32: SB_FLOAT32, torch.uint8: SB_UINT8, torch.complex64: SB_COMPLEX64}
_TORCH = {SB_INT16: torch.int16, SB_FLOAT32: torch.float32, SB_UINT8: torch.uint8, SB_COMPLEX64: torch.complex64}


def _stream() -> C.c_void_p:
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: Optional[torch.Tensor]) -> Optional[C.c_void_p]:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("supra_b200 kernels take CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return C.c_void_p(t.data_ptr())


def dtype_code(t: torch.Tensor) -> int:
    try:
        return _DT[t.dtype]
    except KeyError:
        raise ValueError(f"unsupported dtype {t.dtype}") from None


# RxBeamformerCuda::RxSampleBeamformer (Beamformer/RxBeamformerCuda.h:31-36)
SAMPLE_BEAMFORMERS = {"DelayAndSum": 0, "DelayAndStdDev": 1, "CoherenceFactorDelayAndSum": 2, "TestSignal": 3}


class RxBeamformer:
    """RxBeamformerCuda (Beamformer/RxBeamformerCuda.cu:24-663), DelayAndSum, 2D or 3D."""

    def __init__(self, geometry):
        self.lib = load_library()
        self.geometry = geometry
        g = geometry.ctypes()
        self._plan = C.c_void_p()
        check("sb_das_plan_create", self.lib.sb_das_plan_create(C.byref(g), C.byref(self._plan)))

    def __del__(self):
        if getattr(self, "_plan", None) and self._plan.value:
            self.lib.sb_das_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    @property
    def handle(self) -> C.c_void_p:
        return self._plan

    def beamform(self, rf: torch.Tensor, f_number=1.0, speed_of_sound_mm_s=None, window_type=1, window_parameter=0.0,
                 interpolate_transmits=False, additional_offset=0, out_dtype=torch.float32,
                 out: Optional[torch.Tensor] = None, beamformer="DelayAndSum") -> torch.Tensor:
        """RxBeamformerCuda::performRxBeamforming (Beamformer/RxBeamformerCuda.cu:540-662): [num_depths][num_rx].
        beamformer: a name of BeamformingNode's "beamformerType" (DelayAndSum, DelayAndStdDev,
        CoherenceFactorDelayAndSum, TestSignal) or its index."""
        g = self.geometry
        c = g.speed_of_sound_mm_s if speed_of_sound_mm_s is None else speed_of_sound_mm_s
        bf = SAMPLE_BEAMFORMERS[beamformer] if isinstance(beamformer, str) else int(beamformer)
        if out is None:
            out = torch.empty((g.num_depths, g.num_rx), dtype=out_dtype, device=rf.device)
        if bf == 0:
            check("sb_das_run", self.lib.sb_das_run(self._plan, _ptr(rf), dtype_code(rf), _ptr(out), dtype_code(out),
                                                    float(f_number), float(c), int(window_type), float(window_parameter),
                                                    int(bool(interpolate_transmits)), int(additional_offset), _stream()))
        else:
            check("sb_das_run_beamformer",
                  self.lib.sb_das_run_beamformer(self._plan, bf, _ptr(rf), dtype_code(rf), _ptr(out), dtype_code(out),
                                                 float(f_number), float(c), int(window_type), float(window_parameter),
                                                 int(bool(interpolate_transmits)), int(additional_offset), _stream()))
        return out

    def raw_delay(self, rf: torch.Tensor, f_number=1.0, speed_of_sound_mm_s=None, window_type=1, window_parameter=0.0,
                  out_dtype=torch.float32) -> torch.Tensor:
        """RawDelay::performDelay (Beamformer/RawDelay.cu:556-650): [num_rx][num_channels][num_depths]."""
        g = self.geometry
        c = g.speed_of_sound_mm_s if speed_of_sound_mm_s is None else speed_of_sound_mm_s
        out = torch.empty((g.num_rx, g.num_channels, g.num_depths), dtype=out_dtype, device=rf.device)
        check("sb_rawdelay_run", self.lib.sb_rawdelay_run(self._plan, _ptr(rf), dtype_code(rf), _ptr(out),
                                                          dtype_code(out), float(f_number), float(c), int(window_type),
                                                          float(window_parameter), _stream()))
        return out


    def forward_apod(self, rf: torch.Tensor, apod: Optional[torch.Tensor], speed_of_sound_mm_s: float, f_number=1.0,
                     window_type=1, window_parameter=0.0) -> torch.Tensor:
        """Differentiable-path forward: rf FP32 [frames][num_tx][num_channels][num_samples] (or without the
        frame axis), per-element apodisation apod [num_elements] (None = 1) -> [frames][num_depths][num_rx]."""
        g = self.geometry
        squeeze = rf.dim() == 3
        if squeeze:
            rf = rf.unsqueeze(0)
        if rf.dtype != torch.float32:
            raise ValueError("forward_apod takes float32 channel data")
        frames = rf.shape[0]
        out = torch.empty((frames, g.num_depths, g.num_rx), dtype=torch.float32, device=rf.device)
        check("sb_das_forward_apod", self.lib.sb_das_forward_apod(self._plan, _ptr(rf), _ptr(apod), _ptr(out), frames,
                                                                  float(f_number), float(speed_of_sound_mm_s),
                                                                  int(window_type), float(window_parameter), _stream()))
        return out[0] if squeeze else out

    def adjoint(self, rf: torch.Tensor, apod: Optional[torch.Tensor], grad_out: torch.Tensor, speed_of_sound_mm_s: float,
                forward_out: Optional[torch.Tensor] = None, f_number=1.0, window_type=1, window_parameter=0.0,
                need_rf=True, need_apod=True, need_c=True):
        """Adjoint of forward_apod: returns (grad_rf or None, grad_apod or None, grad_c or None); grad_c is a
        one-element tensor (per mm/s)."""
        squeeze = rf.dim() == 3
        if squeeze:
            rf, grad_out = rf.unsqueeze(0), grad_out.unsqueeze(0)
            forward_out = None if forward_out is None else forward_out.unsqueeze(0)
        frames = rf.shape[0]
        grad_out = grad_out.contiguous()
        g_rf = torch.empty_like(rf) if need_rf else None
        g_ap = torch.empty(self.geometry.num_elements, dtype=torch.float32, device=rf.device) if need_apod else None
        g_c = torch.empty(1, dtype=torch.float32, device=rf.device) if need_c else None
        check("sb_das_adjoint", self.lib.sb_das_adjoint(self._plan, _ptr(rf), _ptr(apod), _ptr(forward_out),
                                                        _ptr(grad_out), _ptr(g_rf), _ptr(g_ap), _ptr(g_c), frames,
                                                        float(f_number), float(speed_of_sound_mm_s), int(window_type),
                                                        float(window_parameter), _stream()))
        if squeeze and g_rf is not None:
            g_rf = g_rf[0]
        return g_rf, g_ap, g_c


class HilbertFirEnvelope:
    """HilbertFirEnvelope(filterLength) (Beamformer/HilbertFirEnvelope.cu:63-104)."""

    def __init__(self, filter_length: int = 65):
        self.lib = load_library()
        self._plan = C.c_void_p()
        check("sb_hilbert_plan_create", self.lib.sb_hilbert_plan_create(int(filter_length), C.byref(self._plan)))

    def __del__(self):
        if getattr(self, "_plan", None) and self._plan.value:
            self.lib.sb_hilbert_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    @property
    def handle(self):
        return self._plan

    def demodulate(self, img: torch.Tensor) -> torch.Tensor:
        nS, nL = img.shape
        out = torch.empty((nS, nL), dtype=torch.float32, device=img.device)
        check("sb_hilbert_env_run", self.lib.sb_hilbert_env_run(self._plan, _ptr(img), dtype_code(img), _ptr(out),
                                                                SB_FLOAT32, nL, nS, _stream()))
        return out

    def adjoint(self, img: torch.Tensor, grad_env: torch.Tensor) -> torch.Tensor:
        """Gradient of the envelope w.r.t. its FP32 input [num_samples][num_scanlines]."""
        nS, nL = img.shape
        grad_env = grad_env.contiguous()
        out = torch.empty_like(img)
        check("sb_hilbert_env_adjoint", self.lib.sb_hilbert_env_adjoint(self._plan, _ptr(img), _ptr(grad_env),
                                                                        _ptr(out), nL, nS, _stream()))
        return out


class HilbertEnvelope:
    """HilbertEnvelope (Beamformer/HilbertEnvelope.cu:27-207): the envelope of the analytic signal of each
    scanline over its whole length (the reference computes it by FFT; here by the exact circular Hilbert
    transform), for images [num_samples][num_scanlines]."""

    def __init__(self, num_samples: int):
        self.lib = load_library()
        self.num_samples = int(num_samples)
        self._plan = C.c_void_p()
        check("sb_analytic_plan_create", self.lib.sb_analytic_plan_create(self.num_samples, C.byref(self._plan)))

    def __del__(self):
        if getattr(self, "_plan", None) and self._plan.value:
            self.lib.sb_analytic_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    def envelope(self, img: torch.Tensor, out_dtype=torch.float32) -> torch.Tensor:
        if img.dim() != 2 or img.shape[0] != self.num_samples or not img.is_contiguous():
            raise ValueError("HilbertEnvelope: a contiguous [num_samples][num_scanlines] image")
        out = torch.empty(img.shape, dtype=out_dtype, device=img.device)
        check("sb_analytic_env_run", self.lib.sb_analytic_env_run(self._plan, _ptr(img), dtype_code(img), _ptr(out),
                                                                  dtype_code(out), img.shape[1], _stream()))
        return out


class LogCompressor:
    """LogCompressor::compress (Beamformer/LogCompressor.cu:44-66)."""

    def __init__(self):
        self.lib = load_library()

    def compress(self, img: torch.Tensor, dynamic_range=80.0, gain=1.0, in_max=1024.0,
                 out_dtype=torch.float32) -> torch.Tensor:
        out = torch.empty(img.shape, dtype=out_dtype, device=img.device)
        check("sb_logcompress_run", self.lib.sb_logcompress_run(_ptr(img), dtype_code(img), _ptr(out), dtype_code(out),
                                                                img.numel(), float(dynamic_range), float(gain),
                                                                float(in_max), _stream()))
        return out


class IQDemodulator:
    """IQDemodulator + IQDemodulatorNode's frequency-compounding list (Beamformer/IQDemodulator.cu,
    Beamformer/IQDemodulatorNode.cpp:126-165)."""

    def __init__(self, sampling_frequency=40e6, cutoff_frequency=2.5e6, lowpass_filter_length=51,
                 bandpass_filter_length=51, reference_frequencies: Sequence[float] = (7e6,),
                 bandwidths: Sequence[float] = (1e6,), weights: Sequence[float] = (1.0,)):
        self.lib = load_library()
        self.fs = sampling_frequency
        self.cutoff = cutoff_frequency
        rf = np.ascontiguousarray(reference_frequencies, np.float64)
        bw = np.ascontiguousarray(bandwidths, np.float64)
        w = np.ascontiguousarray(weights, np.float64)
        self._plan = C.c_void_p()
        check("sb_iq_plan_create", self.lib.sb_iq_plan_create(float(sampling_frequency), float(cutoff_frequency),
                                                              int(lowpass_filter_length), int(bandpass_filter_length),
                                                              len(rf), rf.ctypes.data, bw.ctypes.data, w.ctypes.data,
                                                              C.byref(self._plan)))

    def __del__(self):
        if getattr(self, "_plan", None) and self._plan.value:
            self.lib.sb_iq_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    @staticmethod
    def decimated_length(num_samples: int, decimation: int) -> int:
        return num_samples // decimation if decimation > 1 else num_samples

    def demodulate_magnitude(self, img: torch.Tensor, decimation: int = 8, out_dtype=torch.float32) -> torch.Tensor:
        nS, nL = img.shape
        out = torch.empty((self.decimated_length(nS, decimation), nL), dtype=out_dtype, device=img.device)
        check("sb_iq_magnitude_run", self.lib.sb_iq_magnitude_run(self._plan, _ptr(img), dtype_code(img), _ptr(out),
                                                                  dtype_code(out), nL, nS, int(decimation), _stream()))
        return out


def iq_complex(img: torch.Tensor, sampling_frequency: float, mixing_frequency: float, cutoff_frequency: float,
               lowpass_length: int, decimation: int) -> torch.Tensor:
    """Complex baseband IQ (extension): [num_samples / decimation][num_scanlines] complex64."""
    lib = load_library()
    nS, nL = img.shape
    out = torch.empty((nS // max(decimation, 1), nL), dtype=torch.complex64, device=img.device)
    check("sb_iq_complex_run", lib.sb_iq_complex_run(_ptr(img), dtype_code(img), _ptr(out), nL, nS,
                                                     float(sampling_frequency), float(mixing_frequency),
                                                     float(cutoff_frequency), int(lowpass_length), int(decimation),
                                                     _stream()))
    return out


class ScanConverter:
    """ScanConverter (Beamformer/ScanConverter.cu:436-815). `scanlines` is the SCANLINE_DTYPE array of
    the receive geometry (x fastest)."""

    def __init__(self, scanlines: np.ndarray, layout, num_samples: int, depth_mm: float, resolution_mm: float):
        self.lib = load_library()
        self.layout = tuple(int(v) for v in layout)
        sl = np.ascontiguousarray(scanlines)
        self._plan = C.c_void_p()
        check("sb_scan_plan_create", self.lib.sb_scan_plan_create(sl.ctypes.data, self.layout[0], self.layout[1],
                                                                  int(num_samples), float(depth_mm),
                                                                  float(resolution_mm), C.byref(self._plan)))
        size = (C.c_uint32 * 3)()
        check("sb_scan_image_size", self.lib.sb_scan_image_size(self._plan, size))
        self.image_size = (int(size[0]), int(size[1]), int(size[2]))

    def __del__(self):
        if getattr(self, "_plan", None) and self._plan.value:
            self.lib.sb_scan_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    @property
    def handle(self):
        return self._plan

    @property
    def numel(self) -> int:
        return self.image_size[0] * self.image_size[1] * self.image_size[2]

    def tables(self) -> dict:
        n = self.numel
        mask = np.zeros(n, np.uint8)
        sidx = np.zeros(n, np.uint32)
        wx = np.zeros(n, np.float32)
        wy = np.zeros(n, np.float32)
        wz = np.zeros(n, np.float32)
        check("sb_scan_copy_tables", self.lib.sb_scan_copy_tables(self._plan, mask.ctypes.data, sidx.ctypes.data,
                                                                  wx.ctypes.data, wy.ctypes.data, wz.ctypes.data))
        return dict(size=self.image_size, mask=mask, sample_idx=sidx, weight_x=wx, weight_y=wy, weight_z=wz)

    def _shape(self):
        W, H, D = self.image_size
        return (D, H, W) if D > 1 else (H, W)

    def convert(self, img: torch.Tensor, out_dtype=torch.uint8) -> torch.Tensor:
        out = torch.empty(self._shape(), dtype=out_dtype, device=img.device)
        check("sb_scan_run", self.lib.sb_scan_run(self._plan, _ptr(img), dtype_code(img), _ptr(out), dtype_code(out),
                                                  _stream()))
        return out

    def env_log_convert(self, hilbert: HilbertFirEnvelope, rf: torch.Tensor, dynamic_range=80.0, gain=1.0,
                        in_max=1024.0, out_dtype=torch.uint8) -> torch.Tensor:
        """Fused HilbertFirEnvelope -> LogCompressor -> ScanConverter."""
        out = torch.empty(self._shape(), dtype=out_dtype, device=rf.device)
        check("sb_env_log_scan_run", self.lib.sb_env_log_scan_run(hilbert.handle, self._plan, _ptr(rf), _ptr(out),
                                                                  dtype_code(out), float(dynamic_range), float(gain),
                                                                  float(in_max), _stream()))
        return out


def temporal_filter(images: Sequence[torch.Tensor], weights: Optional[Sequence[float]] = None,
                    out_dtype=torch.float32, out: Optional[torch.Tensor] = None) -> torch.Tensor:
    """TemporalFilter::filter (Beamformer/TemporalFilter.cu:48-110): the weighted mean of equally shaped
    images, images[0] the oldest; weights default to 1 (TemporalFilterNode's)."""
    lib = load_library()
    if not images:
        raise ValueError("temporal_filter: no images")
    shape, dt = images[0].shape, images[0].dtype
    for im in images:
        if im.shape != shape or im.dtype != dt or not im.is_contiguous():
            raise ValueError("temporal_filter: images must be contiguous with one shape and dtype")
    if out is None:
        out = torch.empty(shape, dtype=out_dtype, device=images[0].device)
    ptrs = (C.c_void_p * len(images))(*[im.data_ptr() for im in images])
    w = None if weights is None else (C.c_double * len(images))(*[float(x) for x in weights])
    check("sb_temporal_filter_run",
          lib.sb_temporal_filter_run(C.cast(ptrs, C.c_void_p), len(images), None if w is None else C.cast(w, C.c_void_p),
                                     dtype_code(images[0]), _ptr(out), dtype_code(out), images[0].numel(), _stream()))
    return out


def scan_tables_2d_host(scanlines: np.ndarray, layout_x: int, num_samples: int, depth_mm: float, resolution_mm: float):
    """Host-only 2D table build of the product (no GPU needed)."""
    lib = load_library()
    sl = np.ascontiguousarray(scanlines)
    size = np.zeros(3, np.uint32)
    check("sb_scan_tables_2d_host", lib.sb_scan_tables_2d_host(sl.ctypes.data, layout_x, num_samples, depth_mm,
                                                               resolution_mm, size.ctypes.data, None, None, None, None))
    n = int(size[0]) * int(size[1]) * int(size[2])
    mask = np.zeros(n, np.uint8)
    sidx = np.zeros(n, np.uint32)
    wx = np.zeros(n, np.float32)
    wy = np.zeros(n, np.float32)
    check("sb_scan_tables_2d_host", lib.sb_scan_tables_2d_host(sl.ctypes.data, layout_x, num_samples, depth_mm,
                                                               resolution_mm, size.ctypes.data, mask.ctypes.data,
                                                               sidx.ctypes.data, wx.ctypes.data, wy.ctypes.data))
    return dict(size=tuple(int(v) for v in size), mask=mask, sample_idx=sidx, weight_x=wx, weight_y=wy)


def window_lut(window_type: int, window_parameter: float = 0.0, n: int = 64) -> np.ndarray:
    lib = load_library()
    out = np.zeros(n, np.float32)
    check("sb_window_lut", lib.sb_window_lut(int(window_type), float(window_parameter), n, out.ctypes.data))
    return out


def fir_design(length: int, ftype: int, window: int, fs=2.0, f=0.0, bw=0.0) -> np.ndarray:
    lib = load_library()
    out = np.zeros(length, np.float32)
    check("sb_fir_design", lib.sb_fir_design(int(length), int(ftype), int(window), float(fs), float(f), float(bw),
                                             out.ctypes.data))
    return out


def mv_beamform(raw_delayed: torch.Tensor, subarray_size=0, temporal_smoothing=3, subarray_scaling_power=1.5,
                compute_means=False, loading_scale=1.0, fp64_threshold=1e6, out_dtype=None, with_stats=True):
    """RxBeamformerMV::performRxBeamforming (Beamformer/RxBeamformerMV.cu:382-622).
    raw_delayed [num_rx][num_channels][num_depths] float32, int16 or complex64 -> ([num_depths][num_rx], stats).
    with_stats=False skips the statistics read-back (no host synchronisation; stats is then None)."""
    lib = load_library()
    nRx, nCh, nS = raw_delayed.shape
    if out_dtype is None:
        out_dtype = torch.complex64 if raw_delayed.dtype == torch.complex64 else torch.float32
    out = torch.empty((nS, nRx), dtype=out_dtype, device=raw_delayed.device)
    stats = sb_mv_stats() if with_stats else None
    check("sb_mv_run", lib.sb_mv_run(_ptr(raw_delayed), dtype_code(raw_delayed), _ptr(out), dtype_code(out), nRx, nCh,
                                     nS, int(subarray_size), int(temporal_smoothing), float(subarray_scaling_power),
                                     int(bool(compute_means)), float(loading_scale), float(fp64_threshold),
                                     C.byref(stats) if with_stats else None, _stream()))
    return out, stats


def mv_beamform_pcg(raw_delayed: torch.Tensor, subarray_size=0, temporal_smoothing=3, max_iterations_override=0,
                    convergence_threshold=1e-4, subarray_scaling_power=1.5, compute_means=False, loading_scale=1.0,
                    out_dtype=torch.float32) -> torch.Tensor:
    """RxBeamformerMVpcg::performRxBeamforming (Beamformer/RxBeamformerMVpcg.cu:622-800): minimum variance
    with the weights from Jacobi-PCG. raw_delayed [num_rx][num_channels][num_depths] float32 or int16 ->
    [num_depths][num_rx]."""
    lib = load_library()
    nRx, nCh, nS = raw_delayed.shape
    out = torch.empty((nS, nRx), dtype=out_dtype, device=raw_delayed.device)
    check("sb_mv_pcg_run", lib.sb_mv_pcg_run(_ptr(raw_delayed), dtype_code(raw_delayed), _ptr(out), dtype_code(out), nRx,
                                             nCh, nS, int(subarray_size), int(temporal_smoothing),
                                             int(max_iterations_override), float(convergence_threshold),
                                             float(subarray_scaling_power), int(bool(compute_means)),
                                             float(loading_scale), _stream()))
    return out


class BatchedDasIq:
    """Persistent, graph-captured batched DAS + complex IQ over frames of uneven probes.

    frames: list of (RxBeamformer, rf tensor [num_tx][num_channels][num_samples] int16 on the device).
    Output tensors (complex64 [num_depths / decimation][num_rx]) are allocated here, one per frame.
    """

    def __init__(self, frames, f_number=1.0, speed_of_sound_mm_s=1540e3, window_type=1, window_parameter=0.0,
                 mixing_frequency=5e6, cutoff_frequency=2.5e6, lowpass_length=32, decimation=4, ctas_per_sm=0,
                 depth_tile=0, frames_per_pack=0, staged=0):
        self.lib = load_library()
        self.frames = frames
        self.outputs = []
        arr = (abi.sb_batch_frame * len(frames))()
        for i, (bf, rf) in enumerate(frames):
            g = bf.geometry
            out = torch.empty((g.num_depths // max(decimation, 1), g.num_rx), dtype=torch.complex64, device=rf.device)
            self.outputs.append(out)
            arr[i].probe = bf.handle.value
            arr[i].rf = rf.data_ptr()
            arr[i].iq_out = out.data_ptr()
        prm = abi.sb_batch_params()
        prm.f_number = f_number
        prm.speed_of_sound_mm_s = speed_of_sound_mm_s
        prm.window_type = window_type
        prm.window_parameter = window_parameter
        prm.mixing_frequency_hz = mixing_frequency
        prm.cutoff_frequency_hz = cutoff_frequency
        prm.lowpass_length = lowpass_length
        prm.decimation = decimation
        prm.ctas_per_sm = ctas_per_sm
        prm.depth_tile = depth_tile
        prm.frames_per_pack = frames_per_pack
        prm.staged = staged
        self._plan = C.c_void_p()
        check("sb_batch_plan_create", self.lib.sb_batch_plan_create(arr, len(frames), C.byref(prm), C.byref(self._plan)))
        self.rf_outputs = None

    def __del__(self):
        if getattr(self, "_plan", None) and self._plan.value:
            self.lib.sb_batch_plan_destroy(self._plan)
            self._plan = C.c_void_p()

    def enable_rf_outputs(self):
        """Also write each frame's beamformed RF (FP32 [num_depths][num_rx])."""
        self.rf_outputs = [torch.empty((bf.geometry.num_depths, bf.geometry.num_rx), dtype=torch.float32,
                                       device=rf.device) for bf, rf in self.frames]
        ptrs = (C.c_void_p * len(self.rf_outputs))(*[t.data_ptr() for t in self.rf_outputs])
        check("sb_batch_set_rf_outputs", self.lib.sb_batch_set_rf_outputs(self._plan, ptrs))

    def run(self, use_graph=True):
        check("sb_batch_run", self.lib.sb_batch_run(self._plan, int(bool(use_graph)), _stream()))
        return self.outputs

    def autotune(self, cache_path=None):
        """Times the candidate shapes and keeps the fastest: (ctas_per_sm, depth_tile, frames_per_pack, staged)."""
        c, t, f, g = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        check("sb_batch_autotune", self.lib.sb_batch_autotune(self._plan, cache_path.encode() if cache_path else None,
                                                              C.byref(c), C.byref(t), C.byref(f), C.byref(g),
                                                              _stream()))
        return int(c.value), int(t.value), int(f.value), int(g.value)


def check_device_errors(reset=True):
    lib = load_library()
    check("sb_check_device_errors", lib.sb_check_device_errors(int(bool(reset))))
