"""ORACLE — test infrastructure only.

ctypes wrapper of oracle/liboracle.so (the CPU restatement of SUPRA's receive kernels) and of
oracle/_ref/libsupra_ref.so (the reference's own sources compiled for the CPU, used to pin the
restatement). Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU baseline /
reference arm; the product path never imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional, Sequence

import numpy as np

from supra_b200.abi import sb_geometry, SB_FLOAT32, SB_INT16, SB_UINT8

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libsupra_ref.so")
# the reference's own CUDA kernels built without fast-math or FMA contraction (make -C oracle refgpu)
REF_GPU_LIB = os.path.join(HERE, "_ref", "libsupra_ref_gpu.so")

_vp = C.c_void_p
_lib = None
_ref = None


def reference_root() -> Optional[str]:
    """The reference's source tree (the directory holding src/SupraLib), named by the SUPRA_REF
    environment variable; None when it is unset or holds no such tree."""
    root = os.environ.get("SUPRA_REF", "")
    return root if root and os.path.isdir(os.path.join(root, "src", "SupraLib")) else None


def build(ref: bool = True) -> None:
    """Compile the oracle (and the reference checker when SUPRA_REF names the reference sources)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    root = reference_root()
    if ref and root:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref", f"REF={root}"])
        subprocess.check_call(["make", "-s", "-C", HERE, "refgpu", f"REF={root}"])


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build(ref=False)
        _lib = C.CDLL(LIB)
        _lib.orc_window_get.restype = C.c_float
        _lib.orc_window_get.argtypes = [C.c_int, C.c_float, C.c_uint32, C.c_float]
    return _lib


def ref_lib() -> Optional[C.CDLL]:
    global _ref
    if _ref is None:
        if not os.path.exists(REF_LIB):
            return None
        _ref = C.CDLL(REF_LIB)
        _ref.ref_window_get.restype = C.c_float
        _ref.ref_window_get.argtypes = [C.c_int, C.c_float, C.c_uint32, C.c_float]
    return _ref


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def nthreads() -> int:
    return os.cpu_count() or 1


# ------------------------------------------------------------------------------ design helpers
def window_lut(window_type: int, param: float = 0.0, n: int = 64, ref: bool = False) -> np.ndarray:
    out = np.zeros(n, np.float32)
    L = ref_lib() if ref else lib()
    fn = L.ref_window_lut if ref else L.orc_window_lut
    fn(C.c_int(window_type), C.c_float(param), C.c_uint32(n), _vp(_p(out)))
    return out


def window_get(window_type: int, param: float, n: int, rel: float, ref: bool = False) -> float:
    if ref:
        return ref_lib().ref_window_get(window_type, param, n, rel)
    return lib().orc_window_get(window_type, param, n, rel)


def fir(length: int, ftype: int, window: int, fs: float = 2.0, f: float = 0.0, bw: float = 0.0,
        ref: bool = False) -> np.ndarray:
    out = np.zeros(length, np.float32)
    L = ref_lib() if ref else lib()
    fn = L.ref_fir if ref else L.orc_fir
    fn(C.c_uint32(length), C.c_int(ftype), C.c_int(window), C.c_double(fs), C.c_double(f), C.c_double(bw),
       _vp(_p(out)))
    return out


# ------------------------------------------------------------------------------ kernels
def das(geom, rf: np.ndarray, f_number=1.0, c_mm_s=None, window=1, window_param=0.0, interp_tx=False,
        additional_offset=0, precision=32, apod: Optional[np.ndarray] = None, threads=None,
        ref: bool = False) -> np.ndarray:
    """DAS of one frame; rf [num_tx][num_channels][num_samples] (any dtype, converted to float32)."""
    g = geom.ctypes()
    rf32 = np.ascontiguousarray(rf, dtype=np.float32)
    c = geom.speed_of_sound_mm_s if c_mm_s is None else c_mm_s
    n = geom.num_depths * geom.num_rx
    if ref:
        out = np.full(n, np.nan, np.float32)
        ref_lib().ref_das(C.byref(g), _vp(_p(rf32)), _vp(_p(out)), C.c_double(f_number), C.c_double(c),
                          C.c_int(window), C.c_float(window_param), C.c_int(int(interp_tx)),
                          C.c_int32(additional_offset))
        return out.reshape(geom.num_depths, geom.num_rx)
    if precision == 64:
        out64 = np.full(n, np.nan, np.float64)
        outp32, outp64 = None, _vp(_p(out64))
    else:
        out32 = np.full(n, np.nan, np.float32)
        outp32, outp64 = _vp(_p(out32)), None
    ap = None if apod is None else np.ascontiguousarray(apod, dtype=np.float32)
    st = lib().orc_das(C.byref(g), _vp(_p(rf32)), outp32, outp64, C.c_double(f_number), C.c_double(c),
                       C.c_int(window), C.c_float(window_param), C.c_int(int(interp_tx)), C.c_int32(additional_offset),
                       None if ap is None else _vp(_p(ap)), C.c_int(precision), C.c_int(threads or nthreads()))
    assert st == 0
    out = out64 if precision == 64 else out32
    return out.reshape(geom.num_depths, geom.num_rx)


BEAMFORMERS = {"DelayAndSum": 0, "DelayAndStdDev": 1, "CoherenceFactorDelayAndSum": 2, "TestSignal": 3}


def das_bf(geom, rf: np.ndarray, beamformer, f_number=1.0, c_mm_s=None, window=1, window_param=0.0, interp_tx=False,
           additional_offset=0, threads=None, ref: bool = False) -> np.ndarray:
    """One frame through a sample beamformer (name or RxBeamformerCuda::RxSampleBeamformer index), float
    semantics; ref=True runs the reference's own reducers (oracle/_ref)."""
    bf = BEAMFORMERS[beamformer] if isinstance(beamformer, str) else int(beamformer)
    g = geom.ctypes()
    rf32 = np.ascontiguousarray(rf, dtype=np.float32)
    c = geom.speed_of_sound_mm_s if c_mm_s is None else c_mm_s
    out = np.full(geom.num_depths * geom.num_rx, np.nan, np.float32)
    if ref:
        st = ref_lib().ref_das_bf(C.byref(g), _vp(_p(rf32)), _vp(_p(out)), C.c_double(f_number), C.c_double(c),
                                  C.c_int(window), C.c_float(window_param), C.c_int(int(interp_tx)),
                                  C.c_int32(additional_offset), C.c_int(bf))
    else:
        st = lib().orc_das_bf(C.byref(g), _vp(_p(rf32)), _vp(_p(out)), C.c_double(f_number), C.c_double(c),
                              C.c_int(window), C.c_float(window_param), C.c_int(int(interp_tx)),
                              C.c_int32(additional_offset), C.c_int(bf), C.c_int(threads or nthreads()))
    assert st == 0
    return out.reshape(geom.num_depths, geom.num_rx)


def temporal_filter(images, weights=None, out_dtype=np.float32) -> np.ndarray:
    """TemporalFilter (float work type) over equally shaped images, oldest first."""
    ims = [np.ascontiguousarray(im, dtype=np.float32).ravel() for im in images]
    arr = (C.c_void_p * len(ims))(*[im.ctypes.data for im in ims])
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    out = np.empty(ims[0].size, dtype=out_dtype)
    code = {np.dtype(np.float32): 2, np.dtype(np.int16): 1}[np.dtype(out_dtype)]  # SB_FLOAT32, SB_INT16
    st = lib().orc_temporal_filter(C.cast(arr, C.c_void_p), C.c_uint32(len(ims)), None if w is None else _vp(_p(w)),
                                   C.c_uint64(ims[0].size), _vp(_p(out)), C.c_int(code))
    assert st == 0
    return out.reshape(np.shape(images[0]))


def ref_mock_write(filename: str, geom, ascii_format: bool = False) -> None:
    """The reference's mock metadata for a geometry: writeMetaDataForMock (JSON) or, for the ASCII
    layout, the reference's scanline stream operator (oracle/_ref)."""
    g = geom.ctypes()
    fn = ref_lib().ref_mock_write_ascii if ascii_format else ref_lib().ref_mock_write_json
    assert fn(filename.encode(), C.byref(g), C.c_double(geom.depth_mm), C.c_double(geom.speed_of_sound_mm_s)) == 0


def ref_mock_read(filename: str, max_lines=4096, max_depths=65536, max_elems=65536) -> dict:
    """readMetaDataForMock of the reference (oracle/_ref): sizes, values and arrays."""
    from supra_b200.abi import SCANLINE_DTYPE
    sizes = np.zeros(9, np.uint64)
    vals = np.zeros(3, np.float64)
    lines = np.zeros(max_lines, SCANLINE_DTYPE)
    depths = np.zeros(max_depths, np.float32)
    xs = np.zeros(max_elems, np.float32)
    ys = np.zeros(max_elems, np.float32)
    st = ref_lib().ref_mock_read(filename.encode(), _vp(_p(sizes)), _vp(_p(vals)), _vp(_p(lines)), _vp(_p(depths)),
                                 _vp(_p(xs)), _vp(_p(ys)), C.c_uint64(max_lines), C.c_uint64(max_depths),
                                 C.c_uint64(max_elems))
    assert st == 0, "reference reader failed"
    nE, nD, nL = int(sizes[0]), int(sizes[8]), int(sizes[6] * sizes[7])
    return {"sizes": sizes, "vals": vals, "lines": lines[:nL], "depths": depths[:nD], "xs": xs[:nE], "ys": ys[:nE]}


def analytic_env(img: np.ndarray) -> np.ndarray:
    """HilbertEnvelope (BF/HilbertEnvelope.cu:27-207) in FP64: per scanline (columns of [N][nRx]) the
    FFT, the spectrum mask of maskSpectrum (DC x1; bins 1..N/2-1 x2 and N/2 x1 for even N, bins
    1..(N-1)/2 x2 for odd N; the rest 0), the inverse FFT (numpy's is normalised: the reference's
    unnormalised inverse divided by N) and the magnitude."""
    x = np.asarray(img, np.float64)
    N = x.shape[0]
    m = np.zeros(N)
    m[0] = 1.0
    if N % 2 == 0:
        m[1:N // 2] = 2.0
        if N > 1:
            m[N // 2] = 1.0
    else:
        m[1:(N + 1) // 2] = 2.0
    z = np.fft.ifft(np.fft.fft(x, axis=0) * m[:, None], axis=0)
    return np.abs(z)


# ------------------------------------------------------------------ reference GPU kernels
_refg = None


def refgpu_lib() -> Optional[C.CDLL]:
    """The reference's CUDA kernels (oracle/_ref/libsupra_ref_gpu.so), None when not built."""
    global _refg
    if _refg is None and os.path.exists(REF_GPU_LIB):
        _refg = C.CDLL(REF_GPU_LIB)
    return _refg


def refg_das(geom, rf: np.ndarray, beamformer=0, f_number=1.0, c_mm_s=None, window=1, window_param=0.0,
             interp_tx=False, additional_offset=0) -> np.ndarray:
    """RxBeamformerCuda::performRxBeamforming of the reference on the GPU: [num_depths][num_rx]."""
    g = geom.ctypes()
    x = np.ascontiguousarray(rf, np.int16)
    out = np.zeros(geom.num_depths * geom.num_rx, np.float32)
    c = geom.speed_of_sound_mm_s if c_mm_s is None else c_mm_s
    assert refgpu_lib().refg_das(C.byref(g), _vp(_p(x)), _vp(_p(out)), C.c_double(f_number), C.c_double(c),
                                 C.c_int(window), C.c_float(window_param), C.c_int(int(interp_tx)),
                                 C.c_int32(additional_offset), C.c_int(beamformer), C.c_double(geom.depth_mm)) == 0
    return out.reshape(geom.num_depths, geom.num_rx)


def refg_rawdelay(geom, rf: np.ndarray, f_number=1.0, window=1, window_param=0.0) -> np.ndarray:
    g = geom.ctypes()
    x = np.ascontiguousarray(rf, np.int16)
    out = np.zeros(geom.num_rx * geom.num_channels * geom.num_depths, np.float32)
    assert refgpu_lib().refg_rawdelay(C.byref(g), _vp(_p(x)), _vp(_p(out)), C.c_double(f_number),
                                      C.c_double(geom.speed_of_sound_mm_s), C.c_int(window), C.c_float(window_param),
                                      C.c_double(geom.depth_mm)) == 0
    return out.reshape(geom.num_rx, geom.num_channels, geom.num_depths)


def refg_hilbert(img: np.ndarray, filter_length: int) -> np.ndarray:
    x = np.ascontiguousarray(img, np.float32)
    out = np.zeros_like(x)
    assert refgpu_lib().refg_hilbert(_vp(_p(x)), _vp(_p(out)), C.c_uint32(x.shape[1]), C.c_uint32(x.shape[0]),
                                     C.c_uint32(filter_length)) == 0
    return out


def refg_logcompress(img: np.ndarray, dynamic_range: float, gain: float, in_max: float, uint8=False) -> np.ndarray:
    x = np.ascontiguousarray(img, np.float32)
    out = np.zeros(x.shape, np.uint8 if uint8 else np.float32)
    assert refgpu_lib().refg_logcompress(_vp(_p(x)), _vp(_p(out)), C.c_uint32(x.shape[1]), C.c_uint32(x.shape[0]),
                                         C.c_double(dynamic_range), C.c_double(gain), C.c_double(in_max),
                                         C.c_int(int(uint8))) == 0
    return out


def refg_iq(img: np.ndarray, fs: float, reference_frequency: float, cutoff: float, lowpass_length: int,
            bandpass_length: int, decimation: int, frequencies, bandwidths, weights) -> np.ndarray:
    x = np.ascontiguousarray(img, np.float32)
    nS, nRx = x.shape
    f, b, w = (np.ascontiguousarray(v, np.float64) for v in (frequencies, bandwidths, weights))
    out = np.zeros((nS // decimation if decimation > 1 else nS) * nRx, np.float32)  # decimatedSignalLength
    assert refgpu_lib().refg_iq(_vp(_p(x)), _vp(_p(out)), C.c_uint32(nRx), C.c_uint32(nS), C.c_double(fs),
                                C.c_double(reference_frequency), C.c_double(cutoff), C.c_uint32(lowpass_length),
                                C.c_uint32(bandpass_length), C.c_uint32(decimation), C.c_uint32(len(f)), _vp(_p(f)),
                                _vp(_p(b)), _vp(_p(w))) == 0
    return out.reshape(-1, nRx)


class RefScan:
    """ScanConverter of the reference on the GPU: tables of updateInternals and convert()."""

    def __init__(self, scanlines: np.ndarray, layout, num_samples: int, depth_mm: float, resolution_mm: float,
                 lib=None):
        self.lib = lib or refgpu_lib()
        self.lib.refg_scan_create.restype = _vp
        sl = np.ascontiguousarray(scanlines)
        self.h = _vp(self.lib.refg_scan_create(_vp(_p(sl)), C.c_uint32(layout[0]), C.c_uint32(layout[1]),
                                               C.c_uint32(num_samples), C.c_double(depth_mm),
                                               C.c_double(resolution_mm)))
        size = np.zeros(3, np.uint32)
        self.lib.refg_scan_size(self.h, _vp(_p(size)))
        self.size = tuple(int(v) for v in size)
        self.numel = int(np.prod(self.size))
        self.is2D = layout[0] == 1 or layout[1] == 1
        self.num_rx = int(layout[0]) * int(layout[1])
        self.num_samples = num_samples

    def tables(self) -> dict:
        n = self.numel
        t = {"mask": np.zeros(n, np.uint8), "sample_idx": np.zeros(n, np.uint32), "weight_x": np.zeros(n, np.float32),
             "weight_y": np.zeros(n, np.float32), "weight_z": np.zeros(n, np.float32)}
        assert self.lib.refg_scan_tables(self.h, *(_vp(_p(t[k])) for k in ("mask", "sample_idx", "weight_x",
                                                                            "weight_y", "weight_z"))) == 0
        return t

    def convert(self, img: np.ndarray, uint8=True) -> np.ndarray:
        x = np.ascontiguousarray(img, np.float32)
        assert x.size == self.num_rx * self.num_samples
        out = np.zeros(self.numel, np.uint8 if uint8 else np.float32)
        assert self.lib.refg_scan_convert(self.h, _vp(_p(x)), _vp(_p(out)), C.c_int(int(uint8))) == 0
        return out

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.refg_scan_destroy(self.h)
            self.h = None


def refg_mv(raw: np.ndarray, subarray_size: int, temporal_smoothing: int, scaling_power=1.5) -> np.ndarray:
    """RxBeamformerMV::performRxBeamforming of the reference on the GPU (cuBLAS batched LU), real
    raw-delayed data [scanlines][channels][samples], samples <= 2000: image [samples][scanlines]."""
    x = np.ascontiguousarray(raw, np.float32)
    nRx, nCh, nS = x.shape
    assert nS <= 2000, "the reference's MV handles at most 2000 samples"
    out = np.zeros(nS * nRx, np.float32)
    assert refgpu_lib().refg_mv(_vp(_p(x)), _vp(_p(out)), C.c_uint32(nRx), C.c_uint32(nCh), C.c_uint32(nS),
                                C.c_uint32(subarray_size), C.c_uint32(temporal_smoothing),
                                C.c_double(scaling_power)) == 0
    return out.reshape(nS, nRx)


def refg_mvpcg(raw: np.ndarray, subarray_size: int, temporal_smoothing: int, max_iterations_override=0,
               convergence_threshold=1e-4, scaling_power=1.5) -> np.ndarray:
    """RxBeamformerMVpcg::performRxBeamforming of the reference on the GPU: image [samples][scanlines]."""
    x = np.ascontiguousarray(raw, np.float32)
    nRx, nCh, nS = x.shape
    out = np.zeros(nS * nRx, np.float32)
    assert refgpu_lib().refg_mvpcg(_vp(_p(x)), _vp(_p(out)), C.c_uint32(nRx), C.c_uint32(nCh), C.c_uint32(nS),
                                   C.c_uint32(subarray_size), C.c_uint32(temporal_smoothing),
                                   C.c_uint32(max_iterations_override), C.c_double(convergence_threshold),
                                   C.c_double(scaling_power)) == 0
    return out.reshape(nS, nRx)


def refg_temporal(images, weights) -> np.ndarray:
    """TemporalFilter::filter of the reference on the GPU over float images (oldest first)."""
    ims = [np.ascontiguousarray(a, np.float32) for a in images]
    h, w = ims[0].shape
    ptrs = (C.c_void_p * len(ims))(*[_p(a) for a in ims])
    wt = np.ascontiguousarray(weights, np.float64)
    out = np.zeros((h, w), np.float32)
    assert refgpu_lib().refg_temporal(ptrs, C.c_uint32(len(ims)), _vp(_p(wt)), C.c_uint32(w), C.c_uint32(h),
                                      _vp(_p(out))) == 0
    return out


def refg_fft_env(img: np.ndarray) -> np.ndarray:
    """HilbertEnvelope::computeHilbertEnvelope of the reference on the GPU (cuFFT)."""
    x = np.ascontiguousarray(img, np.float32)
    out = np.zeros_like(x)
    assert refgpu_lib().refg_fft_env(_vp(_p(x)), _vp(_p(out)), C.c_uint32(x.shape[1]), C.c_uint32(x.shape[0])) == 0
    return out


# the same reference sources built with the reference's production flags (--use_fast_math): the
# per-kernel timing baseline on the GPU
REF_GPU_FAST_LIB = os.path.join(HERE, "_ref", "libsupra_ref_gpu_fast.so")
_refgf = None


def refgpu_fast_lib() -> Optional[C.CDLL]:
    global _refgf
    if _refgf is None and os.path.exists(REF_GPU_FAST_LIB):
        _refgf = C.CDLL(REF_GPU_FAST_LIB)
        for name in ("refg_time_das", "refg_time_rawdelay", "refg_time_hilbert", "refg_time_logcompress", "refg_time_iq",
                     "refg_time_scan", "refg_time_mv", "refg_time_mvpcg", "refg_time_fft_env", "refg_time_temporal"):
            getattr(_refgf, name).restype = C.c_float
    return _refgf


def das_adjoint64(geom, rf: np.ndarray, apod, gout: np.ndarray, c_mm_s=None, f_number=1.0, window=1, window_param=0.0):
    """FP64 reference gradient of the apodised 2D DAS: (grad_rf, grad_apod, grad_c)."""
    g = geom.ctypes()
    rf32 = np.ascontiguousarray(rf, dtype=np.float32)
    c = geom.speed_of_sound_mm_s if c_mm_s is None else c_mm_s
    go = np.ascontiguousarray(gout, dtype=np.float64)
    grf = np.zeros(rf32.size, np.float64)
    gap = np.zeros(geom.num_elements, np.float64)
    gc = np.zeros(1, np.float64)
    ap = None if apod is None else np.ascontiguousarray(apod, dtype=np.float32)
    st = lib().orc_das_adjoint64(C.byref(g), _vp(_p(rf32)), None if ap is None else _vp(_p(ap)), _vp(_p(go)),
                                 _vp(_p(grf)), _vp(_p(gap)), _vp(_p(gc)), C.c_double(f_number), C.c_double(c),
                                 C.c_int(window), C.c_float(window_param))
    assert st == 0
    return grf.reshape(rf32.shape), gap, float(gc[0])


def rawdelay(geom, rf: np.ndarray, f_number=1.0, c_mm_s=None, window=1, window_param=0.0, threads=None):
    g = geom.ctypes()
    rf32 = np.ascontiguousarray(rf, dtype=np.float32)
    c = geom.speed_of_sound_mm_s if c_mm_s is None else c_mm_s
    out = np.zeros(geom.num_rx * geom.num_channels * geom.num_depths, np.float32)
    st = lib().orc_rawdelay(C.byref(g), _vp(_p(rf32)), _vp(_p(out)), C.c_double(f_number), C.c_double(c),
                            C.c_int(window), C.c_float(window_param), C.c_int(threads or nthreads()))
    assert st == 0
    return out.reshape(geom.num_rx, geom.num_channels, geom.num_depths)


def hilbert_env(x: np.ndarray, filter_length: int, threads=None) -> np.ndarray:
    """x [num_samples][num_scanlines] float32."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    lib().orc_hilbert_env(_vp(_p(x)), _vp(_p(out)), C.c_uint32(x.shape[1]), C.c_uint32(x.shape[0]),
                          C.c_uint32(filter_length), C.c_int(threads or nthreads()))
    return out


def logcompress(x: np.ndarray, dynamic_range: float, gain: float, in_max: float, out_dtype=np.uint8) -> np.ndarray:
    x = np.ascontiguousarray(x)
    in_code = SB_INT16 if x.dtype == np.int16 else SB_UINT8 if x.dtype == np.uint8 else SB_FLOAT32
    if in_code == SB_FLOAT32:
        x = x.astype(np.float32, copy=False)
    out = np.zeros(x.shape, out_dtype)
    oc = SB_UINT8 if out_dtype == np.uint8 else SB_FLOAT32
    lib().orc_logcompress(_vp(_p(x)), C.c_int(in_code), _vp(_p(out)), C.c_int(oc), C.c_size_t(x.size),
                          C.c_double(dynamic_range), C.c_double(gain), C.c_double(in_max))
    return out


def iq_magnitude(x: np.ndarray, decimation: int, fs: float, cutoff: float, lp_len: int, bp_len: int,
                 ref_freqs: Sequence[float], bandwidths: Sequence[float], weights: Sequence[float], threads=None):
    x = np.ascontiguousarray(x, np.float32)
    nS, nL = x.shape
    n_out = nS // decimation if decimation > 1 else nS
    out = np.zeros((n_out, nL), np.float32)
    rf_ = np.ascontiguousarray(ref_freqs, np.float64)
    bw_ = np.ascontiguousarray(bandwidths, np.float64)
    w_ = np.ascontiguousarray(weights, np.float64)
    st = lib().orc_iq_magnitude(_vp(_p(x)), _vp(_p(out)), C.c_uint32(nL), C.c_uint32(nS), C.c_uint32(decimation),
                                C.c_double(fs), C.c_double(cutoff), C.c_uint32(lp_len), C.c_uint32(bp_len),
                                C.c_uint32(len(rf_)), _vp(_p(rf_)), _vp(_p(bw_)), _vp(_p(w_)),
                                C.c_int(threads or nthreads()))
    assert st == 0
    return out


def iq_complex(x: np.ndarray, fs: float, fmix: float, cutoff: float, lp_len: int, decimation: int, threads=None):
    x = np.ascontiguousarray(x, np.float32)
    nS, nL = x.shape
    out = np.zeros((nS // decimation, nL, 2), np.float64)
    lib().orc_iq_complex(_vp(_p(x)), _vp(_p(out)), C.c_uint32(nL), C.c_uint32(nS), C.c_double(fs), C.c_double(fmix),
                         C.c_double(cutoff), C.c_uint32(lp_len), C.c_uint32(decimation), C.c_int(threads or nthreads()))
    return out[..., 0] + 1j * out[..., 1]


def scan_tables(scanlines: np.ndarray, lx: int, ly: int, num_samples: int, depth: float, resolution: float):
    size = np.zeros(3, np.uint32)
    bb = np.zeros(3, np.float64)
    sl = np.ascontiguousarray(scanlines)
    L = lib()
    L.orc_scan_tables(_vp(_p(sl)), C.c_uint32(lx), C.c_uint32(ly), C.c_uint32(num_samples), C.c_double(depth),
                      C.c_double(resolution), _vp(_p(size)), _vp(_p(bb)), None, None, None, None, None)
    n = int(size[0]) * int(size[1]) * int(size[2])
    mask = np.zeros(n, np.uint8)
    sidx = np.zeros(n, np.uint32)
    wx = np.zeros(n, np.float32)
    wy = np.zeros(n, np.float32)
    wz = np.zeros(n, np.float32)
    L.orc_scan_tables(_vp(_p(sl)), C.c_uint32(lx), C.c_uint32(ly), C.c_uint32(num_samples), C.c_double(depth),
                      C.c_double(resolution), _vp(_p(size)), _vp(_p(bb)), _vp(_p(mask)), _vp(_p(sidx)),
                      _vp(_p(wx)), _vp(_p(wy)), _vp(_p(wz)))
    return dict(size=tuple(int(v) for v in size), bb_min=bb, mask=mask, sample_idx=sidx, weight_x=wx,
                weight_y=wy, weight_z=wz)


def scan_apply(x: np.ndarray, lx: int, ly: int, tables: dict, out_dtype=np.uint8) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    size = np.array(tables["size"], np.uint32)
    n = int(np.prod(size))
    out = np.zeros(n, out_dtype)
    oc = SB_UINT8 if out_dtype == np.uint8 else SB_INT16 if out_dtype == np.int16 else SB_FLOAT32
    lib().orc_scan_apply(_vp(_p(x)), C.c_uint32(lx), C.c_uint32(ly), C.c_uint32(x.shape[0]), _vp(_p(size)),
                         _vp(_p(tables["mask"])), _vp(_p(tables["sample_idx"])), _vp(_p(tables["weight_x"])),
                         _vp(_p(tables["weight_y"])), _vp(_p(tables["weight_z"])), _vp(_p(out)), C.c_int(oc))
    return out.reshape(size[2], size[1], size[0])


def mv_pcg(raw: np.ndarray, L: int, T: int, max_iterations=0, threshold=1e-4, scaling_power=1.5, loading_scale=1.0,
           precision=32, threads=None) -> np.ndarray:
    """RxBeamformerMVpcg on real raw [nRx][nCh][nS] float32 (PCG in float for precision 32, double for
    64); returns [nS][nRx]."""
    nRx, nCh, nS = raw.shape
    r = np.ascontiguousarray(raw, np.float32)
    dt = np.float64 if precision == 64 else np.float32
    out = np.zeros(nS * nRx, dt)
    o32, o64 = (None, _vp(_p(out))) if precision == 64 else (_vp(_p(out)), None)
    st = lib().orc_mv_pcg(_vp(_p(r)), o32, o64, C.c_uint32(nRx), C.c_uint32(nCh), C.c_uint32(nS), C.c_uint32(L),
                          C.c_uint32(T), C.c_double(scaling_power), C.c_float(loading_scale), C.c_uint32(max_iterations),
                          C.c_double(threshold), C.c_int(precision), C.c_int(threads or nthreads()))
    assert st == 0
    return out.reshape(nS, nRx)


def mv(raw: np.ndarray, L: int, T: int, scaling_power=1.5, loading_scale=1.0, precision=32, block=2000,
       threads=None) -> np.ndarray:
    """raw [nRx][nCh][nS] float32 (real) or complex64; returns [nS][nRx]."""
    iscomplex = np.iscomplexobj(raw)
    nRx, nCh, nS = raw.shape
    if iscomplex:
        r = np.ascontiguousarray(raw.astype(np.complex64)).view(np.float32)
    else:
        r = np.ascontiguousarray(raw, np.float32)
    if precision == 64:
        out = np.zeros(nS * nRx * (2 if iscomplex else 1), np.float64)
        st = lib().orc_mv(_vp(_p(r)), C.c_int(int(iscomplex)), None, _vp(_p(out)), C.c_uint32(nRx), C.c_uint32(nCh),
                          C.c_uint32(nS), C.c_uint32(L), C.c_uint32(T), C.c_double(scaling_power),
                          C.c_float(loading_scale), C.c_int(64), C.c_uint32(block), C.c_int(threads or nthreads()))
    else:
        out = np.zeros(nS * nRx * (2 if iscomplex else 1), np.float32)
        st = lib().orc_mv(_vp(_p(r)), C.c_int(int(iscomplex)), _vp(_p(out)), None, C.c_uint32(nRx), C.c_uint32(nCh),
                          C.c_uint32(nS), C.c_uint32(L), C.c_uint32(T), C.c_double(scaling_power),
                          C.c_float(loading_scale), C.c_int(32), C.c_uint32(block), C.c_int(threads or nthreads()))
    assert st == 0
    if iscomplex:
        out = out.reshape(nS, nRx, 2)
        return out[..., 0] + 1j * out[..., 1]
    return out.reshape(nS, nRx)
