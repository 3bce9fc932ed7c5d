"""Minimum-variance beamformer (sb_mv_run) against the oracle's restatement of
RxBeamformerMV::performRxBeamforming (Beamformer/RxBeamformerMV.cu:382-622).

The reference solves R a = 1 by a batched FP32 LU (cuBLAS); the kernel uses an FP32 Cholesky. Both
are backward stable on the loaded (symmetric positive definite) systems, so outputs are compared
within a tolerance relative to the frame peak, stated per test:
  * reference mode (real data, loading trace/sz): against the oracle with FP32 covariance and an
    FP64 solve, 1e-4 of the peak;
  * FP64 re-solve forced for every system: against the all-FP64 oracle, 1e-6 of the peak;
  * complex data with loading trace/(100 sz): against the all-FP64 oracle, 1e-3 of the peak (the
    FP32 error grows with the condition number, up to 100 sz + 1 here).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c0_raw():
    from supra_b200 import synth
    from supra_b200.api import RxBeamformer
    g, rf = synth.c0_frame(3, device="cuda")
    raw = RxBeamformer(g).raw_delay(rf, 1.0, window_type=1)
    torch.cuda.synchronize()
    raw = raw[::11].contiguous()  # 12 scanlines x 64 channels x 2048 samples (crosses the 2000 block)
    # RawDelay writes +-FLT_MAX where its weight sum is 0 at depth 0 (clampCast of NaN); MV on such
    # samples overflows in the reference as well, so they are zeroed.
    raw[~(raw.abs() < 1e30)] = 0.0
    return raw


def _peak_err(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _mv(raw, **kw):
    from supra_b200.api import mv_beamform
    out, stats = mv_beamform(raw, **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy(), stats


@pytest.mark.parametrize("L,T", [(32, 3), (16, 0), (48, 7), (0, 3)])
def test_mv_reference_mode_real(oracle, c0_raw, L, T):
    out, stats = _mv(c0_raw, subarray_size=L, temporal_smoothing=T, fp64_threshold=0.0)
    ref = oracle.mv(c0_raw.cpu().numpy(), L or c0_raw.shape[1] // 2, T, precision=32)
    assert out.shape == ref.shape
    assert stats.systems == c0_raw.shape[0] * c0_raw.shape[2]
    assert stats.fp64_systems == 0
    err = _peak_err(out, ref)
    assert err <= 1e-4, err


def test_mv_fp64_resolve_matches_fp64_oracle(oracle, c0_raw):
    raw = c0_raw[:4].contiguous()
    # every estimate is >= 1, so a threshold of 0.5 routes every solved system (samples whose window
    # holds no signal have trace 0 and are written as 0 without a solve)
    out, stats = _mv(raw, subarray_size=32, temporal_smoothing=3, fp64_threshold=0.5)
    assert stats.fp64_systems >= 0.9 * raw.shape[0] * raw.shape[2]
    ref = oracle.mv(raw.cpu().numpy(), 32, 3, precision=64)
    assert _peak_err(out, ref) <= 1e-6


def test_mv_threshold_routes_only_ill_conditioned(oracle, c0_raw):
    raw = c0_raw[:4].contiguous()
    _, s_all = _mv(raw, subarray_size=32, temporal_smoothing=3, fp64_threshold=0.0)
    thr = max(1.0, 0.5 * s_all.max_condition_estimate)
    out, stats = _mv(raw, subarray_size=32, temporal_smoothing=3, fp64_threshold=thr)
    assert 0 < stats.fp64_systems < stats.systems
    ref = oracle.mv(raw.cpu().numpy(), 32, 3, precision=64)
    assert _peak_err(out, ref) <= 1e-4


def test_mv_complex_c3_style(oracle):
    """Complex channel data on a 128-channel aperture, L = 32, +-5 samples, loading trace/(100 sz)."""
    from supra_b200 import synth
    from supra_b200.api import RxBeamformer
    from supra_b200.geometry import linear_probe_geometry
    g = linear_probe_geometry(128, 0.3, 128, 512, 40e6, aperture=128, focus_mm=20.0)
    pts, amps = synth.random_scatterers(20, (-19.05, 19.05), (2.0, 9.0), seed=5)
    rf = synth.channel_data(g, pts, amps, synth.PulseSpec(7e6, 0.6), -40.0, 30000.0, seed=5, device="cuda")
    raw = RxBeamformer(g).raw_delay(rf, 1.0, window_type=1)[::16].contiguous()  # 8 lines
    raw[~(raw.abs() < 1e30)] = 0.0
    n = torch.arange(raw.shape[2], device="cuda", dtype=torch.float32)
    mix = torch.exp(-2j * np.pi * 5e6 / 40e6 * n.to(torch.complex64))
    x = (raw.to(torch.complex64) * mix).contiguous()
    out, stats = _mv(x, subarray_size=32, temporal_smoothing=5, loading_scale=0.01, fp64_threshold=0.0)
    ref = oracle.mv(x.cpu().numpy(), 32, 5, loading_scale=0.01, precision=64)
    err = _peak_err(out, ref)
    assert err <= 1e-3, err
    assert stats.max_condition_estimate < 1e6


@pytest.mark.parametrize("in_dtype,out_dtype", [(torch.int16, torch.float32), (torch.float32, torch.int16),
                                                (torch.int16, torch.int16)])
def test_mv_dtypes(oracle, c0_raw, in_dtype, out_dtype):
    raw = c0_raw[:3]
    if in_dtype == torch.int16:
        raw = (raw / raw.abs().max() * 20000).round().to(torch.int16)
    raw = raw.contiguous()
    out, _ = _mv(raw, subarray_size=32, temporal_smoothing=2, fp64_threshold=0.0, out_dtype=out_dtype)
    ref = oracle.mv(raw.float().cpu().numpy(), 32, 2, precision=32)
    if out_dtype == torch.int16:
        exp = np.clip(ref, -32767, 32767).astype(np.int16).astype(np.float32)
        assert np.max(np.abs(out.astype(np.float32) - exp)) <= 1e-4 * np.max(np.abs(ref)) + 1
    else:
        assert _peak_err(out, ref) <= 1e-4


def test_mv_zero_and_narrow_aperture(oracle):
    rng = np.random.Generator(np.random.PCG64(1))
    raw = rng.standard_normal((3, 40, 300)).astype(np.float32)
    raw[0] = 0.0                      # no signal at all
    raw[1, :, :100] = 0.0
    raw[1, 10:14, :100] = 1.0 + rng.random((4, 100))  # 4-channel aperture (sz < L)
    raw[2, :25, 150:] = 0.0           # aperture narrower than L on the deep half
    x = torch.from_numpy(raw).cuda()
    out, _ = _mv(x, subarray_size=16, temporal_smoothing=2, fp64_threshold=0.0)
    ref = oracle.mv(raw, 16, 2, precision=32)
    assert np.all(out[:, 0] == 0.0)
    assert _peak_err(out, ref) <= 1e-4


def test_mv_rejects_unsupported():
    from supra_b200.abi import SupraError
    from supra_b200.api import mv_beamform
    x = torch.zeros((2, 130, 64), device="cuda", dtype=torch.float32)
    with pytest.raises(SupraError):
        mv_beamform(x, subarray_size=65)
    with pytest.raises(SupraError):
        mv_beamform(x, subarray_size=8, compute_means=True)
    xc = torch.zeros((2, 80, 64), device="cuda", dtype=torch.complex64)
    with pytest.raises(SupraError):
        mv_beamform(xc, subarray_size=40)


def test_mv_c3_shape_error_vs_fp64(oracle):
    """The c3 workload (complex raw-delayed [128 lines][128 channels][2048 depths] with two interferers,
    L = 32, +-5, loading trace/(100 L), FP64 re-solve above a condition estimate of 1e6) against the
    all-FP64 restatement on every 16th scanline; the measured error and the number of FP64 re-solves
    are printed."""
    from supra_b200 import workloads as W
    g3, x3 = W.c3_raw_delayed()
    out, stats = _mv(x3, subarray_size=W.C3_L, temporal_smoothing=W.C3_T, loading_scale=W.C3_LOADING,
                     fp64_threshold=1e6)
    sub = x3[::16].contiguous()
    ref = oracle.mv(sub.cpu().numpy(), W.C3_L, W.C3_T, loading_scale=W.C3_LOADING, precision=64)
    err = _peak_err(out[:, ::16], ref)
    print(f"c3 MV vs FP64 (16 of 128 scanlines, 2048 depths): {err:.3g} of the peak; FP64 re-solves "
          f"{stats.fp64_systems} of {stats.systems}; largest condition estimate {stats.max_condition_estimate:.4g}")
    assert err <= 1e-3
