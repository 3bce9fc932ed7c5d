"""DAS and raw delay on the GPU against the oracle (CPU restatement pinned to the reference)."""
import numpy as np
import pytest
import torch

from conftest import random_rf, small_linear, small_matrix

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative to the frame peak


def compare(got, ref, tol=TOL):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    big = np.finfo(np.float32).max
    same_clamp = (got == ref) & (np.abs(ref) >= big)
    got = np.where(same_clamp, 0.0, got)
    ref = np.where(same_clamp, 0.0, ref)
    both_nan = np.isnan(got) & np.isnan(ref)
    assert not (np.isnan(got) ^ np.isnan(ref)).any(), "NaN pattern differs"
    peak = np.nanmax(np.abs(ref))
    err = np.nanmax(np.abs(np.where(both_nan, 0, got - ref)))
    assert err <= tol * peak, f"max error {err} > {tol} x peak {peak}"
    exact = np.mean((got == ref) | both_nan)
    return err / peak, exact


@pytest.mark.parametrize("case", range(5))
def test_das_golden_cases(oracle, case):
    from golden.cases import DAS_CASES
    from supra_b200.api import RxBeamformer
    gname, F, w, wp, itx, off = DAS_CASES[case]
    g = small_linear() if gname == "lin" else small_matrix()
    rf = random_rf(g, seed=100 + case)
    ref = oracle.das(g, rf, F, window=w, window_param=wp, interp_tx=bool(itx), additional_offset=off)
    bf = RxBeamformer(g)
    out = bf.beamform(torch.from_numpy(rf).cuda(), F, None, w, wp, bool(itx), off)
    rel, exact = compare(out.cpu().numpy(), ref)
    assert exact > 0.999, f"only {exact:.4f} bit-identical"


@pytest.mark.parametrize("rf_dtype,out_dtype", [(torch.int16, torch.float32), (torch.float32, torch.float32),
                                                (torch.int16, torch.int16), (torch.float32, torch.int16)])
def test_das_dtypes(oracle, rf_dtype, out_dtype):
    from supra_b200.api import RxBeamformer
    g = small_linear()
    rf = random_rf(g, seed=5, amp=2000)
    ref = oracle.das(g, rf, 1.0, window=1)
    out = RxBeamformer(g).beamform(torch.from_numpy(rf).to(rf_dtype).cuda(), 1.0, window_type=1, out_dtype=out_dtype)
    got = out.float().cpu().numpy()
    if out_dtype == torch.int16:
        r = np.nan_to_num(ref)
        expect = np.trunc(np.clip(r, -32767, 32767))
        assert np.max(np.abs(got - expect)) <= 1
    else:
        compare(got, ref)


def test_das_c0_full_frame(oracle):
    """Config 0: 128 lines x 2048 depths from a 128x64x2048 int16 frame (20 scatterers, -40 dB)."""
    from supra_b200 import synth
    from supra_b200.api import RxBeamformer
    g, rf = synth.c0_frame(seed=0, device="cuda")
    ref = oracle.das(g, rf.cpu().numpy(), 1.0, window=1)
    out = RxBeamformer(g).beamform(rf, 1.0, window_type=1)
    rel, exact = compare(out.cpu().numpy(), ref)
    assert exact > 0.999


def test_das_3d_mid(oracle):
    """3D: 16x16 matrix, 8x8 scanlines, 8x8 sub-aperture, 64 channels (element e -> channel e % 64)."""
    from supra_b200.api import RxBeamformer
    from supra_b200.geometry import matrix_probe_geometry
    g = matrix_probe_geometry(nx=16, ny=16, pitch_mm=0.3, num_channels=64, num_samples=512, fs_hz=20e6,
                              lines=(8, 8), aperture=(8, 8), focus_mm=20.0)
    rf = random_rf(g, seed=11)
    ref = oracle.das(g, rf, 1.0, window=1)
    out = RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), 1.0, window_type=1)
    rel, exact = compare(out.cpu().numpy(), ref)
    assert exact > 0.999


def test_das_speed_of_sound_argument(oracle):
    from supra_b200.api import RxBeamformer
    g = small_linear()
    rf = random_rf(g, seed=9)
    bf = RxBeamformer(g)
    x = torch.from_numpy(rf).cuda()
    for c in (1450e3, 1540e3, 1600e3, 1540e3):
        ref = oracle.das(g, rf, 1.0, c_mm_s=c, window=2)
        compare(bf.beamform(x, 1.0, c, 2).cpu().numpy(), ref)


def test_das_channel_map(oracle):
    from supra_b200.api import RxBeamformer
    g = small_linear()
    m = np.arange(g.num_elements, dtype=np.int32) % g.num_channels
    m[5] = -1
    m[17] = -1
    g.element_to_channel = m
    rf = random_rf(g, seed=21)
    ref = oracle.das(g, rf, 1.0, window=1)
    compare(RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), 1.0, window_type=1).cpu().numpy(), ref)


def test_rawdelay(oracle):
    from supra_b200.api import RxBeamformer
    g = small_linear()
    rf = random_rf(g, seed=4)
    ref = oracle.rawdelay(g, rf, 1.0, window=1)
    got = RxBeamformer(g).raw_delay(torch.from_numpy(rf).cuda(), 1.0, window_type=1).cpu().numpy()
    compare(got, ref)
