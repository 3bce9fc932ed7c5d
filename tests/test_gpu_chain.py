"""Envelope, log compression, IQ demodulation and scan conversion on the GPU against the oracle."""
import numpy as np
import pytest
import torch

from conftest import small_linear, small_matrix

pytestmark = pytest.mark.gpu


def rf_image(nS=2048, nL=128, seed=0):
    from supra_b200 import synth
    from supra_b200.api import RxBeamformer
    g, rf = synth.c0_frame(seed=seed, device="cuda", num_samples=nS)
    img = RxBeamformer(g).beamform(rf, 1.0, window_type=1)
    # depth 0 holds the reference's -FLT_MAX quirk (0/0 aperture, clamped); clear it for the chain
    img[~torch.isfinite(img) | (img.abs() > 1e30)] = 0.0
    return g, img


@pytest.mark.parametrize("N", [65, 64, 31])
def test_hilbert(oracle, N):
    from supra_b200.api import HilbertFirEnvelope
    g, img = rf_image()
    img = torch.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0)
    ref = oracle.hilbert_env(img.cpu().numpy(), N)
    got = HilbertFirEnvelope(N).demodulate(img).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-6 * np.max(np.abs(ref))


@pytest.mark.parametrize("out_dtype", [torch.uint8, torch.float32])
def test_logcompress(oracle, out_dtype):
    from supra_b200.api import LogCompressor
    rng = np.random.Generator(np.random.PCG64(1))
    x = (rng.standard_normal(200000) * 3000).astype(np.float32)
    ref = oracle.logcompress(x, 50.0, 1.0, 20000.0, np.uint8 if out_dtype == torch.uint8 else np.float32)
    got = LogCompressor().compress(torch.from_numpy(x).cuda(), 50.0, 1.0, 20000.0, out_dtype).cpu().numpy()
    if out_dtype == torch.uint8:
        assert np.max(np.abs(got.astype(int) - ref.astype(int))) <= 1
    else:
        assert np.max(np.abs(got - ref)) <= 1e-5 * 255


@pytest.mark.parametrize("dec,filters,bp", [(8, 1, 51), (4, 3, 51), (1, 1, 51), (2, 5, 51), (1, 8, 51), (4, 2, 51),
                                            (3, 3, 3), (2, 2, 5), (4, 4, 7)])
def test_iq_magnitude(oracle, dec, filters, bp):
    """One reference frequency (iqMagnitude1Kernel) and 2-8 frequencies (the filter-bank kernel
    specialised on the filter count, band-pass rows in groups of 8, 4 or 2 per thread; band-pass
    filters shorter than a group take the per-row tap test) against the oracle's restatement of
    IQDemodulator.cu:68-175."""
    from supra_b200.api import IQDemodulator
    g, img = rf_image()
    img = torch.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0)
    refs = [7e6, 5e6, 9e6, 6e6, 8e6, 4e6, 10e6, 7.5e6][:filters]
    bws = [1e6, 2e6, 2e6, 1.5e6, 1.5e6, 1e6, 2e6, 1e6][:filters]
    ws = [1.0, 0.5, 0.5, 0.25, 0.25, 0.75, 0.5, 1.0][:filters]
    ref = oracle.iq_magnitude(img.cpu().numpy(), dec, 40e6, 2.5e6, 51, bp, refs, bws, ws)
    got = IQDemodulator(40e6, 2.5e6, 51, bp, refs, bws, ws).demodulate_magnitude(img, dec).cpu().numpy()
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_iq_complex_vs_fp64(oracle):
    from supra_b200.api import iq_complex
    g, img = rf_image()
    img = torch.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0)
    ref = oracle.iq_complex(img.cpu().numpy(), 40e6, 5e6, 2.5e6, 32, 4)
    got = iq_complex(img, 40e6, 5e6, 2.5e6, 32, 4).cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_scan_tables_2d_bit_exact(oracle):
    from supra_b200.api import ScanConverter
    g = small_linear()
    sc = ScanConverter(g.scanlines, g.rx_layout, g.num_depths, g.depth_mm, 0.1)
    t = sc.tables()
    r = oracle.scan_tables(g.scanlines, g.rx_layout[0], 1, g.num_depths, g.depth_mm, 0.1)
    m = r["mask"].astype(bool)
    assert np.array_equal(t["mask"], r["mask"])
    for k in ("sample_idx", "weight_x", "weight_y"):
        assert np.array_equal(t[k][m].view(np.uint32), r[k][m].view(np.uint32)), k


def test_scan_tables_3d(oracle):
    from supra_b200.api import ScanConverter
    g = small_matrix()
    sc = ScanConverter(g.scanlines, g.rx_layout, g.num_depths, g.depth_mm, 0.2)
    t = sc.tables()
    r = oracle.scan_tables(g.scanlines, g.rx_layout[0], g.rx_layout[1], g.num_depths, g.depth_mm, 0.2)
    assert t["size"] == r["size"]
    agree = np.mean(t["mask"] == r["mask"])
    assert agree >= 0.999, agree
    m = (t["mask"] == 1) & (r["mask"] == 1)
    assert np.mean(t["sample_idx"][m] == r["sample_idx"][m]) >= 0.999
    same = t["sample_idx"][m] == r["sample_idx"][m]
    for k in ("weight_x", "weight_y", "weight_z"):
        assert np.max(np.abs(t[k][m][same] - r[k][m][same])) <= 1e-4, k


def test_scan_convert_2d(oracle):
    from supra_b200.api import ScanConverter
    g, img = rf_image()
    img = torch.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0).abs()
    sc = ScanConverter(g.scanlines, g.rx_layout, g.num_depths, g.depth_mm, 0.1)
    r = oracle.scan_tables(g.scanlines, g.rx_layout[0], 1, g.num_depths, g.depth_mm, 0.1)
    ref = oracle.scan_apply(img.cpu().numpy(), g.rx_layout[0], 1, r, np.float32)[0]
    got = sc.convert(img, torch.float32).cpu().numpy()
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref))


def test_fused_env_log_scan_c0(oracle):
    """Config 0 chain after DAS: 64-tap Hilbert, 50 dB log, 0.1 mm uint8 scan conversion."""
    from supra_b200.api import HilbertFirEnvelope, ScanConverter
    g, img = rf_image()
    img = torch.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0)
    x = img.cpu().numpy()
    env = oracle.hilbert_env(x, 64)
    in_max = float(env.max())
    logc = oracle.logcompress(env, 50.0, 1.0, in_max, np.float32)
    r = oracle.scan_tables(g.scanlines, g.rx_layout[0], 1, g.num_depths, g.depth_mm, 0.1)
    ref = oracle.scan_apply(logc, g.rx_layout[0], 1, r, np.uint8)[0]
    sc = ScanConverter(g.scanlines, g.rx_layout, g.num_depths, g.depth_mm, 0.1)
    got = sc.env_log_convert(HilbertFirEnvelope(64), img, 50.0, 1.0, in_max, torch.uint8).cpu().numpy()
    assert got.shape == ref.shape == (396, 383)
    d = np.abs(got.astype(int) - ref.astype(int))
    assert d.max() <= 1, d.max()


def test_env_log_scan_3d(oracle):
    """The 3D chain after DAS (c2's processing): 65-tap envelope, log compression and trilinear scan
    conversion, against the oracle's envelope, log and gather applied with the plan's own tables (the
    3D tables themselves are compared in test_scan_tables_3d); uint8 within 1 LSB."""
    from supra_b200.api import HilbertFirEnvelope, ScanConverter
    g = small_matrix(num_samples=512)
    rng = np.random.Generator(np.random.PCG64(12))
    vol = (rng.standard_normal((g.num_depths, g.num_rx)) * 1000).astype(np.float32)
    env = oracle.hilbert_env(vol, 65)
    in_max = float(env.max())
    logc = oracle.logcompress(env, 50.0, 1.0, in_max, np.float32)
    sc = ScanConverter(g.scanlines, g.rx_layout, g.num_depths, g.depth_mm, 0.25)
    ref = oracle.scan_apply(logc, g.rx_layout[0], g.rx_layout[1], sc.tables(), np.uint8)
    got = sc.env_log_convert(HilbertFirEnvelope(65), torch.from_numpy(vol).cuda(), 50.0, 1.0, in_max,
                             torch.uint8).cpu().numpy()
    assert got.shape == ref.shape and ref.any()
    assert np.abs(got.astype(int) - ref.astype(int)).max() <= 1
