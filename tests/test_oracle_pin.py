"""The oracle against the reference's own code: golden fixtures made from oracle/_ref (the reference
sources compiled for the CPU) and, where oracle/_ref is built, a live comparison."""
import os

import numpy as np
import pytest

from conftest import bf_geometries, random_rf, small_linear, small_matrix
from oracle.oracle import reference_root

GOLD = os.path.join(os.path.dirname(__file__), "golden", "ref_pins.npz")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_fir_bit_exact_vs_reference(oracle, gold):
    i = 0
    while f"fir_{i}" in gold:
        L, t, w, fs, f, bw = gold[f"fir_{i}_case"]
        got = oracle.fir(int(L), int(t), int(w), fs, f, bw)
        assert np.array_equal(bits(got), bits(gold[f"fir_{i}"])), f"FIR case {i}"
        i += 1
    assert i >= 8


def test_window_lut_bit_exact_vs_reference(oracle, gold):
    i = 0
    while f"win_{i}" in gold:
        t, p = gold[f"win_{i}_case"]
        got = oracle.window_lut(int(t), float(p), 64)
        assert np.array_equal(bits(got), bits(gold[f"win_{i}"])), f"window case {i}"
        i += 1


def test_das_bit_exact_vs_reference(oracle, gold):
    from golden.cases import DAS_CASES as cases
    geoms = {"lin": small_linear(), "mat": small_matrix()}
    for i, (gname, F, w, wp, itx, off) in enumerate(cases):
        g = geoms[gname]
        rf = random_rf(g, seed=100 + i)
        got = oracle.das(g, rf, F, window=w, window_param=wp, interp_tx=bool(itx), additional_offset=off)
        ref = gold[f"das_{i}"].copy()
        # the CPU build of the reference's clampCast passes NaN through; on the GPU (fmaxf) the
        # reference writes -FLT_MAX there, which is what the oracle models
        ref[np.isnan(ref)] = -np.finfo(np.float32).max
        same = bits(got) == bits(ref)
        assert same.all(), f"DAS case {i}: {np.count_nonzero(~same)} differ"


def test_sample_beamformers_bit_exact_vs_reference(oracle, gold):
    """DelayAndStdDev, CoherenceFactorDelayAndSum and TestSignal (2D and 3D, highest-weight and
    interpolated transmits) against the reference's own reducers."""
    from golden.cases import DAS_BF_CASES as cases
    geoms = bf_geometries()
    for i, (gname, bf, F, w, wp, itx, off) in enumerate(cases):
        g = geoms[gname]
        rf = random_rf(g, seed=200 + i)
        got = oracle.das_bf(g, rf, bf, F, window=w, window_param=wp, interp_tx=bool(itx), additional_offset=off)
        ref = gold[f"dasbf_{i}"].copy()
        ref[np.isnan(ref)] = -np.finfo(np.float32).max  # the GPU clampCast (see the DAS pin)
        same = bits(got) == bits(ref)
        assert same.all(), f"sample beamformer case {i}: {np.count_nonzero(~same)} differ"
    # beamformer 0 is the delay-and-sum path
    g = geoms["lin"]
    rf = random_rf(g, seed=5)
    assert np.array_equal(bits(oracle.das_bf(g, rf, 0)), bits(oracle.das(g, rf)))


@pytest.mark.skipif(reference_root() is None, reason="reference sources not named by SUPRA_REF")
def test_live_reference_checker(oracle):
    """Rebuilds oracle/_ref from the reference sources and compares a c0-sized DAS frame."""
    oracle.build(ref=True)
    from supra_b200.geometry import linear_probe_geometry
    g = linear_probe_geometry(128, 0.3, 64, 2048, 40e6, aperture=64, focus_mm=20.0)
    rf = random_rf(g, seed=7, amp=30000)
    a = oracle.das(g, rf, 1.0, window=1)
    b = oracle.das(g, rf, 1.0, window=1, ref=True)
    b[np.isnan(b)] = -np.finfo(np.float32).max
    same = bits(a) == bits(b)
    assert same.all()
    for n in (65, 64, 31):
        assert np.array_equal(bits(oracle.fir(n, 3, 2)), bits(oracle.fir(n, 3, 2, ref=True)))


def test_oracle_fp64_close_to_fp32(oracle):
    """FP32 reference semantics vs FP64 on band-limited echo data. The float delay (ulp(500 samples)
    = 3e-5 samples) alone moves a 7 MHz echo by ~1e-5 of its peak, so the bound is 5e-5."""
    from supra_b200 import synth
    g = small_linear()
    pts, amps = synth.random_scatterers(8, (-4.0, 4.0), (2.0, 9.0), seed=1)
    rf = synth.channel_data(g, pts, amps, synth.PulseSpec(7e6, 0.6), seed=1).numpy()
    a = oracle.das(g, rf, 1.0, window=1)
    b = oracle.das(g, rf, 1.0, window=1, precision=64)
    m = np.isfinite(b)
    assert np.nanmax(np.abs(a[m] - b[m])) <= 5e-5 * np.nanmax(np.abs(b[m]))


def test_oracle_hilbert_is_envelope(oracle):
    """A sinusoid's Hilbert envelope is flat away from the edges."""
    n = 1024
    t = np.arange(n)
    x = np.cos(2 * np.pi * 0.1 * t)[:, None].repeat(4, 1).astype(np.float32)
    env = oracle.hilbert_env(x, 65)
    assert np.allclose(env[100:-100], 1.0, atol=0.02)


def test_oracle_scan_tables_cover_image(oracle):
    g = small_linear()
    t = oracle.scan_tables(g.scanlines, g.rx_layout[0], g.rx_layout[1], g.num_depths, g.depth_mm, 0.1)
    W, H, D = t["size"]
    assert D == 1 and W > 10 and H > 10
    m = t["mask"].astype(bool)
    assert m.mean() > 0.9
    assert t["weight_x"][m].min() >= -1e-6 and t["weight_x"][m].max() <= 1 + 1e-6
    # weightY is stored in mm (quirk Q5): below one sample distance
    assert t["weight_y"][m].max() <= g.sample_distance_mm * (1 + 1e-6)


def test_oracle_mv_reference_vs_fp64(oracle):
    rng = np.random.Generator(np.random.PCG64(0))
    raw = rng.standard_normal((3, 16, 64)).astype(np.float32)
    raw[:, :3, :10] = 0  # narrower aperture at shallow depths
    a = oracle.mv(raw, 8, 2, precision=32)
    b = oracle.mv(raw, 8, 2, precision=64)
    assert np.max(np.abs(a - b)) <= 1e-3 * np.max(np.abs(b))


def test_oracle_mv_pcg_converges_to_direct_solve(oracle):
    """The PCG restatement (RxBeamformerMVpcg) with enough iterations and a tight threshold gives the
    direct solve (Cholesky) of the same systems; with the reference's defaults it is close to it."""
    rng = np.random.Generator(np.random.PCG64(0))
    raw = rng.standard_normal((3, 16, 64)).astype(np.float32)
    raw[:, :3, :10] = 0
    direct = oracle.mv(raw, 8, 2, precision=64, block=64)  # one block: the PCG reference has none
    pcg = oracle.mv_pcg(raw, 8, 2, max_iterations=64, threshold=1e-9, precision=64)
    assert np.max(np.abs(pcg - direct)) <= 1e-7 * np.max(np.abs(direct))
    default = oracle.mv_pcg(raw, 8, 2, precision=32)
    assert np.max(np.abs(default - direct)) <= 1e-3 * np.max(np.abs(direct))


def test_oracle_analytic_envelope(oracle):
    """HilbertEnvelope's FFT envelope: a periodic tone's envelope is its amplitude, and it equals
    sqrt(x^2 + (k (*) x)^2) with the circular Hilbert kernel k[n] = (2/N) sum_{j=1..J} sin(2 pi j n / N)
    in the closed form the library's plan uses, for even and odd lengths."""
    for N in (64, 63, 1000, 7):
        n = np.arange(N)
        x = 3.0 * np.cos(2 * np.pi * 5 * n / N + 0.3)
        env = oracle.analytic_env(x[:, None])[:, 0]
        if N > 11:
            assert np.max(np.abs(env - 3.0)) < 1e-9
        J = N // 2 - 1 if N % 2 == 0 else (N - 1) // 2
        t = 2 * np.pi * n[1:] / N
        k = np.zeros(N)
        k[1:] = 2.0 / N * np.sin(J * t / 2) * np.sin((J + 1) * t / 2) / np.sin(t / 2)
        rng = np.random.Generator(np.random.PCG64(N))
        y = rng.standard_normal((N, 3))
        h = np.stack([[np.sum(k[(i - np.arange(N)) % N] * y[:, c]) for i in range(N)] for c in range(3)], axis=1)
        assert np.max(np.abs(np.sqrt(y * y + h * h) - oracle.analytic_env(y))) < 1e-9
