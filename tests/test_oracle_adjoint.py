"""Pins the oracle's FP64 reference gradient of the apodised DAS (used by the GPU adjoint tests):
against central differences of an FP64 forward that is smooth in the speed of sound
(tests/adjoint_model.py), central differences of the oracle's FP64 forward in the apodisation,
and the adjoint identity in the channel data. CPU only.
"""
import numpy as np
import pytest

from conftest import small_linear


@pytest.fixture(scope="module")
def small_case():
    from supra_b200 import synth
    g = small_linear(num_samples=256)
    pts, amps = synth.random_scatterers(8, (-4.5, 4.5), (1.0, 4.5), seed=9)
    rf = synth.channel_data(g, pts, amps, synth.PulseSpec(7e6, 0.6), -40.0, 1.0, seed=9, quantize=False)
    rf = rf.numpy().astype(np.float32)
    rng = np.random.Generator(np.random.PCG64(5))
    apod = rng.uniform(0.5, 1.5, g.num_elements).astype(np.float32)
    gout = rng.standard_normal((g.num_depths, g.num_rx))
    gout[0] = 0.0  # depth 0 is not finite (zero-width aperture)
    return g, rf, apod, gout


def _dot(s, g):
    m = np.isfinite(s)
    return float(np.sum(np.where(m, s, 0.0) * np.where(m, g, 0.0)))


def test_grad_c_against_smooth_fp64_differences(oracle, small_case):
    import adjoint_model as M
    g, rf, apod, gout = small_case
    c0 = g.speed_of_sound_mm_s
    _, _, gc = oracle.das_adjoint64(g, rf, apod, gout)
    dec = M.decisions(g, c0, oracle.window_lut(1))
    rf64 = rf.astype(np.float64)
    assert abs(M.grad_c(g, rf64, apod, dec, c0, gout) - gc) <= 1e-7 * abs(gc)
    h = 0.1  # mm/s: converged (larger steps cross sample boundaries of the linear interpolation)
    fd = (_dot(M.forward(g, rf64, apod, dec, c0 + h), gout) - _dot(M.forward(g, rf64, apod, dec, c0 - h), gout)) / (2 * h)
    assert abs(fd - gc) <= 1e-6 * abs(gc)


def test_grad_apod_against_fp64_differences(oracle, small_case):
    g, rf, apod, gout = small_case
    _, gap, _ = oracle.das_adjoint64(g, rf, apod, gout)
    h = 1e-3
    for e in range(0, g.num_elements, 5):
        ap = apod.copy()
        ap[e] = apod[e] + h
        lp = _dot(oracle.das(g, rf, 1.0, window=1, apod=ap, precision=64), gout)
        hp = float(ap[e])
        ap[e] = apod[e] - h
        lm = _dot(oracle.das(g, rf, 1.0, window=1, apod=ap, precision=64), gout)
        fd = (lp - lm) / (hp - float(ap[e]))
        assert abs(fd - gap[e]) <= 1e-6 * max(1.0, np.max(np.abs(gap)))


def test_adjoint_identity_rf(oracle, small_case):
    g, rf, apod, gout = small_case
    d = np.random.Generator(np.random.PCG64(2)).standard_normal(rf.shape).astype(np.float32)
    grf, _, _ = oracle.das_adjoint64(g, d, apod, gout)
    lhs = _dot(oracle.das(g, d, 1.0, window=1, apod=apod, precision=64), gout)
    rhs = float(np.sum(d.astype(np.float64) * grf))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_vectorised_smooth_model_matches_loops(oracle, small_case):
    """SmoothModelTorch (used for the c4-size finite differences on the GPU) against the loop model on
    the CPU: the same decisions and the same FP64 forward at c0 and at c0 + 10 mm/s."""
    import torch
    import adjoint_model as M
    g, rf, apod, _ = small_case
    c0 = g.speed_of_sound_mm_s
    lut = oracle.window_lut(1)
    dec = M.decisions(g, c0, lut)
    tm = M.SmoothModelTorch(g, c0, lut, device="cpu")
    rf64 = rf.astype(np.float64)
    for c in (c0, c0 + 10.0):
        want = M.forward(g, rf64, apod, dec, c)
        got = tm.forward(torch.from_numpy(rf), c, torch.from_numpy(apod)).numpy()
        both = np.isfinite(want) & np.isfinite(got)
        assert np.array_equal(np.isfinite(want), np.isfinite(got))
        assert np.max(np.abs(got[both] - want[both])) <= 1e-9 * np.max(np.abs(want[both]))
