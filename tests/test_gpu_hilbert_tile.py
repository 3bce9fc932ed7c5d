"""The tiled Hilbert envelope kernel against the oracle's restatement of HilbertFirEnvelope
(Beamformer/HilbertFirEnvelope.cu:28-61), bit for bit: both tile sizes (8 x 4 and 8 x 16 outputs per
warp row), odd and even filter lengths, ragged images (scanlines not a multiple of 32, samples not a
multiple of the tile), records shorter than the filter, int16 input, a filter too long for the tile
(the one-thread-per-output kernel), and tiles holding an infinity or NaN (every tap summed, NaN where
the reference's zero taps meet the infinity)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _image(nS, nL, seed, dtype=np.float32):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.standard_normal((nS, nL)) * 2000.0
    return x.astype(np.int16) if dtype == np.int16 else x.astype(np.float32)


def _check(oracle, x, N):
    from supra_b200.api import HilbertFirEnvelope
    got = HilbertFirEnvelope(N).demodulate(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = oracle.hilbert_env(x.astype(np.float32), N)
    assert got.shape == ref.shape
    nan_g, nan_r = np.isnan(got), np.isnan(ref)
    assert np.array_equal(nan_g, nan_r)
    same = bits(got)[~nan_g] == bits(ref)[~nan_r]
    assert same.all(), f"{np.count_nonzero(~same)} of {same.size} differ"


@pytest.mark.parametrize("nS,nL", [(2048, 128), (4096, 1024), (1000, 77), (10, 6), (129, 33)])
@pytest.mark.parametrize("N", [65, 64, 31])
def test_tile_bit_exact(oracle, nS, nL, N):
    _check(oracle, _image(nS, nL, seed=nS + nL + N), N)


def test_tile_int16_input(oracle):
    _check(oracle, _image(3000, 100, seed=3, dtype=np.int16), 65)


@pytest.mark.parametrize("N", [301, 1001])
def test_long_filters(oracle, N):
    """301 taps fit the small tile; 1001 taps exceed every tile and take the per-output kernel."""
    _check(oracle, _image(2048, 64, seed=N), N)


def test_non_finite_tiles(oracle):
    x = _image(4096, 256, seed=9)
    x[100, 5] = np.inf
    x[2000, 40] = -np.inf
    x[3000, 200] = np.nan
    _check(oracle, x, 65)
