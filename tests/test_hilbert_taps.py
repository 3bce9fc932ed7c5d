"""The two facts the tiled Hilbert envelope kernel rests on, checked on the CPU.

1. The Hilbert designs (FirFilterFactory, Hilbert type with a Hamming window) have their nonzero
   taps at one parity only (odd offsets from the centre) and exact zeros in between, for odd and even
   lengths (tap N of an even-length filter is taken as 0, as the reference reads it).
2. A float32 sum taken in tap order with separately rounded products is unchanged, bit for bit, when
   the zero taps are left out, as long as the inputs are finite: a sum that starts at +0 never
   becomes -0, and a finite value times +-0 is +-0. An infinity meets a zero tap as NaN, so tiles
   holding one must sum every tap.
"""
import numpy as np
import pytest

HILBERT, HAMMING = 3, 2


@pytest.mark.parametrize("N", [3, 4, 7, 31, 32, 64, 65, 128, 301])
def test_hilbert_taps_alternate_with_exact_zeros(N):
    from supra_b200.api import fir_design
    h = np.append(fir_design(N, HILBERT, HAMMING), np.float32(0.0)) if N % 2 == 0 else fir_design(N, HILBERT, HAMMING)
    taps = h[:2 * (N // 2) + 1]
    nz = np.flatnonzero(taps)
    assert nz.size > 0
    assert np.all(np.diff(nz) == 2)                      # one parity, no gaps
    zero = np.setdiff1d(np.arange(taps.size), nz)
    assert np.all(taps[zero] == 0.0)


def _fir_sum(x, h, skip_zero_taps):
    """sum_j x[j] h[j] in tap order, float32 products and additions (round to nearest each)."""
    acc = np.float32(0.0)
    for xv, hv in zip(x, h):
        if skip_zero_taps and hv == 0.0:
            continue
        acc = np.float32(acc + np.float32(xv * hv))
    return acc


def test_zero_taps_leave_finite_sums_bit_identical():
    from supra_b200.api import fir_design
    h = fir_design(65, HILBERT, HAMMING)
    rng = np.random.Generator(np.random.PCG64(17))
    for scale in (1e-30, 1.0, 3000.0, 3e30):
        for _ in range(40):
            x = (rng.standard_normal(h.size) * scale).astype(np.float32)
            x[rng.integers(0, h.size, 5)] = 0.0         # zeros and exact cancellations included
            full, skip = _fir_sum(x, h, False), _fir_sum(x, h, True)
            assert np.array_equal(np.array([full]).view(np.uint32), np.array([skip]).view(np.uint32))


def test_infinity_needs_every_tap():
    from supra_b200.api import fir_design
    h = fir_design(65, HILBERT, HAMMING)
    x = np.ones(h.size, np.float32)
    x[np.flatnonzero(h == 0.0)[0]] = np.inf            # an infinity on a zero tap
    with np.errstate(invalid="ignore"):
        assert np.isnan(_fir_sum(x, h, False))
        assert np.isfinite(_fir_sum(x, h, True))
