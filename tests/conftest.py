import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libsupra_b200.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    if not os.path.exists(O.LIB):
        O.build(ref=False)
    return O


def small_linear(num_samples=512, seed=0):
    from supra_b200.geometry import linear_probe_geometry
    return linear_probe_geometry(num_elements=32, pitch_mm=0.3, num_channels=16, num_samples=num_samples,
                                 fs_hz=40e6, aperture=16, focus_mm=10.0)


def small_matrix(num_samples=256):
    from supra_b200.geometry import matrix_probe_geometry
    return matrix_probe_geometry(nx=8, ny=8, pitch_mm=0.3, num_channels=32, num_samples=num_samples, fs_hz=20e6,
                                 lines=(4, 4), aperture=(4, 4), focus_mm=15.0)


def bf_geometries():
    """Geometries of the sample-beamformer cases; the deep ones reach the test signal's 30 mm cylinders."""
    return {"lin": small_linear(), "mat": small_matrix(), "lin_deep": small_linear(num_samples=2048),
            "mat_deep": small_matrix(num_samples=1024)}


def random_rf(geom, seed=0, dtype=np.int16, amp=3000):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.integers(-amp, amp + 1, size=(geom.num_tx, geom.num_channels, geom.num_samples))
    return x.astype(dtype)
