"""The other sample beamformers of RxBeamformerCuda (DelayAndStdDev, CoherenceFactorDelayAndSum,
TestSignal) on the GPU against the oracle, which is pinned bit for bit to the reference's own reducers
(tests/test_oracle_pin.py). The kernels follow the reference's float operations in order, so results
are compared bit for bit."""
import numpy as np
import pytest
import torch

from conftest import bf_geometries, random_rf

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def geoms():
    return bf_geometries()


@pytest.mark.parametrize("case", range(9))
def test_sample_beamformer_golden_cases(oracle, geoms, case):
    from golden.cases import DAS_BF_CASES
    from supra_b200.api import RxBeamformer
    gname, bf, F, w, wp, itx, off = DAS_BF_CASES[case]
    g = geoms[gname]
    rf = random_rf(g, seed=200 + case)
    ref = oracle.das_bf(g, rf, bf, F, window=w, window_param=wp, interp_tx=bool(itx), additional_offset=off)
    out = RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), F, None, w, wp, bool(itx), off, beamformer=bf)
    got = out.cpu().numpy()
    same = bits(got) == bits(ref)
    assert same.all(), f"case {case}: {np.count_nonzero(~same)} of {same.size} differ"


@pytest.mark.parametrize("name", ["DelayAndStdDev", "CoherenceFactorDelayAndSum"])
@pytest.mark.parametrize("rf_dtype,out_dtype", [(torch.float32, torch.float32), (torch.int16, torch.int16),
                                                (torch.float32, torch.int16)])
def test_sample_beamformer_dtypes(oracle, geoms, name, rf_dtype, out_dtype):
    from supra_b200.api import RxBeamformer
    g = geoms["lin"]
    rf = random_rf(g, seed=31, amp=2000)
    ref = oracle.das_bf(g, rf, name, 1.0, window=1)
    out = RxBeamformer(g).beamform(torch.from_numpy(rf).to(rf_dtype).cuda(), 1.0, window_type=1, out_dtype=out_dtype,
                                   beamformer=name)
    got = out.cpu().numpy()
    if out_dtype == torch.int16:
        # clampCast<int16_t> of the same float sum: clamp to +-32767 (NaN to the lower bound), truncate
        expect = np.trunc(np.fmin(np.fmax(ref, -32767.0), 32767.0)).astype(np.int16)
        assert np.array_equal(got, expect)
    else:
        assert np.array_equal(bits(got), bits(ref))


@pytest.mark.parametrize("name", ["DelayAndStdDev", "CoherenceFactorDelayAndSum"])
def test_sample_beamformer_channel_map(oracle, geoms, name):
    """Unconnected elements (map entry -1) are skipped by both passes."""
    from supra_b200.api import RxBeamformer
    from supra_b200.geometry import linear_probe_geometry
    g = linear_probe_geometry(num_elements=32, pitch_mm=0.3, num_channels=16, num_samples=512, fs_hz=40e6,
                              aperture=16, focus_mm=10.0)
    m = np.arange(g.num_elements, dtype=np.int32) % g.num_channels
    m[5] = -1
    m[17] = -1
    g.element_to_channel = m
    rf = random_rf(g, seed=41)
    ref = oracle.das_bf(g, rf, name, 1.0, window=1)
    got = RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), 1.0, window_type=1, beamformer=name).cpu().numpy()
    assert np.array_equal(bits(got), bits(ref))


def test_test_signal_phantom(geoms):
    """The phantom's cylinders: 1000 inside, 0 elsewhere, and the RF is not read (a zero frame gives the
    same image)."""
    from supra_b200.api import RxBeamformer
    g = geoms["lin_deep"]
    bf = RxBeamformer(g)
    a = bf.beamform(torch.from_numpy(random_rf(g, seed=3)).cuda(), beamformer="TestSignal").cpu().numpy()
    b = bf.beamform(torch.zeros((g.num_tx, g.num_channels, g.num_samples), dtype=torch.int16, device="cuda"),
                    beamformer="TestSignal").cpu().numpy()
    assert np.array_equal(a, b)
    assert set(np.unique(a).tolist()) == {0.0, 1000.0}
    # a 2 mm cylinder at 30 mm under x = 0: rows within +-2 mm of 30 mm are lit on the central lines
    depths = np.asarray(g.depths, np.float64)
    lit_rows = np.nonzero(a.max(axis=1) == 1000.0)[0]
    assert abs(depths[lit_rows].mean() - 30.0) < 0.5 and depths[lit_rows].max() - depths[lit_rows].min() <= 4.01


def test_sample_beamformer_rejects_unknown(geoms):
    from supra_b200.abi import SupraError
    from supra_b200.api import RxBeamformer
    g = geoms["lin"]
    with pytest.raises(SupraError):
        RxBeamformer(g).beamform(torch.zeros((g.num_tx, g.num_channels, g.num_samples), dtype=torch.int16,
                                             device="cuda"), beamformer=7)
