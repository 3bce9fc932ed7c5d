"""Edge cases of the GPU paths against the oracle: ragged sizes (sample counts that break the staged
path's 16-byte rows, depth grids unlike the sample grid, odd scanline counts), degenerate geometries
(two scanlines and two depths, apertures wider than the shared-memory element table), a batch of one
frame, records shorter than the Hilbert filter, MV on single-channel apertures, and empty inputs.
DAS results are compared bit for bit as in the other DAS tests."""
import numpy as np
import pytest
import torch

from conftest import random_rf

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def das_both(oracle, g, rf, **kw):
    from supra_b200.api import RxBeamformer
    ref = oracle.das(g, rf, 1.0, window=1, **kw)
    ref = np.where(np.isnan(ref), -np.float32(3.4028235e38), ref)
    out = RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), 1.0, window_type=1, **kw).cpu().numpy()
    return out, ref


@pytest.mark.parametrize("ne,nch,ns,nd,ntx", [
    (32, 16, 509, None, None),   # 1018-byte rows: not a multiple of 16, the unstaged path
    (32, 16, 512, 333, None),    # depth grid unlike the sample grid
    (7, 7, 300, 101, 7),         # odd element / scanline counts, aperture = all channels
    (16, 8, 64, 2, 2),           # two scanlines, two depths
])
def test_das_ragged_sizes_bit_exact(oracle, ne, nch, ns, nd, ntx):
    from supra_b200.geometry import linear_probe_geometry
    g = linear_probe_geometry(num_elements=ne, pitch_mm=0.3, num_channels=nch, num_samples=ns, fs_hz=40e6,
                              aperture=min(ne, nch), focus_mm=8.0, num_depths=nd, num_tx=ntx)
    rf = random_rf(g, seed=ns + ne)
    out, ref = das_both(oracle, g, rf)
    assert out.shape == ref.shape
    assert np.array_equal(bits(out), bits(ref))


def test_das_aperture_wider_than_element_table(oracle):
    """320-element apertures exceed the staged kernels' 256-entry element table: the generic path runs
    and stays bit-exact."""
    from supra_b200.geometry import linear_probe_geometry
    g = linear_probe_geometry(num_elements=384, pitch_mm=0.1, num_channels=320, num_samples=256, fs_hz=40e6,
                              aperture=320, focus_mm=10.0, num_tx=4)
    rf = random_rf(g, seed=11)
    out, ref = das_both(oracle, g, rf)
    assert np.array_equal(bits(out), bits(ref))


def test_batch_of_one_frame(oracle):
    """One frame in a 4-frame pack (the narrowest loop); records of 504 samples (the batched plan takes
    multiples of 8: 500 is refused with a clear error)."""
    from supra_b200.abi import SupraError
    from supra_b200.api import BatchedDasIq, RxBeamformer
    from supra_b200.geometry import linear_probe_geometry
    g500 = linear_probe_geometry(num_elements=32, pitch_mm=0.3, num_channels=16, num_samples=500, fs_hz=40e6,
                                 aperture=16, focus_mm=10.0)
    with pytest.raises(SupraError, match="multiple of 8"):
        BatchedDasIq([(RxBeamformer(g500), torch.from_numpy(random_rf(g500, seed=2)).cuda())])
    g = linear_probe_geometry(num_elements=32, pitch_mm=0.3, num_channels=16, num_samples=504, fs_hz=40e6,
                              aperture=16, focus_mm=10.0)
    rf = random_rf(g, seed=2)
    b = BatchedDasIq([(RxBeamformer(g), torch.from_numpy(rf).cuda())], 1.0, g.speed_of_sound_mm_s, 1, 0.0, 5e6, 2.5e6,
                     32, 4, frames_per_pack=4)
    b.enable_rf_outputs()
    b.run(use_graph=False)
    torch.cuda.synchronize()
    ref = oracle.das(g, rf, 1.0, window=1)
    ref = np.where(np.isnan(ref), -np.float32(3.4028235e38), ref)
    got = b.rf_outputs[0].cpu().numpy()
    big = np.abs(ref) > 1e30
    assert np.array_equal(got[big], ref[big])
    assert np.max(np.abs(got[~big] - ref[~big])) <= 1e-6 * np.max(np.abs(ref[~big]))
    iq = oracle.iq_complex(got, 40e6, 5e6, 2.5e6, 32, 4)
    assert np.max(np.abs(b.outputs[0].cpu().numpy() - iq)) <= 2e-6 * np.max(np.abs(iq))


def test_hilbert_record_shorter_than_filter(oracle):
    from supra_b200.api import HilbertFirEnvelope
    x = np.random.Generator(np.random.PCG64(4)).standard_normal((10, 6)).astype(np.float32) * 100
    got = HilbertFirEnvelope(65).demodulate(torch.from_numpy(x).cuda()).cpu().numpy()
    ref = oracle.hilbert_env(x, 65)
    assert np.array_equal(bits(got), bits(ref))


def test_mv_single_channel_apertures(oracle):
    """Samples whose aperture is one channel (sz = 1, one subarray) and all-zero samples (no solve)."""
    from supra_b200.api import mv_beamform
    rng = np.random.Generator(np.random.PCG64(8))
    raw = np.zeros((2, 16, 96), np.float32)
    raw[:, 5, 0:32] = rng.standard_normal((2, 32))
    raw[:, :, 32:64] = rng.standard_normal((2, 16, 32))
    out, _ = mv_beamform(torch.from_numpy(raw).cuda(), 8, 2, 1.5, False, 1.0, 0.0)
    torch.cuda.synchronize()
    ref = oracle.mv(raw, 8, 2, precision=32)
    assert np.max(np.abs(out.cpu().numpy() - ref)) <= 1e-4 * np.max(np.abs(ref))
    assert np.all(out.cpu().numpy()[64:] == 0.0)


def test_empty_inputs_rejected_or_noop():
    from supra_b200.abi import SupraError
    from supra_b200.api import BatchedDasIq, temporal_filter
    with pytest.raises((SupraError, ValueError)):
        BatchedDasIq([], 1.0, 1540e3, 1, 0.0, 5e6, 2.5e6, 32, 4)
    empty = torch.empty(0, device="cuda")
    assert temporal_filter([empty, empty]).numel() == 0
