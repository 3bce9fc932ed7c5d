"""The library's kernels against the reference's own CUDA kernels on the same GPU and the same inputs.

oracle/_ref/libsupra_ref_gpu.so is built (make -C oracle refgpu) from the reference's sources
RxBeamformerCuda.cu, RawDelay.cu, HilbertFirEnvelope.cu, IQDemodulator.cu and LogCompressor.cu
without fast-math and without FMA contraction, so every float operation of the
reference's kernels is a separately rounded IEEE operation (the semantics this library follows; the
reference's production build adds --use_fast_math, SupraLib/CMakeLists.txt:65). Expected:
  * DAS (all four sample beamformers), RawDelay, Hilbert FIR envelope, log compression: bit-identical;
  * IQ magnitude: within 1e-5 of the peak (the mixer's cos/sin argument is formed in a different order).
Inputs avoid the reference's out-of-range reads (odd filter lengths).
"""
import numpy as np
import pytest
import torch

from conftest import bf_geometries, random_rf, small_linear

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def ref(oracle):
    if oracle.refgpu_lib() is None:
        pytest.skip("reference GPU kernels not built (make -C oracle refgpu needs the reference sources)")
    return oracle


@pytest.mark.parametrize("gname,bf,itx,off", [("lin", 0, 0, 0), ("lin", 0, 1, 3), ("mat", 0, 0, 0), ("lin", 1, 0, 0),
                                              ("lin", 2, 1, -2), ("mat", 1, 0, 0), ("mat", 2, 0, 0),
                                              ("lin_deep", 3, 0, 0)])
def test_das_bit_identical_to_reference_kernel(ref, gname, bf, itx, off):
    from supra_b200.api import RxBeamformer
    g = bf_geometries()[gname]
    rf = random_rf(g, seed=300 + bf)
    want = ref.refg_das(g, rf, bf, 1.0, window=1, interp_tx=bool(itx), additional_offset=off)
    got = RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), 1.0, None, 1, 0.0, bool(itx), off,
                                   beamformer=bf).cpu().numpy()
    same = bits(got) == bits(want)
    assert same.all(), f"{np.count_nonzero(~same)} of {same.size} differ"


def _rawdelay_written(g):
    """[line][channel] mask of the slots the reference's RawDelay kernel writes: local elements
    0 .. last - first of the highest-weight transmit (first maximum, as float), lines whose weight is
    positive (Beamformer/RawDelay.cu:372-385, 268-310). Its other slots keep whatever the freshly
    allocated output held; the library writes zeros there (checked against the oracle elsewhere)."""
    lines = np.asarray(g.scanlines)
    mask = np.zeros((lines.shape[0], g.num_channels), bool)
    for i, s in enumerate(lines):
        w = s["tx_weights"].astype(np.float32)
        k = int(np.argmax(w))
        if w[k] > 0.0:
            mask[i, :max(int(s["tx"][k]["last"][0]) - int(s["tx"][k]["first"][0]), 0)] = True
    return mask


def test_rawdelay_bit_identical_to_reference_kernel(ref):
    from supra_b200.api import RxBeamformer
    g = small_linear()
    rf = random_rf(g, seed=21)
    want = ref.refg_rawdelay(g, rf, 1.0, window=1)
    got = RxBeamformer(g).raw_delay(torch.from_numpy(rf).cuda(), 1.0, window_type=1).cpu().numpy()
    written = _rawdelay_written(g)
    assert written.any() and got.shape == want.shape
    assert np.array_equal(bits(got[written]), bits(want[written]))
    assert np.all(got[~written] == 0.0)


@pytest.fixture(scope="module")
def rf_image():
    from supra_b200.api import RxBeamformer
    g = small_linear(num_samples=1024)
    rf = random_rf(g, seed=5, amp=20000)
    img = RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), 1.0, window_type=1)
    return torch.nan_to_num(img, nan=0.0, posinf=0.0, neginf=0.0).contiguous()


def test_hilbert_bit_identical_to_reference_kernel(ref, rf_image):
    from supra_b200.api import HilbertFirEnvelope
    want = ref.refg_hilbert(rf_image.cpu().numpy(), 65)
    got = HilbertFirEnvelope(65).demodulate(rf_image).cpu().numpy()
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("uint8", [False, True])
def test_logcompress_identical_to_reference_kernel(ref, rf_image, uint8):
    from supra_b200.api import HilbertFirEnvelope, LogCompressor
    env = HilbertFirEnvelope(65).demodulate(rf_image)
    want = ref.refg_logcompress(env.cpu().numpy(), 50.0, 1.0, 30000.0, uint8=uint8)
    got = LogCompressor().compress(env, 50.0, 1.0, 30000.0,
                                   out_dtype=torch.uint8 if uint8 else torch.float32).cpu().numpy()
    if uint8:
        assert np.array_equal(got, want)
    else:
        assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("dec,filters", [(4, 1), (8, 3), (4, 2)])
def test_iq_magnitude_matches_reference_kernel(ref, rf_image, dec, filters):
    from supra_b200.api import IQDemodulator
    refs = [7e6, 5e6, 9e6][:filters]
    bws = [1e6, 2e6, 2e6][:filters]
    ws = [1.0, 0.5, 0.5][:filters]
    want = ref.refg_iq(rf_image.cpu().numpy(), 40e6, refs[0], 2.5e6, 51, 33, dec, refs, bws, ws)
    got = IQDemodulator(40e6, 2.5e6, 51, 33, refs, bws, ws).demodulate_magnitude(rf_image, dec).cpu().numpy()
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-5 * np.max(np.abs(want))


def test_c1_batched_path_matches_reference_kernel(ref):
    """The headline path: one frame of each c1 probe (P64, P128, P192) through the batched pack kernel,
    its RF against the reference's own DAS kernel on the same frames (within 1e-6 of the peak: the pack
    kernel contracts the per-frame sums into FMAs; the +-FLT_MAX of empty apertures equal)."""
    from supra_b200.api import BatchedDasIq, RxBeamformer
    from supra_b200.workloads import c1_workload
    wl = c1_workload(num_frames=3, device="cuda")
    plans = [RxBeamformer(g) for g in wl.geometries]
    b = BatchedDasIq([(plans[p], rf) for p, rf in zip(wl.frame_probe, wl.rf)], 1.0, 1540e3, 1, 0.0, 5e6, 2.5e6, 32, 4,
                     ctas_per_sm=8, depth_tile=128, frames_per_pack=4)
    b.enable_rf_outputs()
    b.run(use_graph=False)
    torch.cuda.synchronize()
    for k, p in enumerate(wl.frame_probe):
        g = wl.geometries[p]
        want = ref.refg_das(g, wl.rf[k].cpu().numpy(), 0, 1.0, c_mm_s=1540e3, window=1)
        got = b.rf_outputs[k].cpu().numpy()
        big = np.abs(want) > 1e30
        assert np.array_equal(got[big], want[big])
        assert np.max(np.abs(got[~big] - want[~big])) <= 1e-6 * np.max(np.abs(want[~big])), f"probe {p}"
