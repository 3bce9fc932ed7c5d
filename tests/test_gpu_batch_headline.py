"""The batched DAS + complex IQ path at the exact shape the benchmark times.

The workload is 64 frames of three linear probes: 22 frames of P64 (64 elements, 1024 samples), 21 of
P128 (2048 samples) and 21 of P192 (3072 samples), int16, with one focused transmit per element and a
64-channel receive aperture. The IQ stage mixes at 5 MHz, applies a 32-tap low-pass and decimates by
4. The frames are the benchmark's own seeded frames.

With 8 frames per pack, P64 forms packs of 8, 8 and 6 frames and the other probes packs of 8, 8 and 5.
So the pack kernel's 8-frame loop and its 6-frame loop both run, as they do in the benchmark. Both
loops carry the L2 prefetch of the gathers two elements ahead.

Each frame is checked twice:
  * its RF against the reference's own DAS kernel (rxBeamformingDTSPACEKernel,
    Beamformer/RxBeamformerCuda.cu:238-323), built into the checker. The tolerance is 1e-6 of the
    frame peak, since the pack kernel contracts the per-frame sums into FMAs. The +-FLT_MAX pixels of
    empty apertures must be equal. Without the checker, the RF is compared with sb_das_run, which
    the other tests pin bit-exactly to that kernel.
  * its IQ against the oracle's FP64 mixing and low-pass of that RF, within 2e-6 of the IQ peak.

Two tile shapes run: the benchmark's autotuned <8 frames, 256 threads, 4 CTAs/SM> forced, and the
autotuner's own choice on this workload.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

RF_TOL = 1e-6
IQ_TOL = 2e-6


@pytest.fixture(scope="module")
def headline():
    from supra_b200.api import RxBeamformer
    from supra_b200.workloads import c1_workload
    wl = c1_workload(num_frames=64, device="cuda", seed0=1000)  # the benchmark's frames (rank 0)
    plans = [RxBeamformer(g) for g in wl.geometries]
    return wl, plans


@pytest.fixture(scope="module")
def expected_rf(headline, oracle):
    """RF of every frame from the reference's own DAS kernel (or sb_das_run without the checker)."""
    wl, plans = headline
    use_ref = oracle.refgpu_lib() is not None
    out = []
    for k, p in enumerate(wl.frame_probe):
        if use_ref:
            out.append(oracle.refg_das(wl.geometries[p], wl.rf[k].cpu().numpy(), 0, 1.0, c_mm_s=1540e3, window=1))
        else:
            out.append(plans[p].beamform(wl.rf[k], 1.0, 1540e3, 1).cpu().numpy())
    return out


def _pack_sizes(frame_probe, fp):
    sizes = []
    for p in sorted(set(frame_probe)):
        n = frame_probe.count(p)
        sizes += [min(fp, n - b) for b in range(0, n, fp)]
    return sizes


def test_headline_pack_shape_reaches_wide_loops(headline):
    """The 8-frame packs of the benchmark: full packs (8-frame loop) and packs of 6 and 5 (6-frame loop)."""
    wl, _ = headline
    sizes = _pack_sizes(wl.frame_probe, 8)
    assert sorted(sizes) == sorted([8, 8, 6, 8, 8, 5, 8, 8, 5])


def _check(b, wl, expected_rf, oracle):
    torch.cuda.synchronize()
    worst_rf = worst_iq = 0.0
    for k, p in enumerate(wl.frame_probe):
        want = expected_rf[k]
        got = b.rf_outputs[k].cpu().numpy()
        big = np.abs(want) > 1e30
        assert np.array_equal(got[big], want[big]), f"frame {k}: clamped pixels differ"
        peak = np.max(np.abs(want[~big]))
        err = np.max(np.abs(got[~big].astype(np.float64) - want[~big]))
        assert err <= RF_TOL * peak, f"frame {k} (probe {p}): RF error {err / peak:.3g} of peak"
        iq_want = oracle.iq_complex(got, 40e6, 5e6, 2.5e6, 32, 4)
        iq_got = b.outputs[k].cpu().numpy()
        assert iq_got.shape == iq_want.shape
        ierr = np.max(np.abs(iq_got - iq_want))
        assert ierr <= IQ_TOL * np.max(np.abs(iq_want)), f"frame {k} (probe {p}): IQ error {ierr:.3g}"
        worst_rf = max(worst_rf, err / peak)
        worst_iq = max(worst_iq, ierr / np.max(np.abs(iq_want)))
    print(f"c1 64 frames: RF vs the reference kernel {worst_rf:.3g} of the frame peak (worst frame), "
          f"IQ vs FP64 {worst_iq:.3g} of the IQ peak")


@pytest.mark.parametrize("use_graph", [False, True])
def test_headline_forced_8_frame_packs(headline, expected_rf, oracle, use_graph):
    from supra_b200.api import BatchedDasIq
    wl, plans = headline
    b = BatchedDasIq([(plans[p], rf) for p, rf in zip(wl.frame_probe, wl.rf)], 1.0, 1540e3, 1, 0.0, 5e6, 2.5e6, 32, 4,
                     ctas_per_sm=4, depth_tile=256, frames_per_pack=8)
    b.enable_rf_outputs()
    b.run(use_graph=use_graph)
    b.run(use_graph=use_graph)  # a replay gives the same outputs
    _check(b, wl, expected_rf, oracle)
    from supra_b200.api import check_device_errors
    check_device_errors()


def test_headline_autotuned_shape(headline, expected_rf, oracle, tmp_path):
    from supra_b200.api import BatchedDasIq
    wl, plans = headline
    b = BatchedDasIq([(plans[p], rf) for p, rf in zip(wl.frame_probe, wl.rf)], 1.0, 1540e3, 1, 0.0, 5e6, 2.5e6, 32, 4)
    shape = b.autotune(str(tmp_path / "tune.txt"))
    b.enable_rf_outputs()
    b.run(use_graph=True)
    _check(b, wl, expected_rf, oracle)
    print("autotuned shape", shape)
