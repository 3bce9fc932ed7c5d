"""Batched persistent DAS + complex IQ against the per-frame path and the FP64 IQ oracle."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small_batch():
    from supra_b200.api import BatchedDasIq, RxBeamformer
    from supra_b200.workloads import c1_frame, c1_geometries
    geoms = c1_geometries()
    plans = [RxBeamformer(g) for g in geoms]
    probe = [0, 1, 2, 1, 0]
    rfs = [c1_frame(geoms[p], 500 + k) for k, p in enumerate(probe)]
    return geoms, plans, probe, rfs


@pytest.mark.parametrize("shape", [(1, 256, 1, 0), (1, 384, 1, 0), (2, 128, 1, 0), (4, 256, 4, 0), (4, 256, 8, 0),
                                   (6, 128, 8, 0), (3, 128, 2, 0), (1, 128, 4, 1), (1, 128, 2, 1), (2, 128, 2, 1)])
@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_rf_matches_per_frame(small_batch, shape, use_graph):
    from supra_b200.api import BatchedDasIq
    geoms, plans, probe, rfs = small_batch
    b = BatchedDasIq([(plans[p], rf) for p, rf in zip(probe, rfs)], ctas_per_sm=shape[0], depth_tile=shape[1],
                     frames_per_pack=shape[2], staged=shape[3])
    b.enable_rf_outputs()
    b.run(use_graph=use_graph)
    b.run(use_graph=use_graph)  # a second replay must give the same result
    torch.cuda.synchronize()
    for k, p in enumerate(probe):
        ref = plans[p].beamform(rfs[k], 1.0, 1540e3, 1).cpu().numpy().astype(np.float64)
        got = b.rf_outputs[k].cpu().numpy().astype(np.float64)
        if shape[2] == 1:  # per-frame pipeline: same arithmetic as sb_das_run, bit-identical
            assert np.array_equal(got, ref), f"frame {k}"
        else:  # frame packs: FMA-contracted sums, identical decisions
            big = np.abs(ref) >= np.finfo(np.float32).max
            assert np.array_equal(got[big], ref[big])
            peak = np.max(np.abs(ref[~big]))
            assert np.max(np.abs(got[~big] - ref[~big])) <= 1e-6 * peak, f"frame {k}"


def test_batch_iq_vs_fp64(small_batch, oracle):
    from supra_b200.api import BatchedDasIq
    geoms, plans, probe, rfs = small_batch
    b = BatchedDasIq([(plans[p], rf) for p, rf in zip(probe, rfs)])
    b.enable_rf_outputs()
    b.run()
    torch.cuda.synchronize()
    for k, p in enumerate(probe):
        rf = b.rf_outputs[k].cpu().numpy()
        ref = oracle.iq_complex(rf, 40e6, 5e6, 2.5e6, 32, 4)
        got = b.outputs[k].cpu().numpy()
        assert got.shape == ref.shape
        err = np.max(np.abs(got - ref))
        assert err <= 2e-6 * np.max(np.abs(ref)), (k, err, np.max(np.abs(ref)))


@pytest.mark.parametrize("decimation,lowpass", [(1, 16), (2, 31), (3, 32), (5, 20), (8, 64), (40, 8)])
@pytest.mark.parametrize("frames_per_pack", [4, 8])
def test_batch_iq_decimations(small_batch, oracle, decimation, lowpass, frames_per_pack):
    """The pack kernel keeps an item's rows in shared memory ordered by decimation phase; every
    decimation (up to 32 phases, row order above) and low-pass length gives the FP64 IQ of its RF."""
    from supra_b200.api import BatchedDasIq
    geoms, plans, probe, rfs = small_batch
    b = BatchedDasIq([(plans[p], rf) for p, rf in zip(probe, rfs)], 1.0, 1540e3, 1, 0.0, 5e6, 2.5e6, lowpass,
                     decimation, ctas_per_sm=4, depth_tile=256, frames_per_pack=frames_per_pack)
    b.enable_rf_outputs()
    b.run(use_graph=True)
    torch.cuda.synchronize()
    for k, p in enumerate(probe):
        rf = b.rf_outputs[k].cpu().numpy()
        ref = oracle.iq_complex(rf, 40e6, 5e6, 2.5e6, lowpass, decimation)
        got = b.outputs[k].cpu().numpy()
        assert got.shape == ref.shape
        err = np.max(np.abs(got - ref))
        assert err <= 2e-6 * np.max(np.abs(ref)), (k, err, np.max(np.abs(ref)))


def test_batch_autotune_and_cache(small_batch, tmp_path):
    from supra_b200.api import BatchedDasIq
    geoms, plans, probe, rfs = small_batch
    b = BatchedDasIq([(plans[p], rf) for p, rf in zip(probe, rfs)])
    cache = str(tmp_path / "tune.txt")
    c, t, f, g = b.autotune(cache)
    assert 1 <= c <= 12 and t in (128, 256, 384, 512) and f in (1, 2, 4, 8) and g in (0, 1)
    b2 = BatchedDasIq([(plans[p], rf) for p, rf in zip(probe, rfs)])
    assert b2.autotune(cache) == (c, t, f, g)
    b2.run()
    torch.cuda.synchronize()


def test_device_error_flag_clear():
    from supra_b200.api import check_device_errors
    check_device_errors()
