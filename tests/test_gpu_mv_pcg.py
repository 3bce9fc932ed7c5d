"""Minimum variance with the PCG solve (sb_mv_pcg_run) against the oracle's restatement of
RxBeamformerMVpcg::performRxBeamforming (Beamformer/RxBeamformerMVpcg.cu:450-800).

The reference's matrix-vector and dot products sum with atomics in arbitrary order, so it is not
bit-reproducible itself; the kernel (warp sums) and the oracle (sums in order) run the same iteration
with the same stopping rules and are compared within a tolerance relative to the frame peak.
The reference iterates in FP32 from a = 1 while the solution is of order 1 / |R|: on int16-scale data
the first step cancels almost all of a's digits, and on a fraction of the systems (about 0.5% at
subarray size 16 on the c0 frame) the subarray-size iterations do not recover. The oracle's FP32
restatement shows the same. So on the c0 frame:
  * of the systems that the reference's own FP32 iteration (oracle, precision 32) solves to within
    1e-4 of the peak of the FP64 PCG, at least 99.9% are within 2e-4 of the peak of the FP64 PCG
    (which systems are lost depends on the summation order, as it does in the reference);
  * the kernel loses no more systems than the FP32 restatement (twice its count plus 0.1%).
On unit-variance data (little cancellation) the iterates themselves are compared: two iterations
against the oracle's FP32 PCG at 1e-4 of the peak. The temporal window is clipped only at the
record ends (no 2000-sample blocks), checked across sample 2000.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c0_raw():
    from supra_b200 import synth
    from supra_b200.api import RxBeamformer
    g, rf = synth.c0_frame(3, device="cuda")
    raw = RxBeamformer(g).raw_delay(rf, 1.0, window_type=1)
    torch.cuda.synchronize()
    raw = raw[::16].contiguous()  # 8 scanlines x 64 channels x 2048 samples
    raw[~(raw.abs() < 1e30)] = 0.0  # +-FLT_MAX of RawDelay at depth 0 (see the MV tests)
    return raw


def _peak_err(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _pcg(raw, **kw):
    from supra_b200.api import mv_beamform_pcg
    out = mv_beamform_pcg(raw, **kw)
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _compare(oracle, raw, L, T, out):
    r = raw.cpu().numpy() if torch.is_tensor(raw) else raw
    ref64 = oracle.mv_pcg(r, L, T, precision=64)
    ref32 = oracle.mv_pcg(r, L, T, precision=32)
    pk = np.max(np.abs(ref64))
    stable = np.abs(ref32 - ref64) <= 1e-4 * pk
    bad = np.abs(out - ref64) > 2e-4 * pk
    assert np.mean(~bad[stable]) >= 0.999, (int((bad & stable).sum()), int(stable.sum()))
    assert bad.sum() <= 2 * (~stable).sum() + 1e-3 * out.size, (int(bad.sum()), int((~stable).sum()))


@pytest.mark.parametrize("L,T", [(32, 3), (16, 0), (48, 5), (0, 3)])
def test_mv_pcg_matches_oracle(oracle, c0_raw, L, T):
    out = _pcg(c0_raw, subarray_size=L, temporal_smoothing=T)
    assert out.shape == (c0_raw.shape[2], c0_raw.shape[0])
    _compare(oracle, c0_raw, L, T, out)


@pytest.fixture(scope="module")
def unit_raw():
    rng = np.random.Generator(np.random.PCG64(5))
    raw = rng.standard_normal((3, 32, 2100)).astype(np.float32)
    raw[:, :2, :100] = 0.0  # a narrower aperture at the start
    return raw


def test_mv_pcg_no_sample_blocks(oracle, unit_raw):
    """Across sample 2000 the PCG reference smooths over the whole window (the Cholesky reference
    clips it at its 2000-sample blocks)."""
    out = _pcg(torch.from_numpy(unit_raw).cuda(), subarray_size=16, temporal_smoothing=5)
    ref = oracle.mv_pcg(unit_raw, 16, 5, precision=64)
    blocked = oracle.mv(unit_raw, 16, 5, precision=64, block=2000)
    rows = slice(1990, 2010)
    pk = np.max(np.abs(ref))
    assert _peak_err(out, ref) <= 1e-4
    assert np.max(np.abs(ref[rows] - blocked[rows])) > 1e-3 * pk  # the two references differ there


def test_mv_pcg_early_stop(oracle, unit_raw):
    out = _pcg(torch.from_numpy(unit_raw).cuda(), subarray_size=16, temporal_smoothing=3, max_iterations_override=2)
    ref = oracle.mv_pcg(unit_raw, 16, 3, max_iterations=2, precision=32)
    assert _peak_err(out, ref) <= 1e-4
    full = oracle.mv_pcg(unit_raw, 16, 3, precision=64)
    assert _peak_err(ref, full) > 1e-2  # two iterations are not the converged result


def test_mv_pcg_int16_in_and_out(oracle, c0_raw):
    raw = c0_raw[:3]
    raw16 = torch.clamp(raw, -32767, 32767).to(torch.int16).contiguous()
    out = _pcg(raw16, subarray_size=32, temporal_smoothing=3)
    _compare(oracle, raw16.float(), 32, 3, out)
    ref = oracle.mv_pcg(raw16.float().cpu().numpy(), 32, 3, precision=64)
    out16 = _pcg(raw16, subarray_size=32, temporal_smoothing=3, out_dtype=torch.int16)
    diff = np.abs(out16.astype(np.float64) - np.trunc(np.clip(ref, -32767, 32767)))
    assert np.mean(diff <= 1 + 2e-4 * np.abs(ref).max()) >= 0.995


def test_mv_pcg_node(c0_raw):
    from supra_b200.api import mv_beamform_pcg
    from supra_b200.nodes import Node
    from conftest import small_linear
    g = small_linear()
    raw = c0_raw[:2].contiguous()
    n = Node("BeamformingMVpcgNode", "PCG")
    n.set("subArraySize", 16)
    n.set("convergenceThresholdExponent", -5)
    out, state = n.process_raw(g, raw, delayed=True)
    ref = mv_beamform_pcg(raw, subarray_size=16, convergence_threshold=1e-5)
    torch.cuda.synchronize()
    assert state == "rf" and torch.equal(out, ref)


def test_mv_pcg_rejects_complex():
    from supra_b200.abi import SupraError
    x = torch.zeros((2, 16, 64), dtype=torch.complex64, device="cuda")
    with pytest.raises(SupraError):
        _pcg(x, subarray_size=8, out_dtype=torch.complex64)
