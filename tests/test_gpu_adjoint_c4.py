"""The differentiable DAS at its stated shape: 16 frames of the 128-element c0 geometry (FP32 channel
data [16][128 transmits][64 channels][2048 samples], 1 GiB), the loss 1/2 ||env(DAS(rf; apod, c)) -
target||^2 with the 64-tap Hilbert FIR envelope, and the target rendered at a seeded true speed of
sound c_true ~ U[1450, 1600] m/s. The forward and the gradients run through the libtorch autograd
Functions (torch.ops.supra_b200.das_apod / .envelope) at c = 1540 m/s.

Checks, with the tolerances written here:
  * all three gradients against the FP64 reference chain (the FP64 envelope backward, then the
    oracle's FP64 transpose of the DAS with the same discrete decisions), per frame for the channel
    data: 1e-3 of the largest entry (grad_rf, grad_apod), 1e-3 relative (grad_c);
  * grad_apod against central differences of the FP64 forward + envelope + loss, step 1e-4, for
    eight elements: 1e-3 of the largest entry;
  * grad_c against central differences at the stated step 1e-2 m/s (10 mm/s). The forward
    interpolates linearly between samples, so it is only piecewise smooth in c: a 10 mm/s step
    moves a delay of ~4000 samples by ~0.03 samples, and the terms whose delay crosses a sample
    boundary inside the step make the central difference deviate from the derivative at c. The
    deviation is printed; the test bounds it by 2e-2 relative.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N_TAPS = 64


def _env64(x, taps):
    """Hilbert FIR envelope in float64 torch over the depth axis of [depth][line] (tap N of an
    even-length filter reads 0, as the kernel)."""
    N = len(taps)
    hh = torch.zeros(2 * (N // 2) + 1, dtype=torch.float64)
    hh[:min(N, len(hh))] = torch.from_numpy(np.asarray(taps[:len(hh)], np.float64))
    nS = x.shape[0]
    acc = torch.zeros_like(x)
    for fe in range(len(hh)):
        sh = fe - N // 2
        if sh >= 0:
            acc[:nS - sh] = acc[:nS - sh] + x[sh:] * hh[fe]
        else:
            acc[-sh:] = acc[-sh:] + x[:nS + sh] * hh[fe]
    return torch.sqrt(torch.clamp(x * x + acc * acc, min=1e-300))


@pytest.fixture(scope="module")
def c4():
    from supra_b200 import workloads as W
    from supra_b200.api import HilbertFirEnvelope, RxBeamformer
    from supra_b200.autograd import das_apod, envelope
    g, rf = W.c4_batch(frames=16, device="cuda")
    bf = RxBeamformer(g)
    hil = HilbertFirEnvelope(N_TAPS)
    rng = np.random.Generator(np.random.PCG64(44))
    c_true = float(rng.uniform(1450.0, 1600.0)) * 1e3  # mm/s
    apod = torch.ones(g.num_elements, device="cuda")
    with torch.no_grad():
        t = das_apod(bf, rf, apod, torch.tensor(c_true, dtype=torch.float64, device="cuda"))
        t = torch.where(t.abs() < 1e30, t, torch.zeros_like(t))
        target = envelope(t, hil)
    c0 = 1540e3
    rf_g = rf.clone().requires_grad_(True)
    ap = apod.clone().requires_grad_(True)
    c = torch.tensor(c0, dtype=torch.float64, device="cuda", requires_grad=True)
    s = das_apod(bf, rf_g, ap, c)
    valid = s.detach().abs() < 1e30  # no gradient through the reference's clamped 0/0 pixels
    s = torch.where(valid, s, torch.zeros_like(s))
    loss = 0.5 * ((envelope(s, hil) - target) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return {"g": g, "rf": rf.cpu().numpy(), "target": target.double().cpu(), "valid": valid.cpu(), "c0": c0,
            "c_true": c_true, "loss": float(loss), "grad_rf": rf_g.grad, "grad_apod": ap.grad.cpu().numpy(),
            "grad_c": float(c.grad)}


def _loss64(oracle, case, apod, c_mm_s, taps):
    """The FP64 forward + envelope + loss over the 16 frames (the same valid-pixel mask)."""
    g = case["g"]
    tot = 0.0
    for f in range(case["rf"].shape[0]):
        s = torch.from_numpy(oracle.das(g, case["rf"][f], 1.0, c_mm_s=c_mm_s, window=1, apod=apod, precision=64))
        s = torch.where(case["valid"][f], s, torch.zeros_like(s))
        tot += 0.5 * float(((_env64(s, taps) - case["target"][f]) ** 2).sum())
    return tot


def test_c4_gradients_vs_fp64_chain(oracle, c4):
    from supra_b200.api import fir_design
    g = c4["g"]
    taps = fir_design(N_TAPS, 3, 2)
    apod = np.ones(g.num_elements, np.float32)
    tot_ap = np.zeros(g.num_elements)
    tot_c = 0.0
    worst_rf = 0.0
    for f in range(c4["rf"].shape[0]):
        s64 = torch.from_numpy(oracle.das(g, c4["rf"][f], 1.0, c_mm_s=c4["c0"], window=1, apod=apod,
                                          precision=64)).requires_grad_(True)
        vf = c4["valid"][f]
        e64 = _env64(torch.where(vf, s64, torch.zeros_like(s64)), taps)
        (0.5 * ((e64 - c4["target"][f]) ** 2).sum()).backward()
        gs = torch.where(vf, s64.grad, torch.zeros_like(s64.grad)).numpy()
        grf, gap, gc = oracle.das_adjoint64(g, c4["rf"][f], apod, gs, c_mm_s=c4["c0"])
        got = c4["grad_rf"][f].cpu().numpy()
        worst_rf = max(worst_rf, float(np.max(np.abs(got - grf)) / np.max(np.abs(grf))))
        tot_ap += gap
        tot_c += gc
    err_ap = float(np.max(np.abs(c4["grad_apod"] - tot_ap)) / np.max(np.abs(tot_ap)))
    err_c = abs(c4["grad_c"] - tot_c) / abs(tot_c)
    print(f"c4 vs FP64 chain (c_true {c4['c_true'] / 1e3:.2f} m/s): grad_rf {worst_rf:.3g} of peak (worst frame), "
          f"grad_apod {err_ap:.3g} of peak, grad_c {err_c:.3g} relative")
    assert worst_rf <= 1e-3
    assert err_ap <= 1e-3
    assert err_c <= 1e-3


def test_c4_grad_apod_finite_differences(oracle, c4):
    from supra_b200.api import fir_design
    g = c4["g"]
    taps = fir_design(N_TAPS, 3, 2)
    h = 1e-4
    elements = [8, 30, 50, 63, 64, 77, 100, 120]
    fd = []
    for e in elements:
        ap = np.ones(g.num_elements, np.float32)
        ap[e] = np.float32(1.0 + h)
        lp = _loss64(oracle, c4, ap, c4["c0"], taps)
        ap[e] = np.float32(1.0 - h)
        lm = _loss64(oracle, c4, ap, c4["c0"], taps)
        fd.append((lp - lm) / (float(np.float32(1.0 + h)) - float(np.float32(1.0 - h))))
    fd = np.array(fd)
    got = c4["grad_apod"][elements]
    err = float(np.max(np.abs(got - fd)) / np.max(np.abs(c4["grad_apod"])))
    print(f"c4 grad_apod vs central differences (step 1e-4, 8 elements): {err:.3g} of the largest entry")
    assert err <= 1e-3


def test_c4_grad_c_finite_differences_at_stated_step(oracle, c4):
    from supra_b200.api import fir_design
    taps = fir_design(N_TAPS, 3, 2)
    h = 10.0  # mm/s = 1e-2 m/s
    apod = np.ones(c4["g"].num_elements, np.float32)
    fd = (_loss64(oracle, c4, apod, c4["c0"] + h, taps) - _loss64(oracle, c4, apod, c4["c0"] - h, taps)) / (2 * h)
    dev = abs(c4["grad_c"] - fd) / abs(fd)
    print(f"c4 grad_c {c4['grad_c']:.6g} vs central difference at 1e-2 m/s {fd:.6g}: deviation {dev:.3g} relative")
    assert dev <= 2e-2
