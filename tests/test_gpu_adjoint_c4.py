"""The differentiable DAS at its stated shape: 16 frames of the 128-element c0 geometry (FP32 channel
data [16][128 transmits][64 channels][2048 samples], 1 GiB), the loss 1/2 ||env(DAS(rf; apod, c)) -
target||^2 with the 64-tap Hilbert FIR envelope, and the target rendered at a seeded true speed of
sound c_true ~ U[1450, 1600] m/s. The loss covers the pixels whose aperture delays stay inside the
record (where a delay crosses the record's end, a term jumps between 0 and a sample value and the
loss is not continuous in c) and whose window weights average at least 0.25 (shallow pixels whose
aperture holds only elements at the window's edge are amplified without bound by the normalisation). The forward and the gradients run through the libtorch autograd
Functions (torch.ops.supra_b200.das_apod / .envelope) at c = 1540 m/s.

Checks, with the tolerances written here:
  * all three gradients against the FP64 reference chain (the FP64 envelope backward, then the
    oracle's FP64 transpose of the DAS with the same discrete decisions), per frame for the channel
    data. Two chains: (a) evaluated at the library's own FP32 forward output, so that only the
    backward pass differs: 1e-3 of the largest entry (grad_rf, grad_apod), 1e-3 relative (grad_c);
    (b) the all-FP64 chain from the channel data. In (b) the forward's FP32 rounding (about 1e-7 of
    the peak) enters the envelope derivative s / env, which is ill-conditioned at pixels whose
    envelope is far below |env - target|; the measured deviation is printed and bounded by 1e-2 of
    the largest entry (grad_rf) and 1e-2 relative (grad_c);
  * grad_apod against central differences of the FP64 forward + envelope + loss, step 1e-4, for
    eight elements: 1e-3 of the largest entry;
  * grad_c against central differences at the stated step 1e-2 m/s (10 mm/s) of an FP64 model with
    the decisions and sample cells of c0 kept (smooth in c, the same derivative at c0): 1e-3
    relative. The forward itself interpolates linearly between samples, so it is only piecewise
    smooth in c: a 10 mm/s step moves a delay of ~4000 samples by ~0.03 samples, and the terms whose
    delay crosses a sample boundary inside the step make its central difference deviate from the
    derivative at c; that deviation is printed.
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
    hh = torch.zeros(2 * (N // 2) + 1, dtype=torch.float64, device=x.device)
    hh[:min(N, len(hh))] = torch.from_numpy(np.asarray(taps[:len(hh)], np.float64)).to(x.device)
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
    # The loss covers the pixels whose aperture delays all stay inside the record (1 <= tau <= nS - 3 at
    # c0): where a delay crosses the record's end a term jumps between 0 and a sample value, so the loss
    # would not be continuous in c there (a finite difference in c would pick up the jumps)
    import adjoint_model as M
    from oracle import oracle as O
    model = M.SmoothModelTorch(g, c0, O.window_lut(1), device="cuda")
    tlo, thi = model.tau_range(c0)
    # and whose aperture weights average at least 0.25: at shallow depths an aperture of elements at
    # the window's edge has weights near 0, and the normalisation n / D makes such a pixel, and its
    # derivatives, arbitrarily large
    inrec = (tlo >= 1.0) & (thi <= g.num_samples - 3.0) & (model.weight_ratio() >= 0.25)
    rf_g = rf.clone().requires_grad_(True)
    ap = apod.clone().requires_grad_(True)
    c = torch.tensor(c0, dtype=torch.float64, device="cuda", requires_grad=True)
    s = das_apod(bf, rf_g, ap, c)
    # no gradient through the reference's clamped 0/0 pixels, nor through pixels outside the record
    valid = (s.detach().abs() < 1e30) & inrec[None]
    s = torch.where(valid, s, torch.zeros_like(s))
    loss = 0.5 * ((envelope(s, hil) - target) ** 2).sum()
    loss.backward()
    torch.cuda.synchronize()
    return {"g": g, "rf": rf.cpu().numpy(), "target": target.double().cpu(), "valid": valid.cpu(), "c0": c0,
            "s32": s.detach().double().cpu(),
            "c_true": c_true, "loss": float(loss.detach()), "grad_rf": rf_g.grad, "grad_apod": ap.grad.cpu().numpy(),
            "grad_c": float(c.grad), "model": model, "inrec_frac": float(inrec.float().mean())}


def _loss64(oracle, case, apod, c_mm_s, taps):
    """The FP64 forward + envelope + loss over the 16 frames (the same valid-pixel mask)."""
    g = case["g"]
    tot = 0.0
    for f in range(case["rf"].shape[0]):
        s = torch.from_numpy(oracle.das(g, case["rf"][f], 1.0, c_mm_s=c_mm_s, window=1, apod=apod, precision=64))
        # the pixels the forward at c0 clamps, and any 0/0 of the FP64 forward at a shifted c (depth 0)
        s = torch.where(case["valid"][f] & torch.isfinite(s), s, torch.zeros_like(s))
        tot += 0.5 * float(((_env64(s, taps) - case["target"][f]) ** 2).sum())
    return tot


def test_c4_gradients_vs_fp64_chain(oracle, c4):
    from supra_b200.api import fir_design
    g = c4["g"]
    taps = fir_design(N_TAPS, 3, 2)
    apod = np.ones(g.num_elements, np.float32)
    res = {}
    for chain in ("at_fp32_forward", "all_fp64"):
        tot_ap = np.zeros(g.num_elements)
        tot_c = 0.0
        worst_rf = 0.0
        for f in range(c4["rf"].shape[0]):
            vf = c4["valid"][f]
            if chain == "all_fp64":
                s0 = torch.from_numpy(oracle.das(g, c4["rf"][f], 1.0, c_mm_s=c4["c0"], window=1, apod=apod,
                                                 precision=64))
            else:
                s0 = c4["s32"][f].clone()
            s64 = s0.requires_grad_(True)
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
        res[chain] = (worst_rf, err_ap, err_c)
        print(f"c4 vs FP64 chain {chain} (c_true {c4['c_true'] / 1e3:.2f} m/s): grad_rf {worst_rf:.3g} of peak "
              f"(worst frame), grad_apod {err_ap:.3g} of peak, grad_c {err_c:.3g} relative")
    rf_a, ap_a, c_a = res["at_fp32_forward"]
    assert rf_a <= 1e-3 and ap_a <= 1e-3 and c_a <= 1e-3
    rf_b, ap_b, c_b = res["all_fp64"]
    assert rf_b <= 1e-2 and ap_b <= 1e-3 and c_b <= 1e-2


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
    """Central differences in c at the stated step 1e-2 m/s (10 mm/s) of three forwards:
    (1) the FP64 model with the decisions of c0 and each term's sample cell of c0 kept (every term
        linear in its delay, the image smooth in c; its derivative at c0 is the forward's): must match
        the gradient within 1e-3;
    (2) the same model with the sample cells recomputed at each c (the forward's own linear
        interpolation), and (3) the oracle's forward, which also recomputes the FP32 decisions and
        DT-space positions at each c: printed. The interpolation's slope jumps at every sample
        boundary (a 7 MHz carrier sampled at 40 MHz changes slope by about as much as its slope), and
        a 10 mm/s step moves the delays by up to ~0.03 samples, so the terms that cross a boundary
        inside the step make (2) and (3) deviate from the derivative; that deviation shrinks only as
        the step approaches the distance from the delays to their nearest sample boundary."""
    from supra_b200.api import fir_design
    taps = fir_design(N_TAPS, 3, 2)
    g = c4["g"]
    apod = np.ones(g.num_elements, np.float32)
    gc = c4["grad_c"]
    c0 = c4["c0"]
    h = 10.0  # mm/s = 1e-2 m/s
    model = c4["model"]
    valid = c4["valid"].cuda()
    target = c4["target"].cuda()
    rfs = [torch.from_numpy(c4["rf"][f]).cuda() for f in range(c4["rf"].shape[0])]

    def loss_model(c, cells_of):
        tot = 0.0
        for f, rf in enumerate(rfs):
            s = model.forward(rf, c, cells_of=cells_of)
            s = torch.where(valid[f] & torch.isfinite(s), s, torch.zeros_like(s))
            tot += 0.5 * float(((_env64(s, taps) - target[f]) ** 2).sum())
        return tot

    fd_cells = (loss_model(c0 + h, c0) - loss_model(c0 - h, c0)) / (2 * h)
    fd_smooth = (loss_model(c0 + h, None) - loss_model(c0 - h, None)) / (2 * h)
    fd_oracle = (_loss64(oracle, c4, apod, c0 + h, taps) - _loss64(oracle, c4, apod, c0 - h, taps)) / (2 * h)
    dev_cells = abs(gc - fd_cells) / abs(fd_cells)
    dev_smooth = abs(gc - fd_smooth) / abs(fd_smooth)
    dev_oracle = abs(gc - fd_oracle) / abs(fd_oracle)
    print(f"c4 loss over {c4['inrec_frac'] * 100:.1f}% of the pixels (aperture delays inside the record)")
    print(f"c4 grad_c {gc:.6g}; central differences at 1e-2 m/s: cells of c0 kept {fd_cells:.6g} (deviation "
          f"{dev_cells:.3g}), cells recomputed {fd_smooth:.6g} (deviation {dev_smooth:.3g}), the oracle's "
          f"FP32-decision forward {fd_oracle:.6g} (deviation {dev_oracle:.3g})")
    assert dev_cells <= 1e-3
