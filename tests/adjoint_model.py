"""FP64 model of the apodised 2D DAS that is smooth in the speed of sound, for finite differences.

The library (and the reference it follows) converts positions to DT space in FP32, so its output
moves in steps of one float rounding as c changes: a 10 mm/s step shifts a 4 mm position by about
100 ulp, and the rounding of each evaluation leaves ~1% noise in a finite difference. This model
takes the discrete decisions (aperture membership, window weight, highest-weight transmit) exactly
as the FP32 path does at the nominal c, then evaluates delays in FP64 directly from the mm
geometry, tau = t0 / dt + (|e - p(d)| + d) / (c dt), so that central differences in c are clean.
"""
import numpy as np


def _f32(x):
    return np.float32(x)


def decisions(geom, c_mm_s, lut, f_number=1.0):
    """Per (line, depth): list of (element, channel, w) with the FP32 path's aperture test and
    nearest-LUT window weight."""
    dt = 1.0 / geom.sampling_frequency_hz
    factor = 1.0 / (c_mm_s * dt)
    xe = (geom.element_x.astype(np.float64) * factor).astype(np.float32)
    dep = (geom.depths.astype(np.float64) * factor).astype(np.float32)
    F = _f32(f_number)
    cf, dtf = _f32(c_mm_s), _f32(dt)
    out = []
    for l, s in enumerate(geom.scanlines):
        k = int(np.argmax(s["tx_weights"]))
        x = _f32(s["position"][0] * factor)
        maxd = _f32(s["max_element_distance"][0] * factor)
        first, last = int(s["tx"][k]["first"][0]), int(s["tx"][k]["last"][0])
        per_depth = []
        for r in range(geom.num_depths):
            d = dep[r]
            aDT = _f32(_f32(_f32(_f32(_f32(d * dtf) * cf) / _f32(2 * F)) / cf) / dtf)
            with np.errstate(divide="ignore"):
                inv = _f32(_f32(1.0) / min(aDT, maxd))
            terms = []
            for e in range(first, last):
                ch = e % geom.num_channels
                dx = _f32(xe[e] - x)
                if abs(dx) <= aDT:
                    rel = _f32(dx * inv) if abs(dx) > 0 or np.isfinite(inv) else _f32(np.nan)
                    # fminf(fmaxf(NaN, -1), 1) = -1 on the device (depth 0: 0 * inf)
                    rel = _f32(-1) if np.isnan(rel) else min(max(rel, _f32(-1)), _f32(1))
                    idx = int(np.floor(_f32(31.5) * _f32(rel + _f32(1)) + 0.5))
                    terms.append((e, ch, float(lut[idx])))
            per_depth.append(terms)
        out.append((k, per_depth))
    return out


def forward(geom, rf, apod, dec, c_mm_s):
    """FP64 forward [num_depths][num_rx] with the given decisions."""
    dt = 1.0 / geom.sampling_frequency_hz
    nS = geom.num_samples
    out = np.zeros((geom.num_depths, geom.num_rx))
    for l, (k, per_depth) in enumerate(dec):
        s = geom.scanlines[l]
        t0 = s["tx"][k]["initial_delay"] / dt
        tx = int(s["tx"][k]["tx_idx"])
        px, dirx, diry = s["position"][0], s["direction"][0], s["direction"][1]
        for r, terms in enumerate(per_depth):
            if not terms:
                continue
            d = float(geom.depths[r])
            num = den = 0.0
            for e, ch, w in terms:
                W = w * float(apod[e])
                den += W
                dx = float(geom.element_x[e]) - (px + dirx * d)
                tau = t0 + (np.hypot(dx, diry * d) + d) / (c_mm_s * dt)
                i = int(np.floor(tau))
                f = tau - i
                if 0 <= i < nS - 1:
                    num += W * ((1 - f) * rf[tx, ch, i] + f * rf[tx, ch, i + 1])
            out[r, l] = num / den * len(terms) if den != 0.0 else np.nan
    return out


def grad_c(geom, rf, apod, dec, c_mm_s, gout):
    """d/dc of sum(gout * forward): sum g n / D sum_e W_e (rf[i+1] - rf[i]) dtau/dc."""
    dt = 1.0 / geom.sampling_frequency_hz
    nS = geom.num_samples
    total = 0.0
    for l, (k, per_depth) in enumerate(dec):
        s = geom.scanlines[l]
        t0 = s["tx"][k]["initial_delay"] / dt
        tx = int(s["tx"][k]["tx_idx"])
        px, dirx, diry = s["position"][0], s["direction"][0], s["direction"][1]
        for r, terms in enumerate(per_depth):
            g = gout[r, l]
            if not terms or g == 0.0:
                continue
            d = float(geom.depths[r])
            den = sum(w * float(apod[e]) for e, _, w in terms)
            acc = 0.0
            for e, ch, w in terms:
                dx = float(geom.element_x[e]) - (px + dirx * d)
                path = np.hypot(dx, diry * d) + d
                tau = t0 + path / (c_mm_s * dt)
                i = int(np.floor(tau))
                if 0 <= i < nS - 1:
                    acc += w * float(apod[e]) * (rf[tx, ch, i + 1] - rf[tx, ch, i]) * (-path / (c_mm_s * c_mm_s * dt))
            total += g * len(terms) / den * acc
    return total


class SmoothModelTorch:
    """The same FP64 model as forward() (decisions of the FP32 path at the nominal c, delays in FP64
    from the mm geometry), vectorised with torch over every (scanline, depth, element) of the
    highest-weight transmit, for geometries where the Python loops are too slow. Linear arrays
    (the element's lateral position and the scanline's lateral direction only)."""

    def __init__(self, geom, c_mm_s, lut, f_number=1.0, device="cuda"):
        import torch
        f32, f64 = torch.float32, torch.float64
        dt = 1.0 / geom.sampling_frequency_hz
        factor = 1.0 / (c_mm_s * dt)
        self.geom, self.dt, self.device = geom, dt, device
        nE, nD, nRx, nCh = geom.num_elements, geom.num_depths, geom.num_rx, geom.num_channels
        xe = torch.tensor(geom.element_x.astype(np.float64) * factor, dtype=f64, device=device).to(f32)
        dep = torch.tensor(geom.depths.astype(np.float64) * factor, dtype=f64, device=device).to(f32)
        dtf = torch.tensor(np.float32(dt), device=device)
        cf = torch.tensor(np.float32(c_mm_s), device=device)
        two_f = torch.tensor(np.float32(2 * np.float32(f_number)), device=device)
        aDT = (((dep * dtf) * cf) / two_f / cf) / dtf  # [nD], float32, one rounding per operation
        lut_t = torch.tensor(np.asarray(lut, np.float32), device=device)
        lines = geom.scanlines
        ks = [int(np.argmax(s["tx_weights"])) for s in lines]
        first = np.array([int(s["tx"][k]["first"][0]) for s, k in zip(lines, ks)])
        last = np.array([int(s["tx"][k]["last"][0]) for s, k in zip(lines, ks)])
        nA = int(max(1, (last - first).max()))
        e_idx = torch.tensor(first, device=device)[:, None] + torch.arange(nA, device=device)[None, :]  # [nRx][nA]
        in_ap = e_idx < torch.tensor(last, device=device)[:, None]
        e_c = torch.clamp(e_idx, max=nE - 1)
        x = torch.tensor([np.float32(s["position"][0] * factor) for s in lines], device=device)
        maxd = torch.tensor([np.float32(s["max_element_distance"][0] * factor) for s in lines], device=device)
        dx = xe[e_c] - x[:, None]  # [nRx][nA] float32
        inv = 1.0 / torch.minimum(aDT[None, :], maxd[:, None])  # [nRx][nD]
        member = (dx.abs()[:, None, :] <= aDT[None, :, None]) & in_ap[:, None, :]  # [nRx][nD][nA]
        rel = dx[:, None, :] * inv[:, :, None]
        rel = torch.where(torch.isnan(rel), torch.full_like(rel, -1.0), rel).clamp(-1.0, 1.0)
        v = (rel + 1.0) * torch.tensor(np.float32(31.5), device=device)
        idx = torch.floor(v.to(f64) + 0.5).long()  # roundf of a non-negative float
        w = lut_t[idx].to(f64) * member.to(f64)
        self.member, self.w = member, w
        self.count = member.sum(dim=2).to(f64)  # [nRx][nD]
        self.e = e_c
        self.ch = (e_c % nCh)
        self.tx = torch.tensor([int(s["tx"][k]["tx_idx"]) for s, k in zip(lines, ks)], device=device)
        self.t0 = torch.tensor([s["tx"][k]["initial_delay"] / dt for s, k in zip(lines, ks)], dtype=f64,
                               device=device)
        self.px = torch.tensor([s["position"][0] for s in lines], dtype=f64, device=device)
        self.dirx = torch.tensor([s["direction"][0] for s in lines], dtype=f64, device=device)
        self.diry = torch.tensor([s["direction"][1] for s in lines], dtype=f64, device=device)
        self.xe_mm = torch.tensor(geom.element_x.astype(np.float64), device=device)
        self.d_mm = torch.tensor(geom.depths.astype(np.float64), device=device)

    def weight_ratio(self):
        """Sum of the aperture's window weights over the number of aperture elements, per pixel:
        [num_depths][num_rx] (0 for an empty aperture). The normalisation n / D amplifies every term
        of a pixel whose ratio is small."""
        import torch
        den = self.w.sum(dim=2)
        r = torch.where(self.count > 0, den / torch.clamp(self.count, min=1.0), torch.zeros_like(den))
        return r.T.contiguous()

    def tau_range(self, c_mm_s):
        """(smallest, largest) delay in samples over each pixel's aperture elements at c:
        [num_depths][num_rx] each (+inf / -inf for an empty aperture)."""
        import torch
        lat = self.xe_mm[self.e][:, None, :] - (self.px[:, None, None] + self.dirx[:, None, None] * self.d_mm[None, :, None])
        path = torch.hypot(lat, (self.diry[:, None] * self.d_mm[None, :])[:, :, None]) + self.d_mm[None, :, None]
        tau = self.t0[:, None, None] + path / (c_mm_s * self.dt)
        inf = torch.full_like(tau, float("inf"))
        lo = torch.where(self.member, tau, inf).amin(dim=2)
        hi = torch.where(self.member, tau, -inf).amax(dim=2)
        return lo.T.contiguous(), hi.T.contiguous()

    def forward(self, rf, c_mm_s, apod=None, cells_of=None):
        """rf [num_tx][num_channels][num_samples] (torch, any float type, on the model's device) ->
        FP64 image [num_depths][num_rx] (0 where no element is in the aperture, NaN where the weights
        of the aperture's elements sum to 0). cells_of: a speed of sound whose sample cells (the
        interpolation's index i = floor(tau)) are kept for every term, so that each term is linear in
        tau and the image is smooth in c; its derivative at c = cells_of is the forward's."""
        import torch
        g = self.geom
        nS = g.num_samples
        W = self.w if apod is None else self.w * apod.to(torch.float64)[self.e][:, None, :]
        den = W.sum(dim=2)
        lat = self.xe_mm[self.e][:, None, :] - (self.px[:, None, None] + self.dirx[:, None, None] * self.d_mm[None, :, None])
        path = torch.hypot(lat, (self.diry[:, None] * self.d_mm[None, :])[:, :, None]) + self.d_mm[None, :, None]
        tau = self.t0[:, None, None] + path / (c_mm_s * self.dt)
        if cells_of is None:
            i = torch.floor(tau)
        else:
            i = torch.floor(self.t0[:, None, None] + path / (cells_of * self.dt))
        fr = tau - i
        i = i.long()
        ok = (i >= 0) & (i < nS - 1)
        ic = torch.clamp(i, 0, nS - 2)
        base = (self.tx[:, None, None] * g.num_channels + self.ch[:, None, :]) * nS
        flat = rf.reshape(-1).to(torch.float64)
        v0 = flat[base + ic]
        v1 = flat[base + ic + 1]
        num = (W * torch.where(ok, (1 - fr) * v0 + fr * v1, torch.zeros_like(fr))).sum(dim=2)
        out = num / den * self.count  # [nRx][nD]
        out = torch.where(self.count == 0, torch.zeros_like(out), out)  # no element in the aperture: 0
        return out.T.contiguous()
