"""Seeded synthetic channel data for the receive path (stand-in for SUPRA's recorded mock data).

SUPRA's sample recordings are downloaded at build time and are not available here, so tests and the
benchmark use seeded synthetic raw data of the same shapes: point scatterers (and, where asked, a
fully developed speckle background) echoing a Gaussian-modulated pulse, additive Gaussian noise and
int16 quantisation. Works on CPU or GPU tensors (torch); the geometry comes from geometry.py.

Echo model (per transmit t, channel ch, scatterer p): the channel carries the element e of t's
receive aperture with e % num_channels == ch (the first one in the beamformer's element loop order,
x outer / y inner); arrival sample = (|p - s_t| + |p - e|) / (c dt) + initialDelay_t / dt, with s_t
the transmit line origin; amplitude = a_p * exp(-r_perp^2 / (2 w^2)) (Gaussian transmit beam).
Speckle: band-limited Gaussian noise with the pulse's spectrum (the limit of many random-amplitude
scatterers per resolution cell), scaled to `speckle_rms` of the point amplitude.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np


@dataclass
class PulseSpec:
    fc_hz: float = 7e6
    frac_bw: float = 0.6


def element_channel_table(geom) -> np.ndarray:
    """[num_tx, num_channels] element index feeding each channel (-1 = none)."""
    nE, nCh = geom.num_elements, geom.num_channels
    lx = geom.element_layout[0]
    table = np.full((geom.num_tx, nCh), -1, np.int64)
    # transmit t uses the aperture of the receive line whose highest-weight tx is t (subdivision 1)
    for line in geom.scanlines:
        k = int(np.argmax(line["tx_weights"]))
        t = int(line["tx"][k]["tx_idx"])
        fx, fy = (int(v) for v in line["tx"][k]["first"])
        lx_, ly_ = (int(v) for v in line["tx"][k]["last"])
        if (table[t] >= 0).any():
            continue
        for ex in range(fx, lx_ + 1):
            for ey in range(fy, ly_ + 1):
                e = ex + ey * lx
                if geom.element_to_channel is not None:
                    ch = int(geom.element_to_channel[e])
                else:
                    ch = e % nCh
                if ch >= 0 and table[t, ch] < 0:
                    table[t, ch] = e
    return table


def tx_origins(geom) -> np.ndarray:
    """[num_tx, 4]: origin x, origin elevation, initialDelay [s], lateral beam width [mm]."""
    out = np.zeros((geom.num_tx, 4))
    for line in geom.scanlines:
        k = int(np.argmax(line["tx_weights"]))
        t = int(line["tx"][k]["tx_idx"])
        out[t, 0] = line["position"][0]
        out[t, 1] = line["position"][2]
        out[t, 2] = line["tx"][k]["initial_delay"]
        out[t, 3] = 1.5
    return out


def random_scatterers(n: int, x_range, z_range, y_range=(0.0, 0.0), seed: int = 0, amplitude=1.0):
    rng = np.random.Generator(np.random.PCG64(seed))
    x = rng.uniform(*x_range, n)
    y = rng.uniform(*y_range, n) if y_range[1] > y_range[0] else np.zeros(n)
    z = rng.uniform(*z_range, n)
    a = np.full(n, amplitude, np.float64)
    return np.stack([x, y, z], 1), a


def channel_data(geom, points: np.ndarray, amps: np.ndarray, pulse: PulseSpec = PulseSpec(), noise_db: float = -40.0,
                 peak: float = 30000.0, seed: int = 0, speckle_rms: float = 0.0, device: str = "cpu",
                 quantize: bool = True, chunk: int = 16):
    """Returns a torch tensor [num_tx, num_channels, num_samples] (int16 if quantize else float32)."""
    import torch

    nTx, nCh, nS = geom.num_tx, geom.num_channels, geom.num_samples
    fs = geom.sampling_frequency_hz
    c = geom.speed_of_sound_mm_s
    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    table = torch.as_tensor(element_channel_table(geom), device=dev)
    org = torch.as_tensor(tx_origins(geom), device=dev, dtype=torch.float64)
    ec = torch.as_tensor(geom.element_centers, device=dev, dtype=torch.float64)  # x, elevation, 0
    pts = torch.as_tensor(points, device=dev, dtype=torch.float64)  # x, elevation, depth
    amp = torch.as_tensor(amps, device=dev, dtype=torch.float64)
    sigma_f = pulse.frac_bw * pulse.fc_hz / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    sigma_t = 1.0 / (2.0 * math.pi * sigma_f)
    half = int(math.ceil(3.5 * sigma_t * fs))
    offs = torch.arange(-half, half + 1, device=dev, dtype=torch.float64)
    rf = torch.zeros(nTx * nCh * nS, device=dev, dtype=torch.float32)
    valid_ch = table >= 0
    e_idx = table.clamp(min=0)
    for t0 in range(0, nTx, chunk):
        t1 = min(nTx, t0 + chunk)
        tt = torch.arange(t0, t1, device=dev)
        el = ec[e_idx[t0:t1]]                      # [T, nCh, 3]
        o = org[t0:t1]                             # [T, 4]
        # transmit path: origin (x_t, 0, elev_t) to point; receive path: point to element
        dx_t = pts[None, :, 0] - o[:, None, 0]     # [T, P]
        dy_t = pts[None, :, 1] - o[:, None, 1]
        tx_path = torch.sqrt(dx_t * dx_t + dy_t * dy_t + pts[None, :, 2] ** 2)
        beam = torch.exp(-(dx_t * dx_t + dy_t * dy_t) / (2.0 * o[:, None, 3] ** 2)) * amp[None, :]
        rx_path = torch.sqrt((pts[None, None, :, 0] - el[:, :, None, 0]) ** 2 +
                             (pts[None, None, :, 1] - el[:, :, None, 1]) ** 2 +
                             pts[None, None, :, 2] ** 2)  # [T, nCh, P]
        arrival = (tx_path[:, None, :] + rx_path) / c * fs + o[:, None, None, 2] * fs  # samples
        base = torch.floor(arrival)
        idx = base[..., None] + offs                # [T, nCh, P, K]
        tau = (idx - arrival[..., None]) / fs
        val = torch.exp(-tau * tau / (2 * sigma_t * sigma_t)) * torch.cos(2 * math.pi * pulse.fc_hz * tau)
        val = val * beam[:, None, :, None] * valid_ch[t0:t1, :, None, None]
        ok = (idx >= 0) & (idx < nS)
        lin = ((tt[:, None, None, None] * nCh + torch.arange(nCh, device=dev)[None, :, None, None]) * nS +
               idx.clamp(0, nS - 1).long())
        rf.index_add_(0, lin[ok].reshape(-1), val[ok].reshape(-1).float())
    rf = rf.view(nTx, nCh, nS)
    if speckle_rms > 0:
        white = torch.randn(nTx * nCh, 1, nS, generator=g, device=dev, dtype=torch.float32)
        k = torch.arange(-half, half + 1, device=dev, dtype=torch.float32) / fs
        kern = (torch.exp(-k * k / (2 * sigma_t * sigma_t)) * torch.cos(2 * math.pi * pulse.fc_hz * k)).view(1, 1, -1)
        kern = kern / kern.square().sum().sqrt()
        sp = torch.nn.functional.conv1d(white, kern, padding=half).view(nTx, nCh, nS)
        rf += speckle_rms * sp * valid_ch[:, :, None]
    pk = float(rf.abs().max().item()) or 1.0
    noise_std = pk * 10.0 ** (noise_db / 20.0)
    rf += noise_std * torch.randn(rf.shape, generator=g, device=dev, dtype=torch.float32)
    if not quantize:
        return rf
    scale = peak / float(rf.abs().max().item())
    return torch.round(rf * scale).clamp(-32767, 32767).to(torch.int16)


def c0_frame(seed: int = 0, device: str = "cpu", num_samples: int = 2048):
    """Config 0: 128-element linear probe, 0.3 mm, 7 MHz, 40 MHz, 64-channel aperture, 20 scatterers
    at x ~ U(array), z ~ U[5, 50] mm, -40 dB noise, int16 (peak 30000)."""
    from .geometry import linear_probe_geometry

    geom = linear_probe_geometry(128, 0.3, 64, num_samples, 40e6, aperture=64, focus_mm=20.0)
    pts, amps = random_scatterers(20, (-19.05, 19.05), (5.0, 50.0), seed=seed)
    rf = channel_data(geom, pts, amps, PulseSpec(7e6, 0.6), -40.0, 30000.0, seed=seed, device=device)
    return geom, rf
