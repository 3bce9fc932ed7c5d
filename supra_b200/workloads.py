"""Synthetic workloads of the named benchmark configurations.

c1 ("batched streaming 2D DAS + IQ"): 64 frames per launch drawn from three linear probes — 64
elements / 1024 samples, 128 / 2048, 192 / 3072 — all 0.3 mm pitch, 7 MHz, fs 40 MHz, one focused
transmit per element, 64-channel receive aperture, int16. Frame k uses probe k mod 3 (22 + 21 + 21
frames). Each frame: 30 seeded point scatterers and a fully developed speckle background (the
many-scatterer limit of 200k random-amplitude scatterers: band-limited Gaussian noise with the
pulse spectrum), -40 dB noise, int16. IQ: 5 MHz mixing, 32-tap low-pass (2.5 MHz), decimation 4.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import torch

from . import synth
from .geometry import linear_probe_geometry

C1_PROBES = [(64, 1024), (128, 2048), (192, 3072)]
C1_FRAMES = 64


@dataclass
class C1Workload:
    geometries: list
    frame_probe: List[int]
    rf: List[torch.Tensor]

    @property
    def beamformed_px(self) -> int:
        return sum(self.geometries[p].num_rx * self.geometries[p].num_depths for p in self.frame_probe)

    @property
    def rf_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.rf)

    def iq_bytes(self, decimation=4) -> int:
        return sum(self.geometries[p].num_rx * (self.geometries[p].num_depths // decimation) * 8 for p in self.frame_probe)


def c1_geometries():
    return [linear_probe_geometry(n, 0.3, 64, ns, 40e6, aperture=64, focus_mm=20.0) for n, ns in C1_PROBES]


def c1_frame(geom, seed: int, device="cuda") -> torch.Tensor:
    half = geom.element_centers[-1, 0]
    depth = geom.depth_mm
    pts, amps = synth.random_scatterers(30, (-half, half), (2.0, depth), seed=seed)
    return synth.channel_data(geom, pts, amps, synth.PulseSpec(7e6, 0.6), noise_db=-40.0, peak=30000.0, seed=seed,
                              speckle_rms=0.1, device=device)


def c1_workload(num_frames: int = C1_FRAMES, device="cuda", seed0: int = 1000) -> C1Workload:
    geoms = c1_geometries()
    probe = [k % 3 for k in range(num_frames)]
    rf = [c1_frame(geoms[p], seed0 + k, device) for k, p in enumerate(probe)]
    return C1Workload(geoms, probe, rf)


# c2 ("3D matrix-probe DAS"): 32 x 32 elements at 0.3 mm, fs 20 MHz, 32 x 32 focused scanlines,
# 16 x 16-channel receive sub-aperture, 1024 samples, int16 (1024 transmits x 256 channels x 1024
# samples = 512 MB per volume). Timing only: seeded uniform int16 channel data of that shape.
def c2_geometry():
    from .geometry import matrix_probe_geometry
    return matrix_probe_geometry()


def c2_volume(geom, seed: int = 0, device="cuda") -> torch.Tensor:
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    return torch.randint(-3000, 3001, (geom.num_tx, geom.num_channels, geom.num_samples), generator=gen,
                         dtype=torch.int16, device=device)


# c3 ("2D minimum variance on complex IQ"): 128-element probe received on all 128 channels, c0's
# scatterer generator plus two off-axis interferers at +6 dB, raw-delayed (RawDelay, FP32
# [128 lines][128 channels][2048 depths]) and mixed to complex baseband at 7 MHz (zeros outside the
# aperture stay exactly zero, so the per-sample aperture of the reference is kept). L = 32, +-5
# samples, loading trace / (100 L).
C3_L, C3_T, C3_LOADING = 32, 5, 0.01


def c3_raw_delayed(seed: int = 0, device="cuda"):
    from .api import RxBeamformer
    geom = linear_probe_geometry(128, 0.3, 128, 2048, 40e6, aperture=128, focus_mm=20.0)
    pts, amps = synth.random_scatterers(20, (-19.05, 19.05), (5.0, 39.0), seed=seed)
    inter = torch.tensor([[-15.0, 0.0, 20.0], [14.0, 0.0, 30.0]], dtype=torch.float64).numpy()
    import numpy as np
    pts = np.concatenate([pts, inter])
    amps = np.concatenate([amps, np.full(2, 2.0 * float(np.max(np.abs(amps))))])
    rf = synth.channel_data(geom, pts, amps, synth.PulseSpec(7e6, 0.6), -40.0, 30000.0, seed=seed, device=device)
    raw = RxBeamformer(geom).raw_delay(rf, 1.0, window_type=1)
    raw[~(raw.abs() < 1e30)] = 0.0  # RawDelay's clamped 0/0 samples at depth 0
    n = torch.arange(raw.shape[2], device=raw.device, dtype=torch.float64)
    mix = torch.exp(-2j * np.pi * 7e6 / 40e6 * n).to(torch.complex64)
    return geom, (raw.to(torch.complex64) * mix).contiguous()


# c4 ("differentiable DAS"): 16 frames on c0's geometry, FP32 channel data.
def c4_batch(frames: int = 16, device="cuda"):
    g, rf0 = synth.c0_frame(0, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(4)
    rf = rf0.float().unsqueeze(0).repeat(frames, 1, 1, 1)
    rf = rf + 30.0 * torch.randn(rf.shape, generator=gen, device=device)
    return g, rf.contiguous()
