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
