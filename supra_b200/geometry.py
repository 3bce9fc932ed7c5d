"""Receive geometry for the B200 beamformers, built the way SUPRA's Beamformer builds it.

SUPRA computes its receive scanline parameters on the host (Beamformer/Beamformer.cpp:409-1184,
element centres Beamformer/USTransducer.cpp:179-245) and hands them to the receive nodes through
RxBeamformerParameters. This module restates that construction for linear (2D) and biphased
(matrix, 3D) scans so that callers of the C ABI, the tests and the benchmark get the same
ScanlineRxParameters3D layout; `Geometry.ctypes()` produces the `sb_geometry` struct.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import numpy as np

from .abi import SCANLINE_DTYPE, sb_geometry

M_EPS = 2.2204e-16  # SupraLib/utilities/utility.h:43


def _cround(x: float) -> float:
    """C's round(): halves away from zero (Python's round() rounds halves to even)."""
    return math.copysign(math.floor(abs(x) + 0.5), x)


def _norm(v):
    return math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])


def _normalize(v):
    n = _norm(v)
    return (v[0] / n, v[1] / n, v[2] / n)


def _dot(a, b):
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _slerp3(a, b, t):
    """SupraLib/vec.h:424-445."""
    omega = math.acos(max(-1.0, min(1.0, _dot(a, b))))
    if omega < M_EPS or t < M_EPS:
        return a
    if 1.0 - t < M_EPS:
        return b
    s = math.sin(omega)
    ka = math.sin((1.0 - t) * omega) / s
    kb = math.sin(t * omega) / s
    return (a[0] * ka + b[0] * kb, a[1] * ka + b[1] * kb, a[2] * ka + b[2] * kb)


def linear_element_centers(num_elements: int, pitch_mm: float) -> np.ndarray:
    """USTransducer::computeInternals, Linear (Beamformer/USTransducer.cpp:190-207)."""
    width = 0.0
    for _ in range(num_elements - 1):
        width += pitch_mm
    pos = -width / 2
    out = np.zeros((num_elements, 3))
    for i in range(num_elements):
        out[i] = (pos, 0.0, 0.0)
        if i < num_elements - 1:
            pos += pitch_mm
    return out


def planar_element_centers(nx: int, ny: int, pitch_x: float, pitch_y: float) -> np.ndarray:
    """USTransducer::computeInternals, Planar (Beamformer/USTransducer.cpp:209-240)."""
    wx = 0.0
    for _ in range(nx - 1):
        wx += pitch_x
    wy = 0.0
    for _ in range(ny - 1):
        wy += pitch_y
    out = np.zeros((nx * ny, 3))
    cy = -wy / 2
    for y in range(ny):
        cx = -wx / 2
        for x in range(nx):
            out[x + nx * y] = (cx, cy, 0.0)
            if x < nx - 1:
                cx += pitch_x
        if y < ny - 1:
            cy += pitch_y
    return out


def compute_aperture(layout: Tuple[int, int], size: Tuple[int, int], rel: Tuple[float, float]):
    """Beamformer::computeAperture (Beamformer/Beamformer.cpp:1147-1184); end is inclusive."""
    bx = rel[0] - (size[0] - 1) / 2
    ex = rel[0] + (size[0] - 1) / 2
    by = rel[1] - (size[1] - 1) / 2
    ey = rel[1] + (size[1] - 1) / 2
    if _cround(bx) < 0:
        bx, ex = 0.0, float(size[0] - 1)
    elif _cround(ex) > layout[0] - 1:
        ex = float(layout[0] - 1)
        bx = ex - (size[0] - 1)
    if _cround(by) < 0:
        by, ey = 0.0, float(size[1] - 1)
    elif _cround(ey) > layout[1] - 1:
        ey = float(layout[1] - 1)
        by = ey - (size[1] - 1)
    return (int(_cround(bx)), int(_cround(by))), (int(_cround(ex)), int(_cround(ey)))


@dataclass
class _Tx:
    first: Tuple[int, int]
    last: Tuple[int, int]
    position: Tuple[float, float, float]
    direction: Tuple[float, float, float]
    max_delay: float


@dataclass
class ScanSpec:
    """Parameters of SUPRA's Beamformer (the ones its XML exposes)."""
    scan_type: str = "linear"          # "linear" | "biphased"
    num_tx: Tuple[int, int] = (128, 1)
    max_aperture: Tuple[int, int] = (64, 1)
    tx_max_aperture: Tuple[int, int] = (64, 1)
    tx_focus_active: bool = True
    tx_focus_depth_mm: float = 20.0
    tx_focus_width_mm: float = 0.0
    steering_deg: Tuple[float, float] = (0.0, 0.0)
    sector_deg: Tuple[float, float] = (0.0, 0.0)
    speed_of_sound_m_s: float = 1540.0


@dataclass
class Geometry:
    """Receive geometry (RxBeamformerParameters + USRawData sizes) in host memory."""
    element_centers: np.ndarray          # [num_elements, 3] mm (double)
    element_layout: Tuple[int, int]
    num_channels: int
    num_samples: int
    num_tx: int
    rx_layout: Tuple[int, int]
    depth_mm: float
    num_depths: int
    sampling_frequency_hz: float
    speed_of_sound_mm_s: float
    scanlines: np.ndarray                # SCANLINE_DTYPE [num_rx], x fastest
    element_to_channel: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def num_elements(self) -> int:
        return int(self.element_centers.shape[0])

    @property
    def num_rx(self) -> int:
        return int(self.rx_layout[0] * self.rx_layout[1])

    @property
    def is3d(self) -> bool:
        return self.rx_layout[0] > 1 and self.rx_layout[1] > 1

    @property
    def element_x(self) -> np.ndarray:
        return self.element_centers[:, 0].astype(np.float32)

    @property
    def element_y(self) -> np.ndarray:
        return self.element_centers[:, 1].astype(np.float32)

    @property
    def depths(self) -> np.ndarray:
        """RxBeamformerParameters depth grid (Beamformer/RxBeamformerParameters.cpp:61-64)."""
        n = self.num_depths
        return np.array([np.float32(z * self.depth_mm / (n - 1)) for z in range(n)], dtype=np.float32)

    @property
    def sample_distance_mm(self) -> float:
        return self.depth_mm / (self.num_depths - 1)

    def ctypes(self) -> sb_geometry:
        ex = np.ascontiguousarray(self.element_x)
        ey = np.ascontiguousarray(self.element_y)
        dp = np.ascontiguousarray(self.depths)
        sl = np.ascontiguousarray(self.scanlines)
        keep = [ex, ey, dp, sl]
        g = sb_geometry()
        g.num_elements = self.num_elements
        g.element_layout[0], g.element_layout[1] = self.element_layout
        g.num_channels = self.num_channels
        g.num_samples = self.num_samples
        g.num_tx = self.num_tx
        g.num_rx = self.num_rx
        g.rx_layout[0], g.rx_layout[1] = self.rx_layout
        g.num_depths = self.num_depths
        g.sampling_frequency_hz = self.sampling_frequency_hz
        g.element_x_mm = ex.ctypes.data_as(C.POINTER(C.c_float))
        g.element_y_mm = ey.ctypes.data_as(C.POINTER(C.c_float))
        g.depths_mm = dp.ctypes.data_as(C.POINTER(C.c_float))
        g.scanlines = sl.ctypes.data
        if self.element_to_channel is not None:
            m = np.ascontiguousarray(self.element_to_channel, dtype=np.int32)
            keep.append(m)
            g.element_to_channel = m.ctypes.data_as(C.POINTER(C.c_int32))
        else:
            g.element_to_channel = C.POINTER(C.c_int32)()
        self._keep = keep
        return g


def _tx_scanline(centers, layout, spec: ScanSpec, active, tx_ap, start, angle) -> _Tx:
    """Beamformer::getTxScanline3D (Beamformer/Beamformer.cpp:840-1066), the parts the receive side
    uses: aperture, position, direction and the largest focusing delay (initialDelay)."""
    c_mm_s = spec.speed_of_sound_m_s * 1000.0
    (bx, by), (ex, ey) = tx_ap
    E = lambda ix, iy: tuple(centers[ix + iy * layout[0]])
    if bx == ex and by == ey:
        corners = [((0.5, 0.5), E(bx, by))]
    elif bx == ex:
        corners = [((0.5, 0.0), E(bx, by)), ((0.5, 1.0), E(ex, ey))]
    elif by == ey:
        corners = [((0.0, 0.5), E(bx, by)), ((1.0, 0.5), E(ex, ey))]
    else:
        corners = [((0.0, 0.0), E(bx, by)), ((0.0, 1.0), E(bx, ey)), ((1.0, 0.0), E(ex, by)), ((1.0, 1.0), E(ex, ey))]
    start3 = (start[0], start[1], 0.0)
    d = _normalize((math.tan(angle[0]), math.tan(angle[1]), 1.0))
    px = _normalize(tuple(u - d[i] * _dot((1.0, 0.0, 0.0), d) for i, u in enumerate((1.0, 0.0, 0.0))))
    py = _normalize(tuple(u - d[i] * _dot((0.0, 1.0, 0.0), d) for i, u in enumerate((0.0, 1.0, 0.0))))
    fd, fw = spec.tx_focus_depth_mm, spec.tx_focus_width_mm

    def focus_vec(rel, pos):
        off = tuple(((rel[0] - 0.5) * fw) * px[i] + ((rel[1] - 0.5) * fw) * py[i] for i in range(3))
        return tuple(start3[i] + fd * d[i] + off[i] - pos[i] for i in range(3))

    max_delay = 0.0
    if spec.tx_focus_active:
        max_tt = 0.0
        for rel, pos in corners:
            max_tt = max(max_tt, _norm(focus_vec(rel, pos)) / c_mm_s)
        for ix in range(bx, ex + 1):
            for iy in range(by, ey + 1):
                rx_ = (ix - bx) / max(ex - bx, 1)
                ry_ = (iy - by) / max(ey - by, 1)
                if ex == bx:
                    rx_ = 0.5
                if ey == by:
                    ry_ = 0.5
                tt = _norm(focus_vec((rx_, ry_), E(ix, iy))) / c_mm_s
                max_delay = max(max_delay, max_tt - tt)
    else:
        max_tt = 0.0
        for _, pos in corners:
            v = tuple((start3[i] - pos[i]) * d[i] for i in range(3))
            max_tt = max(max_tt, (v[0] + v[1] + v[2] + fd) / c_mm_s)
        for ix in range(bx, ex + 1):
            for iy in range(by, ey + 1):
                pos = E(ix, iy)
                v = tuple((start3[i] - pos[i]) * d[i] for i in range(3))
                tt = (v[0] + v[1] + v[2] + fd) / c_mm_s
                max_delay = max(max_delay, max_tt - tt)
    return _Tx(first=active[0], last=active[1], position=(start[0], 0.0, start[1]),
               direction=(d[0], d[2], d[1]), max_delay=max_delay)


def _rx_interpolated(centers, layout, idx, txs: List[_Tx], interp):
    """Beamformer::getRxScanline3DInterpolated (Beamformer/Beamformer.cpp:1068-1135)."""
    rec = np.zeros((), dtype=SCANLINE_DTYPE)
    ix, iy = interp
    w = ((1 - ix) * (1 - iy), ix * (1 - iy), (1 - ix) * iy, ix * iy)
    for k in range(4):
        t = txs[k]
        rec["tx"][k]["first"] = t.first
        rec["tx"][k]["last"] = t.last
        rec["tx"][k]["tx_idx"] = idx[k]
        rec["tx"][k]["initial_delay"] = t.max_delay
        rec["tx_weights"][k] = w[k]
    p = [tuple(t.position) for t in txs]
    pos = tuple((1 - iy) * ((1 - ix) * p[0][i] + ix * p[1][i]) + iy * ((1 - ix) * p[2][i] + ix * p[3][i])
                for i in range(3))
    dirv = _slerp3(_slerp3(txs[0].direction, txs[1].direction, ix), _slerp3(txs[2].direction, txs[3].direction, ix), iy)
    rec["position"] = pos
    rec["direction"] = dirv
    md = [0.0, 0.0]
    for t in txs:
        for (ax, ay) in ((t.first[0], t.first[1]), (t.first[0], t.last[1]), (t.last[0], t.first[1]), (t.last[0], t.last[1])):
            e = centers[ax + ay * layout[0]]
            md[0] = max(md[0], abs(e[0] - pos[0]))
            md[1] = max(md[1], abs(e[1] - pos[2]))
    rec["max_element_distance"] = md
    return rec


def build_geometry(centers: np.ndarray, element_layout: Tuple[int, int], num_channels: int, num_samples: int,
                   sampling_frequency_hz: float, spec: ScanSpec, depth_mm: Optional[float] = None,
                   num_depths: Optional[int] = None, element_to_channel: Optional[np.ndarray] = None) -> Geometry:
    """Beamformer::computeTxParameters (Beamformer/Beamformer.cpp:409-760) with receive scanline
    subdivision 1 (one receive line per transmit, txWeights = {1, 0, 0, 0})."""
    layout = element_layout
    nE = centers.shape[0]
    c_mm_s = spec.speed_of_sound_m_s * 1000.0
    if depth_mm is None:
        depth_mm = (num_samples - 1) * c_mm_s / sampling_frequency_hz / 2.0
    if num_depths is None:
        num_depths = num_samples
    steer = (math.radians(spec.steering_deg[0]), math.radians(spec.steering_deg[1]))
    sector = (math.radians(spec.sector_deg[0]), math.radians(spec.sector_deg[1]))
    nx, ny = spec.num_tx
    txs: List[_Tx] = []
    if spec.scan_type == "linear":
        first, last = centers[0], centers[nE - 1]
        for i in range(nx):
            pos = first[0] + i / (nx - 1) * (last[0] - first[0])
            rel = i / (nx - 1) * (nE - 1)
            act = compute_aperture(layout, spec.max_aperture, (rel, 0.0))
            txa = compute_aperture(layout, spec.tx_max_aperture, (rel, 0.0))
            ang = steer[0] - sector[0] / 2 + i / (nx - 1) * sector[0]
            txs.append(_tx_scanline(centers, layout, spec, act, txa, (pos, 0.0), (ang, 0.0)))
    elif spec.scan_type == "biphased":
        for y in range(ny):
            for x in range(nx):
                rel = (x / (nx - 1) * (layout[0] - spec.max_aperture[0]) + (spec.max_aperture[0] - 1) / 2,
                       y / (ny - 1) * (layout[1] - spec.max_aperture[1]) + (spec.max_aperture[1] - 1) / 2)
                act = compute_aperture(layout, spec.max_aperture, rel)
                txa = compute_aperture(layout, spec.tx_max_aperture, rel)
                sx = (centers[act[0][0]][0] + centers[act[1][0]][0]) / 2
                sy = (centers[act[0][1] * layout[0]][1] + centers[act[1][1] * layout[0]][1]) / 2
                ang = (steer[0] + (x / (nx - 1) - 0.5) * sector[0], steer[1] + (y / (ny - 1) - 0.5) * sector[1])
                txs.append(_tx_scanline(centers, layout, spec, act, txa, (sx, sy), ang))
    else:
        raise ValueError(f"unsupported scan type {spec.scan_type}")

    T = lambda x, y: x + y * nx
    rx = {}
    if ny > 1:
        for y in range(ny - 1):
            for x in range(nx - 1):
                ids = (T(x, y), T(x + 1, y), T(x, y + 1), T(x + 1, y + 1))
                rx[(x, y)] = _rx_interpolated(centers, layout, ids, [txs[i] for i in ids], (0.0, 0.0))
            x = nx - 1
            ids = (T(x, y), T(x, y), T(x, y + 1), T(x, y + 1))
            rx[(x, y)] = _rx_interpolated(centers, layout, ids, [txs[i] for i in ids], (0.0, 0.0))
            i = T(nx - 1, y)
            rx[(nx - 1, y)] = _rx_interpolated(centers, layout, (i,) * 4, [txs[i]] * 4, (0.0, 0.0))
        y = ny - 1
        for x in range(nx - 1):
            ids = (T(x, y), T(x + 1, y), T(x, y), T(x + 1, y))
            rx[(x, y)] = _rx_interpolated(centers, layout, ids, [txs[i] for i in ids], (0.0, 0.0))
        i = T(nx - 1, ny - 1)
        rx[(nx - 1, ny - 1)] = _rx_interpolated(centers, layout, (i,) * 4, [txs[i]] * 4, (0.0, 0.0))
    else:
        for x in range(nx - 1):
            ids = (x, x + 1, x, x + 1)
            rx[(x, 0)] = _rx_interpolated(centers, layout, ids, [txs[i] for i in ids], (0.0, 0.0))
        i = nx - 1
        rx[(i, 0)] = _rx_interpolated(centers, layout, (i,) * 4, [txs[i]] * 4, (0.0, 0.0))
    lines = np.zeros(nx * ny, dtype=SCANLINE_DTYPE)
    k = 0
    for y in range(ny):  # RxBeamformerParameters ctor, Beamformer/RxBeamformerParameters.cpp:65-74
        for x in range(nx):
            lines[k] = rx[(x, y)]
            k += 1
    return Geometry(element_centers=centers, element_layout=tuple(layout), num_channels=num_channels,
                    num_samples=num_samples, num_tx=nx * ny, rx_layout=(nx, ny), depth_mm=float(depth_mm),
                    num_depths=int(num_depths), sampling_frequency_hz=float(sampling_frequency_hz),
                    speed_of_sound_mm_s=c_mm_s, scanlines=lines, element_to_channel=element_to_channel)


def linear_probe_geometry(num_elements=128, pitch_mm=0.3, num_channels=64, num_samples=2048, fs_hz=40e6,
                          aperture=64, focus_mm=20.0, c_m_s=1540.0, num_depths=None, depth_mm=None,
                          num_tx=None) -> Geometry:
    """Linear array, one focused transmit per element, `aperture`-element receive aperture."""
    centers = linear_element_centers(num_elements, pitch_mm)
    spec = ScanSpec(scan_type="linear", num_tx=(num_tx or num_elements, 1), max_aperture=(aperture, 1),
                    tx_max_aperture=(aperture, 1), tx_focus_active=True, tx_focus_depth_mm=focus_mm,
                    speed_of_sound_m_s=c_m_s)
    return build_geometry(centers, (num_elements, 1), num_channels, num_samples, fs_hz, spec,
                          depth_mm=depth_mm, num_depths=num_depths)


def matrix_probe_geometry(nx=32, ny=32, pitch_mm=0.3, num_channels=256, num_samples=1024, fs_hz=20e6,
                          lines=(32, 32), aperture=(16, 16), focus_mm=40.0, c_m_s=1540.0,
                          num_depths=None, depth_mm=None) -> Geometry:
    """Matrix array, biphased focused scanlines on a lines[0] x lines[1] grid, sub-aperture receive."""
    centers = planar_element_centers(nx, ny, pitch_mm, pitch_mm)
    spec = ScanSpec(scan_type="biphased", num_tx=lines, max_aperture=aperture, tx_max_aperture=aperture,
                    tx_focus_active=True, tx_focus_depth_mm=focus_mm, speed_of_sound_m_s=c_m_s)
    return build_geometry(centers, (nx, ny), num_channels, num_samples, fs_hz, spec, depth_mm=depth_mm,
                          num_depths=num_depths)
