"""Recorded raw data in SUPRA's mock format: metadata (.mock ASCII / .json) and int16 frame files.

MockMetadata mirrors RxBeamformerParameters::readMetaDataForMock (Beamformer/RxBeamformerParameters.cpp:
164-450) and can stand wherever a geometry is taken (RxBeamformer, nodes); MockReader replays the frame
files as UltrasoundInterfaceRawDataMock does (SupraLib/InputOutput/UltrasoundInterfaceRawDataMock.cpp:
47-204), asynchronously into device memory; write_mock_json is writeMetaDataForMock.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Tuple

import numpy as np
import torch

from .abi import SCANLINE_DTYPE, check, load_library, sb_geometry
from .api import _ptr, _stream


class MockMetadata:
    """The geometry of a recorded-data metadata file (read by the library)."""

    def __init__(self, filename: str):
        self.lib = load_library()
        self._h = C.c_void_p()
        check("sb_mock_meta_read", self.lib.sb_mock_meta_read(filename.encode(), C.byref(self._h)))
        self._g = sb_geometry()
        depth, c = C.c_double(), C.c_double()
        check("sb_mock_meta_geometry", self.lib.sb_mock_meta_geometry(self._h, C.byref(self._g), C.byref(depth),
                                                                      C.byref(c)))
        self.depth_mm = depth.value
        self.speed_of_sound_mm_s = c.value
        self.element_to_channel = None

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            self.lib.sb_mock_meta_destroy(self._h)
            self._h = C.c_void_p()

    def ctypes(self) -> sb_geometry:
        return self._g

    num_elements = property(lambda self: int(self._g.num_elements))
    element_layout = property(lambda self: (int(self._g.element_layout[0]), int(self._g.element_layout[1])))
    num_channels = property(lambda self: int(self._g.num_channels))
    num_samples = property(lambda self: int(self._g.num_samples))
    num_tx = property(lambda self: int(self._g.num_tx))
    num_rx = property(lambda self: int(self._g.num_rx))
    rx_layout = property(lambda self: (int(self._g.rx_layout[0]), int(self._g.rx_layout[1])))
    num_depths = property(lambda self: int(self._g.num_depths))
    sampling_frequency_hz = property(lambda self: float(self._g.sampling_frequency_hz))

    @property
    def is3d(self) -> bool:
        return self.rx_layout[0] > 1 and self.rx_layout[1] > 1

    @property
    def depths(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._g.depths_mm, (self.num_depths,)).copy()

    @property
    def element_x(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._g.element_x_mm, (self.num_elements,)).copy()

    @property
    def element_y(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._g.element_y_mm, (self.num_elements,)).copy()

    @property
    def scanlines(self) -> np.ndarray:
        raw = (C.c_char * (self.num_rx * SCANLINE_DTYPE.itemsize)).from_address(self._g.scanlines)
        return np.frombuffer(bytes(raw), dtype=SCANLINE_DTYPE).copy()


def write_mock_json(filename: str, geometry) -> None:
    """writeMetaDataForMock (Beamformer/RxBeamformerParameters.cpp:93-162) for a geometry."""
    lib = load_library()
    g = geometry.ctypes()
    check("sb_mock_write_json", lib.sb_mock_write_json(filename.encode(), C.byref(g), float(geometry.depth_mm),
                                                       float(geometry.speed_of_sound_mm_s)))


class MockReader:
    """Replays int16 frame files [num_tx][num_channels][num_samples] into device memory."""

    def __init__(self, meta: MockMetadata, data_filenames: str, single_image=False, stream_sequence_once=False):
        self.lib = load_library()
        self.meta = meta
        self._h = C.c_void_p()
        check("sb_mock_reader_create", self.lib.sb_mock_reader_create(meta._h, data_filenames.encode(),
                                                                      int(single_image), int(stream_sequence_once),
                                                                      C.byref(self._h)))
        fb, n = C.c_uint64(), C.c_uint32()
        check("sb_mock_reader_info", self.lib.sb_mock_reader_info(self._h, C.byref(fb), C.byref(n), None))
        lens = (C.c_uint64 * n.value)()
        check("sb_mock_reader_info", self.lib.sb_mock_reader_info(self._h, None, None, lens))
        self.frame_bytes = fb.value
        self.sequence_lengths = list(lens)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            self.lib.sb_mock_reader_destroy(self._h)
            self._h = C.c_void_p()

    def next(self, out: Optional[torch.Tensor] = None, device="cuda") -> Tuple[torch.Tensor, bool]:
        """The next frame (asynchronous on the current stream) and whether it is the last one."""
        m = self.meta
        if out is None:
            out = torch.empty((m.num_tx, m.num_channels, m.num_samples), dtype=torch.int16, device=device)
        last = C.c_int(0)
        check("sb_mock_reader_next", self.lib.sb_mock_reader_next(self._h, _ptr(out), _stream(), C.byref(last)))
        return out, bool(last.value)
