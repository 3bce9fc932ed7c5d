"""Python view of the node layer (SUPRA's receive-path nodes re-hosted on the C ABI).

    node = Node("BeamformingNode", "BEAM")
    node.set("windowType", "Hann")            # validated against the reference's value range
    out = node.process_raw(geometry, rf)       # USRawData in -> USImage out (torch view of the device buffer)
    env = Node("HilbertFirEnvelopeNode", "ENV").process_after(node)

    graph = Graph(open("config.xml").read())  # SUPRA XML configuration: nodes, params, connections
    img = graph.process_raw(geometry, rf)

Outputs are torch tensors that alias memory owned by the node (or graph) until its next call;
clone them to keep them.
"""
from __future__ import annotations

import collections
import ctypes as C
from typing import Dict, List, Optional

import torch

from .abi import SB_OK, check, load_library, sb_record
from .api import _TORCH, _ptr, _stream, dtype_code

STATES = ["raw", "raw_delayed", "rf", "envelope", "log_compressed", "scan_converted"]


def node_types() -> List[str]:
    lib = load_library()
    out = []
    buf = C.create_string_buffer(128)
    for i in range(lib.sb_node_type_count()):
        check("sb_node_type_name", lib.sb_node_type_name(i, buf, 128))
        out.append(buf.value.decode())
    return out


def _record_tensor(rec: sb_record, device) -> torch.Tensor:
    """Zero-copy torch view of a node output (device memory owned by the node)."""
    dt = _TORCH[rec.dtype]
    if rec.is_image:
        shape = (rec.size[1], rec.size[0]) if rec.size[2] <= 1 else (rec.size[2], rec.size[1], rec.size[0])
    else:
        shape = (rec.size[2], rec.size[1], rec.size[0])
    n = 1
    for d in shape:
        n *= d
    return _from_pointer(rec.data, shape, dt, n * torch.empty((), dtype=dt).element_size(), device)


def _from_pointer(ptr: int, shape, dtype, nbytes: int, device) -> torch.Tensor:
    class _Holder:
        __cuda_array_interface__ = {
            "shape": tuple(shape), "typestr": _typestr(dtype), "data": (ptr, False), "version": 2, "strides": None,
        }
    return torch.as_tensor(_Holder(), device=device)


def _typestr(dtype) -> str:
    return {torch.float32: "<f4", torch.int16: "<i2", torch.uint8: "|u1", torch.complex64: "<c8"}[dtype]


class Node:
    def __init__(self, node_type: str, node_id: str):
        self.lib = load_library()
        self._h = C.c_void_p()
        check("sb_node_create", self.lib.sb_node_create(node_type.encode(), node_id.encode(), C.byref(self._h)))
        self.type, self.id = node_type, node_id
        self._geometry_keep = None
        self._inputs = collections.deque(maxlen=50)

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            self.lib.sb_node_destroy(self._h)
            self._h = C.c_void_p()

    def set(self, name: str, value) -> bool:
        """Sets a parameter; returns False (and stores the default) if the value is not valid."""
        if isinstance(value, bool):
            value = "true" if value else "false"
        return self.lib.sb_node_set_param(self._h, name.encode(), str(value).encode()) == SB_OK

    def get(self, name: str) -> str:
        buf = C.create_string_buffer(256)
        check("sb_node_get_param", self.lib.sb_node_get_param(self._h, name.encode(), buf, 256))
        return buf.value.decode()

    def params(self) -> Dict[str, dict]:
        out = {}
        bufs = [C.create_string_buffer(512) for _ in range(4)]
        for i in range(self.lib.sb_node_param_count(self._h)):
            check("sb_node_param_info", self.lib.sb_node_param_info(self._h, i, *bufs, 512))
            name, typ, rng, dflt = (b.value.decode() for b in bufs)
            out[name] = {"type": typ, "range": rng, "default": dflt}
        return out

    def process_raw(self, geometry, data: torch.Tensor, delayed: bool = False, image_resolution_mm: float = 0.1):
        g = geometry.ctypes()
        self._geometry_keep = g
        rec = sb_record()
        if delayed:
            n_tx, n_ch, n_s = data.shape
        else:
            n_tx, n_ch, n_s = geometry.num_tx, geometry.num_channels, geometry.num_samples
        check("sb_node_process_raw", self.lib.sb_node_process_raw(self._h, C.byref(g), _ptr(data), dtype_code(data),
                                                                  int(delayed), n_tx, n_ch, n_s,
                                                                  float(geometry.depth_mm), float(image_resolution_mm),
                                                                  _stream(), C.byref(rec)))
        return _record_tensor(rec, data.device), STATES[rec.state]

    def process_image(self, image: torch.Tensor, state: str = "rf", geometry=None, depth_mm: float = 0.0,
                      image_resolution_mm: float = 0.1):
        """Runs the node on a device image [(depth,) samples, scanlines] in image state `state`. The last
        50 inputs are kept referenced here, since the C entry point borrows them (TemporalFilterNode
        reads its stored images again on later calls)."""
        if not image.is_contiguous() or image.dim() not in (2, 3):
            raise ValueError("process_image: a contiguous 2D or 3D image")
        size = (C.c_uint32 * 3)(image.shape[-1], image.shape[-2], image.shape[0] if image.dim() == 3 else 1)
        g = None if geometry is None else geometry.ctypes()
        if g is not None:
            self._geometry_keep = g
        self._inputs.append(image)
        rec = sb_record()
        check("sb_node_process_image",
              self.lib.sb_node_process_image(self._h, None if g is None else C.byref(g), _ptr(image), dtype_code(image),
                                             STATES.index(state), size, float(depth_mm), float(image_resolution_mm),
                                             _stream(), C.byref(rec)))
        return _record_tensor(rec, image.device), STATES[rec.state]

    def process_after(self, upstream: "Node", device="cuda"):
        rec = sb_record()
        check("sb_node_process_last", self.lib.sb_node_process_last(self._h, upstream._h, C.byref(rec)))
        return _record_tensor(rec, device), STATES[rec.state]


class Graph:
    def __init__(self, xml_text: str):
        self.lib = load_library()
        self._h = C.c_void_p()
        check("sb_graph_create_xml", self.lib.sb_graph_create_xml(xml_text.encode(), C.byref(self._h)))
        self._geometry_keep = None

    def __del__(self):
        if getattr(self, "_h", None) and self._h.value:
            self.lib.sb_graph_destroy(self._h)
            self._h = C.c_void_p()

    def chain(self) -> List[str]:
        buf = C.create_string_buffer(4096)
        n = self.lib.sb_graph_chain(self._h, buf, 4096)
        return buf.value.decode().split(",") if n > 0 else []

    def get(self, node_id: str, name: str) -> str:
        buf = C.create_string_buffer(256)
        check("sb_graph_node_get_param", self.lib.sb_graph_node_get_param(self._h, node_id.encode(), name.encode(),
                                                                          buf, 256))
        return buf.value.decode()

    def process_next(self, image_resolution_mm: float = 0.1, device="cuda"):
        """Next frame of the configuration's UltrasoundInterfaceRawDataMock input through the chain:
        (output tensor, state, last_frame)."""
        rec = sb_record()
        last = C.c_int(0)
        check("sb_graph_process_next", self.lib.sb_graph_process_next(self._h, float(image_resolution_mm), _stream(),
                                                                      C.byref(last), C.byref(rec)))
        return _record_tensor(rec, device), STATES[rec.state], bool(last.value)

    def process_raw(self, geometry, rf: torch.Tensor, image_resolution_mm: float = 0.1):
        g = geometry.ctypes()
        self._geometry_keep = g
        rec = sb_record()
        check("sb_graph_process_raw", self.lib.sb_graph_process_raw(self._h, C.byref(g), _ptr(rf), dtype_code(rf),
                                                                    geometry.num_tx, geometry.num_channels,
                                                                    geometry.num_samples, float(geometry.depth_mm),
                                                                    float(image_resolution_mm), _stream(), C.byref(rec)))
        return _record_tensor(rec, rf.device), STATES[rec.state]
