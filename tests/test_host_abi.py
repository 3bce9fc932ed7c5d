"""The C ABI library without a GPU: it loads, exports every entry point the header declares, its
host-side design code matches the oracle bit for bit, and bad arguments are rejected."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import small_linear
from supra_b200 import abi, api

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "supra_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(sb_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    names = declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(abi.EXPORTED) | {"sb_last_error"}


def test_window_lut_matches_oracle(oracle):
    for t, p in [(0, 0.0), (1, 0.0), (1, 0.3), (2, 0.0), (3, 0.4)]:
        assert np.array_equal(api.window_lut(t, p).view(np.uint32), oracle.window_lut(t, p).view(np.uint32))


def test_fir_matches_oracle(oracle):
    for c in [(65, 3, 2, 2.0, 0, 0), (64, 3, 2, 2.0, 0, 0), (51, 0, 2, 40e6, 2.5e6, 0), (32, 0, 2, 40e6, 2.5e6, 0),
              (51, 2, 3, 40e6, 7e6, 1e6), (51, 1, 1, 40e6, 3e6, 0)]:
        assert np.array_equal(api.fir_design(*c).view(np.uint32), oracle.fir(*c).view(np.uint32)), c


@pytest.mark.parametrize("res", [0.1, 0.05, 0.23])
def test_scan_tables_2d_bit_exact(oracle, res):
    g = small_linear()
    mine = api.scan_tables_2d_host(g.scanlines, g.rx_layout[0], g.num_depths, g.depth_mm, res)
    ref = oracle.scan_tables(g.scanlines, g.rx_layout[0], 1, g.num_depths, g.depth_mm, res)
    assert mine["size"] == ref["size"]
    assert np.array_equal(mine["mask"], ref["mask"])
    m = ref["mask"].astype(bool)
    assert np.array_equal(mine["sample_idx"][m], ref["sample_idx"][m])
    assert np.array_equal(mine["weight_x"][m].view(np.uint32), ref["weight_x"][m].view(np.uint32))
    assert np.array_equal(mine["weight_y"][m].view(np.uint32), ref["weight_y"][m].view(np.uint32))


def test_scan_tables_2d_c0_size(oracle):
    from supra_b200.geometry import linear_probe_geometry
    g = linear_probe_geometry(128, 0.3, 64, 2048, 40e6, aperture=64)
    mine = api.scan_tables_2d_host(g.scanlines, 128, 2048, g.depth_mm, 0.1)
    W, H, D = mine["size"]
    assert (W, H, D) == (383, 396, 1)


def test_invalid_arguments_rejected_without_gpu():
    lib = abi.load_library()
    plan = C.c_void_p()
    g = small_linear().ctypes()
    g.num_rx = 7  # inconsistent with rx_layout
    st = lib.sb_das_plan_create(C.byref(g), C.byref(plan))
    assert st == abi.SB_ERR_INVALID_ARG and not plan.value
    assert b"num_rx" in lib.sb_last_error()
    assert lib.sb_window_lut(9, 0.0, 64, None) == abi.SB_ERR_INVALID_ARG
    assert lib.sb_fir_design(0, 0, 0, 1.0, 0.1, 0.0, None) == abi.SB_ERR_INVALID_ARG
    assert lib.sb_das_run(None, None, 1, None, 2, 1.0, 1540e3, 1, 0.0, 0, 0, None) == abi.SB_ERR_INVALID_ARG
    assert lib.sb_hilbert_plan_create(0, C.byref(plan)) == abi.SB_ERR_INVALID_ARG


def test_bad_transmit_index_rejected():
    lib = abi.load_library()
    geom = small_linear()
    sl = geom.scanlines.copy()
    sl[3]["tx"][0]["tx_idx"] = 999
    geom.scanlines = sl
    g = geom.ctypes()
    plan = C.c_void_p()
    assert lib.sb_das_plan_create(C.byref(g), C.byref(plan)) == abi.SB_ERR_INVALID_ARG
    assert b"transmit index" in lib.sb_last_error()


def test_libtorch_autograd_operators_load():
    """The libtorch autograd Functions (torch.ops.supra_b200.*) load and register without a GPU."""
    import torch
    from supra_b200.autograd import load_torch_ops
    load_torch_ops()
    assert hasattr(torch.ops.supra_b200, "das_apod") and hasattr(torch.ops.supra_b200, "envelope")
