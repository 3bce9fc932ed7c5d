"""The allocation-free DAS entry point (sb_das_run_static), for callers that cannot allocate device
memory (hosts that hand out buffers only from their own pre-reserved pool, real-time frame loops
that cannot afford cudaMalloc/cudaFree). Called through the C ABI and compared with the planned
entry point (sb_das_plan_create + sb_das_run) on two calls in a row. Named to be collected last."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import random_rf, small_linear

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative to the frame peak, as the other DAS parity tests


def planned(lib, geom, rf, **kw):
    from supra_b200 import abi
    g = geom.ctypes()
    plan = C.c_void_p()
    assert lib.sb_das_plan_create(C.byref(g), C.byref(plan)) == abi.SB_OK
    out = torch.empty((geom.num_depths, geom.num_rx), dtype=torch.float32, device="cuda")
    st = lib.sb_das_run(plan, C.c_void_p(rf.data_ptr()), abi.SB_INT16, C.c_void_p(out.data_ptr()), abi.SB_FLOAT32,
                        kw["F"], kw["c"], kw["w"], 0.0, 0, 0, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.SB_OK, lib.sb_last_error()
    torch.cuda.synchronize()
    lib.sb_das_plan_destroy(plan)
    return out


def static(lib, geom, rf, **kw):
    from supra_b200 import abi
    g = geom.ctypes()
    out = torch.full((geom.num_depths, geom.num_rx), float("nan"), dtype=torch.float32, device="cuda")
    st = lib.sb_das_run_static(C.byref(g), C.c_void_p(rf.data_ptr()), abi.SB_INT16, C.c_void_p(out.data_ptr()),
                               abi.SB_FLOAT32, kw["F"], kw["c"], kw["w"], 0.0, 0, 0,
                               C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.SB_OK, lib.sb_last_error()
    torch.cuda.synchronize()
    return out


def close(a, b):
    a = a.cpu().numpy().astype(np.float64)
    b = b.cpu().numpy().astype(np.float64)
    same = (a == b) | (np.isnan(a) & np.isnan(b))
    peak = np.nanmax(np.abs(b[np.abs(b) < 1e30]))
    err = np.nanmax(np.abs(np.where(same, 0.0, a - b)))
    return err <= TOL * peak


def test_static_das_matches_planned_two_calls():
    from supra_b200 import abi
    from supra_b200.geometry import linear_probe_geometry
    lib = abi.load_library()
    # two calls in a row with different geometries and data: the shared scratch must be refreshed
    g1 = linear_probe_geometry(128, 0.3, 64, 2048, 40e6, aperture=64, focus_mm=20.0)
    g2 = small_linear()
    rf1 = torch.from_numpy(random_rf(g1, seed=31, amp=30000)).cuda()
    rf2 = torch.from_numpy(random_rf(g2, seed=32)).cuda()
    ref1 = planned(lib, g1, rf1, F=1.0, c=1540e3, w=1)
    ref2 = planned(lib, g2, rf2, F=0.8, c=1500e3, w=2)
    out1 = static(lib, g1, rf1, F=1.0, c=1540e3, w=1)
    out2 = static(lib, g2, rf2, F=0.8, c=1500e3, w=2)
    assert close(out1, ref1)
    assert close(out2, ref2)
    # and once more the first geometry after the second
    assert close(static(lib, g1, rf1, F=1.0, c=1540e3, w=1), ref1)
    assert lib.sb_check_device_errors(1) == abi.SB_OK


def test_static_das_rejects_oversized_geometry():
    from supra_b200 import abi
    from supra_b200.geometry import linear_probe_geometry
    lib = abi.load_library()
    g = linear_probe_geometry(128, 0.3, 64, 2048, 40e6, aperture=64, num_depths=abi_max_depths() + 1)
    rf = torch.zeros((g.num_tx, g.num_channels, g.num_samples), dtype=torch.int16, device="cuda")
    out = torch.empty((g.num_depths, g.num_rx), dtype=torch.float32, device="cuda")
    st = lib.sb_das_run_static(C.byref(g.ctypes()), C.c_void_p(rf.data_ptr()), abi.SB_INT16,
                               C.c_void_p(out.data_ptr()), abi.SB_FLOAT32, 1.0, 1540e3, 1, 0.0, 0, 0, None)
    assert st == abi.SB_ERR_INVALID_ARG
    assert b"static limits" in lib.sb_last_error()


def abi_max_depths():
    import os
    import re
    hdr = open(os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "supra_b200.h")).read()
    return int(re.search(r"#define SB_DAS_STATIC_MAX_DEPTHS (\d+)", hdr).group(1))
