"""The allocation-free DAS entry point (sb_das_run_static), for callers that cannot allocate device
memory (hosts that hand out buffers only from their own pre-reserved pool, real-time frame loops
that cannot afford cudaMalloc/cudaFree). Called through the C ABI and compared with the planned
entry point (sb_das_plan_create + sb_das_run) on calls in a row, on every branch the static entry
point takes: 2D int16 -> float (the single-frame pack kernel, also bit-exact against the oracle),
3D, interpolated transmits, float channel data, int16 output and a channel map. Both entry points
run kernels with the reference's exact arithmetic, so results are compared bit for bit. Named to be
collected last."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import random_rf, small_linear, small_matrix

pytestmark = pytest.mark.gpu

_OUT = {"f32": torch.float32, "i16": torch.int16}


def _codes(rf, out_dtype):
    from supra_b200 import abi
    rfc = abi.SB_INT16 if rf.dtype == torch.int16 else abi.SB_FLOAT32
    oc = abi.SB_FLOAT32 if out_dtype == torch.float32 else abi.SB_INT16
    return rfc, oc


def planned(lib, geom, rf, F, c, w, itx=0, off=0, out_dtype=torch.float32):
    from supra_b200 import abi
    g = geom.ctypes()
    plan = C.c_void_p()
    assert lib.sb_das_plan_create(C.byref(g), C.byref(plan)) == abi.SB_OK
    out = torch.empty((geom.num_depths, geom.num_rx), dtype=out_dtype, device="cuda")
    rfc, oc = _codes(rf, out_dtype)
    st = lib.sb_das_run(plan, C.c_void_p(rf.data_ptr()), rfc, C.c_void_p(out.data_ptr()), oc, F, c, w, 0.0, itx, off,
                        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.SB_OK, lib.sb_last_error()
    torch.cuda.synchronize()
    lib.sb_das_plan_destroy(plan)
    return out


def static(lib, geom, rf, F, c, w, itx=0, off=0, out_dtype=torch.float32):
    from supra_b200 import abi
    g = geom.ctypes()
    # start from a value no path writes, so a pixel left unwritten shows
    fill = float("nan") if out_dtype == torch.float32 else 12345
    out = torch.full((geom.num_depths, geom.num_rx), fill, dtype=out_dtype, device="cuda")
    rfc, oc = _codes(rf, out_dtype)
    st = lib.sb_das_run_static(C.byref(g), C.c_void_p(rf.data_ptr()), rfc, C.c_void_p(out.data_ptr()), oc, F, c, w,
                               0.0, itx, off, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == abi.SB_OK, lib.sb_last_error()
    torch.cuda.synchronize()
    return out


def same_bits(a, b):
    a = a.cpu().numpy()
    b = b.cpu().numpy()
    if a.dtype == np.float32:
        a, b = a.view(np.uint32), b.view(np.uint32)
    return a.shape == b.shape and np.array_equal(a, b)


def test_static_das_matches_planned_two_calls(oracle):
    from supra_b200 import abi
    from supra_b200.geometry import linear_probe_geometry
    lib = abi.load_library()
    # two calls in a row with different geometries and data: the shared scratch must be refreshed
    g1 = linear_probe_geometry(128, 0.3, 64, 2048, 40e6, aperture=64, focus_mm=20.0)
    g2 = small_linear()
    rf1 = torch.from_numpy(random_rf(g1, seed=31, amp=30000)).cuda()
    rf2 = torch.from_numpy(random_rf(g2, seed=32)).cuda()
    ref1 = planned(lib, g1, rf1, 1.0, 1540e3, 1)
    ref2 = planned(lib, g2, rf2, 0.8, 1500e3, 2)
    out1 = static(lib, g1, rf1, 1.0, 1540e3, 1)
    out2 = static(lib, g2, rf2, 0.8, 1500e3, 2)
    assert same_bits(out1, ref1)
    assert same_bits(out2, ref2)
    # the oracle (the reference's FP32 semantics; 0/0 pixels clamp to -FLT_MAX)
    exp = oracle.das(g2, rf2.cpu().numpy(), 0.8, c_mm_s=1500e3, window=2)
    exp = np.where(np.isnan(exp), -np.float32(3.4028235e38), exp).astype(np.float32)
    assert np.array_equal(out2.cpu().numpy().view(np.uint32), exp.view(np.uint32))
    # and once more the first geometry after the second
    assert same_bits(static(lib, g1, rf1, 1.0, 1540e3, 1), ref1)
    assert lib.sb_check_device_errors(1) == abi.SB_OK


def _channel_mapped():
    g = small_linear()
    m = np.arange(g.num_elements, dtype=np.int32) % g.num_channels
    m[5] = -1
    m[17] = -1
    g.element_to_channel = m
    return g


@pytest.mark.parametrize("case", ["3d", "interp_tx", "float_rf", "int16_out", "channel_map", "offset"])
def test_static_das_other_branches(case):
    """Each branch twice in a row (second call with other data), bit for bit against sb_das_run."""
    from supra_b200 import abi
    lib = abi.load_library()
    g = small_matrix() if case == "3d" else _channel_mapped() if case == "channel_map" else small_linear()
    kw = {"F": 1.0, "c": 1540e3, "w": 1}
    if case == "interp_tx":
        kw["itx"] = 1
    if case == "offset":
        kw["off"] = 3
    if case == "int16_out":
        kw["out_dtype"] = torch.int16
    for seed in (41, 42):
        x = random_rf(g, seed=seed, amp=3000 if case != "int16_out" else 300)
        rf = torch.from_numpy(x.astype(np.float32) if case == "float_rf" else x).cuda()
        ref = planned(lib, g, rf, **kw)
        got = static(lib, g, rf, **kw)
        assert same_bits(got, ref), (case, seed)
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
