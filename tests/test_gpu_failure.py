"""Failure detection without a GPU fault: a bounded device-side wait that runs out (an mbarrier nothing
arrives at) raises the device error flag, the host reads SB_ERR_TIMEOUT from sb_check_device_errors,
the flag clears, and the context stays usable (a DAS call afterwards is bit-exact)."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import random_rf, small_linear

pytestmark = pytest.mark.gpu


def test_bounded_wait_timeout_is_reported_and_cleared(oracle):
    from supra_b200 import abi
    from supra_b200.api import RxBeamformer
    lib = abi.load_library()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.sb_check_device_errors(1) == abi.SB_OK
    done = C.c_int(-1)
    # the wait completes when its barrier is arrived at: no flag
    assert lib.sb_selftest_bounded_wait(1000, 1, C.byref(done), stream) == abi.SB_OK
    assert done.value == 1 and lib.sb_check_device_errors(1) == abi.SB_OK
    # nothing arrives: the wait gives up after its polls, the kernel returns, the flag is raised
    assert lib.sb_selftest_bounded_wait(1000, 0, C.byref(done), stream) == abi.SB_OK
    assert done.value == 0
    assert lib.sb_check_device_errors(1) == abi.SB_ERR_TIMEOUT
    assert b"bounded wait" in lib.sb_last_error()
    assert lib.sb_check_device_errors(1) == abi.SB_OK  # cleared by the reset above
    # the context is intact
    g = small_linear()
    rf = random_rf(g, seed=9)
    out = RxBeamformer(g).beamform(torch.from_numpy(rf).cuda(), 1.0, window_type=1).cpu().numpy()
    ref = oracle.das(g, rf, 1.0, window=1)
    ref = np.where(np.isnan(ref), -np.float32(3.4028235e38), ref)
    assert np.array_equal(out.view(np.uint32), ref.astype(np.float32).view(np.uint32))


def test_bounded_wait_rejects_bad_limits():
    from supra_b200 import abi
    lib = abi.load_library()
    assert lib.sb_selftest_bounded_wait(0, 0, None, None) == abi.SB_ERR_INVALID_ARG
