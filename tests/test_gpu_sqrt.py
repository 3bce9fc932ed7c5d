"""The 3D delay kernel's Newton square root (one step from the hardware reciprocal square root) equals
__fsqrt_rn on every float in [2^-102, FLT_MAX], the range the kernel uses it in (depths whose q = r2 +
ay2 provably lies there); that keeps the 3D DAS bit-identical to the reference's sampleBeamform3D."""
import ctypes as C

import pytest
import torch

pytestmark = pytest.mark.gpu


def test_newton_sqrt_equals_ieee_on_its_range():
    from supra_b200 import abi
    lib = abi.load_library()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    bad, first = C.c_uint64(123), C.c_uint32(0)
    # bit patterns of 2^-102 ... FLT_MAX (0x7F7FFFFF), all 1.9e9 of them
    assert lib.sb_selftest_sqrt(0x0C800000, 0x7F800000, C.byref(bad), C.byref(first), stream) == abi.SB_OK
    assert bad.value == 0, f"{bad.value} mismatches, lowest bit pattern {first.value:#010x}"
    assert first.value == 0xFFFFFFFF


def test_sqrt_selftest_rejects_bad_ranges():
    from supra_b200 import abi
    lib = abi.load_library()
    bad = C.c_uint64(0)
    assert lib.sb_selftest_sqrt(0, (1 << 32) + 1, C.byref(bad), None, None) == abi.SB_ERR_INVALID_ARG
    assert lib.sb_selftest_sqrt(5, 4, C.byref(bad), None, None) == abi.SB_ERR_INVALID_ARG
