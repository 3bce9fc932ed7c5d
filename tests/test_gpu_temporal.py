"""Temporal filter (TemporalFilter / TemporalFilterNode) on the GPU against the oracle, bit for bit:
both follow the reference's float operations in order."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def images(n, shape, dtype, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    if dtype == np.int16:
        return [rng.integers(-32768, 32768, size=shape).astype(np.int16) for _ in range(n)]
    return [(rng.standard_normal(shape) * 1e4).astype(np.float32) for _ in range(n)]


@pytest.mark.parametrize("in_dtype", [np.int16, np.float32])
@pytest.mark.parametrize("out_dtype", [np.float32, np.int16])
@pytest.mark.parametrize("n", [1, 3, 50])
def test_temporal_filter_bit_exact(oracle, in_dtype, out_dtype, n):
    from supra_b200.api import temporal_filter
    ims = images(n, (2048, 129), in_dtype, seed=n)  # 264,192 elements: whole vectors plus a tail
    rng = np.random.Generator(np.random.PCG64(7))
    w = rng.uniform(0.1, 2.0, n)
    ref = oracle.temporal_filter(ims, w, out_dtype)
    t_out = torch.float32 if out_dtype == np.float32 else torch.int16
    got = temporal_filter([torch.from_numpy(x).cuda() for x in ims], w, out_dtype=t_out).cpu().numpy()
    if out_dtype == np.float32:
        assert np.array_equal(bits(got), bits(ref))
    else:
        assert np.array_equal(got, ref)
    # default weights (the node's: all 1)
    ref1 = oracle.temporal_filter(ims, None, out_dtype)
    got1 = temporal_filter([torch.from_numpy(x).cuda() for x in ims], out_dtype=t_out).cpu().numpy()
    assert np.array_equal(got1.view(np.uint8), ref1.view(np.uint8))


@pytest.mark.parametrize("numel", [1, 7, 8, 9, 1001])
def test_temporal_filter_unaligned_and_small(oracle, numel):
    """Views starting 2 bytes into a buffer take the element path; tiny sizes only the tail."""
    from supra_b200.api import temporal_filter
    ims = images(3, (numel + 1,), np.int16, seed=numel)
    dev = [torch.from_numpy(x).cuda()[1:] for x in ims]  # offset by one int16: not 16-byte aligned
    ref = oracle.temporal_filter([x[1:] for x in ims], None, np.float32)
    got = temporal_filter(dev).cpu().numpy()
    assert np.array_equal(bits(got), bits(ref))


def test_temporal_filter_rejects_bad_arguments():
    from supra_b200.abi import SupraError
    from supra_b200.api import temporal_filter
    x = torch.zeros(16, dtype=torch.float32, device="cuda")
    with pytest.raises(SupraError):
        temporal_filter([x] * 51)
    with pytest.raises(SupraError):
        temporal_filter([x.to(torch.uint8)])


def test_temporal_filter_node_queue(oracle):
    """The node averages the last numImages images; a size change empties the store; uint16 output is
    refused as in the reference."""
    from supra_b200.abi import SupraError
    from supra_b200.nodes import Node
    node = Node("TemporalFilterNode", "FILT")
    node.set("numImages", 2)
    ims = images(4, (64, 32), np.float32, seed=3)
    outs = [node.process_image(torch.from_numpy(x).cuda(), state="rf")[0].cpu().numpy() for x in ims]
    assert np.array_equal(bits(outs[0]), bits(oracle.temporal_filter(ims[:1])))
    for k in range(1, 4):
        assert np.array_equal(bits(outs[k]), bits(oracle.temporal_filter(ims[k - 1:k + 1])))
    other = images(1, (32, 32), np.float32, seed=9)[0]
    o, _ = node.process_image(torch.from_numpy(other).cuda(), state="rf")
    assert np.array_equal(bits(o.cpu().numpy()), bits(other))  # store emptied: the image itself
    node.set("outputType", "uint16")
    with pytest.raises(SupraError):
        node.process_image(torch.from_numpy(other).cuda(), state="rf")
