"""Node layer on the GPU: every node's output equals the direct C-ABI call it wraps (bit-identical),
node chains equal the same calls in sequence, and a graph built from an XML configuration equals
the node chain."""
import numpy as np
import pytest
import torch

from conftest import small_linear
from test_nodes import CONFIG

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def frame():
    from supra_b200 import synth
    g = small_linear(num_samples=512)
    pts, amps = synth.random_scatterers(10, (-4.5, 4.5), (1.5, 9.0), seed=21)
    rf = synth.channel_data(g, pts, amps, synth.PulseSpec(7e6, 0.6), -40.0, 30000.0, seed=21, device="cuda")
    return g, rf


def _eq(a, b):
    a, b = a.cpu().numpy(), b.cpu().numpy()
    return a.shape == b.shape and np.array_equal(a, b)


def test_beamforming_node_equals_das(frame):
    from supra_b200.api import RxBeamformer
    from supra_b200.nodes import Node
    g, rf = frame
    n = Node("BeamformingNode", "BEAM")
    n.set("windowType", "Hann")
    n.set("speedOfSound", 1500)
    n.set("fNumber", 1.5)
    out, state = n.process_raw(g, rf)
    ref = RxBeamformer(g).beamform(rf, 1.5, 1500e3, window_type=1)
    torch.cuda.synchronize()
    assert state == "rf" and _eq(out, ref)
    n.set("outputType", "int16")
    out16, _ = n.process_raw(g, rf)
    ref16 = RxBeamformer(g).beamform(rf, 1.5, 1500e3, window_type=1, out_dtype=torch.int16)
    torch.cuda.synchronize()
    assert out16.dtype == torch.int16 and _eq(out16, ref16)
    n.set("outputType", "float")
    for name in ("CoherenceFactorDelayAndSum", "DelayAndStdDev", "TestSignal"):
        n.set("beamformerType", name)
        outv, _ = n.process_raw(g, rf)
        refv = RxBeamformer(g).beamform(rf, 1.5, 1500e3, window_type=1, beamformer=name)
        torch.cuda.synchronize()
        assert _eq(outv, refv), name


def test_envelope_log_scan_chain(frame):
    from supra_b200.api import HilbertFirEnvelope, LogCompressor, RxBeamformer, ScanConverter
    from supra_b200.nodes import Node
    g, rf = frame
    beam, env, logc, scan = (Node("BeamformingNode", "B"), Node("HilbertFirEnvelopeNode", "E"),
                             Node("LogCompressorNode", "L"), Node("ScanConverterNode", "S"))
    beam.set("windowType", "Hamming")
    env.set("filterLength", 64)
    logc.set("dynamicRange", 50)
    logc.set("inMax", 30000)
    logc.set("outputType", "uint8")
    scan.set("outputType", "uint8")
    beam.process_raw(g, rf)
    e, st_e = env.process_after(beam)
    l, st_l = logc.process_after(env)
    s, st_s = scan.process_after(logc)
    torch.cuda.synchronize()
    # the same calls directly
    r = RxBeamformer(g).beamform(rf, 1.0, window_type=2)
    e_ref = HilbertFirEnvelope(64).demodulate(r)
    l_ref = LogCompressor().compress(e_ref, 50.0, 1.0, 30000.0, out_dtype=torch.uint8)
    sc = ScanConverter(g.scanlines, g.rx_layout, g.num_depths, g.depth_mm, 0.1)
    s_ref = sc.convert(l_ref, out_dtype=torch.uint8)
    torch.cuda.synchronize()
    assert (st_e, st_l, st_s) == ("envelope", "log_compressed", "scan_converted")
    assert _eq(e, e_ref) and _eq(l, l_ref) and _eq(s, s_ref)


def test_envelope_int16_output_is_clampcast(frame):
    from supra_b200.nodes import Node
    g, rf = frame
    beam, env = Node("BeamformingNode", "B"), Node("HilbertFirEnvelopeNode", "E")
    beam.process_raw(g, rf)
    e32, _ = env.process_after(beam)
    e32 = e32.clone()
    env.set("outputType", "int16")
    e16, _ = env.process_after(beam)
    torch.cuda.synchronize()
    exp = torch.clamp(e32, -32767, 32767).to(torch.int16)  # clamp then truncate toward zero
    assert _eq(e16, exp)


def test_iq_demodulator_node(frame):
    from supra_b200.api import IQDemodulator, RxBeamformer
    from supra_b200.nodes import Node
    g, rf = frame
    beam, iq = Node("BeamformingNode", "B"), Node("IQDemodulatorNode", "D")
    for k, v in {"decimation": 2, "referenceFrequency": 7e6, "bandwidth": 3e6, "weight": 1,
                 "referenceFrequencyAdd0": 6.5e6, "weightAdd0": 1, "bandwidthAdd0": 3e6}.items():
        assert iq.set(k, v)
    beam.process_raw(g, rf)
    out, state = iq.process_after(beam)
    r = RxBeamformer(g).beamform(rf, 1.0, window_type=0)
    ref = IQDemodulator(40e6, 2.5e6, 51, 51, (7e6, 6.5e6), (3e6, 3e6), (1.0, 1.0)).demodulate_magnitude(r, 2)
    torch.cuda.synchronize()
    assert state == "envelope" and _eq(out, ref)


def test_rawdelay_then_mv_node(frame):
    from supra_b200.api import RxBeamformer, mv_beamform
    from supra_b200.nodes import Node
    g, rf = frame
    rd, mv = Node("RawDelayNode", "RD"), Node("BeamformingMVNode", "MV")
    rd.set("windowType", "Hann")
    mv.set("subArraySize", 8)
    mv.set("temporalSmoothing", 2)
    raw, st = rd.process_raw(g, rf)
    assert st == "raw_delayed"
    ref_raw = RxBeamformer(g).raw_delay(rf, 1.0, window_type=1)
    torch.cuda.synchronize()
    assert _eq(raw, ref_raw)
    # MV on RawDelay output needs the clamped 0/0 samples removed (they overflow in the reference too)
    clean = torch.where(ref_raw.abs() < 1e30, ref_raw, torch.zeros_like(ref_raw)).contiguous()
    out, st2 = mv.process_raw(g, clean, delayed=True)
    ref, _ = mv_beamform(clean, 8, 2, 1.5, False, 1.0, 1e6)
    torch.cuda.synchronize()
    assert st2 == "rf" and _eq(out, ref)
    # MV refuses data that was not raw-delayed (BeamformingMVNode.cpp:131)
    from supra_b200.abi import SupraError
    with pytest.raises(SupraError):
        mv.process_raw(g, rf)


def test_graph_from_xml_equals_node_chain(frame):
    from supra_b200.nodes import Graph, Node
    g, rf = frame
    graph = Graph(CONFIG)
    img, state = graph.process_raw(g, rf)
    img = img.clone()
    beam, env, logc, scan = (Node("BeamformingNode", "B"), Node("HilbertFirEnvelopeNode", "E"),
                             Node("LogCompressorNode", "L"), Node("ScanConverterNode", "S"))
    beam.set("windowType", "Hamming")
    beam.set("windowParameter", 0.5)
    beam.set("speedOfSound", 1500)
    env.set("filterLength", 64)
    logc.set("dynamicRange", 50)
    logc.set("inMax", 30000)
    logc.set("outputType", "uint8")
    scan.set("outputType", "uint8")
    beam.process_raw(g, rf)
    env.process_after(beam)
    logc.process_after(env)
    s, _ = scan.process_after(logc)
    torch.cuda.synchronize()
    assert state == "scan_converted" and img.dtype == torch.uint8 and _eq(img, s)
