"""Replay of recorded frames (UltrasoundInterfaceRawDataMock semantics) into device memory, and a
graph whose XML input is the recorded-data mock."""
import os

import numpy as np
import pytest
import torch

from conftest import random_rf, small_linear

pytestmark = pytest.mark.gpu


@pytest.fixture()
def recording(tmp_path):
    """Metadata plus two frame files: 3 frames and 2 frames (a partial trailing frame is ignored)."""
    from supra_b200.mock import MockMetadata, write_mock_json
    g = small_linear()
    meta_fn = str(tmp_path / "probe.json")
    write_mock_json(meta_fn, g)
    frames = [random_rf(g, seed=50 + k) for k in range(5)]
    f0, f1 = str(tmp_path / "seq0.raw"), str(tmp_path / "seq1.raw")
    with open(f0, "wb") as f:
        for x in frames[:3]:
            f.write(x.tobytes())
    with open(f1, "wb") as f:
        for x in frames[3:]:
            f.write(x.tobytes())
        f.write(b"\x00" * 100)
    return g, MockMetadata(meta_fn), f0, f1, frames


def test_reader_plays_files_in_order_and_wraps(recording):
    from supra_b200.mock import MockReader
    g, meta, f0, f1, frames = recording
    r = MockReader(meta, f"{f0}, {f1}")
    assert r.sequence_lengths == [3, 2] and r.frame_bytes == frames[0].nbytes
    got = []
    for _ in range(12):
        x, last = r.next()
        got.append(x.cpu().numpy())
        assert not last
    order = [0, 1, 2, 3, 4] * 3
    for k, x in enumerate(got):
        assert np.array_equal(x, frames[order[k]]), k


def test_reader_stream_once_and_single_image(recording):
    from supra_b200.abi import SupraError
    from supra_b200.mock import MockReader
    g, meta, f0, f1, frames = recording
    r = MockReader(meta, f"{f0},{f1}", stream_sequence_once=True)
    out = torch.empty((g.num_tx, g.num_channels, g.num_samples), dtype=torch.int16, device="cuda")
    for k in range(5):
        x, last = r.next(out)
        assert np.array_equal(x.cpu().numpy(), frames[k]) and last == (k == 4)
    with pytest.raises(SupraError):
        r.next(out)
    s = MockReader(meta, f1, single_image=True)
    for _ in range(3):
        x, last = s.next()
        assert np.array_equal(x.cpu().numpy(), frames[3]) and not last


def test_reader_rejects_bad_files(recording, tmp_path):
    from supra_b200.abi import SupraError
    from supra_b200.mock import MockReader
    g, meta, f0, f1, frames = recording
    short = tmp_path / "short.raw"
    short.write_bytes(b"\x00" * 10)
    with pytest.raises(SupraError):
        MockReader(meta, str(short))
    with pytest.raises(SupraError):
        MockReader(meta, str(tmp_path / "missing.raw"))


def test_graph_replays_mock_input(recording):
    """A configuration in the reference's layout (configRawDataMock.xml): the mock input feeds
    BeamformingNode -> HilbertFirEnvelopeNode -> LogCompressorNode; each frame equals the same nodes
    run on that frame directly."""
    from supra_b200.nodes import Graph, Node
    g, meta, f0, f1, frames = recording
    xml = f"""<?xml version="1.0"?>
<supra_config>
  <devices>
    <inputs>
      <input type="UltrasoundInterfaceRawDataMock" id="US-Mock">
        <param name="frequency" type="int">10</param>
        <param name="mockMetaDataFilename" type="string">{meta_path(meta, f0)}</param>
        <param name="mockDataFilename" type="string">{f0}, {f1}</param>
        <param name="singleImage" type="bool">0</param>
        <param name="streamSequenceOnce" type="bool">1</param>
      </input>
    </inputs>
    <nodes>
      <node type="BeamformingNode" id="BEAM"><param name="windowType" type="string">Hann</param></node>
      <node type="HilbertFirEnvelopeNode" id="ENV"/>
      <node type="LogCompressorNode" id="LOGC"><param name="inMax" type="double">30000</param></node>
    </nodes>
  </devices>
  <connections>
    <connection><from id="US-Mock" port="0"/><to id="BEAM" port="0"/></connection>
    <connection><from id="BEAM" port="0"/><to id="ENV" port="0"/></connection>
    <connection><from id="ENV" port="0"/><to id="LOGC" port="0"/></connection>
  </connections>
</supra_config>"""
    graph = Graph(xml)
    beam, env, logc = Node("BeamformingNode", "B"), Node("HilbertFirEnvelopeNode", "E"), Node("LogCompressorNode", "L")
    beam.set("windowType", "Hann")
    logc.set("inMax", 30000)
    for k in range(5):
        img, state, last = graph.process_next()
        img = img.clone()
        beam.process_raw(meta, torch.from_numpy(frames[k]).cuda())
        env.process_after(beam)
        ref, _ = logc.process_after(env)
        torch.cuda.synchronize()
        assert state == "log_compressed" and last == (k == 4)
        assert torch.equal(img, ref), k


def meta_path(meta, f0):
    return os.path.join(os.path.dirname(f0), "probe.json")


def test_graph_without_mock_input_refuses_next():
    from supra_b200.abi import SupraError
    from supra_b200.nodes import Graph
    from test_nodes import CONFIG
    with pytest.raises(SupraError):
        Graph(CONFIG).process_next()
