"""Node layer, host side (no GPU): parameter tables against the reference's constructors (fixture
tests/golden/node_params.json, made by tests/golden/make_node_params.py from the reference sources),
validation with fallback to the default, and graphs built from SUPRA's XML configuration format."""
import json
import os

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def ref_params():
    with open(os.path.join(HERE, "golden", "node_params.json")) as f:
        return json.load(f)


def _num(s):
    return float(s)


def test_node_types_cover_the_receive_path(ref_params):
    from supra_b200.nodes import node_types
    assert set(ref_params) <= set(node_types())


def test_parameter_tables_match_the_reference(ref_params):
    from supra_b200.nodes import Node
    for node_type, params in ref_params.items():
        ours = Node(node_type, "N").params()
        for name, spec in params.items():
            assert name in ours, (node_type, name)
            o = ours[name]
            assert o["type"] == spec["type"], (node_type, name)
            if "min" in spec:
                lo, hi = (float(v) for v in o["range"].split(".."))
                assert (lo, hi) == pytest.approx((spec["min"], spec["max"]), rel=1e-12), (node_type, name)
                assert _num(o["default"]) == pytest.approx(spec["default"], rel=1e-12), (node_type, name)
            else:
                if "choices" in spec:
                    want = {str(c).lower() if isinstance(c, bool) else c for c in spec["choices"]}
                    assert set(o["range"].split("|")) == want, (node_type, name)
                d = spec["default"]
                assert o["default"] == (str(d).lower() if isinstance(d, bool) else d), (node_type, name)


def test_invalid_values_fall_back_to_the_default():
    from supra_b200.nodes import Node
    n = Node("BeamformingNode", "B")
    assert n.set("windowType", "Hann") and n.get("windowType") == "Hann"
    assert not n.set("fNumber", 9) and n.get("fNumber") == "1"            # out of range [0.1, 4]
    assert not n.set("windowType", "Blackman") and n.get("windowType") == "Rectangular"
    assert not n.set("outputType", "uint8") and n.get("outputType") == "float"  # not in {float, int16}
    assert n.set("outputType", "int16_t") and n.get("outputType") == "int16"    # SUPRA's alias
    assert n.set("interpolateTransmits", True) and n.get("interpolateTransmits") == "true"
    assert not n.set("additionalOffset", 1.5)                                   # int32_t
    m = Node("BeamformingMVNode", "MV")
    assert m.set("subArraySize", 48) and m.get("subArraySize") == "48"
    assert not m.set("temporalSmoothing", 11) and m.get("temporalSmoothing") == "3"


CONFIG = """<?xml version="1.0"?>
<!-- receive chain in SUPRA's configuration format -->
<supra_config>
  <devices>
    <inputs>
      <input type="UltrasoundInterfaceRawDataMock" id="SRC">
        <param name="frequency" type="int">10</param>
      </input>
    </inputs>
    <outputs>
      <output type="MetaImageOutputDevice" id="OUT"/>
    </outputs>
    <nodes>
      <node type="BeamformingNode" id="BEAM">
        <param name="windowType" type="string">
          Hamming
        </param>
        <param name="windowParameter" type="double">0.5</param>
        <param name="speedOfSound" type="double">1500</param>
      </node>
      <node type="TimeGainCompensationNode" id="TGC"/>
      <node type="TemporalFilterNode" id="FILT"/>
      <node type="HilbertFirEnvelopeNode" id="ENV">
        <param name="filterLength" type="uint32_t">64</param>
      </node>
      <node type="LogCompressorNode" id="LOGC">
        <param name="dynamicRange" type="double">50</param>
        <param name="inMax" type="double">30000</param>
        <param name="outputType" type="DataType">uint8_t</param>
      </node>
      <node type="ScanConverterNode" id="SCAN">
        <param name="outputType" type="DataType">uint8_t</param>
        <param name="notAParameter" type="double">1</param>
      </node>
    </nodes>
  </devices>
  <connections>
    <connection><from id="SRC" port="0"/><to id="BEAM" port="0"/></connection>
    <connection><from id="BEAM" port="0"/><to id="TGC" port="0"/></connection>
    <connection><from id="TGC" port="0"/><to id="FILT" port="0"/></connection>
    <connection><from id="FILT" port="0"/><to id="ENV" port="0"/></connection>
    <connection><from id="ENV" port="0"/><to id="LOGC" port="0"/></connection>
    <connection><from id="LOGC" port="0"/><to id="SCAN" port="0"/></connection>
    <connection><from id="SCAN" port="0"/><to id="OUT" port="0"/></connection>
  </connections>
</supra_config>
"""


def test_graph_from_xml():
    from supra_b200.nodes import Graph
    g = Graph(CONFIG)
    # TimeGainCompensationNode (post-processing) is not built: bypassed
    assert g.chain() == ["BEAM", "FILT", "ENV", "LOGC", "SCAN"]
    assert g.get("FILT", "numImages") == "3"
    assert g.get("BEAM", "windowType") == "Hamming"
    assert float(g.get("BEAM", "speedOfSound")) == 1500.0
    assert g.get("ENV", "filterLength") == "64"
    assert g.get("LOGC", "outputType") == "uint8"
    assert g.get("SCAN", "outputType") == "uint8"
    assert g.get("BEAM", "fNumber") == "1"  # default


def test_graph_xml_errors():
    from supra_b200.abi import SupraError
    from supra_b200.nodes import Graph
    with pytest.raises(SupraError):
        Graph("<supra_config><devices></supra_config>")
    with pytest.raises(SupraError):
        Graph("<other/>")
