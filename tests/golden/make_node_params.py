"""Regenerates tests/golden/node_params.json: the parameter tables (name, type, range or choices,
default) that the reference's receive-path node constructors declare with
m_valueRangeDictionary.set<T>(...), read from the reference sources as text.

    python tests/golden/make_node_params.py [reference root, default $SUPRA_REF]

The fixture lets tests check the node layer's tables where the reference tree is absent.
"""
import ast
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NODES = {
    "BeamformingNode": "BeamformingNode.cpp",
    "RawDelayNode": "RawDelayNode.cpp",
    "BeamformingMVNode": "BeamformingMVNode.cpp",
    "BeamformingMVpcgNode": "BeamformingMVpcgNode.cpp",
    "HilbertFirEnvelopeNode": "HilbertFirEnvelopeNode.cpp",
    "HilbertEnvelopeNode": "HilbertEnvelopeNode.cpp",
    "IQDemodulatorNode": "IQDemodulatorNode.cpp",
    "LogCompressorNode": "LogCompressorNode.cpp",
    "ScanConverterNode": "ScanConverterNode.cpp",
    "TemporalFilterNode": "TemporalFilterNode.cpp",
}
DTYPES = {"TypeFloat": "float", "TypeInt16": "int16", "TypeUint8": "uint8", "TypeUint16": "uint16"}
CALL = re.compile(r'm_valueRangeDictionary\.set<\s*(\w+)\s*>\((.*)\);')


def split_args(s):
    """Top-level comma split (braces and quotes kept together)."""
    out, depth, cur, q = [], 0, "", False
    for ch in s:
        if ch == '"':
            q = not q
        if not q and ch == "{":
            depth += 1
        if not q and ch == "}":
            depth -= 1
        if ch == "," and depth == 0 and not q:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    out.append(cur.strip())
    return out


def value(tok, typ):
    tok = tok.strip()
    if typ == "DataType":
        return DTYPES[tok]
    if typ == "bool":
        return tok == "true"
    if typ == "string":
        return ast.literal_eval(tok)
    return float(eval(tok, {"__builtins__": {}}, {}))  # numeric literals and products such as 20 * 1e6


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SUPRA_REF", "")
    if not root:
        sys.exit("name the reference's source tree: argument or SUPRA_REF")
    bf = os.path.join(root, "src", "SupraLib", "Beamformer")
    out = {}
    for node, fname in NODES.items():
        text = open(os.path.join(bf, fname)).read()
        params = {}
        for m in CALL.finditer(text):
            typ, args = m.group(1), split_args(m.group(2))
            name = ast.literal_eval(args[0])
            if len(args) == 3:  # set<T>(name, default, label): no range
                params[name] = {"type": typ, "default": value(args[1], typ)}
            elif args[1].startswith("{"):
                choices = [value(t, typ) for t in split_args(args[1][1:-1])]
                params[name] = {"type": typ, "choices": choices, "default": value(args[2], typ)}
            else:
                params[name] = {"type": typ, "min": value(args[1], typ), "max": value(args[2], typ),
                                "default": value(args[3], typ)}
        out[node] = params
    with open(os.path.join(HERE, "node_params.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print({k: len(v) for k, v in out.items()})


if __name__ == "__main__":
    main()
