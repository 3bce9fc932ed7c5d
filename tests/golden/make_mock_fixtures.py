"""Regenerates tests/golden/mock/: metadata files written by the reference's own writers (JSON by
RxBeamformerParameters::writeMetaDataForMock; ASCII in the layout of readMetaDataForMockAscii with
the reference's scanline stream operator) for a 2D and a 3D geometry, and what the reference's reader
(readMetaDataForMock) makes of each, in mock_parsed.npz.

    make -C oracle ref && python tests/golden/make_mock_fixtures.py

The fixtures pin the library's metadata reader (tests/test_mock.py) where oracle/_ref is not built.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))

from conftest import small_linear, small_matrix  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(HERE, "mock")


def main():
    assert O.ref_lib() is not None, "build oracle/_ref first: make -C oracle ref"
    os.makedirs(OUT, exist_ok=True)
    parsed = {}
    for name, geom in (("linear", small_linear()), ("matrix", small_matrix())):
        for ext, ascii_format in ((".json", False), (".mock", True)):
            fn = os.path.join(OUT, name + ext)
            O.ref_mock_write(fn, geom, ascii_format=ascii_format)
            r = O.ref_mock_read(fn)
            key = name + ext.replace(".", "_")
            for k, v in r.items():
                parsed[f"{key}_{k}"] = v
    np.savez_compressed(os.path.join(OUT, "mock_parsed.npz"), **parsed)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
