"""Regenerates tests/golden/ref_pins.npz from the reference's own code compiled in oracle/_ref
(FirFilterFactory, WindowFunction, and the per-sample reducers of the four sample beamformers,
RxSampleBeamformerDelayAndSum.h, ...DelayAndStdDev.h, ...CoherenceFactorDelayAndSum.h, ...TestSignal.h).

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures pin the oracle (tests/test_oracle_pin.py) even where oracle/_ref is not built.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from conftest import bf_geometries, random_rf, small_linear, small_matrix  # noqa: E402
from oracle import oracle as O  # noqa: E402

from golden.cases import DAS_BF_CASES, DAS_CASES, FIR_CASES, WIN_CASES  # noqa: E402


def main():
    assert O.ref_lib() is not None, "build oracle/_ref first: make -C oracle ref"
    out = {}
    for i, c in enumerate(FIR_CASES):
        out[f"fir_{i}"] = O.fir(*c, ref=True)
        out[f"fir_{i}_case"] = np.array(c, np.float64)
    for i, (t, p) in enumerate(WIN_CASES):
        out[f"win_{i}"] = O.window_lut(t, p, 64, ref=True)
        out[f"win_{i}_case"] = np.array([t, p], np.float64)
    geoms = {"lin": small_linear(), "mat": small_matrix()}
    for i, (gname, F, w, wp, itx, off) in enumerate(DAS_CASES):
        g = geoms[gname]
        rf = random_rf(g, seed=100 + i)  # regenerated from the seed by the test
        out[f"das_{i}"] = O.das(g, rf, F, window=w, window_param=wp, interp_tx=bool(itx), additional_offset=off,
                                ref=True)
    bgeoms = bf_geometries()
    for i, (gname, bf, F, w, wp, itx, off) in enumerate(DAS_BF_CASES):
        g = bgeoms[gname]
        rf = random_rf(g, seed=200 + i)
        out[f"dasbf_{i}"] = O.das_bf(g, rf, bf, F, window=w, window_param=wp, interp_tx=bool(itx),
                                     additional_offset=off, ref=True)
    np.savez_compressed(os.path.join(HERE, "ref_pins.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_pins.npz"))


if __name__ == "__main__":
    main()
