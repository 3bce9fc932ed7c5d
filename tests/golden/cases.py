"""Parameter sets of the golden fixtures (shared by make_golden.py and tests/test_oracle_pin.py)."""
FIR_CASES = [(65, 3, 2, 2.0, 0.0, 0.0), (64, 3, 2, 2.0, 0.0, 0.0), (51, 0, 2, 40e6, 2.5e6, 0.0),
             (32, 0, 2, 40e6, 2.5e6, 0.0), (51, 2, 3, 40e6, 7e6, 1e6), (51, 1, 1, 40e6, 3e6, 0.0),
             (33, 2, 3, 20e6, 5e6, 2e6), (17, 0, 0, 20e6, 4e6, 0.0)]
WIN_CASES = [(0, 0.0), (1, 0.0), (1, 0.25), (2, 0.0), (2, 0.5), (3, 0.3), (3, 1.0)]
DAS_CASES = [  # (geometry, f-number, window, window param, interpolate transmits, offset)
    ("lin", 1.0, 1, 0.0, 0, 0), ("lin", 0.7, 2, 0.1, 1, 3), ("lin", 2.0, 0, 0.0, 0, -2),
    ("mat", 1.0, 1, 0.0, 0, 0), ("mat", 1.5, 3, 0.5, 1, 1),
]
DAS_BF_CASES = [  # (geometry, sample beamformer, f-number, window, window param, interpolate transmits, offset)
    ("lin", 1, 1.0, 1, 0.0, 0, 0), ("lin", 2, 1.0, 1, 0.0, 0, 0), ("lin", 1, 0.7, 2, 0.1, 1, 3),
    ("lin", 2, 2.0, 0, 0.0, 1, -2), ("mat", 1, 1.0, 1, 0.0, 0, 0), ("mat", 2, 1.5, 3, 0.5, 1, 1),
    ("lin_deep", 3, 1.0, 1, 0.0, 0, 0), ("mat_deep", 3, 1.0, 1, 0.0, 1, 0), ("lin_deep", 1, 1.0, 1, 0.0, 0, 0),
]
