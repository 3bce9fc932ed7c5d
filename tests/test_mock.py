"""Recorded-data metadata (SUPRA's .mock / .json) without a GPU: the library's reader against what the
reference's reader made of files written by the reference's writers (tests/golden/mock, generated by
tests/golden/make_mock_fixtures.py from oracle/_ref), and the library's JSON writer round trip."""
import os

import numpy as np
import pytest

from conftest import small_linear, small_matrix
from oracle.oracle import reference_root

MOCK = os.path.join(os.path.dirname(__file__), "golden", "mock")


def f32bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def check_meta(meta, ref):
    sizes, vals = ref["sizes"], ref["vals"]
    assert (meta.num_elements, *meta.element_layout, meta.num_channels, meta.num_samples, meta.num_tx,
            *meta.rx_layout, meta.num_depths) == tuple(int(x) for x in sizes)
    assert np.array_equal(np.array([meta.depth_mm, meta.sampling_frequency_hz, meta.speed_of_sound_mm_s]).view(np.uint64),
                          np.asarray(vals, np.float64).view(np.uint64))
    assert meta.scanlines.tobytes() == np.ascontiguousarray(ref["lines"]).tobytes()
    assert np.array_equal(f32bits(meta.depths), f32bits(ref["depths"]))
    assert np.array_equal(f32bits(meta.element_x), f32bits(ref["xs"]))
    assert np.array_equal(f32bits(meta.element_y), f32bits(ref["ys"]))


@pytest.mark.parametrize("name", ["linear.json", "linear.mock", "matrix.json", "matrix.mock"])
def test_metadata_reader_matches_reference(name):
    from supra_b200.mock import MockMetadata
    gold = np.load(os.path.join(MOCK, "mock_parsed.npz"))
    key = name.replace(".", "_")
    ref = {k: gold[f"{key}_{k}"] for k in ("sizes", "vals", "lines", "depths", "xs", "ys")}
    check_meta(MockMetadata(os.path.join(MOCK, name)), ref)


@pytest.mark.parametrize("make", [small_linear, small_matrix])
def test_json_writer_round_trip(tmp_path, make):
    """writeMetaDataForMock then readMetaDataForMock gives back the geometry (depths derived as the
    reference does, which is how the geometry builds them)."""
    from supra_b200.mock import MockMetadata, write_mock_json
    g = make()
    fn = str(tmp_path / "probe.json")
    write_mock_json(fn, g)
    m = MockMetadata(fn)
    assert (m.num_elements, m.num_channels, m.num_samples, m.num_tx, m.rx_layout, m.num_depths) == \
        (g.num_elements, g.num_channels, g.num_samples, g.num_tx, tuple(g.rx_layout), g.num_depths)
    assert m.depth_mm == g.depth_mm and m.speed_of_sound_mm_s == g.speed_of_sound_mm_s
    assert m.sampling_frequency_hz == g.sampling_frequency_hz
    assert m.scanlines.tobytes() == np.ascontiguousarray(g.scanlines).tobytes()
    assert np.array_equal(f32bits(m.depths), f32bits(g.depths))
    assert np.array_equal(f32bits(m.element_x), f32bits(g.element_x))
    assert np.array_equal(f32bits(m.element_y), f32bits(g.element_y))


@pytest.mark.skipif(reference_root() is None, reason="reference sources not named by SUPRA_REF")
def test_reference_reads_library_json(tmp_path, oracle):
    """The reference's reader on the library's JSON gives what the library's reader gives."""
    from supra_b200.mock import MockMetadata, write_mock_json
    oracle.build(ref=True)
    for make in (small_linear, small_matrix):
        fn = str(tmp_path / "probe.json")
        write_mock_json(fn, make())
        check_meta(MockMetadata(fn), oracle.ref_mock_read(fn))


def test_metadata_errors(tmp_path):
    from supra_b200.abi import SupraError
    from supra_b200.mock import MockMetadata
    with pytest.raises(SupraError):
        MockMetadata(str(tmp_path / "missing.json"))
    bad = tmp_path / "probe.txt"
    bad.write_text("{}")
    with pytest.raises(SupraError):
        MockMetadata(str(bad))  # unknown suffix
    trunc = tmp_path / "probe.mock"
    trunc.write_text("rawDataMockMetadata v 1\n32 32 1 16 512")
    with pytest.raises(SupraError):
        MockMetadata(str(trunc))
    broken = tmp_path / "broken.json"
    broken.write_text('{"numElements": 3,')
    with pytest.raises(SupraError):
        MockMetadata(str(broken))
