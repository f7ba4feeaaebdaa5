"""USC-HairSalon .data files (kami_usc_info / kami_usc_read / kami_usc_write), against an
independent restatement of the format with `struct`: a uint32 strand count, then per strand a
uint32 vertex count and that many float32 xyz triples (importers/USCHairsalonImporter.cpp:56-80,
exporters/USCHairsalonExporter.cpp:6-18)."""
import struct

import numpy as np
import pytest

from kamisimulator_b200 import synth, vbd


def _struct_bytes(counts, packed):
    out = [struct.pack("<I", len(counts))]
    k = 0
    for n in counts:
        out.append(struct.pack("<I", int(n)))
        out.append(struct.pack("<%df" % (3 * n), *packed[k:k + n].ravel()))
        k += n
    return b"".join(out)


def _groom():
    g = synth.groom_strands(np.random.default_rng(3), np.array([5, 1, 12, 0, 7, 3]))
    return np.diff(g.strand_begin).astype(np.int32), g.positions.astype(np.float32)


def test_written_bytes_match_the_format(tmp_path):
    counts, packed = _groom()
    path = tmp_path / "hair.data"
    vbd.write_usc(path, counts, packed)
    assert path.read_bytes() == _struct_bytes(counts, packed)


def test_read_packed_and_padded(tmp_path):
    counts, packed = _groom()
    path = tmp_path / "hair.data"
    path.write_bytes(_struct_bytes(counts, packed))
    c, x = vbd.read_usc(path)
    np.testing.assert_array_equal(c, counts)
    np.testing.assert_array_equal(x, packed)
    c, xp = vbd.read_usc(path, max_verts=16)
    assert xp.shape == (len(counts), 16, 3)
    k = 0
    for s, n in enumerate(counts):
        np.testing.assert_array_equal(xp[s, :n], packed[k:k + n])
        assert not xp[s, n:].any()
        k += n
    # a padded array writes back to the same file
    vbd.write_usc(tmp_path / "again.data", c, xp, max_verts=16)
    assert (tmp_path / "again.data").read_bytes() == path.read_bytes()


def test_bad_files_are_reported(tmp_path):
    counts, packed = _groom()
    data = _struct_bytes(counts, packed)
    with pytest.raises(vbd.KamiError, match="KAMI_ERR_IO"):
        vbd.read_usc(tmp_path / "missing.data")
    (tmp_path / "cut.data").write_bytes(data[:-5])
    with pytest.raises(vbd.KamiError, match="KAMI_ERR_IO"):
        vbd.read_usc(tmp_path / "cut.data")
    (tmp_path / "huge.data").write_bytes(struct.pack("<I", 1 << 30))
    with pytest.raises(vbd.KamiError, match="KAMI_ERR_IO"):
        vbd.read_usc(tmp_path / "huge.data")
    (tmp_path / "ok.data").write_bytes(data)
    with pytest.raises(vbd.KamiError, match="max_verts"):
        vbd.read_usc(tmp_path / "ok.data", max_verts=8)  # a strand of 12 vertices
    (tmp_path / "empty.data").write_bytes(struct.pack("<I", 0))
    c, x = vbd.read_usc(tmp_path / "empty.data")
    assert c.shape == (0,) and x.shape == (0, 3)
