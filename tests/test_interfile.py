"""Interfile projection data headers (InterfilePDFSHeader's data-addressing keys) and the oracle's stream reader."""
import os

import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import interfile

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scatter_cylinder.npz")


def test_segment_sequence():
    assert interfile.segment_sequence([-4, -3, -2, -1, 0, 1, 2, 3, 4], [-4, -3, -2, -1, 0, 1, 2, 3, 4]) == list(range(-4, 5))
    assert interfile.segment_sequence([0, -2, 1], [0, -1, 2]) == [0, -1, 1]
    with pytest.raises(ValueError, match="segment 0"):
        interfile.segment_sequence([1, 2], [1, 2])


def _header(tmp_path, body):
    p = tmp_path / "h.hs"
    p.write_text(body)
    (tmp_path / "h.s").write_bytes(b"")
    return str(p)


def test_parse_keys_and_storage_orders(tmp_path):
    common = """!INTERFILE :=
name of data file := h.s
!number format := signed integer
!number of bytes per pixel := 2
number of dimensions := 4
matrix axis label [4] := segment
!matrix size [4] := 3
matrix axis label [1] := tangential coordinate
!matrix size [1] := 5
minimum ring difference per segment := {-2, 0, 1}   ; comment
maximum ring difference per segment := {-1, 0, 2}
data offset in bytes [1] := 16
image scaling factor [1] := 0.5
"""
    savt = common + """matrix axis label [2] := view
!matrix size [2] := 6
matrix axis label [3] := axial coordinate
!matrix size [3] := {3, 4, 3}
"""
    h = interfile.InterfileProjDataHeader(_header(tmp_path, savt))
    assert h.storage_order == _abi.STORAGE_SEGMENT_AXIAL_VIEW_TANG
    assert (h.num_views, h.num_tangential_poss, h.num_axial_poss) == (6, 5, [3, 4, 3])
    assert h.segment_sequence == [-1, 0, 1]
    assert h.number_type == "short" and h.big_endian  # Interfile's default byte order
    assert h.data_offset == 16 and h.scale_factor == 0.5 and h.num_timing_poss == 1
    svat = common.replace("signed integer", "float").replace("!number of bytes per pixel := 2",
                                                              "!number of bytes per pixel := 4") + """imagedata byte order := LITTLEENDIAN
matrix axis label [3] := view
!matrix size [3] := 6
matrix axis label [2] := axial coordinate
!matrix size [2] := {3, 4, 3}
"""
    h = interfile.InterfileProjDataHeader(_header(tmp_path, svat))
    assert h.storage_order == _abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG and h.number_type == "float" and not h.big_endian
    with pytest.raises(ValueError):
        interfile.InterfileProjDataHeader(_header(tmp_path, common))  # no view / axial labels


def test_reads_stir_test_pack_header(oracle_lib, tmp_path):
    """scatter_cylinder.hs of STIR's recon_test_pack (header text and data bytes in a fixture written by
    golden/make_fixtures.py): 1 segment, 32 views, 8 rings, 35 bins, float LE, view-major."""
    fx = np.load(GOLDEN)
    (tmp_path / "scatter_cylinder.hs").write_bytes(fx["header"].tobytes())
    (tmp_path / "scatter_cylinder.s").write_bytes(fx["data"].tobytes())
    h = interfile.InterfileProjDataHeader(str(tmp_path / "scatter_cylinder.hs"))
    assert h.storage_order == _abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG
    assert (h.num_views, h.num_axial_poss, h.num_tangential_poss) == (32, [8], 35)
    assert h.segment_sequence == [0] and h.number_type == "float" and not h.big_endian
    raw = np.fromfile(h.data_file, dtype=np.uint8, offset=h.data_offset)
    assert raw.size == 32 * 8 * 35 * 4
    geo = _abi.Geometry(num_views=32, num_tangential_poss=35, max_segment_num=0)
    pd = oracle_lib.projdata_from_stream(raw, geo, h.storage_order, h.number_type, h.big_endian, h.scale_factor,
                                         h.segment_sequence, h.num_axial_poss)
    # ProjDataInMemory order is [axial][view][tangential]: element (a, v, t) is the file's (v, a, t)
    f = np.frombuffer(raw.tobytes(), "<f4").reshape(32, 8, 35)
    assert np.array_equal(pd.reshape(8, 32, 35), f.transpose(1, 0, 2))
