"""Projection data streams on the GPU (b200rt_projdata_from/to_stream_dev, stir_b200.interfile) against the
oracle's element-by-element restatement of ProjDataFromStream::get_offset."""
import numpy as np
import pytest

from stir_b200 import _abi
from stir_b200 import geometry as G

pytestmark = pytest.mark.gpu

NP = {"schar": "i1", "uchar": "u1", "short": "i2", "ushort": "u2", "int": "i4", "uint": "u4", "float": "f4",
      "double": "f8"}
FORMAT = {"schar": ("signed integer", 1), "uchar": ("unsigned integer", 1), "short": ("signed integer", 2),
          "ushort": ("unsigned integer", 2), "int": ("signed integer", 4), "uint": ("unsigned integer", 4),
          "float": ("float", 4), "double": ("float", 8)}


def _write_stream(tmp_path, g, order, ntype, big, scale, seq, extra_seg, offset, rng, ntof=1):
    """A header and data file with segments in the order `seq` (the file may hold one more segment pair than the
    projector uses), random values of the number type."""
    S = g.max_segment_num
    nv, nt = g.num_views, g.num_tangential_poss
    nax = {s: g.num_axial_poss[s + S] for s in range(-S, S + 1)}
    if extra_seg:
        nax[S + 1] = max(1, nax[S] - 2)
        nax[-S - 1] = max(1, nax[S] - 2)
    naxs = [nax[s] for s in seq]
    n = sum(naxs) * nv * nt * ntof
    dt = np.dtype(NP[ntype]).newbyteorder(">" if big else "<")
    if ntype in ("float", "double"):
        vals = rng.uniform(-5, 5, n)
    else:
        info = np.iinfo(NP[ntype])
        vals = rng.integers(info.min, info.max, n, endpoint=True)
    data = vals.astype(dt)
    (tmp_path / "p.s").write_bytes(b"\x07" * offset + data.tobytes())
    # ring differences that give the sequence: ring difference = segment number
    labels = (["matrix axis label [3] := view", f"!matrix size [3] := {nv}", "matrix axis label [2] := axial coordinate",
               "!matrix size [2] := {" + ",".join(map(str, naxs)) + "}"]
              if order == _abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG else
              ["matrix axis label [2] := view", f"!matrix size [2] := {nv}", "matrix axis label [3] := axial coordinate",
               "!matrix size [3] := {" + ",".join(map(str, naxs)) + "}"])
    fmt, nb = FORMAT[ntype]
    hdr = ["!INTERFILE :=", "name of data file := p.s", f"!number format := {fmt}", f"!number of bytes per pixel := {nb}",
           f"imagedata byte order := {'BIGENDIAN' if big else 'LITTLEENDIAN'}", f"data offset in bytes[1] := {offset}",
           f"image scaling factor[1] := {scale}", f"number of dimensions := {5 if ntof > 1 else 4}",
           "matrix axis label [4] := segment", f"!matrix size [4] := {len(seq)}",
           "matrix axis label [1] := tangential coordinate", f"!matrix size [1] := {nt}"] + labels
    if ntof > 1:
        hdr += ["matrix axis label [5] := timing positions", f"!matrix size [5] := {ntof}"]
    hdr += ["minimum ring difference per segment := {" + ",".join(map(str, seq)) + "}",
            "maximum ring difference per segment := {" + ",".join(map(str, seq)) + "}", "!END OF INTERFILE :="]
    (tmp_path / "p.hs").write_text("\n".join(hdr) + "\n")
    return str(tmp_path / "p.hs"), naxs


@pytest.fixture(scope="module")
def small(cuda_device):
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.small_3d_pet()
    return RayTracingProjector(pdi, img, device=cuda_device)


@pytest.mark.parametrize("order", [_abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG, _abi.STORAGE_SEGMENT_AXIAL_VIEW_TANG])
@pytest.mark.parametrize("ntype,big,scale", [("float", False, 1.0), ("float", True, 1.0), ("short", True, 0.25),
                                             ("ushort", False, 2.0), ("uchar", False, 1.5), ("schar", True, 1.0),
                                             ("int", False, 1e-3), ("uint", True, 1.0), ("double", True, 1.0)])
@pytest.mark.parametrize("sequence", ["ascending", "stir_memory", "extra_segments"])
def test_read_matches_oracle(tmp_path, small, oracle_lib, order, ntype, big, scale, sequence):
    from stir_b200 import interfile
    proj = small
    g = proj.geometry
    S = g.max_segment_num
    rng = np.random.default_rng(3)
    if sequence == "ascending":
        seq, extra = list(range(-S, S + 1)), False
    elif sequence == "stir_memory":
        seq, extra = [0] + [s for k in range(1, S + 1) for s in (k, -k)], False
    else:
        seq, extra = [S + 1] + list(range(S, -S - 2, -1)), True
    offset = 13 if sequence == "extra_segments" else 0
    path, naxs = _write_stream(tmp_path, g, order, ntype, big, scale, seq, extra, offset, rng)
    got = proj.projdata_from_device_layout(interfile.read_projdata(path, proj)).cpu().numpy()
    raw = np.fromfile(str(tmp_path / "p.s"), np.uint8, offset=offset)
    ref = oracle_lib.projdata_from_stream(raw, g, order, ntype, big, scale, seq, naxs)
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_write_read_round_trip_and_layout(tmp_path, small, oracle_lib):
    import torch
    from stir_b200 import interfile
    proj = small
    g = proj.geometry
    S = g.max_segment_num
    y = torch.rand(proj.projdata_size, device="cuda")
    hs = interfile.write_projdata(str(tmp_path / "w.hs"), proj, y)
    back = interfile.read_projdata(hs, proj)
    assert torch.equal(back, y)
    h = interfile.InterfileProjDataHeader(hs)
    assert h.storage_order == _abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG and h.segment_sequence == list(range(-S, S + 1))
    raw = np.fromfile(h.data_file, np.uint8)
    ref = oracle_lib.projdata_from_stream(raw, g, h.storage_order, "float", False, 1.0, h.segment_sequence,
                                          h.num_axial_poss)
    assert np.array_equal(ref, proj.projdata_from_device_layout(y).cpu().numpy())


def test_tof_stream(tmp_path, cuda_device, oracle_lib):
    from stir_b200 import interfile
    from stir_b200.projectors import RayTracingProjector
    pdi, img = G.tof_small_3d_pet(num_tof_bins=5, timing_bin_ps=250.0, num_views=48)
    proj = RayTracingProjector(pdi, img, device=cuda_device)
    g = proj.geometry
    S = g.max_segment_num
    ntof = proj.info.num_tof_bins
    seq = list(range(-S, S + 1))
    path, naxs = _write_stream(tmp_path, g, _abi.STORAGE_SEGMENT_AXIAL_VIEW_TANG, "float", False, 1.0, seq, False, 0,
                               np.random.default_rng(9), ntof=ntof)
    got = proj.projdata_from_device_layout(interfile.read_projdata(path, proj)).cpu().numpy()
    raw = np.fromfile(str(tmp_path / "p.s"), np.uint8)
    ref = oracle_lib.projdata_from_stream(raw, g, _abi.STORAGE_SEGMENT_AXIAL_VIEW_TANG, "float", False, 1.0, seq, naxs,
                                          num_timing_poss=ntof)
    assert np.array_equal(got, ref)


def test_stream_errors(tmp_path, small):
    from stir_b200 import interfile
    proj = small
    g = proj.geometry
    S = g.max_segment_num
    # a stream without the projector's outermost segments
    path, _ = _write_stream(tmp_path, g, _abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG, "float", False, 1.0,
                            list(range(-S + 1, S)), False, 0, np.random.default_rng(1))
    with pytest.raises(_abi.B200Error, match="missing"):
        interfile.read_projdata(path, proj)
