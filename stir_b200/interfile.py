"""Interfile projection data (STIR's ".hs" + ".s") read into and written from device-resident projection data.

The header is parsed on the host as STIR's InterfilePDFSHeader does for the keys that address the data
(src/IO/InterfileHeader.cxx: "name of data file", "number format" / "number of bytes per pixel",
"imagedata byte order" (default BIGENDIAN), "data offset in bytes", "image scaling factor", "matrix axis label" /
"matrix size" (the storage order, InterfilePDFSHeader::find_storage_order), "minimum/maximum ring difference
per segment" (the segment sequence, find_segment_sequence), "TOF bin order"); the file's bytes are copied to
the GPU as they are and converted there (b200rt_projdata_from_stream_dev).  Writing produces a float
Segment_View_AxialPos_TangPos stream with a header STIR reads back.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import Dict, List, Optional

import numpy as np

from . import _abi
from .projectors import RayTracingProjector, _stream_ptr

_NUMBER_TYPES = {("signed integer", 1): "schar", ("signed integer", 2): "short", ("signed integer", 4): "int",
                 ("unsigned integer", 1): "uchar", ("unsigned integer", 2): "ushort", ("unsigned integer", 4): "uint",
                 ("float", 4): "float", ("float", 8): "double"}


def _norm_key(k: str) -> str:
    k = k.strip().lstrip("!").strip().lower()
    return re.sub(r"\s+", " ", k)


def _value(v: str):
    v = v.strip()
    if v.startswith("{") and v.endswith("}"):
        return [x.strip() for x in v[1:-1].split(",") if x.strip()]
    return v


def parse_interfile(text: str) -> Dict[str, object]:
    """key := value lines; keys case-insensitive without "!" and with single spaces; "key [i]" kept with its index;
    comments after ";" dropped; {a, b} lists become lists of strings."""
    out: Dict[str, object] = {}
    for line in text.splitlines():
        line = line.split(";", 1)[0]
        if ":=" not in line:
            continue
        k, v = line.split(":=", 1)
        k = _norm_key(k)
        m = re.match(r"^(.*?)\s*\[\s*(\d+)\s*\]$", k)
        if m:
            k = f"{m.group(1)} [{int(m.group(2))}]"
        out[k] = _value(v)
    return out


def _ints(v) -> List[int]:
    return [int(float(x)) for x in (v if isinstance(v, list) else [v])]


def segment_sequence(min_ring_diff: List[int], max_ring_diff: List[int]) -> List[int]:
    """find_segment_sequence (InterfileHeader.cxx:795-935): segments numbered by sorting the sums of the ring
    differences, 0 where the sum is 0; returns the segment number of each segment in the file's order."""
    n = len(min_ring_diff)
    sums = sorted(((float(min_ring_diff[i] + max_ring_diff[i]), i) for i in range(n)), key=lambda p: p[0])
    zero = 0
    while zero < n and sums[zero][0] < -1e-3:
        zero += 1
    if zero == n or sums[zero][0] > 1e-3:
        raise ValueError("This data does not seem to contain segment 0.")
    seq = [0] * n
    for rank, (_, loc) in enumerate(sums):
        seq[loc] = rank - zero
    return seq


class InterfileProjDataHeader:
    """The data-addressing part of an Interfile projection data header."""

    def __init__(self, path: str):
        self.path = path
        with open(path, "r", errors="replace") as f:
            keys = parse_interfile(f.read())
        self.keys = keys
        data_file = str(keys.get("name of data file", ""))
        if not data_file:
            raise ValueError("Interfile header without 'name of data file'")
        self.data_file = data_file if os.path.isabs(data_file) else os.path.join(os.path.dirname(path), data_file)
        fmt = str(keys.get("number format", "unsigned integer")).lower()
        nbytes = int(keys.get("number of bytes per pixel", 2 if fmt != "float" else 4))
        if (fmt, nbytes) not in _NUMBER_TYPES:
            raise ValueError(f"unsupported number format {fmt!r} with {nbytes} bytes per pixel")
        self.number_type = _NUMBER_TYPES[(fmt, nbytes)]
        self.big_endian = str(keys.get("imagedata byte order", "BIGENDIAN")).upper() != "LITTLEENDIAN"
        off = keys.get("data offset in bytes [1]", keys.get("data offset in bytes", 0))
        self.data_offset = int(float(off[0] if isinstance(off, list) else off))
        sf = keys.get("image scaling factor [1]", keys.get("image scaling factor", 1.0))
        self.scale_factor = float(sf[0] if isinstance(sf, list) else sf)
        ndim = int(keys.get("number of dimensions", 0))
        if ndim not in (4, 5):
            raise ValueError("Interfile error: expecting 4D structure or 5D in case of TOF information")
        labels = [str(keys.get(f"matrix axis label [{i}]", "")).lower() for i in range(1, ndim + 1)]
        sizes = [keys.get(f"matrix size [{i}]") for i in range(1, ndim + 1)]
        if labels[0] != "tangential coordinate":
            raise ValueError("Interfile error: expecting 'matrix axis label[1] := tangential coordinate'")
        if labels[3] != "segment":
            raise ValueError("Interfile error: matrix labels not in expected (or supported) format")
        self.num_tangential_poss = _ints(sizes[0])[0]
        if labels[1] == "axial coordinate" and labels[2] == "view":
            self.storage_order = _abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG
            self.num_views = _ints(sizes[2])[0]
            self.num_axial_poss = _ints(sizes[1])
        elif labels[1] == "view" and labels[2] == "axial coordinate":
            self.storage_order = _abi.STORAGE_SEGMENT_AXIAL_VIEW_TANG
            self.num_views = _ints(sizes[1])[0]
            self.num_axial_poss = _ints(sizes[2])
        else:
            raise ValueError("Interfile error: matrix labels not in expected (or supported) format")
        nseg = _ints(sizes[3])[0]
        if ndim == 5:
            if labels[4] != "timing positions":
                raise ValueError("Interfile header parsing: currently need 'matrix axis label [5] := timing positions'")
            self.num_timing_poss = _ints(sizes[4])[0]
        else:
            self.num_timing_poss = 1
        self.min_ring_difference = _ints(keys.get("minimum ring difference per segment", [0] * nseg))
        self.max_ring_difference = _ints(keys.get("maximum ring difference per segment", [0] * nseg))
        if not (len(self.num_axial_poss) == len(self.min_ring_difference) == len(self.max_ring_difference) == nseg):
            raise ValueError("Interfile error: per-segment lists of the wrong length")
        self.segment_sequence = segment_sequence(self.min_ring_difference, self.max_ring_difference)
        order = keys.get("tof bin order")
        self.timing_poss_sequence = _ints(order) if order is not None and self.num_timing_poss > 1 else None

    def stream_format(self):
        """(b200rt_stream_format, the arrays it points to)"""
        seq = (ctypes.c_int32 * len(self.segment_sequence))(*self.segment_sequence)
        nax = (ctypes.c_int32 * len(self.num_axial_poss))(*self.num_axial_poss)
        tps = None
        if self.timing_poss_sequence is not None:
            tps = (ctypes.c_int32 * len(self.timing_poss_sequence))(*self.timing_poss_sequence)
        f = _abi.StreamFormat(storage_order=self.storage_order, number_type=_abi.NUMBER_TYPES[self.number_type],
                              swap_bytes=int(self.big_endian), scale_factor=self.scale_factor,
                              num_segments=len(self.segment_sequence),
                              segment_sequence=ctypes.cast(seq, ctypes.POINTER(ctypes.c_int32)),
                              num_axial_poss=ctypes.cast(nax, ctypes.POINTER(ctypes.c_int32)),
                              num_timing_poss=self.num_timing_poss,
                              timing_poss_sequence=None if tps is None else ctypes.cast(tps, ctypes.POINTER(ctypes.c_int32)))
        return f, (seq, nax, tps)


def read_projdata(header_path: str, projector: RayTracingProjector, out=None, stream=None):
    """The projection data of an Interfile header as a device-layout CUDA tensor for `projector` (views and
    tangential positions must match; segments the projector does not use are skipped)."""
    import torch
    hdr = InterfileProjDataHeader(header_path)
    if hdr.num_views != projector.geometry.num_views or hdr.num_tangential_poss != projector.geometry.num_tangential_poss:
        raise ValueError("the file's views or tangential positions differ from the projector's")
    fmt, keep = hdr.stream_format()
    nbytes = ctypes.c_int64()
    _abi.check(projector.lib.b200rt_stream_bytes(projector.h, ctypes.byref(fmt), ctypes.byref(nbytes)), projector.h,
               "b200rt_stream_bytes")
    raw = np.fromfile(hdr.data_file, dtype=np.uint8, count=nbytes.value, offset=hdr.data_offset)
    if raw.size < nbytes.value:
        raise ValueError(f"{hdr.data_file}: {raw.size} bytes after the data offset, the header needs {nbytes.value}")
    dev = torch.from_numpy(raw).to(torch.device("cuda", projector.device))
    out = projector.empty_projdata(zero=False) if out is None else out
    _abi.check(projector.lib.b200rt_projdata_from_stream_dev(projector.h, ctypes.c_void_p(dev.data_ptr()), dev.numel(),
                                                             ctypes.byref(fmt), ctypes.c_void_p(out.data_ptr()),
                                                             _stream_ptr(stream)),
               projector.h, "b200rt_projdata_from_stream_dev")
    torch.cuda.synchronize(projector.device)  # the staged bytes are released on return
    del keep
    return out


def write_projdata(header_path: str, projector: RayTracingProjector, projdata_dev, stream=None):
    """Writes device-layout projection data as Interfile: `header_path` (".hs") and the float little-endian
    Segment_View_AxialPos_TangPos data beside it (".s"), segments in increasing order, as ProjDataInterfile
    writes by default."""
    import torch
    g = projector.geometry
    S = g.max_segment_num
    segs = list(range(-S, S + 1))
    nax = [g.num_axial_poss[s + S] for s in segs]
    ntof = projector.info.num_tof_bins
    seq = (ctypes.c_int32 * len(segs))(*segs)
    naxa = (ctypes.c_int32 * len(segs))(*nax)
    fmt = _abi.StreamFormat(storage_order=_abi.STORAGE_SEGMENT_VIEW_AXIAL_TANG, number_type=_abi.NUMBER_TYPES["float"],
                            swap_bytes=0, scale_factor=1.0, num_segments=len(segs),
                            segment_sequence=ctypes.cast(seq, ctypes.POINTER(ctypes.c_int32)),
                            num_axial_poss=ctypes.cast(naxa, ctypes.POINTER(ctypes.c_int32)), num_timing_poss=ntof,
                            timing_poss_sequence=None)
    nbytes = ctypes.c_int64()
    _abi.check(projector.lib.b200rt_stream_bytes(projector.h, ctypes.byref(fmt), ctypes.byref(nbytes)), projector.h,
               "b200rt_stream_bytes")
    dev = torch.empty(nbytes.value, dtype=torch.uint8, device=projdata_dev.device)
    _abi.check(projector.lib.b200rt_projdata_to_stream_dev(projector.h, ctypes.c_void_p(projdata_dev.data_ptr()),
                                                           ctypes.byref(fmt), ctypes.c_void_p(dev.data_ptr()),
                                                           dev.numel(), _stream_ptr(stream)),
               projector.h, "b200rt_projdata_to_stream_dev")
    torch.cuda.synchronize(projector.device)
    data_path = os.path.splitext(header_path)[0] + ".s"
    dev.cpu().numpy().tofile(data_path)
    mins = [g.min_ring_diff[s + S] for s in segs]
    maxs = [g.max_ring_diff[s + S] for s in segs]
    fmtl = lambda v: "{" + ",".join(str(x) for x in v) + "}"
    lines = [
        "!INTERFILE  :=",
        "!imaging modality := PT",
        f"name of data file := {os.path.basename(data_path)}",
        "!version of keys := STIR4.0",
        "!GENERAL DATA :=",
        "!GENERAL IMAGE DATA :=",
        "!type of data := PET",
        "imagedata byte order := LITTLEENDIAN",
        "!PET STUDY (General) :=",
        "!PET data type := Emission",
        "applied corrections := {None}",
        "!number format := float",
        "!number of bytes per pixel := 4",
        f"number of dimensions := {5 if ntof > 1 else 4}",
        "matrix axis label [4] := segment",
        f"!matrix size [4] := {len(segs)}",
        "matrix axis label [3] := view",
        f"!matrix size [3] := {g.num_views}",
        "matrix axis label [2] := axial coordinate",
        f"!matrix size [2] := {fmtl(nax)}",
        "matrix axis label [1] := tangential coordinate",
        f"!matrix size [1] := {g.num_tangential_poss}",
    ]
    if ntof > 1:
        lines += ["matrix axis label [5] := timing positions", f"!matrix size [5] := {ntof}"]
    lines += [
        f"minimum ring difference per segment := {fmtl(mins)}",
        f"maximum ring difference per segment := {fmtl(maxs)}",
        "Scanner parameters:=",
        "Scanner type := unknown",
        f"Number of rings := {g.num_rings}",
        f"Number of detectors per ring := {g.num_detectors_per_ring}",
        f"Inner ring diameter (cm) := {2 * g.inner_ring_radius_mm / 10:.6g}",
        f"Average depth of interaction (cm) := {g.average_depth_of_interaction_mm / 10:.6g}",
        f"Distance between rings (cm) := {g.ring_spacing_mm / 10:.6g}",
        f"Default bin size (cm) := {g.default_bin_size_mm / 10:.6g}",
        f"View offset (degrees) := {np.degrees(g.intrinsic_azimuthal_tilt_rad):.6g}",
        f"Maximum number of non-arc-corrected bins := {g.num_tangential_poss}",
        "end scanner parameters:=",
        f"effective central bin size (cm) := {(g.arccorr_bin_size_mm if g.arc_corrected else g.default_bin_size_mm) / 10:.6g}",
        "number of time frames := 1",
        "!END OF INTERFILE :=",
    ]
    with open(header_path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return header_path
