"""Subsets of views (detail::find_basic_vs_nums_in_subset, src/recon_buildblock/find_basic_vs_nums_in_subset.cxx:32-70).

A subset holds the basic views v with v % num_subsets == subset_num together with every view
related to them by the projector's symmetries
(DataSymmetriesForBins_PET_CartesianGrid::get_related_view_segment_numbers, .inl:735-782).
"""
from __future__ import annotations

from typing import List

SYM_90 = 1
SYM_180 = 2


def _is_basic(view: int, num_views: int, bits: int) -> bool:
    v90 = num_views >> 1
    v45 = v90 >> 1
    if bits & SYM_90:
        return view <= v45
    if bits & SYM_180:
        return view <= v90
    return True


def related_views(view: int, num_views: int, bits: int) -> List[int]:
    nv = num_views
    out = [view]
    s90, s180 = bool(bits & SYM_90), bool(bits & SYM_180)
    if s180 and s90 and view % (nv // 2) != nv // 4:
        out.append(view + nv // 2 if view < nv // 2 else view - nv // 2)
    if s180 and view % (nv // 2) != 0:
        out.append(nv - view)
    if s90 and view % (nv // 4) != 0:
        out.append((nv // 2 - view + nv) % nv)
    return out


def basic_views_in_subset(num_views: int, bits: int, subset_num: int, num_subsets: int) -> List[int]:
    return [v for v in range(subset_num, num_views, num_subsets) if _is_basic(v, num_views, bits)]


def views_in_subset(geometry, subset_num: int, num_subsets: int, bits: int = None) -> List[int]:
    """All views of the subset.  `geometry` is a b200rt_geometry; `bits` the symmetries in use
    (b200rt_info.symmetries_used), defaulting to what the geometry requests."""
    nv = geometry.num_views
    if bits is None:
        bits = 0
        if geometry.do_symmetry_90degrees_min_phi and nv % 4 == 0:
            bits |= SYM_90 | SYM_180
        elif (geometry.do_symmetry_90degrees_min_phi or geometry.do_symmetry_180degrees_min_phi) and nv % 2 == 0:
            bits |= SYM_180
    views = []
    for v in basic_views_in_subset(nv, bits, subset_num, num_subsets):
        views += related_views(v, nv, bits)
    return sorted(set(views))
