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


class SubsetOrder:
    """IterativeReconstruction::get_subset_num (src/recon_buildblock/IterativeReconstruction.cxx:628-640).

    In order: subset (subiteration_num + start_subset_num - 1) mod num_subsets.  With
    `uniformly_randomise_subset_order` ("uniformly randomise subset order", :87): a new random permutation of the
    subsets at the first sub-iteration of every full iteration ((subiteration_num - 1) mod num_subsets == 0), drawn
    as randomly_permute_subset_order does (:577-600: repeatedly pick one of the remaining subsets uniformly and
    remove it), and sub-iteration k takes entry (k - 1) mod num_subsets.  STIR seeds rand() with the time
    (:495-498); `seed` makes the order reproducible (None: seeded from the time, as STIR).  The permutation is
    made once per full iteration, however often the subset of one sub-iteration is asked for."""

    def __init__(self, num_subsets: int, start_subset_num: int = 0, uniformly_randomise_subset_order: bool = False,
                 seed=None):
        import random
        import time
        self.num_subsets = num_subsets
        self.start_subset_num = start_subset_num
        self.randomise = bool(uniformly_randomise_subset_order)
        self._rng = random.Random(int(time.time()) if seed is None else seed)
        self._perm = None
        self._perm_iteration = None

    def randomly_permute_subset_order(self):
        remaining = list(range(self.num_subsets))
        out = []
        for i in range(self.num_subsets):
            index = int(self._rng.random() * (self.num_subsets - i))
            index = min(index, self.num_subsets - i - 1)
            out.append(remaining.pop(index))
        return out

    def __call__(self, subiteration_num: int) -> int:
        if not self.randomise:
            return (subiteration_num + self.start_subset_num - 1) % self.num_subsets
        iteration = (subiteration_num - 1) // self.num_subsets
        if self._perm is None or iteration != self._perm_iteration:
            self._perm = self.randomly_permute_subset_order()
            self._perm_iteration = iteration
        return self._perm[(subiteration_num - 1) % self.num_subsets]
