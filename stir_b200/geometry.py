"""Scanner / projection-data / image descriptions, mirroring STIR's objects.

These build the `b200rt_geometry` descriptor passed through the C ABI.  Only
primary parameters are stored; everything STIR derives from them (azimuthal
sampling, m offsets, tan(theta), symmetry tables) is derived by the library.

Mirrors:
  Scanner                      src/include/stir/Scanner.h
  ProjDataInfo::ProjDataInfoCTI src/buildblock/ProjDataInfo.cxx:487-600
  VoxelsOnCartesianGrid(projdata_info, zoom, origin, sizes)
                               src/buildblock/VoxelsOnCartesianGrid.cxx:56-130, 230-289
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np

from . import _abi


@dataclasses.dataclass
class Scanner:
    num_rings: int
    num_detectors_per_ring: int
    inner_ring_radius: float            # mm
    average_depth_of_interaction: float  # mm
    ring_spacing: float                  # mm
    default_bin_size: float              # mm
    intrinsic_tilt: float = 0.0          # rad
    timing_resolution: float = 0.0       # ps (TOF)
    size_of_timing_pos: float = 0.0      # ps (TOF)
    max_num_timing_poss: int = 0

    def get_effective_ring_radius(self) -> float:
        return float(np.float32(self.inner_ring_radius) + np.float32(self.average_depth_of_interaction))


@dataclasses.dataclass
class ProjDataInfo:
    """ProjDataInfoCylindrical{NoArcCorr,ArcCorr}: segments -S..S."""

    scanner: Scanner
    num_views: int
    num_tangential_poss: int
    min_ring_diff: List[int]   # index seg+S
    max_ring_diff: List[int]
    num_axial_poss: List[int]
    arc_corrected: bool = False
    arccorr_bin_size: float = 0.0
    tof_mash_factor: int = 0

    @property
    def max_segment_num(self) -> int:
        return (len(self.num_axial_poss) - 1) // 2

    @property
    def segment_sequence(self) -> List[int]:
        """ProjDataInMemory storage order of segments (ProjData.cxx:641-661)."""
        seq = [0]
        for s in range(1, self.max_segment_num + 1):
            seq += [s, -s]
        return seq

    def get_num_axial_poss(self, seg: int) -> int:
        return self.num_axial_poss[seg + self.max_segment_num]

    @property
    def num_tof_bins(self) -> int:
        if self.tof_mash_factor <= 0:
            return 1
        return self.scanner.max_num_timing_poss // self.tof_mash_factor

    @property
    def num_sinograms(self) -> int:
        return int(sum(self.num_axial_poss))

    @property
    def size(self) -> int:
        return self.num_sinograms * self.num_views * self.num_tangential_poss * self.num_tof_bins

    @property
    def min_tangential_pos_num(self) -> int:
        return -(self.num_tangential_poss // 2)

    def reduce_segment_range(self, max_seg: int) -> "ProjDataInfo":
        S = self.max_segment_num
        sl = slice(S - max_seg, S + max_seg + 1)
        return dataclasses.replace(self, min_ring_diff=self.min_ring_diff[sl], max_ring_diff=self.max_ring_diff[sl],
                                   num_axial_poss=self.num_axial_poss[sl])

    def sinogram_shape(self):
        """(segment, axial, view, tangential) extents in STIR order for each segment of the sequence."""
        return [(s, self.get_num_axial_poss(s), self.num_views, self.num_tangential_poss) for s in self.segment_sequence]


def ProjDataInfoCTI(scanner: Scanner, span: int, max_delta: int, num_views: int, num_tangential_poss: int,
                    arc_corrected: bool = False, tof_mash_factor: int = 0) -> ProjDataInfo:
    """ProjDataInfo::ProjDataInfoCTI (src/buildblock/ProjDataInfo.cxx:487-600)."""
    num_ring = scanner.num_rings
    if max_delta > num_ring - 1:
        raise ValueError(f"max_ring_difference {max_delta} is too large, number of rings is {num_ring}")
    if span < 1 or span > 2 * num_ring - 1:
        raise ValueError(f"invalid span {span}")
    if max_delta < (span - 1) // 2:
        raise ValueError("max_ring_difference has to be at least (span-1)/2")
    rdmin = [0] * num_ring
    rdmax = [0] * num_ring
    if span % 2 == 1:
        rdmin[0] = -((span - 1) // 2)
        rdmax[0] = rdmin[0] + span - 1
    else:
        rdmin[0] = -(span // 2)
        rdmax[0] = rdmin[0] + span
    seg = 0
    while rdmax[seg] < max_delta:
        seg += 1
        rdmin[seg] = rdmax[seg - 1] + 1
        rdmax[seg] = rdmin[seg] + span - 1
    if rdmax[seg] > max_delta:
        rdmax[seg] = max_delta
    S = seg
    mins = [0] * (2 * S + 1)
    maxs = [0] * (2 * S + 1)
    nax = [0] * (2 * S + 1)
    mins[S] = rdmin[0]
    maxs[S] = rdmax[0]
    for i in range(1, S + 1):
        maxs[S - i] = -rdmin[i]
        maxs[S + i] = rdmax[i]
        mins[S - i] = -rdmax[i]
        mins[S + i] = rdmin[i]
    if span == 1:
        nax[S] = num_ring
        for i in range(1, S + 1):
            nax[S + i] = nax[S - i] = num_ring - i
    else:
        nax[S] = 2 * num_ring - 1
        for i in range(1, S + 1):
            nax[S + i] = nax[S - i] = 2 * num_ring - 1 - 2 * rdmin[i]
    return ProjDataInfo(scanner, num_views, num_tangential_poss, mins, maxs, nax, arc_corrected,
                        scanner.default_bin_size if arc_corrected else 0.0, tof_mash_factor)


@dataclasses.dataclass
class ImageGeometry:
    """VoxelsOnCartesianGrid<float> index ranges and grid: z 0..nz-1, y/x centred."""

    nz: int
    ny: int
    nx: int
    voxel_size: Sequence[float]          # (z, y, x) mm
    origin: Sequence[float] = (0.0, 0.0, 0.0)
    min_z: int = 0
    min_y: Optional[int] = None
    min_x: Optional[int] = None

    def __post_init__(self):
        if self.min_y is None:
            self.min_y = -(self.ny // 2)
        if self.min_x is None:
            self.min_x = -(self.nx // 2)

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    @property
    def size(self) -> int:
        return self.nz * self.ny * self.nx


def image_from_projdata(pdi: ProjDataInfo, zoom: float = 1.0, xy_size: int = -1, z_size: int = -1,
                        origin=(0.0, 0.0, 0.0)) -> ImageGeometry:
    """VoxelsOnCartesianGrid(proj_data_info, zoom, origin, sizes) (VoxelsOnCartesianGrid.cxx:56-130, 230-289)."""
    f32 = np.float32
    z_sampling = f32(pdi.scanner.ring_spacing) / f32(2)
    S = pdi.max_segment_num
    if z_size < 0:
        z_size = pdi.num_axial_poss[S] if pdi.max_ring_diff[S] > pdi.min_ring_diff[S] else 2 * pdi.num_axial_poss[S] - 1
    s_sampling = f32(pdi.scanner.default_bin_size)
    vz = f32(z_sampling / f32(1.0))
    vxy = f32(s_sampling / f32(zoom))
    if xy_size < 0:
        raise ValueError("give xy_size explicitly")
    return ImageGeometry(z_size, xy_size, xy_size, (float(vz), float(vxy), float(vxy)), origin)


def make_geometry(pdi: ProjDataInfo, img: ImageGeometry, num_tangential_LORs: int = 1,
                  restrict_to_cylindrical_FOV: bool = True, symmetries: Sequence[bool] = (True,) * 5,
                  tof_kernel_truncation_sigmas: float = 0.0) -> _abi.Geometry:
    """The C ABI's geometry.  tof_kernel_truncation_sigmas: 0 keeps STIR's TOF kernel cut-off; k > 0 truncates the
    Gaussian at +-k sigma (no STIR counterpart)."""
    g = _abi.Geometry()
    sc = pdi.scanner
    g.num_rings = sc.num_rings
    g.num_detectors_per_ring = sc.num_detectors_per_ring
    g.inner_ring_radius_mm = sc.inner_ring_radius
    g.average_depth_of_interaction_mm = sc.average_depth_of_interaction
    g.ring_spacing_mm = sc.ring_spacing
    g.default_bin_size_mm = sc.default_bin_size
    g.intrinsic_azimuthal_tilt_rad = sc.intrinsic_tilt
    g.timing_resolution_ps = sc.timing_resolution
    g.size_of_timing_pos_ps = sc.size_of_timing_pos
    g.max_num_timing_poss = sc.max_num_timing_poss
    g.arc_corrected = 1 if pdi.arc_corrected else 0
    g.arccorr_bin_size_mm = pdi.arccorr_bin_size
    g.num_views = pdi.num_views
    g.num_tangential_poss = pdi.num_tangential_poss
    g.max_segment_num = pdi.max_segment_num
    g.tof_mash_factor = pdi.tof_mash_factor
    if len(pdi.num_axial_poss) > _abi.MAX_SEGMENTS:
        raise ValueError("too many segments")
    for i, (a, b, c) in enumerate(zip(pdi.min_ring_diff, pdi.max_ring_diff, pdi.num_axial_poss)):
        g.min_ring_diff[i] = a
        g.max_ring_diff[i] = b
        g.num_axial_poss[i] = c
    g.nz, g.ny, g.nx = img.nz, img.ny, img.nx
    g.min_z, g.min_y, g.min_x = img.min_z, img.min_y, img.min_x
    g.voxel_size_z, g.voxel_size_y, g.voxel_size_x = img.voxel_size
    g.origin_z, g.origin_y, g.origin_x = img.origin
    g.num_tangential_LORs = num_tangential_LORs
    g.restrict_to_cylindrical_FOV = 1 if restrict_to_cylindrical_FOV else 0
    (g.do_symmetry_90degrees_min_phi, g.do_symmetry_180degrees_min_phi, g.do_symmetry_swap_segment,
     g.do_symmetry_swap_s, g.do_symmetry_shift_z) = [1 if s else 0 for s in symmetries]
    g.tof_kernel_truncation_sigmas = float(tof_kernel_truncation_sigmas)
    return g


# ---------------------------------------------------------------------------
# Workloads (seeded synthetic data stands in for measured data)
# ---------------------------------------------------------------------------

def small_3d_pet():
    """8 rings x 288 detectors, R 300 mm, ring spacing 4 mm, span 1 (max ring difference 7),
    144 views x 64 tangential; image 64x64x15 at 4x4x2 mm."""
    sc = Scanner(8, 288, 300.0, 0.0, 4.0, float(np.float32(2 * math.pi * 300.0 / 288 / 2)))
    pdi = ProjDataInfoCTI(sc, 1, 7, 144, 64)
    img = ImageGeometry(15, 64, 64, (2.0, 4.0, 4.0))
    return pdi, img


def clinical_3d_pet():
    """64 rings x 504 detectors, R 328 mm, ring spacing 4.06 mm, span 11, max ring difference 60,
    252 views x 344 tangential; image 344x344x127 at 2.09x2.09x2.03 mm."""
    sc = Scanner(64, 504, 328.0, 0.0, 4.06, 2.09)
    pdi = ProjDataInfoCTI(sc, 11, 60, 252, 344)
    img = ImageGeometry(127, 344, 344, (2.03, 2.09, 2.09))
    return pdi, img


def clinical_3d_pet_half():
    """The clinical scanner with an image at half the transaxial resolution: 172x172x127 at 4.18 mm."""
    pdi, _ = clinical_3d_pet()
    img = ImageGeometry(127, 172, 172, (2.03, 4.18, 4.18))
    return pdi, img


def tof_small_3d_pet(num_tof_bins: int = 33, fwhm_ps: float = 550.0, timing_bin_ps: float = 50.0, num_views: int = 144):
    """small_3d_pet with TOF: `num_tof_bins` timing bins of `timing_bin_ps` (33 x 50 ps cover the 248 mm FOV)
    and a Gaussian kernel of `fwhm_ps` FWHM."""
    pdi, img = small_3d_pet()
    sc = dataclasses.replace(pdi.scanner, timing_resolution=fwhm_ps, size_of_timing_pos=timing_bin_ps,
                             max_num_timing_poss=num_tof_bins)
    pdi = dataclasses.replace(pdi, scanner=sc, tof_mash_factor=1, num_views=num_views)
    return pdi, img


def non_tof(pdi: ProjDataInfo) -> ProjDataInfo:
    """ProjDataInfo::create_non_tof_clone: the same projection data without timing bins."""
    return dataclasses.replace(pdi, tof_mash_factor=0)


def rpt_sensitivity_test():
    """Geometry of STIR's recon_test_pack sensitivity test (OSMAPOSL_test_PM_for_sensitivity.par):
    Utahscat600k_ca_seg4.hs (PRT-1 scanner, arc-corrected, 96 views x 128 bins, span 1, segments -4..4
    of which -3..3 are processed), image zoom 0.7 with 60x60 pixels, 2 rays per bin tangentially.
    Values follow the Interfile parsing round trips of src/IO/InterfileHeader.cxx:1066-1072,1368-1420."""
    f32, f64 = np.float32, np.float64
    inner_cm = f64(f32(373.0)) * 2 / 10.
    doi_cm = f64(f32(f32(7.0) / f32(10)))
    ring_cm = f64(0.675)
    bin_cm = f64(f32(f32(3.1088) / f32(10)))
    tilt = float(f32(f64(-0.46875) * math.pi / 180))
    sc = Scanner(16, 384, float(f32(inner_cm * 10. / 2)), float(f32(doi_cm * 10)), float(f32(ring_cm * 10.)),
                 float(f32(bin_cm * 10)), tilt)
    eff_bin_cm = f64(f32(sc.default_bin_size) / f32(10))
    arc_bin = float(f32(eff_bin_cm * 10.))
    nax = [12, 13, 14, 15, 16, 15, 14, 13, 12]
    rd = [-4, -3, -2, -1, 0, 1, 2, 3, 4]
    pdi = ProjDataInfo(sc, 96, 128, rd, rd, nax, True, arc_bin)
    pdi = pdi.reduce_segment_range(3)
    img = image_from_projdata(pdi, zoom=0.7, xy_size=60)
    return pdi, img
