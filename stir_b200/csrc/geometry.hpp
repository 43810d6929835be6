// Host-side geometry of the projector pair: everything STIR derives from the
// scanner / projection-data / image description, evaluated with STIR's float
// arithmetic, plus the symmetry tables that drive the device kernels.
//
// STIR sources restated here (paths relative to the STIR tree):
//   ProjDataInfoCylindrical{,.inl}       azimuthal sampling/offset, m offsets, tan(theta), t
//   ProjDataInfoCylindricalNoArcCorr/ArcCorr  get_s
//   DataSymmetriesForBins_PET_CartesianGrid{.cxx,.inl}  basic bins and symmetry operations
//   ProjMatrixByBinUsingRayTracing.cxx   ray end points of each basic bin (:438-829)
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/stir_b200.h"

namespace b200 {

// A symmetry operation of SymmetryOperations_PET_CartesianGrid, reduced to
//   x' = (swap ? y : x) * sx,  y' = (swap ? x : y) * sy,  z' = (zq ? q - z : z) + npa * axial
struct SymOp {
  int swap = 0, sx = 1, sy = 1, zq = 0, q = 0;
};

// One ray of a basic bin, in voxel units (start has the smaller z; see
// ProjMatrixByBinUsingRayTracing.cxx:549-565).
struct Ray {
  float start[3];  // z, y, x
  float stop[3];
  float norm_const;
};

// Everything needed to build the row of one basic bin on the device.
struct BasicBin {
  int view, seg, tang, tof;
  int first_ray, num_rays;     // into rays[]
  int direct;                  // tan(theta)==0 -> add_adjacent_z
  int num_lors_per_axial_pos;  // z copies for oblique bins
  float z_origin_in_planes;    // origin.z/vz               (add_adjacent_z, :800)
  float z_centre;              // (max_z+min_z)/2          (:800)
  float left_edge;             // (t - sdz/2)/vz           (:801)
  float tor_width;             // right_edge - left_edge   (:802-804)
  int capacity;                // upper bound of the row length
};

// A viewgram related to a basic view-segment by a symmetry (get_related_view_segment_numbers),
// for one sign of the tangential position.
struct RelatedLine {
  int view, seg, tang_sign;
  SymOp op;
};

class Geometry {
 public:
  explicit Geometry(const b200rt_geometry& d);  // throws std::runtime_error with STIR's messages

  const b200rt_geometry& desc() const { return d_; }
  int S() const { return S_; }
  int num_views() const { return d_.num_views; }
  int num_tang() const { return d_.num_tangential_poss; }
  int min_tang() const { return min_tang_; }
  int max_tang() const { return max_tang_; }
  int nax(int seg) const { return d_.num_axial_poss[seg + S_]; }
  int npa(int seg) const { return npa_[seg + S_]; }
  int num_tof() const { return num_tof_; }
  int min_tof() const { return min_tof_; }
  int64_t projdata_size() const { return projdata_size_; }
  int64_t image_size() const { return static_cast<int64_t>(d_.nz) * d_.ny * d_.nx; }
  int symmetry_bits() const;

  // STIR ProjDataInMemory index of a bin, and the device-layout index
  int64_t stir_index(int seg, int view, int ax, int tang, int tof) const;
  int64_t dev_index(int seg, int view, int ax, int tang, int tof) const;
  int64_t stir_segment_offset(int seg) const { return stir_seg_off_[seg + S_]; }
  int64_t dev_segment_offset(int seg) const { return dev_seg_off_[seg + S_]; }
  int64_t tof_stride() const { return tof_stride_; }

  // symmetry structure
  bool is_basic_vs(int view, int seg) const;
  std::vector<int> basic_views() const;
  std::vector<int> basic_segments() const;
  std::vector<int> basic_tangs() const;
  void related_lines(int view_b, int seg_b, bool tang_zero, std::vector<RelatedLine>& out) const;
  // operation mapping the basic bin of (seg,view,ax,tang) to it, and the basic bin itself
  SymOp find_op(int seg, int view, int ax, int tang) const;
  void find_basic_bin(int& seg, int& view, int& ax, int& tang, int& tof) const;

  // ray end points of a basic bin (ProjMatrixByBinUsingRayTracing.cxx:581-782)
  BasicBin make_basic_bin(int view, int seg, int tang, int tof, std::vector<Ray>& rays) const;

  // TOF (ProjDataInfo.cxx:174-255, ProjMatrixByBin.cxx:66-75)
  float tof_low(int k) const { return tof_low_[k - min_tof_]; }
  float tof_high(int k) const { return tof_high_[k - min_tof_]; }
  float r_sqrt2_gauss_sigma() const { return r_sqrt2_sigma_; }
  // TOF kernel cut-off k / sqrt(2) for truncation at +-k sigma; 0: STIR's cut-off
  float tof_truncation_n() const { return tof_trunc_n_; }
  // LOR mid point and unit direction of a basic bin, in scanner coordinates (mm) (ProjMatrixByBin.inl:117-133)
  void lor_middle_and_direction(int seg, int view, int tang, float mid[3], float unit[3]) const;
  float scanner_z_offset() const;

  // STIR geometry accessors
  float get_phi(int view) const;
  float get_s(int tang) const;
  float get_tantheta(int seg, int tang) const;
  float get_costheta(int seg, int tang) const;
  float get_m(int seg, int ax) const;
  float get_t(int seg, int ax, int tang) const;
  float axial_sampling(int seg) const;
  float get_sampling_in_s(int tang) const;

 private:
  b200rt_geometry d_;
  int S_ = 0, min_tang_ = 0, max_tang_ = 0;
  int num_tof_ = 1, min_tof_ = 0;
  float azim_sampling_ = 0, azim_offset_ = 0, ring_radius_ = 0, ring_spacing_ = 0, angular_inc_ = 0, arc_bin_ = 0;
  std::vector<float> m_offset_, ax_to_z_, deltas_;
  std::vector<int> npa_;
  int planes_per_ring_ = 0;
  bool sym90_ = true, sym180_ = true, symseg_ = true, syms_ = true, symz_ = true;
  std::vector<int64_t> stir_seg_off_, dev_seg_off_;
  int64_t tof_stride_ = 0, projdata_size_ = 0;
  std::vector<float> tof_low_, tof_high_;
  float r_sqrt2_sigma_ = 0;
  float tof_trunc_n_ = 0;

  float average_ring_difference(int seg) const;
  int transform_z(int abs_seg, int ax) const;
  SymOp op_bin0(int seg, int view) const;
  SymOp op_general(int s, int seg, int view) const;
};

}  // namespace b200
