// Host-side geometry of the projector pair (see geometry.hpp).
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <stdexcept>

namespace b200 {

namespace {
constexpr double kPi = 3.14159265358979323846264338327950288;
inline float sq(float v) { return v * v; }
// stir::round (src/buildblock/round.inl:59-73)
inline int round_half_away(float x) { return x >= 0 ? static_cast<int>(x + 0.5F) : -static_cast<int>(-x + 0.5F); }
// stir::modulo for floats (src/include/stir/modulo.h:51-78)
inline float modulo_f(float a, float b) {
  double r = std::fmod(static_cast<double>(a), static_cast<double>(b));
  if (r < 0) r += std::fabs(static_cast<double>(b));
  float res = static_cast<float>(r);
  const float ab = b >= 0 ? b : -b;
  if (res >= ab) res -= ab;
  return res;
}
// float inner product z,y,x order then sqrt in double (BasicCoordinate.inl:413-429)
inline double norm_zyx(float z, float y, float x) {
  float s = 0.f;
  s = s + z * z;
  s = s + y * y;
  s = s + x * x;
  return std::sqrt(static_cast<double>(s));
}
[[noreturn]] void fail(const std::string& m) { throw std::runtime_error(m); }
}  // namespace

Geometry::Geometry(const b200rt_geometry& d) : d_(d) {
  S_ = d.max_segment_num;
  if (S_ < 0 || 2 * S_ + 1 > B200RT_MAX_SEGMENTS) fail("max_segment_num out of range");
  if (d.num_views < 1 || d.num_tangential_poss < 1) fail("empty projection data");
  if (d.num_detectors_per_ring < 1 || d.num_rings < 1) fail("invalid scanner");
  if (d.nz < 1 || d.ny < 1 || d.nx < 1) fail("empty image");
  if (d.nx > 1024 || d.ny > 1024 || d.nz > 4096) fail("image larger than 1024 x 1024 x 4096 voxels");
  if (!(d.voxel_size_x > 0 && d.voxel_size_y > 0 && d.voxel_size_z > 0)) fail("voxel sizes must be positive");
  // ProjDataInfo::set_num_tangential_poss (ProjDataInfo.cxx:124-129)
  min_tang_ = -(d.num_tangential_poss / 2);
  max_tang_ = min_tang_ + d.num_tangential_poss - 1;
  // ProjDataInfoCylindrical constructor (ProjDataInfoCylindrical.cxx:55-116)
  azim_sampling_ = static_cast<float>(kPi / d.num_views);
  azim_offset_ = d.intrinsic_azimuthal_tilt_rad;
  {
    const int ndet = d.num_detectors_per_ring;
    if (ndet > 2 && d.num_views * 2 != ndet && ndet % (d.num_views * 2) == 0) {
      const int mash = ndet / 2 / d.num_views;
      azim_offset_ += static_cast<float>(kPi / (ndet / 2) * (mash - 1) / 2.F);
    }
  }
  ring_radius_ = d.inner_ring_radius_mm + d.average_depth_of_interaction_mm;  // Scanner.inl:91-95
  ring_spacing_ = d.ring_spacing_mm;
  angular_inc_ = static_cast<float>(kPi / d.num_detectors_per_ring);  // NoArcCorr.cxx:75-88
  arc_bin_ = d.arccorr_bin_size_mm;
  if (d.arc_corrected && !(arc_bin_ > 0)) fail("arc-corrected data needs a positive bin size");
  m_offset_.assign(2 * S_ + 1, 0.f);
  for (int s = -S_; s <= S_; ++s) {
    if (d.num_axial_poss[s + S_] < 1) fail("segment without axial positions");
    if (d.min_ring_diff[s + S_] > d.max_ring_diff[s + S_])
      fail("ProjDataInfoCylindrical: min_ring_difference is larger than max_ring_difference");
    // ProjDataInfoCylindrical.cxx:135-145
    m_offset_[s + S_] = (static_cast<float>(d.num_axial_poss[s + S_] - 1) * axial_sampling(s)) / 2;
  }
  // storage offsets: STIR order 0,+1,-1,... (ProjData.cxx:641-661); device order -S..S
  stir_seg_off_.assign(2 * S_ + 1, 0);
  dev_seg_off_.assign(2 * S_ + 1, 0);
  int64_t off = 0;
  for (int i = 0; i <= 2 * S_; ++i) {
    const int s = (i == 0) ? 0 : ((i % 2) ? (i + 1) / 2 : -(i / 2));
    stir_seg_off_[s + S_] = off;
    off += static_cast<int64_t>(nax(s)) * d.num_views * d.num_tangential_poss;
  }
  tof_stride_ = off;
  off = 0;
  for (int s = -S_; s <= S_; ++s) {
    dev_seg_off_[s + S_] = off;
    off += static_cast<int64_t>(nax(s)) * d.num_views * d.num_tangential_poss;
  }
  // TOF bins (ProjDataInfo.cxx:174-255), kernel width (ProjMatrixByBin.cxx:66-75)
  num_tof_ = 1;
  min_tof_ = 0;
  if (d.tof_mash_factor > 0) {
    if (d.max_num_timing_poss < 1 || d.size_of_timing_pos_ps <= 0 || d.timing_resolution_ps <= 0)
      fail("TOF data needs a TOF-ready scanner");
    if (d.tof_mash_factor > d.max_num_timing_poss || d.max_num_timing_poss % d.tof_mash_factor)
      fail("TOF mashing factor must divide the scanner's number of timing positions");
    num_tof_ = d.max_num_timing_poss / d.tof_mash_factor;
    min_tof_ = -num_tof_ / 2;
    const double c_half = 0.299792458 * 0.5;
    const float inc = static_cast<float>(static_cast<double>(d.tof_mash_factor * d.size_of_timing_pos_ps) * c_half);
    auto get_k = [&](int k) { return (num_tof_ % 2) ? static_cast<float>(k) * inc : static_cast<float>(k) * inc + inc / 2.f; };
    tof_low_.resize(num_tof_);
    tof_high_.resize(num_tof_);
    for (int k = min_tof_; k < min_tof_ + num_tof_; ++k) {
      const float sampling = (get_k(k + 1) - get_k(k - 1)) / 2.f;
      const float centre = get_k(k);
      tof_low_[k - min_tof_] = centre - sampling / 2.f;
      tof_high_[k - min_tof_] = centre + sampling / 2.f;
    }
    const float sigma = static_cast<float>(static_cast<double>(d.timing_resolution_ps) * c_half) / 2.355f;
    r_sqrt2_sigma_ = 1.0f / (sigma * static_cast<float>(std::sqrt(2.0)));
    if (!(d.tof_kernel_truncation_sigmas >= 0.f)) fail("tof_kernel_truncation_sigmas must be 0 (STIR's cut-off) or > 0");
    // +-k sigma in the kernel's units (distance times 1 / (sqrt(2) sigma))
    tof_trunc_n_ = static_cast<float>(static_cast<double>(d.tof_kernel_truncation_sigmas) / std::sqrt(2.0));
  }
  projdata_size_ = tof_stride_ * num_tof_;

  // ProjMatrixByBinUsingRayTracing::set_up (ProjMatrixByBinUsingRayTracing.cxx:272-277)
  if (std::fabs(d.origin_x) > .05F || std::fabs(d.origin_y) > .05F)
    fail("ProjMatrixByBinUsingRayTracing sadly doesn't support shifted x/y origin yet");
  if (d.num_tangential_LORs < 1) fail("num_tangential_LORs should be at least 1");

  // DataSymmetriesForBins_PET_CartesianGrid constructor (DataSymmetriesForBins_PET_CartesianGrid.cxx:223-420)
  sym90_ = d.do_symmetry_90degrees_min_phi != 0;
  sym180_ = sym90_ || d.do_symmetry_180degrees_min_phi != 0;
  symseg_ = d.do_symmetry_swap_segment != 0;
  syms_ = d.do_symmetry_swap_s != 0;
  symz_ = d.do_symmetry_shift_z != 0;
  if (!symz_) fail("do_symmetry_shift_z=0 is not supported by the B200 projector");
  {
    const float zop = d.origin_z / d.voxel_size_z;
    if (std::fabs(round_half_away(zop) - zop) > 1.E-3F)
      fail("DataSymmetriesForBins_PET_CartesianGrid: the z origin should be a multiple of the plane separation");
  }
  if (std::fabs(d.voxel_size_y - d.voxel_size_x) > 2.E-3F) sym90_ = false;
  if (d.num_views % 4 != 0) sym90_ = false;
  if (d.num_views % 2 != 0) sym180_ = false;
  if (std::fabs(get_tantheta(0, 0)) > 1.E-4F)
    fail("DataSymmetriesForBins_PET_CartesianGrid can only handle projection data with segment 0 corresponding to direct planes");
  for (int s = 1; s <= S_; ++s)
    if (std::fabs(get_tantheta(s, 0) + get_tantheta(-s, 0)) > 1.E-4F)
      fail("DataSymmetriesForBins_PET_CartesianGrid: negative segments must correspond to -theta of the positive segments");
  if (std::fabs(get_s(1) + get_s(-1)) > 1.E-4F) fail("DataSymmetriesForBins_PET_CartesianGrid: s-symmetry violated");
  if (std::fabs(get_phi(0)) > 1.E-4F) sym90_ = sym180_ = false;
  if (num_tof_ > 1) sym90_ = sym180_ = symseg_ = syms_ = false;
  if (std::fabs(d.origin_x) > .01F || std::fabs(d.origin_y) > .01F) sym90_ = sym180_ = symseg_ = syms_ = false;
  // find_relation_between_coordinate_systems (DataSymmetriesForBins_PET_CartesianGrid.cxx:49-115)
  {
    const float plane = d.voxel_size_z;
    const float pr = ring_spacing_ / plane;
    planes_per_ring_ = round_half_away(pr);
    if (std::fabs(pr - planes_per_ring_) > 1.E-2)
      fail("DataSymmetriesForBins_PET_CartesianGrid can currently only support z-grid spacing equal to the ring spacing of the scanner divided by an integer");
    npa_.assign(2 * S_ + 1, 0);
    ax_to_z_.assign(2 * S_ + 1, 0.f);
    deltas_.assign(2 * S_ + 1, 0.f);
    const int max_z = d.min_z + d.nz - 1;
    for (int s = -S_; s <= S_; ++s) {
      const float nf = axial_sampling(s) / plane;
      npa_[s + S_] = round_half_away(nf);
      if (std::fabs(nf - npa_[s + S_]) > 1.E-2)
        fail("DataSymmetriesForBins_PET_CartesianGrid can currently only support z-grid spacing equal to the sinogram spacing divided by an integer");
      const float delta = average_ring_difference(s);
      deltas_[s + S_] = delta;
      ax_to_z_[s + S_] = static_cast<float>(max_z + d.min_z) / 2.F - d.origin_z / plane -
                         (static_cast<float>(npa_[s + S_] * (nax(s) - 1)) + static_cast<float>(planes_per_ring_) * delta) / 2;
    }
  }
  // the basic tangential positions must fit next to the others
  if (syms_ && -min_tang_ > max_tang_ + 1) fail("tangential range too asymmetric");
}

int Geometry::symmetry_bits() const {
  return (sym90_ ? 1 : 0) | (sym180_ ? 2 : 0) | (symseg_ ? 4 : 0) | (syms_ ? 8 : 0) | (symz_ ? 16 : 0);
}

float Geometry::axial_sampling(int seg) const {
  const int inc = d_.max_ring_diff[seg + S_] != d_.min_ring_diff[seg + S_] ? 2 : 1;  // ProjDataInfoCylindrical.inl:107-128
  return ring_spacing_ / static_cast<float>(inc);
}
float Geometry::average_ring_difference(int seg) const {
  return static_cast<float>(d_.min_ring_diff[seg + S_] + d_.max_ring_diff[seg + S_]) / 2.F;
}
float Geometry::get_phi(int view) const { return static_cast<float>(view) * azim_sampling_ + azim_offset_; }
float Geometry::get_s(int tang) const {
  if (d_.arc_corrected) return static_cast<float>(tang) * arc_bin_;
  return ring_radius_ * std::sin(static_cast<float>(tang) * angular_inc_);
}
float Geometry::get_tantheta(int seg, int tang) const {
  const float delta = average_ring_difference(seg);
  if (std::fabs(delta) < 0.0001F) return 0.f;
  return delta * ring_spacing_ / (2 * std::sqrt(sq(ring_radius_) - sq(get_s(tang))));
}
float Geometry::get_costheta(int seg, int tang) const { return 1 / std::sqrt(1 + sq(get_tantheta(seg, tang))); }
float Geometry::get_m(int seg, int ax) const { return static_cast<float>(ax) * axial_sampling(seg) - m_offset_[seg + S_]; }
float Geometry::get_t(int seg, int ax, int tang) const { return get_m(seg, ax) * get_costheta(seg, tang); }
float Geometry::get_sampling_in_s(int tang) const { return std::fabs(get_s(tang + 1) - get_s(tang - 1)) / 2; }

int64_t Geometry::stir_index(int seg, int view, int ax, int tang, int tof) const {
  return static_cast<int64_t>(tof - min_tof_) * tof_stride_ + stir_seg_off_[seg + S_] +
         (static_cast<int64_t>(ax) * d_.num_views + view) * d_.num_tangential_poss + (tang - min_tang_);
}
int64_t Geometry::dev_index(int seg, int view, int ax, int tang, int tof) const {
  return static_cast<int64_t>(tof - min_tof_) * tof_stride_ + dev_seg_off_[seg + S_] +
         (static_cast<int64_t>(view) * d_.num_tangential_poss + (tang - min_tang_)) * nax(seg) + ax;
}

// find_basic_view_segment_numbers (DataSymmetriesForBins_PET_CartesianGrid.inl:359-404)
static bool fold_vs(bool sym90, bool sym180, bool symseg, int nv, int& view, int& seg) {
  bool change = false;
  const int v90 = nv >> 1, v45 = v90 >> 1, v135 = v90 + v45;
  if (symseg && seg < 0) {
    seg = -seg;
    change = true;
  }
  if (sym90) {
    if (view >= v135) {
      view = nv - view;
      return true;
    }
    if (view >= v90) {
      view -= v90;
      return true;
    }
    if (view > v45) {
      view = v90 - view;
      return true;
    }
  } else if (sym180 && view > v90) {
    view = nv - view;
    return true;
  }
  return change;
}

bool Geometry::is_basic_vs(int view, int seg) const {
  int v = view, s = seg;
  return !fold_vs(sym90_, sym180_, symseg_, d_.num_views, v, s);
}
std::vector<int> Geometry::basic_views() const {
  std::vector<int> out;
  for (int v = 0; v < d_.num_views; ++v)
    if (is_basic_vs(v, 0)) out.push_back(v);
  return out;
}
std::vector<int> Geometry::basic_segments() const {
  std::vector<int> out;
  for (int s = -S_; s <= S_; ++s)
    if (!symseg_ || s >= 0) out.push_back(s);
  return out;
}
std::vector<int> Geometry::basic_tangs() const {
  std::vector<int> out;
  if (syms_) {
    for (int t = 0; t <= std::max(max_tang_, -min_tang_); ++t) out.push_back(t);
  } else {
    for (int t = min_tang_; t <= max_tang_; ++t) out.push_back(t);
  }
  return out;
}

void Geometry::find_basic_bin(int& seg, int& view, int& ax, int& tang, int& tof) const {
  // DataSymmetriesForBins_PET_CartesianGrid.inl:406-433
  fold_vs(sym90_, sym180_, symseg_, d_.num_views, view, seg);
  if (syms_ && tang < 0) {
    tang = -tang;
    tof = -tof;
  }
  if (symz_) ax = 0;
}

// find_transform_z (DataSymmetriesForBins_PET_CartesianGrid.inl:63-100)
int Geometry::transform_z(int abs_seg, int ax) const {
  const float tz = static_cast<float>(2 * npa_[abs_seg + S_] * ax) + static_cast<float>(planes_per_ring_) * deltas_[abs_seg + S_] +
                   2 * ax_to_z_[abs_seg + S_];
  return static_cast<int>(std::floor(tz + 0.5));
}

static SymOp mk(int swap, int sx, int sy, int zq, int q) {
  SymOp o;
  o.swap = swap;
  o.sx = sx;
  o.sy = sy;
  o.zq = zq;
  o.q = zq ? q : 0;
  return o;
}

// find_sym_op_bin0 (DataSymmetriesForBins_PET_CartesianGrid.inl:102-162); image transforms of
// SymmetryOperations_PET_CartesianGrid.inl (swap_xmy_yx: x'=-y,y'=x; swap_xy_yx: x'=y,y'=x; swap_xmx: x'=-x; ...)
SymOp Geometry::op_bin0(int seg, int view) const {
  const int q = transform_z(std::abs(seg), 0);
  const int v180 = d_.num_views, v135 = v180 / 4 * 3, v90 = v180 / 2, v45 = v180 / 4;
  const bool pos = !symseg_ || seg >= 0;
  if (sym90_ && view > v90 && view <= v135) return pos ? mk(1, -1, 1, 0, q) : mk(1, -1, 1, 1, q);
  if (sym90_ && view > v45 && view <= v90) return pos ? mk(1, 1, 1, 1, q) : mk(1, 1, 1, 0, q);
  if (sym180_ && view > v90) return pos ? mk(0, -1, 1, 1, q) : mk(0, -1, 1, 0, q);
  if (symseg_ && seg < 0) return mk(0, 1, 1, 1, q);
  return mk(0, 1, 1, 0, q);
}

// find_sym_op_general_bin (DataSymmetriesForBins_PET_CartesianGrid.inl:196-326)
SymOp Geometry::op_general(int s, int seg, int view) const {
  const int q = transform_z(std::abs(seg), 0);
  const int v180 = d_.num_views, v135 = v180 / 4 * 3, v90 = v180 / 2, v45 = v180 / 4;
  const bool sp = !syms_ || s > 0;
  if (sym90_ && view > v90 && view <= v135) {
    if (!symseg_ || seg > 0) return sp ? mk(1, -1, 1, 0, q) : mk(1, 1, -1, 1, q);  // xmy_yx | xy_ymx_zq
    if (seg < 0) return sp ? mk(1, -1, 1, 1, q) : mk(1, 1, -1, 0, q);              // xmy_yx_zq | xy_ymx
    return sp ? mk(1, -1, 1, 0, q) : mk(1, 1, -1, 0, q);                           // xmy_yx | xy_ymx
  }
  if (sym90_ && view > v45 && view <= v90) {
    if (!symseg_ || seg > 0) return sp ? mk(1, 1, 1, 1, q) : mk(1, -1, -1, 0, q);  // xy_yx_zq | xmy_ymx
    if (seg < 0) return sp ? mk(1, 1, 1, 0, q) : mk(1, -1, -1, 1, q);              // xy_yx | xmy_ymx_zq
    return sp ? mk(1, 1, 1, 0, q) : mk(1, -1, -1, 0, q);                           // xy_yx | xmy_ymx
  }
  if (sym180_ && view > v90) {
    if (!symseg_ || seg > 0) return sp ? mk(0, -1, 1, 1, q) : mk(0, 1, -1, 0, q);  // xmx_zq | ymy
    return sp ? mk(0, -1, 1, 0, q) : mk(0, 1, -1, 1, q);                           // xmx | ymy_zq
  }
  if (!symseg_ || seg > 0) {
    if (syms_ && s < 0) return mk(0, -1, -1, 1, q);  // xmx_ymy_zq
    return mk(0, 1, 1, 0, q);
  }
  if (seg < 0) {
    if (syms_ && s < 0) return mk(0, -1, -1, 0, q);  // xmx_ymy
    return mk(0, 1, 1, 1, q);                         // zq
  }
  if (syms_ && s < 0) return mk(0, -1, -1, 0, q);
  return mk(0, 1, 1, 0, q);
}

SymOp Geometry::find_op(int seg, int view, int /*ax*/, int tang) const {
  return tang == 0 ? op_bin0(seg, view) : op_general(tang, seg, view);
}

// get_related_view_segment_numbers (DataSymmetriesForBins_PET_CartesianGrid.inl:735-782) crossed with
// the tangential signs of get_related_bins_factorised (:677-697)
void Geometry::related_lines(int view, int seg, bool tang_zero, std::vector<RelatedLine>& out) const {
  out.clear();
  const int nv = d_.num_views;
  const bool symz = symseg_ && seg != 0;
  std::vector<std::pair<int, int>> rel;
  rel.push_back({view, seg});
  if (symz) rel.push_back({view, -seg});
  if (sym180_ && sym90_ && (view % (nv / 2)) != nv / 4) {
    const int rv = view < nv / 2 ? view + nv / 2 : view - nv / 2;
    rel.push_back({rv, seg});
    if (symz) rel.push_back({rv, -seg});
  }
  if (sym180_ && (view % (nv / 2)) != 0) {
    rel.push_back({nv - view, seg});
    if (symz) rel.push_back({nv - view, -seg});
  }
  if (sym90_ && (view % (nv / 4)) != 0) {
    const int rv = (nv / 2 - view + nv) % nv;
    rel.push_back({rv, seg});
    if (symz) rel.push_back({rv, -seg});
  }
  for (const auto& r : rel) {
    if (tang_zero) {
      out.push_back(RelatedLine{r.first, r.second, 0, op_bin0(r.second, r.first)});
    } else {
      out.push_back(RelatedLine{r.first, r.second, +1, op_general(+1, r.second, r.first)});
      if (syms_) out.push_back(RelatedLine{r.first, r.second, -1, op_general(-1, r.second, r.first)});
    }
  }
}

// calculate_proj_matrix_elems_for_one_bin (ProjMatrixByBinUsingRayTracing.cxx:581-829) up to the
// call of RayTraceVoxelsOnCartesianGrid for each ray (ray_trace_one_lor, :438-579)
BasicBin Geometry::make_basic_bin(int view, int seg, int tang, int tof, std::vector<Ray>& rays) const {
  BasicBin b{};
  b.view = view;
  b.seg = seg;
  b.tang = tang;
  b.tof = tof;
  b.first_ray = static_cast<int>(rays.size());
  const float vz = d_.voxel_size_z, vy = d_.voxel_size_y, vx = d_.voxel_size_x;
  const int max_z = d_.min_z + d_.nz - 1, max_y = d_.min_y + d_.ny - 1, max_x = d_.min_x + d_.nx - 1;
  const float s_in_mm = get_s(tang);
  const float phi = get_phi(view);
  const float cphi = std::cos(phi), sphi = std::sin(phi);
  const float tantheta = get_tantheta(seg, tang);
  const float costheta = 1 / std::sqrt(1 + sq(tantheta));
  const float t_in_mm = get_t(seg, 0, tang);
  const float sdz = axial_sampling(seg) * get_costheta(seg, tang) / costheta;
  const int nlz = static_cast<int>(std::ceil(sdz / vz - 1.E-3));
  if (nlz < 1 || std::fabs(sdz / vz - nlz) > 1E-3)
    fail("ProjMatrixByBinUsingRayTracing: currently need sampling distance in axial direction to be an integer multiple of the voxel size");
  const float zfirst = (-sdz / static_cast<float>(2 * nlz) * static_cast<float>(nlz - 1)) - d_.origin_z;
  float offset_in_z = zfirst + static_cast<float>(max_z + d_.min_z) / 2.F * vz;
  if (tantheta == 0 && std::fabs(modulo_f((t_in_mm + offset_in_z) / vz, 1.F) - .5) < .001) offset_in_z -= .1F * vz;
  const float fovrad = std::min(static_cast<float>(std::min(max_x, -d_.min_x)) * vx, static_cast<float>(std::min(max_y, -d_.min_y)) * vy);
  const int ntl = d_.num_tangential_LORs;
  const bool cyl = d_.restrict_to_cylindrical_FOV != 0;

  auto one_lor = [&](float s, int num_LORs) {
    float max_a, min_a;
    if (cyl) {
      if (std::fabs(s) > fovrad) return;
      if (std::fabs(s) == fovrad) {
        max_a = min_a = 0;
      } else {
        max_a = std::sqrt(sq(fovrad) - sq(s));
        min_a = -max_a;
      }
    } else {
      if (std::fabs(cphi) < 1.E-3 || std::fabs(sphi) < 1.E-3) {
        if (fovrad < std::fabs(s)) return;
        max_a = fovrad;
        min_a = -fovrad;
      } else {
        const float sgs = sphi < 0 ? -1.f : 1.f, sgc = cphi < 0 ? -1.f : 1.f;
        max_a = std::min((fovrad * sgs - s * cphi) / sphi, (fovrad * sgc + s * sphi) / cphi);
        min_a = std::max((-fovrad * sgs - s * cphi) / sphi, (-fovrad * sgc + s * sphi) / cphi);
        if (min_a > max_a - 1.E-3 * vx) return;
      }
    }
    float st[3], sp[3];
    st[2] = (s * cphi + max_a * sphi) / vx;
    st[1] = (s * sphi - max_a * cphi) / vy;
    st[0] = (t_in_mm / costheta + offset_in_z - max_a * tantheta) / vz;
    sp[2] = (s * cphi + min_a * sphi) / vx;
    sp[1] = (s * sphi - min_a * cphi) / vy;
    sp[0] = (t_in_mm / costheta + offset_in_z - min_a * tantheta) / vz;
    const bool fwd = st[0] < sp[0] || (st[0] == sp[0] && (st[1] < sp[1] || (st[1] == sp[1] && st[2] <= sp[2])));
    Ray r;
    for (int k = 0; k < 3; ++k) {
      r.start[k] = fwd ? st[k] : sp[k];
      r.stop[k] = fwd ? sp[k] : st[k];
    }
    r.norm_const = 1 / vx / static_cast<float>(num_LORs);
    rays.push_back(r);
  };
  if (ntl == 1) {
    one_lor(s_in_mm, nlz);
  } else {
    const float s_inc = 1 * get_sampling_in_s(tang) / static_cast<float>(ntl);
    float cur = s_in_mm - s_inc * static_cast<float>(ntl - 1) / 2.F;
    for (int k = 1; k <= ntl; ++k, cur += s_inc) one_lor(cur, nlz * ntl);
  }
  b.num_rays = static_cast<int>(rays.size()) - b.first_ray;
  b.direct = tantheta == 0 ? 1 : 0;
  b.num_lors_per_axial_pos = nlz;
  b.z_origin_in_planes = d_.origin_z / vz;
  b.z_centre = static_cast<float>(max_z + d_.min_z) / 2.F;
  const float left = (t_in_mm - sdz / 2) / vz;
  const float right = (t_in_mm + sdz / 2) / vz;
  b.left_edge = left;
  b.tor_width = right - left;
  // capacity: per ray the tracer's own bound (RayTraceVoxelsOnCartesianGrid.cxx:71-73), doubled for
  // rays traced twice on a voxel boundary; times the axial copies
  int64_t cap = 0;
  for (int k = b.first_ray; k < b.first_ray + b.num_rays; ++k) {
    const Ray& r = rays[k];
    cap += 2 * (static_cast<int64_t>(std::ceil(std::fabs(r.stop[0] - r.start[0])) + std::ceil(std::fabs(r.stop[1] - r.start[1])) +
                                     std::ceil(std::fabs(r.stop[2] - r.start[2]))) + 3);
  }
  if (b.direct) {
    cap *= static_cast<int64_t>(std::ceil(b.tor_width)) + 3;
  } else {
    cap *= nlz;
  }
  if (cap > (1 << 20)) fail("row capacity too large");
  b.capacity = static_cast<int>(cap);
  return b;
}

// LOR end points on the ring (ProjDataInfoCylindrical::get_LOR, ProjDataInfoCylindrical.cxx:515-548;
// LORInCylinderCoordinates / LORAs2Points, LORCoordinates.inl:106-120,128-140,288-299) and the
// middle and unit vector of apply_tof_kernel (ProjMatrixByBin.inl:117-133), in scanner coordinates
void Geometry::lor_middle_and_direction(int seg, int view, int tang, float mid[3], float unit[3]) const {
  const float R = ring_radius_;
  const float s = get_s(tang);
  const float m = get_m(seg, 0);
  const float tantheta = get_tantheta(seg, tang);
  float phi = get_phi(view);
  const float max_a = std::sqrt(sq(R) - sq(s));
  const float min_a = -max_a;
  float z1 = m - max_a * tantheta;
  float z2 = m - min_a * tantheta;
  float beta = std::asin(s / R);
  const float two_pi = static_cast<float>(2 * kPi);
  phi = modulo_f(phi, two_pi);  // to_0_2pi (modulo.h:136-140)
  bool swapped = false;
  if (phi >= kPi) {
    phi -= static_cast<float>(kPi);
    beta = -beta;
    std::swap(z1, z2);
    swapped = true;
  }
  float psi1 = modulo_f(phi + beta, two_pi);
  float psi2 = modulo_f(phi - beta + static_cast<float>(kPi), two_pi);
  float pz1 = z1, pz2 = z2;
  if (swapped) {
    std::swap(psi1, psi2);
    std::swap(pz1, pz2);
  }
  const float p1[3] = {pz1, -R * std::cos(psi1), R * std::sin(psi1)};
  const float p2[3] = {pz2, -R * std::cos(psi2), R * std::sin(psi2)};
  float diff[3];
  for (int k = 0; k < 3; ++k) {
    mid[k] = (p1[k] + p2[k]) * 0.5f;
    diff[k] = p2[k] - mid[k];
  }
  const float n = static_cast<float>(norm_zyx(diff[0], diff[1], diff[2]));
  for (int k = 0; k < 3; ++k) unit[k] = diff[k] / n;
}

// image z of the scanner centre (ProjMatrixByBin.inl:125-127)
float Geometry::scanner_z_offset() const { return static_cast<float>(d_.num_rings - 1) / 2.0f * ring_spacing_; }

}  // namespace b200
