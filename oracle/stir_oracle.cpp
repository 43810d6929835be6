/*
 * stir_oracle.cpp -- CPU oracle (test infrastructure, not product code).
 *
 * A restatement of STIR 6.5's ray-tracing projection matrix, its symmetry
 * fold, the projectors built on it and the OSMAPOSL sub-iteration.  It is the
 * parity checker for the CUDA path and the timed CPU baseline.  Each block
 * cites the STIR source (paths relative to the STIR tree) it follows.
 *
 * Precision: templated on T.  T=float evaluates every expression in float in
 * STIR's order (build with -ffp-contract=off so no FMA is formed); T=double
 * is the FP64 oracle.
 */
#include "stir_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPI = 3.14159265358979323846264338327950288;

template <typename T> inline T square(T x) { return x * x; }

/* stir::round (src/buildblock/round.inl:59-73): half away from zero */
inline int stir_round(float x) { return x >= 0 ? static_cast<int>(x + 0.5F) : -static_cast<int>(-x + 0.5F); }
inline int stir_round(double x) { return x >= 0 ? static_cast<int>(x + 0.5) : -static_cast<int>(-x + 0.5); }

/* stir::modulo (src/include/stir/modulo.h:51-78) */
inline double modulo_d(double a, double b) {
  const double res = std::fmod(a, b);
  return res < 0 ? res + std::fabs(b) : res;
}
inline float modulo(float a, float b) {
  float res = static_cast<float>(modulo_d(static_cast<double>(a), static_cast<double>(b)));
  const float abs_b = b >= 0 ? b : -b;
  if (res >= abs_b) res -= abs_b;
  return res;
}
inline double modulo(double a, double b) { return modulo_d(a, b); }

/* ---------------------------------------------------------------------------
 * Row of the projection matrix (ProjMatrixElemsForOneBin)
 * ------------------------------------------------------------------------- */
template <typename T> struct Elem {
  int z, y, x;
  T v;
};
template <typename T> inline bool coords_less(const Elem<T>& a, const Elem<T>& b) {
  /* ProjMatrixElemsForOneBinValue::coordinates_less (ProjMatrixElemsForOneBinValue.inl:121-125) */
  return a.z < b.z || (a.z == b.z && (a.y < b.y || (a.y == b.y && a.x < b.x)));
}
template <typename T> using Row = std::vector<Elem<T>>;

template <typename T> void row_sort(Row<T>& r) { std::sort(r.begin(), r.end(), coords_less<T>); }

/* ProjMatrixElemsForOneBin::merge (src/recon_buildblock/ProjMatrixElemsForOneBin.cxx:162-277):
   sort both, add values of equal coordinates, keep the union sorted. */
template <typename T> void row_merge(Row<T>& a, Row<T>& b) {
  if (b.empty()) return;
  row_sort(a);
  row_sort(b);
  Row<T> out;
  out.reserve(a.size() + b.size());
  size_t i = 0, j = 0;
  while (j < b.size()) {
    if (i == a.size()) {
      out.insert(out.end(), b.begin() + j, b.end());
      break;
    }
    if (a[i].z == b[j].z && a[i].y == b[j].y && a[i].x == b[j].x) {
      Elem<T> e = a[i];
      e.v = a[i].v + b[j].v;
      out.push_back(e);
      ++i;
      ++j;
    } else if (coords_less(b[j], a[i])) {
      out.push_back(b[j]);
      ++j;
    } else {
      out.push_back(a[i]);
      ++i;
    }
  }
  while (i < a.size()) out.push_back(a[i++]);
  a.swap(out);
}

/* ---------------------------------------------------------------------------
 * Siddon tracer: RayTraceVoxelsOnCartesianGrid (src/recon_buildblock/RayTraceVoxelsOnCartesianGrid.cxx:51-269)
 * Coordinates are (z,y,x) in voxel units; voxel_size in mm.
 * ------------------------------------------------------------------------- */
template <typename T> struct C3 {
  T z, y, x;
};

template <typename T> inline bool is_half_integer(T a) {
  /* :47-50 */
  return std::fabs(std::floor(a) + T(.5) - a) < T(.0001);
}

/* norm of a coordinate: inner product in coordT (z first), sqrt in double (BasicCoordinate.inl:413-429) */
template <typename T> inline double norm3(T z, T y, T x) {
  T s = T(0);
  s = s + z * z;
  s = s + y * y;
  s = s + x * x;
  return std::sqrt(static_cast<double>(s));
}

template <typename T>
void ray_trace(Row<T>& lor, const C3<T>& start, const C3<T>& stop, const C3<T>& vox, const T norm_const) {
  const C3<T> diff{stop.z - start.z, stop.y - start.y, stop.x - start.x};
  if (norm3(diff.z, diff.y, diff.x) <= .00001F) return; /* :61-67 */

  /* d12 (:76-79) */
  const T d12 = static_cast<T>(norm3(diff.z * vox.z, diff.y * vox.y, diff.x * vox.x) * norm_const);
  const int sign_x = diff.x >= 0 ? 1 : -1;
  const int sign_y = diff.y >= 0 ? 1 : -1;
  const int sign_z = diff.z >= 0 ? 1 : -1;

  const T small_difference = T(1.E-4F); /* :100-103 */
  const bool zx = std::fabs(diff.x) <= small_difference;
  const bool zy = std::fabs(diff.y) <= small_difference;
  const bool zz = std::fabs(diff.z) <= small_difference;

  /* rays in a plane between voxels: trace twice at +-0.5 with half weight (:105-131) */
  {
    C3<T> inc{0, 0, 0};
    if (zz && is_half_integer(start.z))
      inc = C3<T>{T(.5F), 0, 0};
    else if (zy && is_half_integer(start.y))
      inc = C3<T>{0, T(.5F), 0};
    else if (zx && is_half_integer(start.x))
      inc = C3<T>{0, 0, T(.5F)};
    if (norm3(inc.z, inc.y, inc.x) > .1) {
      ray_trace(lor, C3<T>{start.z - inc.z, start.y - inc.y, start.x - inc.x},
                C3<T>{stop.z - inc.z, stop.y - inc.y, stop.x - inc.x}, vox, norm_const / 2);
      ray_trace(lor, C3<T>{start.z + inc.z, start.y + inc.y, start.x + inc.x},
                C3<T>{stop.z + inc.z, stop.y + inc.y, stop.x + inc.x}, vox, norm_const / 2);
      row_sort(lor);
      return;
    }
  }

  /* increments (:140-142) */
  const T inc_x = zx ? d12 * T(1000000.F) : d12 / std::fabs(diff.x);
  const T inc_y = zy ? d12 * T(1000000.F) : d12 / std::fabs(diff.y);
  const T inc_z = zz ? d12 * T(1000000.F) : d12 / std::fabs(diff.z);

  /* last plane crossings, shortened by .9999 (:146-169) */
  const T xmax = static_cast<T>(stir_round(stop.x)) + static_cast<T>(sign_x) * T(0.5F);
  const T ymax = static_cast<T>(stir_round(stop.y)) + static_cast<T>(sign_y) * T(0.5F);
  const T zmax = static_cast<T>(stir_round(stop.z)) + static_cast<T>(sign_z) * T(0.5F);
  const T axend = zx ? d12 * T(1000000.F) : (xmax - start.x) * inc_x * static_cast<T>(sign_x) * T(.9999F);
  const T ayend = zy ? d12 * T(1000000.F) : (ymax - start.y) * inc_y * static_cast<T>(sign_y) * T(.9999F);
  const T azend = zz ? d12 * T(1000000.F) : (zmax - start.z) * inc_z * static_cast<T>(sign_z) * T(.9999F);
  const T amax = std::min(axend, std::min(ayend, azend));

  /* first voxel and first crossings (:178-213) */
  int cz = stir_round(start.z), cy = stir_round(start.y), cx = stir_round(start.x);
  T az = zz ? -inc_z : ((static_cast<T>(cz) - start.z) - static_cast<T>(sign_z) * T(0.5F)) * inc_z * static_cast<T>(sign_z);
  T ax = zx ? -inc_x : ((static_cast<T>(cx) - start.x) - static_cast<T>(sign_x) * T(0.5F)) * inc_x * static_cast<T>(sign_x);
  T ay = zy ? -inc_y : ((static_cast<T>(cy) - start.y) - static_cast<T>(sign_y) * T(0.5F)) * inc_y * static_cast<T>(sign_y);
  T a = std::max(ax, std::max(ay, az));
  ax = zx ? axend : ax + inc_x;
  ay = zy ? ayend : ay + inc_y;
  az = zz ? azend : az + inc_z;

  /* main loop (:236-267) */
  while (a < amax) {
    if (ax < ay) {
      if (ax < az) {
        lor.push_back(Elem<T>{cz, cy, cx, ax - a});
        a = ax;
        ax += inc_x;
        cx += sign_x;
      } else {
        lor.push_back(Elem<T>{cz, cy, cx, az - a});
        a = az;
        az += inc_z;
        cz += sign_z;
      }
    } else if (ay < az) {
      lor.push_back(Elem<T>{cz, cy, cx, ay - a});
      a = ay;
      ay += inc_y;
      cy += sign_y;
    } else {
      lor.push_back(Elem<T>{cz, cy, cx, az - a});
      a = az;
      az += inc_z;
      cz += sign_z;
    }
  }
}

/* ---------------------------------------------------------------------------
 * Geometry (ProjDataInfoCylindrical{,NoArcCorr,ArcCorr}, Scanner, VoxelsOnCartesianGrid)
 * ------------------------------------------------------------------------- */
enum OpXY { XY_ID = 0 };
/* A symmetry operation of SymmetryOperations_PET_CartesianGrid.inl:38-564, in the form
   x' = (swap ? y : x) * sx,  y' = (swap ? x : y) * sy,  z' = (zq ? q - z : z) + z_shift */
struct SymOp {
  int swap = 0, sx = 1, sy = 1, zq = 0, q = 0, z_shift = 0;
};

template <typename T> struct Geometry {
  b200rt_geometry d;
  int S = 0;  /* max segment */
  int num_views = 0, num_tang = 0, min_tang = 0, max_tang = 0;
  T azimuthal_sampling = 0, azimuthal_offset = 0, ring_radius = 0, ring_spacing = 0, angular_increment = 0, arc_bin = 0;
  std::vector<T> m_offset;                /* per segment index */
  std::vector<int64_t> seg_offset_stir;   /* ProjDataInMemory offset of each segment (index seg+S) */
  int64_t tof_stride = 0;                 /* elements per TOF bin */
  int64_t projdata_size = 0;
  int num_tof = 1, min_tof = 0, max_tof = 0;
  /* image */
  int nz, ny, nx, min_z, min_y, min_x, max_z, max_y, max_x;
  C3<T> vox, origin;
  /* symmetries (DataSymmetriesForBins_PET_CartesianGrid.cxx:223-420) */
  bool sym90 = true, sym180 = true, symseg = true, syms = true, symz = true;
  int num_planes_per_scanner_ring = 0;
  std::vector<int> npa;        /* num_planes_per_axial_pos per segment */
  std::vector<T> ax_to_z;      /* axial_pos_to_z_offset per segment (stored as float in STIR) */
  std::vector<T> deltas;
  /* TOF */
  std::vector<T> tof_low, tof_high; /* bin boundaries in mm */
  T r_sqrt2_gauss_sigma = 0;
  T tof_trunc_n = 0; /* kernel truncated at +-k sigma: k / sqrt(2); 0: STIR's cut-off */

  int nax(int seg) const { return d.num_axial_poss[seg + S]; }
  int min_rd(int seg) const { return d.min_ring_diff[seg + S]; }
  int max_rd(int seg) const { return d.max_ring_diff[seg + S]; }

  /* ProjDataInfoCylindrical.inl:98-128 */
  int num_axial_poss_per_ring_inc(int seg) const { return max_rd(seg) != min_rd(seg) ? 2 : 1; }
  T axial_sampling(int seg) const { return ring_spacing / static_cast<T>(num_axial_poss_per_ring_inc(seg)); }
  T average_ring_difference(int seg) const { return static_cast<T>(min_rd(seg) + max_rd(seg)) / T(2.F); }
  /* get_phi (ProjDataInfoCylindrical.inl:63-67) */
  T get_phi(int view) const { return static_cast<T>(view) * azimuthal_sampling + azimuthal_offset; }
  /* get_s: NoArcCorr (ProjDataInfoCylindricalNoArcCorr.inl:79-82), ArcCorr (ProjDataInfoCylindricalArcCorr.inl:29-33) */
  T get_s(int tang) const {
    if (d.arc_corrected) return static_cast<T>(tang) * arc_bin;
    return ring_radius * std::sin(static_cast<T>(tang) * angular_increment);
  }
  /* get_tantheta (ProjDataInfoCylindrical.inl:83-92) */
  T get_tantheta(int seg, int tang) const {
    const T delta = average_ring_difference(seg);
    if (std::fabs(delta) < T(0.0001F)) return T(0);
    const T R = ring_radius;
    return delta * ring_spacing / (T(2) * std::sqrt(square(R) - square(get_s(tang))));
  }
  /* ProjDataInfo.inl:200-203 */
  T get_costheta(int seg, int tang) const { return T(1) / std::sqrt(T(1) + square(get_tantheta(seg, tang))); }
  /* get_m / get_t (ProjDataInfoCylindrical.inl:69-81) */
  T get_m(int seg, int ax) const { return static_cast<T>(ax) * axial_sampling(seg) - m_offset[seg + S]; }
  T get_t(int seg, int ax, int tang) const { return get_m(seg, ax) * get_costheta(seg, tang); }
  /* get_sampling_in_t (ProjDataInfoCylindrical.inl:100-104) */
  T get_sampling_in_t(int seg, int tang) const { return axial_sampling(seg) * get_costheta(seg, tang); }
  /* ProjDataInfo::get_sampling_in_s (ProjDataInfo.cxx:109-114) */
  T get_sampling_in_s(int tang) const { return std::fabs(get_s(tang + 1) - get_s(tang - 1)) / T(2); }

  /* ProjDataInMemory::get_index (ProjDataInMemory.cxx:190-235) with segment sequence 0,+1,-1,...
     (ProjData.cxx:641-661) */
  int64_t stir_index(int seg, int view, int ax, int tang, int tof) const {
    return static_cast<int64_t>(tof - min_tof) * tof_stride + seg_offset_stir[seg + S] +
           (static_cast<int64_t>(ax) * num_views + view) * num_tang + (tang - min_tang);
  }
};

template <typename T> void setup_geometry(Geometry<T>& g, const b200rt_geometry& d) {
  g.d = d;
  g.S = d.max_segment_num;
  if (g.S < 0 || 2 * g.S + 1 > B200RT_MAX_SEGMENTS) throw std::runtime_error("bad max_segment_num");
  g.num_views = d.num_views;
  g.num_tang = d.num_tangential_poss;
  /* ProjDataInfo::set_num_tangential_poss (ProjDataInfo.cxx:124-129) */
  g.min_tang = -(d.num_tangential_poss / 2);
  g.max_tang = g.min_tang + d.num_tangential_poss - 1;
  /* ProjDataInfoCylindrical constructor (ProjDataInfoCylindrical.cxx:55-116) */
  g.azimuthal_sampling = static_cast<T>(kPI / d.num_views);
  g.azimuthal_offset = static_cast<T>(d.intrinsic_azimuthal_tilt_rad);
  {
    const int ndet = d.num_detectors_per_ring;
    if (ndet > 2 && d.num_views * 2 != ndet && ndet % (d.num_views * 2) == 0) {
      const int view_mashing = ndet / 2 / d.num_views;
      const T offset_inc = static_cast<T>(kPI / (ndet / 2) * (view_mashing - 1) / T(2.F));
      g.azimuthal_offset += offset_inc;
    }
  }
  /* Scanner::get_effective_ring_radius (Scanner.inl:91-95) */
  g.ring_radius = static_cast<T>(d.inner_ring_radius_mm) + static_cast<T>(d.average_depth_of_interaction_mm);
  g.ring_spacing = static_cast<T>(d.ring_spacing_mm);
  /* ProjDataInfoCylindricalNoArcCorr (ProjDataInfoCylindricalNoArcCorr.cxx:75-88) */
  g.angular_increment = static_cast<T>(kPI / d.num_detectors_per_ring);
  g.arc_bin = static_cast<T>(d.arccorr_bin_size_mm);
  /* m_offset (ProjDataInfoCylindrical.cxx:135-145) */
  g.m_offset.assign(2 * g.S + 1, T(0));
  for (int s = -g.S; s <= g.S; ++s) {
    if (d.num_axial_poss[s + g.S] <= 0) throw std::runtime_error("segment without axial positions");
    if (d.min_ring_diff[s + g.S] > d.max_ring_diff[s + g.S]) throw std::runtime_error("min_ring_diff > max_ring_diff");
    g.m_offset[s + g.S] = (static_cast<T>(d.num_axial_poss[s + g.S] - 1 + 0) * g.axial_sampling(s)) / T(2);
  }
  /* storage offsets */
  g.seg_offset_stir.assign(2 * g.S + 1, 0);
  int64_t off = 0;
  std::vector<int> seq;
  seq.push_back(0);
  for (int s = 1; s <= g.S; ++s) {
    seq.push_back(s);
    seq.push_back(-s);
  }
  for (int s : seq) {
    g.seg_offset_stir[s + g.S] = off;
    off += static_cast<int64_t>(g.nax(s)) * g.num_views * g.num_tang;
  }
  g.tof_stride = off;
  /* TOF bins (ProjDataInfo::set_tof_mash_factor, ProjDataInfo.cxx:174-255; get_k / get_sampling_in_k :69-92) */
  g.num_tof = 1;
  g.min_tof = g.max_tof = 0;
  if (d.tof_mash_factor > 0) {
    const int max_poss = d.max_num_timing_poss;
    if (max_poss < 1 || max_poss % d.tof_mash_factor) throw std::runtime_error("bad TOF mashing");
    g.num_tof = max_poss / d.tof_mash_factor;
    g.min_tof = -g.num_tof / 2;
    g.max_tof = g.min_tof + g.num_tof - 1;
    /* tof_delta_time_to_mm (TOF_conversions.h:31-34): speed of light / 2 in mm/ps */
    const double c_half = 0.299792458 * 0.5;
    const float fmash_size = static_cast<float>(d.tof_mash_factor) * d.size_of_timing_pos_ps;
    const T inc = static_cast<T>(static_cast<float>(static_cast<double>(fmash_size) * c_half));
    auto get_k = [&](int k) {
      return (g.num_tof % 2) ? static_cast<T>(k) * inc : static_cast<T>(k) * inc + inc / T(2.f);
    };
    g.tof_low.resize(g.num_tof);
    g.tof_high.resize(g.num_tof);
    for (int k = g.min_tof; k <= g.max_tof; ++k) {
      const T sampling = (get_k(k + 1) - get_k(k - 1)) / T(2.f);
      const T centre = get_k(k);
      g.tof_low[k - g.min_tof] = centre - sampling / T(2.f);
      g.tof_high[k - g.min_tof] = centre + sampling / T(2.f);
    }
    /* ProjMatrixByBin::enable_tof (ProjMatrixByBin.cxx:66-75) */
    const T sigma = static_cast<T>(static_cast<float>(static_cast<double>(d.timing_resolution_ps) * c_half)) / T(2.355f);
    g.r_sqrt2_gauss_sigma = T(1.0f) / (sigma * static_cast<T>(std::sqrt(2.0)));
    if (!(d.tof_kernel_truncation_sigmas >= 0.f)) throw std::runtime_error("tof_kernel_truncation_sigmas must be >= 0");
    g.tof_trunc_n = static_cast<T>(static_cast<double>(d.tof_kernel_truncation_sigmas) / std::sqrt(2.0));
  }
  g.projdata_size = g.tof_stride * g.num_tof;

  /* image */
  g.nz = d.nz;
  g.ny = d.ny;
  g.nx = d.nx;
  g.min_z = d.min_z;
  g.min_y = d.min_y;
  g.min_x = d.min_x;
  g.max_z = d.min_z + d.nz - 1;
  g.max_y = d.min_y + d.ny - 1;
  g.max_x = d.min_x + d.nx - 1;
  g.vox = C3<T>{static_cast<T>(d.voxel_size_z), static_cast<T>(d.voxel_size_y), static_cast<T>(d.voxel_size_x)};
  g.origin = C3<T>{static_cast<T>(d.origin_z), static_cast<T>(d.origin_y), static_cast<T>(d.origin_x)};
  if (g.nz < 1 || g.ny < 1 || g.nx < 1) throw std::runtime_error("empty image");

  /* ProjMatrixByBinUsingRayTracing::set_up checks (ProjMatrixByBinUsingRayTracing.cxx:272-277) */
  if (std::fabs(d.origin_x) > .05F || std::fabs(d.origin_y) > .05F)
    throw std::runtime_error("ProjMatrixByBinUsingRayTracing sadly doesn't support shifted x/y origin yet");
  if (d.num_tangential_LORs < 1) throw std::runtime_error("num_tangential_LORs should be at least 1");

  /* DataSymmetriesForBins_PET_CartesianGrid constructor (DataSymmetriesForBins_PET_CartesianGrid.cxx:223-420) */
  g.sym90 = d.do_symmetry_90degrees_min_phi != 0;
  g.sym180 = d.do_symmetry_90degrees_min_phi != 0 || d.do_symmetry_180degrees_min_phi != 0;
  g.symseg = d.do_symmetry_swap_segment != 0;
  g.syms = d.do_symmetry_swap_s != 0;
  g.symz = d.do_symmetry_shift_z != 0;
  {
    const float zorig_planes = d.origin_z / d.voxel_size_z;
    if (std::fabs(stir_round(zorig_planes) - zorig_planes) > 1.E-3F)
      throw std::runtime_error("z origin should be a multiple of the plane separation");
    if (std::fabs(d.voxel_size_y - d.voxel_size_x) > 2.E-3F) g.sym90 = false;
    if (d.num_views % 4 != 0) g.sym90 = false;
    if (d.num_views % 2 != 0) g.sym180 = false;
    if (std::fabs(g.get_tantheta(0, 0)) > T(1.E-4F))
      throw std::runtime_error("segment 0 must correspond to direct planes (theta==0)");
    for (int s = 1; s <= g.S; ++s)
      if (std::fabs(g.get_tantheta(s, 0) + g.get_tantheta(-s, 0)) > T(1.E-4F))
        throw std::runtime_error("negative segments must correspond to -theta of the positive segments");
    if (std::fabs(g.get_s(1) + g.get_s(-1)) > T(1.E-4F)) throw std::runtime_error("s-symmetry not satisfied");
    if (std::fabs(g.get_phi(0)) > T(1.E-4F) && (g.sym90 || g.sym180)) {
      g.sym90 = false;
      g.sym180 = false;
    }
    if (g.num_tof > 1) {
      g.sym90 = g.sym180 = g.symseg = g.syms = false;
    }
    if (std::fabs(d.origin_x) > .01F || std::fabs(d.origin_y) > .01F) g.sym90 = g.sym180 = g.symseg = g.syms = false;
  }
  /* find_relation_between_coordinate_systems (DataSymmetriesForBins_PET_CartesianGrid.cxx:49-115) */
  {
    const T plane = g.vox.z;
    const T nppsr_f = g.ring_spacing / plane;
    g.num_planes_per_scanner_ring = stir_round(nppsr_f);
    if (std::fabs(nppsr_f - static_cast<T>(g.num_planes_per_scanner_ring)) > T(1.E-2))
      throw std::runtime_error("z-grid spacing must be the ring spacing divided by an integer");
    g.npa.assign(2 * g.S + 1, 0);
    g.ax_to_z.assign(2 * g.S + 1, T(0));
    g.deltas.assign(2 * g.S + 1, T(0));
    for (int s = -g.S; s <= g.S; ++s) {
      const T npa_f = g.axial_sampling(s) / plane;
      g.npa[s + g.S] = stir_round(npa_f);
      if (std::fabs(npa_f - static_cast<T>(g.npa[s + g.S])) > T(1.E-2))
        throw std::runtime_error("z-grid spacing must be the axial sampling divided by an integer");
      const T delta = g.average_ring_difference(s);
      g.deltas[s + g.S] = delta;
      g.ax_to_z[s + g.S] = static_cast<T>(g.max_z + g.min_z) / T(2.F) - g.origin.z / plane -
                           (static_cast<T>(g.npa[s + g.S] * (g.nax(s) - 1 + 0)) +
                            static_cast<T>(g.num_planes_per_scanner_ring) * delta) / T(2);
    }
  }
  if (!g.symz) throw std::runtime_error("do_symmetry_shift_z=0 is not supported");
}

/* ---------------------------------------------------------------------------
 * Symmetries (DataSymmetriesForBins_PET_CartesianGrid.inl)
 * ------------------------------------------------------------------------- */
template <typename T> struct Bin {
  int seg, view, ax, tang, tof;
};

/* find_transform_z (DataSymmetriesForBins_PET_CartesianGrid.inl:63-100) */
template <typename T> int find_transform_z(const Geometry<T>& g, int seg, int ax) {
  const T delta = g.deltas[seg + g.S];
  const T tz = (static_cast<T>(2 * g.npa[seg + g.S] * ax) + static_cast<T>(g.num_planes_per_scanner_ring) * delta +
                T(2) * g.ax_to_z[seg + g.S]);
  return static_cast<int>(std::floor(tz + 0.5));
}

inline SymOp make_op(int swap, int sx, int sy, int zq, int q, int zs) {
  SymOp o;
  o.swap = swap;
  o.sx = sx;
  o.sy = sy;
  o.zq = zq;
  o.q = q;
  o.z_shift = zs;
  return o;
}
/* SymmetryOperations_PET_CartesianGrid.inl transform_image_coordinates, by class */
enum OpClass {
  OP_TRIVIAL, OP_ZSHIFT, OP_XMX_ZQ, OP_XMY_YX_ZQ, OP_XY_YX_ZQ, OP_XMY_YX, OP_XY_YX, OP_XMX, OP_YMY, OP_ZQ,
  OP_XMX_YMY_ZQ, OP_XY_YMX_ZQ, OP_XY_YMX, OP_XMY_YMX, OP_YMY_ZQ, OP_XMX_YMY, OP_XMY_YMX_ZQ
};
inline SymOp op_of(OpClass c, int q, int zs) {
  switch (c) {
    case OP_TRIVIAL: return make_op(0, 1, 1, 0, 0, 0);
    case OP_ZSHIFT: return make_op(0, 1, 1, 0, 0, zs);               /* :48-51 */
    case OP_XMX_ZQ: return make_op(0, -1, 1, 1, q, zs);              /* :72-76 */
    case OP_XMY_YX_ZQ: return make_op(1, -1, 1, 1, q, zs);           /* :100-106 */
    case OP_XY_YX_ZQ: return make_op(1, 1, 1, 1, q, zs);             /* :127-133 */
    case OP_XMY_YX: return make_op(1, -1, 1, 0, 0, zs);              /* :172-178 */
    case OP_XY_YX: return make_op(1, 1, 1, 0, 0, zs);                /* :215-221 */
    case OP_XMX: return make_op(0, -1, 1, 0, 0, zs);                 /* :257-261 */
    case OP_YMY: return make_op(0, 1, -1, 0, 0, zs);                 /* :297-301 */
    case OP_ZQ: return make_op(0, 1, 1, 1, q, zs);                   /* :319-322 */
    case OP_XMX_YMY_ZQ: return make_op(0, -1, -1, 1, q, zs);         /* :339-344 */
    case OP_XY_YMX_ZQ: return make_op(1, 1, -1, 1, q, zs);           /* :383-389 */
    case OP_XY_YMX: return make_op(1, 1, -1, 0, 0, zs);              /* :427-433 */
    case OP_XMY_YMX: return make_op(1, -1, -1, 0, 0, zs);            /* :472-478 */
    case OP_YMY_ZQ: return make_op(0, 1, -1, 1, q, zs);              /* :503-507 */
    case OP_XMX_YMY: return make_op(0, -1, -1, 0, 0, zs);            /* :526-531 */
    case OP_XMY_YMX_ZQ: return make_op(1, -1, -1, 1, q, zs);         /* :556-562 */
  }
  return SymOp();
}

/* find_sym_op_bin0 (DataSymmetriesForBins_PET_CartesianGrid.inl:102-162) */
template <typename T> SymOp find_sym_op_bin0(const Geometry<T>& g, int seg, int view, int ax) {
  const int q = find_transform_z(g, std::abs(seg), g.symz ? 0 : ax);
  const int zs = g.symz ? g.npa[seg + g.S] * ax : 0;
  const int view180 = g.num_views, view135 = view180 / 4 * 3, view90 = view180 / 2, view45 = view180 / 4;
  if (g.sym90 && view > view90 && view <= view135)
    return op_of((!g.symseg || seg >= 0) ? OP_XMY_YX : OP_XMY_YX_ZQ, q, zs);
  if (g.sym90 && view > view45 && view <= view90)
    return op_of((!g.symseg || seg >= 0) ? OP_XY_YX_ZQ : OP_XY_YX, q, zs);
  if (g.sym180 && view > view90) return op_of((!g.symseg || seg >= 0) ? OP_XMX_ZQ : OP_XMX, q, zs);
  if (g.symseg && seg < 0) return op_of(OP_ZQ, q, zs);
  return zs == 0 ? op_of(OP_TRIVIAL, q, zs) : op_of(OP_ZSHIFT, q, zs);
}

/* find_sym_op_general_bin (DataSymmetriesForBins_PET_CartesianGrid.inl:196-326) */
template <typename T> SymOp find_sym_op_general(const Geometry<T>& g, int s, int seg, int view, int ax) {
  const int q = find_transform_z(g, std::abs(seg), g.symz ? 0 : ax);
  const int zs = g.symz ? g.npa[seg + g.S] * ax : 0;
  const int view180 = g.num_views, view135 = view180 / 4 * 3, view90 = view180 / 2, view45 = view180 / 4;
  const bool sp = !g.syms || s > 0;
  if (g.sym90 && view > view90 && view <= view135) {
    if (!g.symseg || seg > 0) return op_of(sp ? OP_XMY_YX : OP_XY_YMX_ZQ, q, zs);
    if (seg < 0) return op_of(sp ? OP_XMY_YX_ZQ : OP_XY_YMX, q, zs);
    return op_of(sp ? OP_XMY_YX : OP_XY_YMX, q, zs);
  }
  if (g.sym90 && view > view45 && view <= view90) {
    if (!g.symseg || seg > 0) return op_of(sp ? OP_XY_YX_ZQ : OP_XMY_YMX, q, zs);
    if (seg < 0) return op_of(sp ? OP_XY_YX : OP_XMY_YMX_ZQ, q, zs);
    return op_of(sp ? OP_XY_YX : OP_XMY_YMX, q, zs);
  }
  if (g.sym180 && view > view90) {
    if (!g.symseg || seg > 0) return op_of(sp ? OP_XMX_ZQ : OP_YMY, q, zs);
    return op_of(sp ? OP_XMX : OP_YMY_ZQ, q, zs);
  }
  if (!g.symseg || seg > 0) {
    if (g.syms && s < 0) return op_of(OP_XMX_YMY_ZQ, q, zs);
    return zs == 0 ? op_of(OP_TRIVIAL, q, zs) : op_of(OP_ZSHIFT, q, zs);
  }
  if (seg < 0) {
    if (g.syms && s < 0) return op_of(OP_XMX_YMY, q, zs);
    return op_of(OP_ZQ, q, zs);
  }
  if (g.syms && s < 0) return op_of(OP_XMX_YMY, q, zs);
  return zs == 0 ? op_of(OP_TRIVIAL, q, zs) : op_of(OP_ZSHIFT, q, zs);
}

/* find_basic_view_segment_numbers (DataSymmetriesForBins_PET_CartesianGrid.inl:359-404) */
template <typename T> bool find_basic_vs(const Geometry<T>& g, int& view, int& seg) {
  bool change = false;
  const int view90 = g.num_views >> 1, view45 = view90 >> 1, view135 = view90 + view45;
  if (g.symseg && seg < 0) {
    seg = -seg;
    change = true;
  }
  if (g.sym90) {
    if (view >= view135) {
      view = g.num_views - view;
      return true;
    } else if (view >= view90) {
      view = view - view90;
      return true;
    } else if (view > view45) {
      view = view90 - view;
      return true;
    }
  } else if (g.sym180) {
    if (view > view90) {
      view = g.num_views - view;
      return true;
    }
  }
  return change;
}

/* find_basic_bin (DataSymmetriesForBins_PET_CartesianGrid.inl:406-433) */
template <typename T> void find_basic_bin(const Geometry<T>& g, Bin<T>& b) {
  find_basic_vs(g, b.view, b.seg);
  if (g.syms && b.tang < 0) {
    b.tang = -b.tang;
    b.tof = -b.tof;
  }
  if (g.symz && b.ax != 0) b.ax = 0;
}

/* find_symmetry_operation_from_basic_bin (DataSymmetriesForBins_PET_CartesianGrid.inl:606-615) */
template <typename T> SymOp find_op_and_basic(const Geometry<T>& g, Bin<T>& b) {
  SymOp op = (b.tang == 0) ? find_sym_op_bin0(g, b.seg, b.view, b.ax) : find_sym_op_general(g, b.tang, b.seg, b.view, b.ax);
  find_basic_bin(g, b);
  return op;
}

/* get_related_view_segment_numbers (DataSymmetriesForBins_PET_CartesianGrid.inl:735-782) */
template <typename T> void related_vs(const Geometry<T>& g, int view, int seg, std::vector<std::pair<int, int>>& rel) {
  const int nv = g.num_views;
  const bool symz = g.symseg && seg != 0;
  rel.clear();
  rel.push_back({view, seg});
  if (symz) rel.push_back({view, -seg});
  if (g.sym180 && g.sym90 && (view % (nv / 2)) != nv / 4) {
    const int rv = view < nv / 2 ? view + nv / 2 : view - nv / 2;
    rel.push_back({rv, seg});
    if (symz) rel.push_back({rv, -seg});
  }
  if (g.sym180 && (view % (nv / 2)) != 0) {
    rel.push_back({nv - view, seg});
    if (symz) rel.push_back({nv - view, -seg});
  }
  if (g.sym90 && (view % (nv / 4)) != 0) {
    const int rv = (nv / 2 - view + nv) % nv;
    rel.push_back({rv, seg});
    if (symz) rel.push_back({rv, -seg});
  }
}

/* detail::find_basic_vs_nums_in_subset (find_basic_vs_nums_in_subset.cxx:32-70) */
template <typename T>
std::vector<std::pair<int, int>> basic_vs_in_subset(const Geometry<T>& g, int subset, int nsub) {
  std::vector<std::pair<int, int>> out;
  for (int seg = -g.S; seg <= g.S; ++seg)
    for (int view = subset; view < g.num_views; view += nsub) {
      int v = view, s = seg;
      if (find_basic_vs(g, v, s)) continue;
      out.push_back({view, seg});
    }
  return out;
}

/* ---------------------------------------------------------------------------
 * Matrix rows (ProjMatrixByBinUsingRayTracing.cxx)
 * ------------------------------------------------------------------------- */
/* ray_trace_one_lor (ProjMatrixByBinUsingRayTracing.cxx:438-579) */
template <typename T>
void ray_trace_one_lor(Row<T>& lor, T s, T t, T cphi, T sphi, T costheta, T tantheta, T offset_in_z, T fovrad,
                       const C3<T>& vox, bool restrict_cyl, int num_LORs) {
  T max_a, min_a;
  if (restrict_cyl) {
    if (std::fabs(s) > fovrad) return;
    if (std::fabs(s) == fovrad) {
      max_a = min_a = 0;
    } else {
      max_a = std::sqrt(square(fovrad) - square(s));
      min_a = -max_a;
    }
  } else {
    if (std::fabs(cphi) < T(1.E-3) || std::fabs(sphi) < T(1.E-3)) {
      if (fovrad < std::fabs(s)) return;
      max_a = fovrad;
      min_a = -fovrad;
    } else {
      auto sign = [](T v) { return v < 0 ? T(-1) : T(1); };
      max_a = std::min((fovrad * sign(sphi) - s * cphi) / sphi, (fovrad * sign(cphi) + s * sphi) / cphi);
      min_a = std::max((-fovrad * sign(sphi) - s * cphi) / sphi, (-fovrad * sign(cphi) + s * sphi) / cphi);
      if (min_a > max_a - T(1.E-3) * vox.x) return;
    }
  }
  C3<T> start, stop;
  start.x = (s * cphi + max_a * sphi) / vox.x;
  start.y = (s * sphi - max_a * cphi) / vox.y;
  start.z = (t / costheta + offset_in_z - max_a * tantheta) / vox.z;
  stop.x = (s * cphi + min_a * sphi) / vox.x;
  stop.y = (s * sphi - min_a * cphi) / vox.y;
  stop.z = (t / costheta + offset_in_z - min_a * tantheta) / vox.z;
  const bool fwd = start.z < stop.z ||
                   (start.z == stop.z && (start.y < stop.y || (start.y == stop.y && (start.x <= stop.x))));
  ray_trace(lor, fwd ? start : stop, !fwd ? start : stop, vox, T(1) / vox.x / static_cast<T>(num_LORs));
}

/* add_adjacent_z (ProjMatrixByBinUsingRayTracing.cxx:831-954) */
template <typename T> void add_adjacent_z(Row<T>& lor, const T zf, const T right) {
  const size_t org = lor.size();
  const int z0 = lor.front().z;
  for (int zi = 1;; ++zi) {
    const T overlap = std::min(right, zf + static_cast<T>(zi) + T(.5F)) - std::max(T(0.F), zf + static_cast<T>(zi) - T(.5F));
    if (overlap <= 0.0001) break;
    const int nz = z0 + zi;
    for (size_t k = 0; k < org; ++k) {
      const Elem<T> e = lor[k];
      lor.push_back(Elem<T>{nz, e.y, e.x, overlap > .9999 ? e.v : e.v * overlap});
    }
  }
  if (zf > 0.5) {
    const T overlap = zf - T(.5F);
    const int nz = z0 - 1;
    for (size_t k = 0; k < org; ++k) {
      const Elem<T> e = lor[k];
      lor.push_back(Elem<T>{nz, e.y, e.x, overlap > .9999 ? e.v : e.v * overlap});
    }
  }
  {
    const T overlap = std::min(right, zf + T(.5F)) - std::max(T(0.F), zf - T(.5F));
    if (overlap < .9999)
      for (size_t k = 0; k < org; ++k) lor[k].v *= overlap;
  }
}

/* calculate_proj_matrix_elems_for_one_bin (ProjMatrixByBinUsingRayTracing.cxx:581-829) for a basic bin */
template <typename T> void calculate_row(const Geometry<T>& g, const Bin<T>& bin, Row<T>& lor) {
  lor.clear();
  const T s_in_mm = g.get_s(bin.tang);
  const T phi = g.get_phi(bin.view);
  const T cphi = std::cos(phi);
  const T sphi = std::sin(phi);
  const T tantheta = g.get_tantheta(bin.seg, bin.tang);
  const T costheta = T(1) / std::sqrt(T(1) + square(tantheta));
  const T t_in_mm = g.get_t(bin.seg, bin.ax, bin.tang);
  const T sdz = g.get_sampling_in_t(bin.seg, bin.tang) / costheta;
  const int nlz = static_cast<int>(std::ceil(sdz / g.vox.z - 1.E-3));
  if (std::fabs(sdz / g.vox.z - nlz) > 1E-3)
    throw std::runtime_error("axial sampling must be an integer multiple of the voxel size");
  const T z_first = (-sdz / static_cast<T>(2 * nlz) * static_cast<T>(nlz - 1)) - g.origin.z;
  T offset_in_z = z_first + static_cast<T>(g.max_z + g.min_z) / T(2.F) * g.vox.z;
  if (tantheta == 0) {
    if (std::fabs(modulo((t_in_mm + offset_in_z) / g.vox.z, T(1.F)) - .5) < .001) offset_in_z -= T(.1F) * g.vox.z;
  }
  const T fovrad = std::min(static_cast<T>(std::min(g.max_x, -g.min_x)) * g.vox.x,
                            static_cast<T>(std::min(g.max_y, -g.min_y)) * g.vox.y);
  const bool rc = g.d.restrict_to_cylindrical_FOV != 0;
  const int ntl = g.d.num_tangential_LORs;
  if (ntl == 1) {
    ray_trace_one_lor(lor, s_in_mm, t_in_mm, cphi, sphi, costheta, tantheta, offset_in_z, fovrad, g.vox, rc, nlz);
  } else {
    Row<T> ray;
    const T s_inc = static_cast<T>(1) * g.get_sampling_in_s(bin.tang) / static_cast<T>(ntl);
    T cur_s = s_in_mm - s_inc * static_cast<T>(ntl - 1) / T(2.F);
    for (int k = 1; k <= ntl; ++k, cur_s += s_inc) {
      ray.clear();
      ray_trace_one_lor(ray, cur_s, t_in_mm, cphi, sphi, costheta, tantheta, offset_in_z, fovrad, g.vox, rc, nlz * ntl);
      row_merge(lor, ray);
    }
  }
  if (!lor.empty()) {
    if (tantheta == 0) {
      const T zfv = static_cast<T>(lor.front().z) + g.origin.z / g.vox.z - static_cast<T>(g.max_z + g.min_z) / T(2.F);
      const T left = (t_in_mm - sdz / T(2)) / g.vox.z;
      const T right = (t_in_mm + sdz / T(2)) / g.vox.z;
      add_adjacent_z(lor, zfv - left, right - left);
    } else if (nlz > 1) {
      Row<T> next = lor;
      for (int zi = 1; zi < nlz; ++zi) {
        for (auto& e : next) e.z += 1;
        row_merge(lor, next);
      }
    }
  }
}

/* FastErf (numerics/FastErf.inl:21-66) as set up by ProjMatrixByBin::set_up (ProjMatrixByBin.cxx:174-176):
   200000 samples of erf on [-5,5] (plus two end samples), linear interpolation in double */
struct FastErf {
  std::vector<double> v;
  double max_v = 5, period = 0;
  FastErf() {
    const int n = 200000;
    period = (2 * max_v) / n;
    v.resize(n + 2);
    for (int i = 0; i < n + 2; ++i) v[i] = std::erf(i * period - max_v);
  }
  double operator()(double xp) const {
    xp = std::max(std::min(max_v, xp), -max_v);
    const double xi = (xp + max_v) / period;
    const int lower = static_cast<int>(std::floor(xi));
    return v[lower] + (xi - lower) * (v[lower + 1] - v[lower]);
  }
};
const FastErf& fast_erf() {
  static const FastErf f;
  return f;
}

/* ProjMatrixByBin::get_tof_value (ProjMatrixByBin.inl:187-197).  With a truncation (tof_trunc_n > 0, no STIR
 * counterpart) the Gaussian is cut at +-k sigma: the bin's ends are clamped to [-k/sqrt2, k/sqrt2] in the kernel's
 * units, so a bin wholly outside gets 0 and a straddling bin the kernel's integral over its inner part. */
template <typename T> T tof_value(const Geometry<T>& g, T d1, T d2) {
  T d1n = d1 * g.r_sqrt2_gauss_sigma, d2n = d2 * g.r_sqrt2_gauss_sigma;
  if (g.tof_trunc_n > T(0)) {
    d1n = std::min(std::max(d1n, -g.tof_trunc_n), g.tof_trunc_n);
    d2n = std::min(std::max(d2n, -g.tof_trunc_n), g.tof_trunc_n);
  } else if ((d1n >= T(4.f) && d2n >= T(4.f)) || (d1n <= T(-4.f) && d2n <= T(-4.f))) {
    return T(0);
  }
  return static_cast<T>(0.5 * (fast_erf()(static_cast<double>(d2n)) - fast_erf()(static_cast<double>(d1n))));
}

/* ---------------------------------------------------------------------------
 * The handle: geometry + basic-row cache (ProjMatrixByBin cache of basic bins)
 * ------------------------------------------------------------------------- */
struct HandleBase {
  virtual ~HandleBase() {}
  int precision = 32;
};

template <typename T> struct Handle : HandleBase {
  Geometry<T> g;
  int basic_tang_max = 0;
  std::vector<Row<T>> cache;
  std::unique_ptr<std::once_flag[]> once;
  size_t cache_n = 0;

  void init_cache() {
    basic_tang_max = std::max(g.max_tang, -g.min_tang);
    cache_n = static_cast<size_t>(g.num_views) * (2 * g.S + 1) * (basic_tang_max - g.min_tang + 1) * g.num_tof;
    cache.assign(cache_n, Row<T>());
    once.reset(new std::once_flag[cache_n]);
  }
  size_t key(const Bin<T>& b) const {
    return ((static_cast<size_t>(b.view) * (2 * g.S + 1) + (b.seg + g.S)) * (basic_tang_max - g.min_tang + 1) +
            (b.tang - g.min_tang)) * g.num_tof + (b.tof - g.min_tof);
  }
  /* basic row, computed once (ProjMatrixByBin.inl:54-78) */
  const Row<T>& basic_row(const Bin<T>& b) {
    const size_t k = key(b);
    std::call_once(once[k], [&]() {
      Row<T> r;
      if (g.num_tof > 1) {
        Bin<T> nt = b;
        nt.tof = 0;
        calculate_row(g, nt, r);
        apply_tof_kernel(b, r);
      } else {
        calculate_row(g, b, r);
      }
      cache[k].swap(r);
    });
    return cache[k];
  }
  /* ProjMatrixByBin::apply_tof_kernel (ProjMatrixByBin.inl:115-185) with the LOR end points of
     ProjDataInfoCylindrical::get_LOR (ProjDataInfoCylindrical.cxx:515-548) converted by
     LORInAxialAndNoArcCorrSinogramCoordinates / LORInCylinderCoordinates / LORAs2Points (LORCoordinates.inl:106-140,288-299) */
  void apply_tof_kernel(const Bin<T>& b, Row<T>& r) {
    const T R = g.ring_radius;
    const T s = g.get_s(b.tang);
    const T m = g.get_m(b.seg, b.ax);
    const T tantheta = g.get_tantheta(b.seg, b.tang);
    T phi = g.get_phi(b.view);
    const T max_a = std::sqrt(square(R) - square(s));
    const T min_a = -max_a;
    T z1 = m - max_a * tantheta, z2 = m - min_a * tantheta;
    T beta = std::asin(s / R);
    const T two_pi = static_cast<T>(2 * kPI);
    phi = modulo(phi, two_pi);
    bool swapped = false;
    if (phi >= kPI) {
      phi -= static_cast<T>(kPI);
      beta = -beta;
      std::swap(z1, z2);
      swapped = true;
    }
    T psi1 = modulo(phi + beta, two_pi);
    T psi2 = modulo(phi - beta + static_cast<T>(kPI), two_pi);
    T pz1 = z1, pz2 = z2;
    if (swapped) {
      std::swap(psi1, psi2);
      std::swap(pz1, pz2);
    }
    const C3<T> p1{pz1, -R * std::cos(psi1), R * std::sin(psi1)};
    const C3<T> p2{pz2, -R * std::cos(psi2), R * std::sin(psi2)};
    const T scanner_z_offset = static_cast<T>(g.d.num_rings - 1) / T(2.0f) * g.ring_spacing;
    const C3<T> mid{(p1.z + p2.z) * T(0.5f), (p1.y + p2.y) * T(0.5f), (p1.x + p2.x) * T(0.5f)};
    const C3<T> diff{p2.z - mid.z, p2.y - mid.y, p2.x - mid.x};
    const T n = static_cast<T>(norm3(diff.z, diff.y, diff.x));
    const C3<T> u{diff.z / n, diff.y / n, diff.x / n};
    const int ti = b.tof - g.min_tof;
    Row<T> out;
    for (const auto& e : r) {
      /* get_physical_coordinates_for_indices: spacing*index + origin, then minus the scanner offset in z */
      const T pz = (static_cast<T>(e.z) * g.vox.z + g.origin.z) - scanner_z_offset;
      const T py = (static_cast<T>(e.y) * g.vox.y + g.origin.y) - T(0.0f);
      const T px = (static_cast<T>(e.x) * g.vox.x + g.origin.x) - T(0.0f);
      T ip = T(0);
      ip = ip + (pz - mid.z) * u.z;
      ip = ip + (py - mid.y) * u.y;
      ip = ip + (px - mid.x) * u.x;
      const T d2 = -ip;
      const T kv = tof_value(g, g.tof_low[ti] - d2, g.tof_high[ti] - d2);
      if (kv > 0 && e.v != 0) out.push_back(Elem<T>{e.z, e.y, e.x, e.v * kv});
    }
    r.swap(out);
  }

  /* forward projection of one bin: ProjMatrixElemsForOneBin::forward_project (ProjMatrixElemsForOneBin.cxx:354-370),
     only z range-checked */
  T fwd_bin(const Bin<T>& bin, const T* img) {
    Bin<T> b = bin;
    const SymOp op = find_op_and_basic(g, b);
    const Row<T>& row = basic_row(b);
    T sum = 0;
    for (const auto& e : row) {
      int z, y, x;
      transform(op, e, z, y, x);
      if (z < g.min_z || z > g.max_z) continue;
      sum += img[img_index(z, y, x)] * e.v;
    }
    return sum;
  }
  /* ProjMatrixElemsForOneBin::back_project (ProjMatrixElemsForOneBin.cxx:333-351) */
  void back_bin(const Bin<T>& bin, T data, T* img) {
    if (data == 0) return;
    Bin<T> b = bin;
    const SymOp op = find_op_and_basic(g, b);
    const Row<T>& row = basic_row(b);
    for (const auto& e : row) {
      int z, y, x;
      transform(op, e, z, y, x);
      if (z < g.min_z || z > g.max_z) continue;
      img[img_index(z, y, x)] += e.v * data;
    }
  }
  static inline void transform(const SymOp& op, const Elem<T>& e, int& z, int& y, int& x) {
    x = (op.swap ? e.y : e.x) * op.sx;
    y = (op.swap ? e.x : e.y) * op.sy;
    z = (op.zq ? op.q - e.z : e.z) + op.z_shift;
  }
  inline int64_t img_index(int z, int y, int x) const {
    if (y < g.min_y || y > g.max_y || x < g.min_x || x > g.max_x)
      throw std::runtime_error("row element outside the image in x/y");
    return (static_cast<int64_t>(z - g.min_z) * g.ny + (y - g.min_y)) * g.nx + (x - g.min_x);
  }

  /* ForwardProjectorByBin::forward_project(ProjData&, subset) (ForwardProjectorByBin.cxx:168-230) with the
     cached-matrix loop of ForwardProjectorByBinUsingProjMatrixByBin::actual_forward_project (:101-137) */
  void forward(const T* img, T* pd, int subset, int nsub, int nthreads) {
    const auto vs = basic_vs_in_subset(g, subset, nsub);
    const int n = static_cast<int>(vs.size());
    std::string err;
#pragma omp parallel for schedule(dynamic) collapse(2) num_threads(nthreads)
    for (int i = 0; i < n; ++i)
      for (int k = g.min_tof; k <= g.max_tof; ++k) {
        try {
          std::vector<std::pair<int, int>> rel;
          related_vs(g, vs[i].first, vs[i].second, rel);
          for (const auto& r : rel)
            for (int t = g.min_tang; t <= g.max_tang; ++t)
              for (int a = 0; a < g.nax(r.second); ++a) {
                Bin<T> b{r.second, r.first, a, t, k};
                pd[g.stir_index(r.second, r.first, a, t, k)] = fwd_bin(b, img);
              }
        } catch (const std::exception& e) {
#pragma omp critical(ORACLE_ERR)
          err = e.what();
        }
      }
    if (!err.empty()) throw std::runtime_error(err);
  }
  /* BackProjectorByBin::back_project(ProjData&, subset) (BackProjectorByBin.cxx:182-229), per-thread images
     reduced as in get_output (:316-346) */
  void back(const T* pd, T* img, int subset, int nsub, int nthreads) {
    const auto vs = basic_vs_in_subset(g, subset, nsub);
    const int n = static_cast<int>(vs.size());
    const int64_t ni = static_cast<int64_t>(g.nz) * g.ny * g.nx;
#ifdef _OPENMP
    const int nt = std::max(1, nthreads);
#else
    const int nt = 1;
#endif
    std::vector<std::vector<T>> local(nt);
    std::string err;
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
      const int tid = omp_get_thread_num();
#else
      const int tid = 0;
#endif
      local[tid].assign(ni, T(0));
      T* mine = local[tid].data();
#pragma omp for schedule(dynamic) collapse(2)
      for (int i = 0; i < n; ++i)
        for (int k = g.min_tof; k <= g.max_tof; ++k) {
          try {
            std::vector<std::pair<int, int>> rel;
            related_vs(g, vs[i].first, vs[i].second, rel);
            for (const auto& r : rel)
              for (int t = g.min_tang; t <= g.max_tang; ++t)
                for (int a = 0; a < g.nax(r.second); ++a) {
                  Bin<T> b{r.second, r.first, a, t, k};
                  back_bin(b, pd[g.stir_index(r.second, r.first, a, t, k)], mine);
                }
          } catch (const std::exception& e) {
#pragma omp critical(ORACLE_ERR)
            err = e.what();
          }
        }
    }
    if (!err.empty()) throw std::runtime_error(err);
    std::fill(img, img + ni, T(0));
    for (int t = 0; t < nt; ++t)
      if (!local[t].empty())
        for (int64_t j = 0; j < ni; ++j) img[j] += local[t][j];
  }
};

/* ---------------------------------------------------------------------------
 * Elementwise pieces of the objective and OSMAPOSL
 * ------------------------------------------------------------------------- */
const float SMALL_NUM = 0.000001F; /* recon_array_functions.cxx:44 */

/* divide_and_truncate (recon_array_functions.cxx:171-266) for one viewgram [ax][tang] of a (seg,view) */
template <typename T, typename Fn> void for_viewgram(const Geometry<T>& g, int seg, int view, int tof, Fn fn) {
  for (int a = 0; a < g.nax(seg); ++a)
    for (int t = g.min_tang; t <= g.max_tang; ++t) fn(a, t, g.stir_index(seg, view, a, t, tof));
}

/* QuadraticPrior / RelativeDifferencePrior weights (QuadraticPrior.cxx:203-230, RelativeDifferencePrior.cxx:251-276) */
void prior_weights(float w[3][3][3], float vz, float vy, float vx, bool only_2D) {
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        if ((only_2D && z != 0) || (z == 0 && y == 0 && x == 0))
          w[z + 1][y + 1][x + 1] = 0;
        else
          w[z + 1][y + 1][x + 1] =
              vx / std::sqrt(square(static_cast<float>(x) * vx) + square(static_cast<float>(y) * vy) +
                             square(static_cast<float>(z) * vz));
      }
}

/* RelativeDifferencePrior::derivative_10 (RelativeDifferencePrior.cxx:287-300) */
inline float rdp_derivative_10(float x, float y, float gamma, float epsilon) {
  if (epsilon == 0.0 && x == 0 && y == 0) return 0.f;
  const double num = (static_cast<double>(x - y) * (gamma * std::abs(x - y) + x + 3 * y + 2 * epsilon));
  const double denom_sqrt = static_cast<double>(x + y) + gamma * std::abs(x - y) + epsilon;
  return static_cast<float>(num / (denom_sqrt * denom_sqrt));
}
/* RelativeDifferencePrior::value (RelativeDifferencePrior.cxx:278-285) */
inline double rdp_value(float x, float y, float gamma, float epsilon) {
  return 0.5 * (square(static_cast<double>(x - y)) / (x + y + gamma * std::abs(x - y) + epsilon));
}

void prior_gradient(const b200rt_prior& p, const float* img, const float* kappa, int nz, int ny, int nx, float vz,
                    float vy, float vx, float* grad) {
  const int64_t ni = static_cast<int64_t>(nz) * ny * nx;
  if (p.type == B200RT_PRIOR_NONE || p.penalisation_factor == 0) {
    std::fill(grad, grad + ni, 0.f);
    return;
  }
  float w[3][3][3];
  prior_weights(w, vz, vy, vx, p.only_2D != 0);
  const int dzmin = p.only_2D ? 0 : -1, dzmax = p.only_2D ? 0 : 1;
  auto at = [&](int z, int y, int x) { return (static_cast<int64_t>(z) * ny + y) * nx + x; };
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const int min_dz = std::max(dzmin, -z), max_dz = std::min(dzmax, nz - 1 - z);
        const int min_dy = std::max(-1, -y), max_dy = std::min(1, ny - 1 - y);
        const int min_dx = std::max(-1, -x), max_dx = std::min(1, nx - 1 - x);
        const float xc = img[at(z, y, x)];
        double gsum = 0.;
        for (int dz = min_dz; dz <= max_dz; ++dz)
          for (int dy = min_dy; dy <= max_dy; ++dy)
            for (int dx = min_dx; dx <= max_dx; ++dx) {
              const float xn = img[at(z + dz, y + dy, x + dx)];
              const float wt = w[dz + 1][dy + 1][dx + 1];
              double cur;
              if (p.type == B200RT_PRIOR_QUADRATIC)
                cur = wt * (xc - xn); /* QuadraticPrior.cxx:355-362 */
              else
                cur = wt * rdp_derivative_10(xc, xn, p.gamma, p.epsilon); /* RelativeDifferencePrior.cxx:432-440 */
              if (kappa) cur *= kappa[at(z, y, x)] * kappa[at(z + dz, y + dy, x + dx)];
              gsum += cur;
            }
        grad[at(z, y, x)] = static_cast<float>(gsum * p.penalisation_factor);
      }
}

double prior_value(const b200rt_prior& p, const float* img, const float* kappa, int nz, int ny, int nx, float vz,
                   float vy, float vx) {
  if (p.type == B200RT_PRIOR_NONE || p.penalisation_factor == 0) return 0.;
  float w[3][3][3];
  prior_weights(w, vz, vy, vx, p.only_2D != 0);
  const int dzmin = p.only_2D ? 0 : -1, dzmax = p.only_2D ? 0 : 1;
  auto at = [&](int z, int y, int x) { return (static_cast<int64_t>(z) * ny + y) * nx + x; };
  double result = 0.;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const int min_dz = std::max(dzmin, -z), max_dz = std::min(dzmax, nz - 1 - z);
        const int min_dy = std::max(-1, -y), max_dy = std::min(1, ny - 1 - y);
        const int min_dx = std::max(-1, -x), max_dx = std::min(1, nx - 1 - x);
        const float xc = img[at(z, y, x)];
        for (int dz = min_dz; dz <= max_dz; ++dz)
          for (int dy = min_dy; dy <= max_dy; ++dy)
            for (int dx = min_dx; dx <= max_dx; ++dx) {
              const float xn = img[at(z + dz, y + dy, x + dx)];
              const float wt = w[dz + 1][dy + 1][dx + 1];
              double cur;
              if (p.type == B200RT_PRIOR_QUADRATIC) {
                cur = wt * square(xc - xn) / 4; /* QuadraticPrior.cxx:283-286 */
              } else {
                if (p.epsilon == 0.0 && xc == 0.0 && xn == 0.0)
                  cur = 0.0;
                else
                  cur = wt * rdp_value(xc, xn, p.gamma, p.epsilon); /* RelativeDifferencePrior.cxx:340-349 */
              }
              if (kappa) cur *= kappa[at(z, y, x)] * kappa[at(z + dz, y + dy, x + dx)];
              result += cur;
            }
      }
  return result * p.penalisation_factor;
}

}  // namespace

/* ---------------------------------------------------------------------------
 * C interface
 * ------------------------------------------------------------------------- */
struct or_handle {
  std::unique_ptr<Handle<float>> f;
  std::unique_ptr<Handle<double>> d;
};

extern "C" {

or_handle* or_create(const b200rt_geometry* g, int precision, char* err, int errlen) {
  try {
    std::unique_ptr<or_handle> h(new or_handle);
    if (precision == 64) {
      h->d.reset(new Handle<double>);
      setup_geometry(h->d->g, *g);
      h->d->init_cache();
    } else {
      h->f.reset(new Handle<float>);
      setup_geometry(h->f->g, *g);
      h->f->init_cache();
    }
    return h.release();
  } catch (const std::exception& e) {
    if (err && errlen > 0) {
      std::strncpy(err, e.what(), errlen - 1);
      err[errlen - 1] = 0;
    }
    return nullptr;
  }
}
void or_destroy(or_handle* h) { delete h; }

#define OR_GEO(h) ((h)->f ? static_cast<const void*>(&(h)->f->g) : static_cast<const void*>(&(h)->d->g))

int64_t or_projdata_size(const or_handle* h) { return h->f ? h->f->g.projdata_size : h->d->g.projdata_size; }
int64_t or_image_size(const or_handle* h) {
  return h->f ? static_cast<int64_t>(h->f->g.nz) * h->f->g.ny * h->f->g.nx
              : static_cast<int64_t>(h->d->g.nz) * h->d->g.ny * h->d->g.nx;
}
int or_num_tof_bins(const or_handle* h) { return h->f ? h->f->g.num_tof : h->d->g.num_tof; }
int or_symmetries_used(const or_handle* h) {
  auto bits = [](bool a, bool b, bool c, bool d, bool e) { return (a ? 1 : 0) | (b ? 2 : 0) | (c ? 4 : 0) | (d ? 8 : 0) | (e ? 16 : 0); };
  if (h->f) return bits(h->f->g.sym90, h->f->g.sym180, h->f->g.symseg, h->f->g.syms, h->f->g.symz);
  return bits(h->d->g.sym90, h->d->g.sym180, h->d->g.symseg, h->d->g.syms, h->d->g.symz);
}
int or_num_basic_views(const or_handle* h) {
  int n = 0;
  if (h->f) {
    for (int v = 0; v < h->f->g.num_views; ++v) {
      int vv = v, s = 0;
      if (!find_basic_vs(h->f->g, vv, s)) ++n;
    }
  } else {
    for (int v = 0; v < h->d->g.num_views; ++v) {
      int vv = v, s = 0;
      if (!find_basic_vs(h->d->g, vv, s)) ++n;
    }
  }
  return n;
}

extern "C++" template <typename T>
int64_t get_row_impl(Handle<T>& H, int seg, int view, int ax, int tang, int tof, int32_t* c, double* v, int64_t cap) {
  Bin<T> b{seg, view, ax, tang, tof};
  const SymOp op = find_op_and_basic(H.g, b);
  const Row<T>& row = H.basic_row(b);
  const int64_t n = static_cast<int64_t>(row.size());
  for (int64_t i = 0; i < n && i < cap; ++i) {
    int z, y, x;
    Handle<T>::transform(op, row[i], z, y, x);
    c[3 * i] = z;
    c[3 * i + 1] = y;
    c[3 * i + 2] = x;
    v[i] = static_cast<double>(row[i].v);
  }
  return n;
}

int64_t or_get_row(or_handle* h, int seg, int view, int ax, int tang, int tof, int32_t* coords, double* values, int64_t cap) {
  try {
    return h->f ? get_row_impl(*h->f, seg, view, ax, tang, tof, coords, values, cap)
                : get_row_impl(*h->d, seg, view, ax, tang, tof, coords, values, cap);
  } catch (...) {
    return -1;
  }
}

extern "C++" template <typename T> int64_t total_nnz_impl(Handle<T>& H, int nthreads) {
  const auto& g = H.g;
  int64_t total = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : total) num_threads(nthreads)
  for (int view = 0; view < g.num_views; ++view)
    for (int seg = -g.S; seg <= g.S; ++seg)
      for (int k = g.min_tof; k <= g.max_tof; ++k)
        for (int t = g.min_tang; t <= g.max_tang; ++t) {
          Bin<T> b{seg, view, 0, t, k};
          find_op_and_basic(g, b);
          total += static_cast<int64_t>(H.basic_row(b).size()) * g.nax(seg);
        }
  return total;
}
int64_t or_total_nnz(or_handle* h, int nthreads) { return h->f ? total_nnz_impl(*h->f, nthreads) : total_nnz_impl(*h->d, nthreads); }

extern "C++" template <typename T> int64_t basic_elems_impl(Handle<T>& H, int nthreads, int64_t* nrows) {
  total_nnz_impl(H, nthreads);
  int64_t n = 0, e = 0;
  for (size_t k = 0; k < H.cache_n; ++k) {
    if (!H.cache[k].empty()) {
      ++n;
      e += static_cast<int64_t>(H.cache[k].size());
    }
  }
  if (nrows) *nrows = n;
  return e;
}
int64_t or_basic_row_elements(or_handle* h, int nthreads, int64_t* nrows) {
  return h->f ? basic_elems_impl(*h->f, nthreads, nrows) : basic_elems_impl(*h->d, nthreads, nrows);
}

int or_forward_project_f32(or_handle* h, const float* img, float* pd, int subset, int nsub, int nthreads) {
  if (!h->f) return -1;
  try {
    h->f->forward(img, pd, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}
int or_back_project_f32(or_handle* h, const float* pd, float* img, int subset, int nsub, int nthreads) {
  if (!h->f) return -1;
  try {
    h->f->back(pd, img, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}
int or_forward_project_f64(or_handle* h, const double* img, double* pd, int subset, int nsub, int nthreads) {
  if (!h->d) return -1;
  try {
    h->d->forward(img, pd, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}
int or_back_project_f64(or_handle* h, const double* pd, double* img, int subset, int nsub, int nthreads) {
  if (!h->d) return -1;
  try {
    h->d->back(pd, img, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}

/* zero_end_sinograms of segment 0 (distributable.cxx:146-158) applied to a full projdata copy */
static void zero_seg0_ends(const Geometry<float>& g, float* pd) {
  for (int k = g.min_tof; k <= g.max_tof; ++k)
    for (int view = 0; view < g.num_views; ++view)
      for (int t = g.min_tang; t <= g.max_tang; ++t) {
        pd[g.stir_index(0, view, 0, t, k)] = 0;
        pd[g.stir_index(0, view, g.nax(0) - 1, t, k)] = 0;
      }
}

int or_sensitivity_f32(or_handle* h, const float* mult, float* sens, int subset, int nsub, int zero_ends, int nthreads) {
  if (!h->f) return -1;
  try {
    const auto& g = h->f->g;
    std::vector<float> m(g.projdata_size, 1.f);
    if (mult) std::copy(mult, mult + g.projdata_size, m.begin());
    if (zero_ends) zero_seg0_ends(g, m.data());
    h->f->back(m.data(), sens, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}

/* gradient-plus-sensitivity of one subset: back-projection of divide_and_truncate(y, A x + a)
   (RPC_process_related_viewgrams_gradient<true>, ...AndProjData.cxx:1421-1481) */
static void subset_ratio(Handle<float>& H, const float* x, const float* y, const float* add, int subset, int nsub,
                         int zero_ends, int nthreads, std::vector<float>& ratio, int* cancelled) {
  auto& g = H.g;
  std::vector<float> est(g.projdata_size, 0.f);
  H.forward(x, est.data(), subset, nsub, nthreads);
  ratio.assign(g.projdata_size, 0.f);
  const auto vs = basic_vs_in_subset(g, subset, nsub);
  int count = 0;
  for (const auto& b : vs)
    for (int k = g.min_tof; k <= g.max_tof; ++k) {
      std::vector<std::pair<int, int>> rel;
      related_vs(g, b.first, b.second, rel);
      for (const auto& r : rel) {
        const int seg = r.second, view = r.first;
        const bool zero_this = zero_ends && seg == 0;
        /* measured viewgram (zeroed end planes) and its max (:185) */
        float vmax = -std::numeric_limits<float>::infinity();
        for_viewgram(g, seg, view, k, [&](int a, int, int64_t i) {
          float yv = y[i];
          if (zero_this && (a == 0 || a == g.nax(0) - 1)) yv = 0;
          vmax = std::max(vmax, yv);
        });
        const float small_value = std::max(vmax * SMALL_NUM, 0.F);
        for_viewgram(g, seg, view, k, [&](int a, int, int64_t i) {
          float num = y[i];
          float av = add ? add[i] : 0.f;
          if (zero_this && (a == 0 || a == g.nax(0) - 1)) {
            num = 0;
            av = 0;
          }
          const float denom = est[i] + av;
          if (num <= small_value) {
            num = 0;
          } else {
            const float max_quotient = 10000.F;
            if (num > max_quotient * denom) {
              ++count;
              num = max_quotient;
            } else {
              num = num / denom;
            }
          }
          ratio[i] = num;
        });
      }
    }
  if (cancelled) *cancelled = count;
}

/* u = A_S^T divide_and_truncate(y, A_S x + a): compute_sub_gradient_without_penalty_plus_sensitivity */
int or_osmaposl_numerator_f32(or_handle* h, const float* x, const float* y, const float* add, int subset, int nsub,
                              int zero_ends, int nthreads, float* u, int* num_cancelled) {
  if (!h->f) return -1;
  try {
    std::vector<float> ratio;
    subset_ratio(*h->f, x, y, add, subset, nsub, zero_ends, nthreads, ratio, num_cancelled);
    h->f->back(ratio.data(), u, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}

/* the rest of OSMAPOSLReconstruction::update_estimate (OSMAPOSLReconstruction.cxx:394-510) given u */
int or_osmaposl_apply_f32(or_handle* h, float* x, float* u, const float* sens, int nsub, int subiter,
                          const b200rt_prior* prior, const float* kappa, float min_rel, float max_rel) {
  if (!h->f) return -1;
  auto& g = h->f->g;
  const int64_t ni = static_cast<int64_t>(g.nz) * g.ny * g.nx;
  const bool no_prior = !prior || prior->type == B200RT_PRIOR_NONE || prior->penalisation_factor == 0;
  std::vector<float> den(ni);
  float small_num;
  if (no_prior) {
    std::copy(sens, sens + ni, den.begin());
    small_num = 0.F;
  } else {
    prior_gradient(*prior, x, kappa, g.nz, g.ny, g.nx, g.d.voxel_size_z, g.d.voxel_size_y, g.d.voxel_size_x, den.data());
    if (prior->map_model == B200RT_MAP_ADDITIVE) {
      for (int64_t i = 0; i < ni; ++i) {
        float dv = den[i] / static_cast<float>(nsub) + sens[i];
        den[i] = std::max(std::min(dv, sens[i] * 10), sens[i] / 10);
      }
    } else {
      for (int64_t i = 0; i < ni; ++i) {
        float dv = den[i] + 1;
        dv = std::max(std::min(dv, 10.F), 1 / 10.F);
        den[i] = dv * sens[i];
      }
    }
    small_num = 0.000001F;
  }
  /* divide (numerics/divide.inl:26-48) */
  {
    float small_value = *std::max_element(u, u + ni) * small_num;
    small_value = (small_value > 0) ? small_value : 0;
    for (int64_t i = 0; i < ni; ++i) {
      if (std::fabs(den[i]) <= small_value && std::fabs(u[i]) <= small_value)
        u[i] = 0;
      else
        u[i] /= den[i];
    }
  }
  /* threshold_upper_lower (:491-507, thresholding.h:45-54) */
  if (subiter != 1)
    for (int64_t i = 0; i < ni; ++i) {
      if (u[i] > max_rel)
        u[i] = max_rel;
      else if (min_rel > u[i])
        u[i] = min_rel;
    }
  /* apply_multiplicative_update (:354-369) */
  for (int64_t i = 0; i < ni; ++i) x[i] *= u[i];
  return 0;
}

int or_osmaposl_update_f32(or_handle* h, float* x, const float* y, const float* add, const float* sens, int subset,
                           int nsub, int subiter, int zero_ends, const b200rt_prior* prior, const float* kappa,
                           float min_rel, float max_rel, int nthreads, int* num_cancelled) {
  if (!h->f) return -1;
  const int64_t ni = static_cast<int64_t>(h->f->g.nz) * h->f->g.ny * h->f->g.nx;
  std::vector<float> u(ni, 0.f);
  if (or_osmaposl_numerator_f32(h, x, y, add, subset, nsub, zero_ends, nthreads, u.data(), num_cancelled) != 0) return -1;
  return or_osmaposl_apply_f32(h, x, u.data(), sens, nsub, subiter, prior, kappa, min_rel, max_rel);
}

/* ---------------------------------------------------------------------------
 * FP64 OSMAPOSL: the same algorithm as the float path above, every quantity in double (the data y, a and m are
 * float inputs, converted once).  It is the "error against an FP64 oracle" reference; the float path is the
 * parity reference.
 * ------------------------------------------------------------------------- */
static void zero_seg0_ends_f64(const Geometry<double>& g, double* pd) {
  for (int k = g.min_tof; k <= g.max_tof; ++k)
    for (int view = 0; view < g.num_views; ++view)
      for (int t = g.min_tang; t <= g.max_tang; ++t) {
        pd[g.stir_index(0, view, 0, t, k)] = 0;
        pd[g.stir_index(0, view, g.nax(0) - 1, t, k)] = 0;
      }
}

int or_sensitivity_f64(or_handle* h, const float* mult, double* sens, int subset, int nsub, int zero_ends,
                       int nthreads) {
  if (!h->d) return -1;
  try {
    const auto& g = h->d->g;
    std::vector<double> m(g.projdata_size, 1.0);
    if (mult) std::copy(mult, mult + g.projdata_size, m.begin());
    if (zero_ends) zero_seg0_ends_f64(g, m.data());
    h->d->back(m.data(), sens, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}

/* RelativeDifferencePrior::derivative_10 (RelativeDifferencePrior.cxx:287-300) in double */
static double rdp_derivative_10_f64(double x, double y, double gamma, double epsilon) {
  if (epsilon == 0.0 && x == 0 && y == 0) return 0.;
  const double d = x + y + gamma * std::abs(x - y) + epsilon;
  return (x - y) * (gamma * std::abs(x - y) + x + 3 * y + 2 * epsilon) / (d * d);
}

/* QuadraticPrior / RelativeDifferencePrior compute_gradient (QuadraticPrior.cxx:303-372,
   RelativeDifferencePrior.cxx:376-452) in double */
static void prior_gradient_f64(const b200rt_prior& p, const double* img, int nz, int ny, int nx, double vz, double vy,
                               double vx, double* grad) {
  const int64_t ni = static_cast<int64_t>(nz) * ny * nx;
  if (p.type == B200RT_PRIOR_NONE || p.penalisation_factor == 0) {
    std::fill(grad, grad + ni, 0.);
    return;
  }
  double w[3][3][3];
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x)
        w[z + 1][y + 1][x + 1] = ((p.only_2D && z != 0) || (z == 0 && y == 0 && x == 0))
                                     ? 0.
                                     : vx / std::sqrt(square(x * vx) + square(y * vy) + square(z * vz));
  const int dzmin = p.only_2D ? 0 : -1, dzmax = p.only_2D ? 0 : 1;
  auto at = [&](int z, int y, int x) { return (static_cast<int64_t>(z) * ny + y) * nx + x; };
#pragma omp parallel for schedule(static)
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const double xc = img[at(z, y, x)];
        double gsum = 0.;
        for (int dz = std::max(dzmin, -z); dz <= std::min(dzmax, nz - 1 - z); ++dz)
          for (int dy = std::max(-1, -y); dy <= std::min(1, ny - 1 - y); ++dy)
            for (int dx = std::max(-1, -x); dx <= std::min(1, nx - 1 - x); ++dx) {
              const double xn = img[at(z + dz, y + dy, x + dx)];
              const double wt = w[dz + 1][dy + 1][dx + 1];
              gsum += p.type == B200RT_PRIOR_QUADRATIC ? wt * (xc - xn)
                                                       : wt * rdp_derivative_10_f64(xc, xn, p.gamma, p.epsilon);
            }
        grad[at(z, y, x)] = gsum * p.penalisation_factor;
      }
}

/* one OSMAPOSL sub-iteration (or_osmaposl_update_f32's steps) in double; no kappa */
int or_osmaposl_update_f64(or_handle* h, double* x, const float* y, const float* add, const double* sens, int subset,
                           int nsub, int subiter, int zero_ends, const b200rt_prior* prior, double min_rel,
                           double max_rel, int nthreads) {
  if (!h->d) return -1;
  try {
    auto& H = *h->d;
    auto& g = H.g;
    const int64_t ni = static_cast<int64_t>(g.nz) * g.ny * g.nx;
    std::vector<double> est(g.projdata_size, 0.), ratio(g.projdata_size, 0.), u(ni, 0.);
    H.forward(x, est.data(), subset, nsub, nthreads);
    for (const auto& b : basic_vs_in_subset(g, subset, nsub))
      for (int k = g.min_tof; k <= g.max_tof; ++k) {
        std::vector<std::pair<int, int>> rel;
        related_vs(g, b.first, b.second, rel);
        for (const auto& r : rel) {
          const int seg = r.second, view = r.first;
          const bool zero_this = zero_ends && seg == 0;
          auto end = [&](int a) { return zero_this && (a == 0 || a == g.nax(0) - 1); };
          double vmax = -std::numeric_limits<double>::infinity();
          for_viewgram(g, seg, view, k, [&](int a, int, int64_t i) { vmax = std::max(vmax, end(a) ? 0. : double(y[i])); });
          const double small_value = std::max(vmax * 0.000001, 0.);
          for_viewgram(g, seg, view, k, [&](int a, int, int64_t i) {
            const double num = end(a) ? 0. : double(y[i]);
            const double denom = est[i] + (add && !end(a) ? double(add[i]) : 0.);
            ratio[i] = num <= small_value ? 0. : (num > 10000. * denom ? 10000. : num / denom);
          });
        }
      }
    H.back(ratio.data(), u.data(), subset, nsub, nthreads);
    const bool no_prior = !prior || prior->type == B200RT_PRIOR_NONE || prior->penalisation_factor == 0;
    std::vector<double> den(sens, sens + ni);
    double small_num = 0.;
    if (!no_prior) {
      prior_gradient_f64(*prior, x, g.nz, g.ny, g.nx, g.d.voxel_size_z, g.d.voxel_size_y, g.d.voxel_size_x, den.data());
      for (int64_t i = 0; i < ni; ++i) {
        if (prior->map_model == B200RT_MAP_ADDITIVE)
          den[i] = std::max(std::min(den[i] / nsub + sens[i], sens[i] * 10), sens[i] / 10);
        else
          den[i] = std::max(std::min(den[i] + 1, 10.), 0.1) * sens[i];
      }
      small_num = 0.000001;
    }
    const double small_value = std::max(*std::max_element(u.begin(), u.end()) * small_num, 0.);
    for (int64_t i = 0; i < ni; ++i) {
      double v = (std::fabs(den[i]) <= small_value && std::fabs(u[i]) <= small_value) ? 0. : u[i] / den[i];
      if (subiter != 1) v = v > max_rel ? max_rel : (min_rel > v ? min_rel : v);
      x[i] *= v;
    }
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}

/* sub-gradient of the log-likelihood without penalty: A^T [divide_and_truncate(y, A x + a) - m]
   (RPC_process_related_viewgrams_gradient<false>, ...AndProjData.cxx:1421-1481) */
int or_loglik_gradient_f32(or_handle* h, const float* x, const float* y, const float* add, const float* mult, int subset,
                           int nsub, int zero_ends, int nthreads, float* grad) {
  if (!h->f) return -1;
  try {
    auto& H = *h->f;
    auto& g = H.g;
    std::vector<float> ratio;
    subset_ratio(H, x, y, add, subset, nsub, zero_ends, nthreads, ratio, nullptr);
    const auto vs = basic_vs_in_subset(g, subset, nsub);
    for (const auto& b : vs)
      for (int k = g.min_tof; k <= g.max_tof; ++k) {
        std::vector<std::pair<int, int>> rel;
        related_vs(g, b.first, b.second, rel);
        for (const auto& r : rel) {
          const int seg = r.second, view = r.first;
          for_viewgram(g, seg, view, k, [&](int a, int, int64_t i) {
            const bool z_here = zero_ends && seg == 0 && (a == 0 || a == g.nax(0) - 1);
            ratio[i] -= z_here ? 0.f : (mult ? mult[i] : 1.f);
          });
        }
      }
    H.back(ratio.data(), grad, subset, nsub, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}

double or_log_likelihood_f32(or_handle* h, const float* x, const float* y, const float* add, const float* mult,
                             int subset, int nsub, int zero_ends, int nthreads) {
  if (!h->f) return std::nan("");
  auto& H = *h->f;
  auto& g = H.g;
  std::vector<float> est(g.projdata_size, 0.f);
  H.forward(x, est.data(), subset, nsub, nthreads);
  const auto vs = basic_vs_in_subset(g, subset, nsub);
  double accum = 0;
  for (const auto& b : vs)
    for (int k = g.min_tof; k <= g.max_tof; ++k) {
      std::vector<std::pair<int, int>> rel;
      related_vs(g, b.first, b.second, rel);
      for (const auto& r : rel) {
        const int seg = r.second, view = r.first;
        const bool zero_this = zero_ends && seg == 0;
        auto yv = [&](int a, int64_t i) { return (zero_this && (a == 0 || a == g.nax(0) - 1)) ? 0.f : y[i]; };
        float vmax = -std::numeric_limits<float>::infinity();
        for_viewgram(g, seg, view, k, [&](int a, int, int64_t i) { vmax = std::max(vmax, yv(a, i)); });
        const float small_value = std::max(vmax * SMALL_NUM, 0.F);
        const float max_quotient = 10000.F;
        double result = 0;
        for (int a = 0; a < g.nax(seg); ++a) {
          double sub = 0;
          for (int t = g.min_tang; t <= g.max_tang; ++t) {
            const int64_t i = g.stir_index(seg, view, a, t, k);
            const bool z_here = zero_this && (a == 0 || a == g.nax(0) - 1);
            /* ybar = (A x + a) * m, with a and m zeroed on the end planes (:1498-1509) */
            float e = est[i] + (add && !z_here ? add[i] : 0.f);
            if (z_here)
              e *= 0.f;
            else if (mult)
              e *= mult[i];
            const float yy = yv(a, i);
            const float ne = std::max(e, yy / max_quotient);
            if (yy <= small_value)
              sub += -double(ne);
            else
              sub += yy * std::log(double(ne)) - double(ne);
          }
          result += sub;
        }
        accum += result;
      }
    }
  return accum;
}

/* RelativeDifferencePrior::derivative_20 / derivative_11 (RelativeDifferencePrior.cxx:623-641): pow of a float
   by an int is evaluated in double, the quotient returned as float */
inline float rdp_derivative_20(float xj, float xk, float gamma, float epsilon) {
  if (xj > 0.0 || xk > 0.0 || epsilon > 0.0)
    return static_cast<float>(2 * std::pow(2 * xk + epsilon, 2) / std::pow(xj + xk + gamma * std::abs(xj - xk) + epsilon, 3));
  return std::numeric_limits<float>::infinity();
}
inline float rdp_derivative_11(float xj, float xk, float gamma, float epsilon) {
  if (xj > 0.0 || xk > 0.0 || epsilon > 0.0)
    return static_cast<float>(-2 * (2 * xj + epsilon) * (2 * xk + epsilon) /
                              std::pow(xj + xk + gamma * std::abs(xj - xk) + epsilon, 3));
  return std::numeric_limits<float>::infinity();
}

/* accumulate_Hessian_times_input (QuadraticPrior.cxx:603-688, RelativeDifferencePrior.cxx:535-621):
   out += beta * sum_k w_k (f20(x_j, x_k) in_j + f11(x_j, x_k) in_k) (kappa_j kappa_k) */
int or_prior_hessian_times_input_f32(const b200rt_prior* p, const float* x, const float* in, const float* kappa, int nz,
                                     int ny, int nx, float vz, float vy, float vx, float* out) {
  if (!p || p->type == B200RT_PRIOR_NONE || p->penalisation_factor == 0) return 0;
  float w[3][3][3];
  prior_weights(w, vz, vy, vx, p->only_2D != 0);
  const int dzmin = p->only_2D ? 0 : -1, dzmax = p->only_2D ? 0 : 1;
  auto at = [&](int z, int y, int xx) { return (static_cast<int64_t>(z) * ny + y) * nx + xx; };
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int xx = 0; xx < nx; ++xx) {
        const int min_dz = std::max(dzmin, -z), max_dz = std::min(dzmax, nz - 1 - z);
        const int min_dy = std::max(-1, -y), max_dy = std::min(1, ny - 1 - y);
        const int min_dx = std::max(-1, -xx), max_dx = std::min(1, nx - 1 - xx);
        const int64_t j = at(z, y, xx);
        float result = 0;
        for (int dz = min_dz; dz <= max_dz; ++dz)
          for (int dy = min_dy; dy <= max_dy; ++dy)
            for (int dx = min_dx; dx <= max_dx; ++dx) {
              float current = w[dz + 1][dy + 1][dx + 1];
              if (current == 0.f) continue;
              const int64_t k = at(z + dz, y + dy, xx + dx);
              float f20, f11;
              if (p->type == B200RT_PRIOR_QUADRATIC) {
                f20 = 1.0;
                f11 = -1.0;
              } else {
                f20 = rdp_derivative_20(x[j], x[k], p->gamma, p->epsilon);
                f11 = rdp_derivative_11(x[j], x[k], p->gamma, p->epsilon);
              }
              if (dz == 0 && dy == 0 && dx == 0)
                current *= f20 * in[j];
              else
                current *= (f20 * in[j] + f11 * in[k]);
              if (kappa) current *= kappa[j] * kappa[k];
              result += current;
            }
        out[j] += result * p->penalisation_factor;
      }
  return 0;
}

/* OSSPS precomputed denominator (OSSPSReconstruction.cxx:184-221): minus the approximate Hessian of the
   log-likelihood times an image of ones, i.e. A^T divide_and_truncate(A 1, (y n) n) over all bins, where n is
   the normalisation's correction (BinNormalisation::apply multiplies by it; NULL: no normalisation)
   (...AndProjData.cxx:955-1064; the small value of divide_and_truncate is taken on A 1) */
int or_ossps_denominator_f32(or_handle* h, const float* y, const float* norm, int nthreads, float* denom) {
  if (!h->f) return -1;
  try {
    auto& H = *h->f;
    auto& g = H.g;
    const int64_t ni = static_cast<int64_t>(g.nz) * g.ny * g.nx;
    std::vector<float> ones(ni, 1.f), fp(g.projdata_size, 0.f);
    H.forward(ones.data(), fp.data(), 0, 1, nthreads);
    const auto vs = basic_vs_in_subset(g, 0, 1);
    for (const auto& b : vs)
      for (int k = g.min_tof; k <= g.max_tof; ++k) {
        std::vector<std::pair<int, int>> rel;
        related_vs(g, b.first, b.second, rel);
        for (const auto& r : rel) {
          const int seg = r.second, view = r.first;
          float vmax = -std::numeric_limits<float>::infinity();
          for_viewgram(g, seg, view, k, [&](int, int, int64_t i) { vmax = std::max(vmax, fp[i]); });
          const float small_value = std::max(vmax * SMALL_NUM, 0.F);
          for_viewgram(g, seg, view, k, [&](int, int, int64_t i) {
            float num = fp[i];
            float den = y[i];
            if (norm) {
              den *= norm[i];
              den *= norm[i];
            }
            if (num <= small_value) {
              num = 0;
            } else {
              const float max_quotient = 10000.F;
              num = (num > max_quotient * den) ? max_quotient : num / den;
            }
            fp[i] = num;
          });
        }
      }
    H.back(fp.data(), denom, 0, 1, nthreads);
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "oracle: %s\n", e.what());
    return -1;
  }
}

/* QuadraticPrior::parabolic_surrogate_curvature (QuadraticPrior.cxx:460-522): beta sum_k w_k (kappa_j kappa_k) */
int or_prior_curvature_f32(const b200rt_prior* p, const float* kappa, int nz, int ny, int nx, float vz, float vy,
                           float vx, float* out) {
  const int64_t ni = static_cast<int64_t>(nz) * ny * nx;
  if (!p || p->type == B200RT_PRIOR_NONE || p->penalisation_factor == 0) {
    std::fill(out, out + ni, 0.f);
    return 0;
  }
  if (p->type != B200RT_PRIOR_QUADRATIC) return -1;
  float w[3][3][3];
  prior_weights(w, vz, vy, vx, p->only_2D != 0);
  const int dzmin = p->only_2D ? 0 : -1, dzmax = p->only_2D ? 0 : 1;
  auto at = [&](int z, int y, int x) { return (static_cast<int64_t>(z) * ny + y) * nx + x; };
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        const int min_dz = std::max(dzmin, -z), max_dz = std::min(dzmax, nz - 1 - z);
        const int min_dy = std::max(-1, -y), max_dy = std::min(1, ny - 1 - y);
        const int min_dx = std::max(-1, -x), max_dx = std::min(1, nx - 1 - x);
        float c = 0;
        for (int dz = min_dz; dz <= max_dz; ++dz)
          for (int dy = min_dy; dy <= max_dy; ++dy)
            for (int dx = min_dx; dx <= max_dx; ++dx) {
              float cur = w[dz + 1][dy + 1][dx + 1] * 1;
              if (kappa) cur *= kappa[at(z, y, x)] * kappa[at(z + dz, y + dy, x + dx)];
              c += cur;
            }
        out[at(z, y, x)] = c * p->penalisation_factor;
      }
  return 0;
}

/* One OSSPS sub-iteration (OSSPSReconstruction.cxx:284-410) on x (in/out).  denom: the precomputed denominator,
   replaced at the first sub-iteration by the thresholded denominator including the prior's curvature (the
   Quadratic prior's does not depend on x, :292-299,325-346).  sens: the total sensitivity, for
   fill_nonidentifiable_target_parameters at the first sub-iteration. */
int or_ossps_update_f32(or_handle* h, float* x, float* denom, const float* y, const float* add, const float* mult,
                        const float* sens, int subset, int nsub, int subiter, int start_subiter, int zero_ends,
                        const b200rt_prior* prior, const float* kappa, float relaxation_parameter,
                        float relaxation_gamma, float upper_bound, int nthreads) {
  if (!h->f) return -1;
  auto& g = h->f->g;
  const int64_t ni = static_cast<int64_t>(g.nz) * g.ny * g.nx;
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  if (subiter == start_subiter)
    for (int64_t i = 0; i < ni; ++i)
      if (sens[i] == 0) x[i] = 0;
  std::vector<float> num(ni, 0.f);
  if (or_loglik_gradient_f32(h, x, y, add, mult, subset, nsub, zero_ends, nthreads, num.data()) != 0) return -1;
  if (has_prior) {
    /* GeneralisedObjectiveFunction::compute_sub_gradient (GeneralisedObjectiveFunction.cxx:139-156) */
    std::vector<float> pg(ni);
    prior_gradient(*prior, x, kappa, g.nz, g.ny, g.nx, g.d.voxel_size_z, g.d.voxel_size_y, g.d.voxel_size_x, pg.data());
    for (int64_t i = 0; i < ni; ++i) num[i] -= pg[i] / nsub;
  }
  for (int64_t i = 0; i < ni; ++i) num[i] = num[i] * nsub;
  if (subiter == start_subiter) {
    if (has_prior) {
      std::vector<float> c(ni);
      if (or_prior_curvature_f32(prior, kappa, g.nz, g.ny, g.nx, g.d.voxel_size_z, g.d.voxel_size_y,
                                 g.d.voxel_size_x, c.data()) != 0)
        return -1;
      for (int64_t i = 0; i < ni; ++i) denom[i] = c[i] * 2 + denom[i];
    }
    /* threshold_min_to_small_positive_value(.., 10.E-6F) (thresholding.h:99-109) */
    float minpos = std::numeric_limits<float>::infinity();
    for (int64_t i = 0; i < ni; ++i)
      if (denom[i] > 0 && denom[i] < minpos) minpos = denom[i];
    if (minpos == std::numeric_limits<float>::infinity()) {
      std::fill(denom, denom + ni, 10.E-6F);
    } else {
      const float lo = minpos * 10.E-6F;
      for (int64_t i = 0; i < ni; ++i)
        if (denom[i] < lo) denom[i] = lo;
    }
  }
  for (int64_t i = 0; i < ni; ++i) num[i] = num[i] / denom[i];
  const float relax = relaxation_parameter / (1 + relaxation_gamma * (subiter / nsub));
  const float alpha = 1.F;
  for (int64_t i = 0; i < ni; ++i) num[i] = num[i] * relax * alpha;
  for (int64_t i = 0; i < ni; ++i) {
    x[i] += num[i];
    /* threshold_upper_lower(.., 0, upper_bound) */
    if (x[i] > upper_bound)
      x[i] = upper_bound;
    else if (0.F > x[i])
      x[i] = 0.F;
  }
  return 0;
}

int or_prior_gradient_f32(const b200rt_prior* p, const float* img, const float* kappa, int nz, int ny, int nx, float vz,
                          float vy, float vx, float* grad) {
  prior_gradient(*p, img, kappa, nz, ny, nx, vz, vy, vx, grad);
  return 0;
}
double or_prior_value_f32(const b200rt_prior* p, const float* img, const float* kappa, int nz, int ny, int nx, float vz,
                          float vy, float vx) {
  return prior_value(*p, img, kappa, nz, ny, nx, vz, vy, vx);
}

/* ---- list mode: LM_gradient_and_value / LM_Hessian
   (PoissonLogLikelihoodWithLinearModelForMeanAndListModeDataWithProjMatrixByBin.cxx:750-820) over the events in order,
   with the subset rule of LM_distributable_computation (distributable.txx:36-140): the basic bin's view mod
   num_subsets.  events: n x 5 ints (segment, view, axial, tangential, timing) with values and additive terms.
   op 0: out += gradient terms; 1: returns the value; 2: out += Hessian times rhs.  Returns the value (op 1), else 0;
   *invalid counts events outside the projection data. */
double or_listmode_f32(or_handle* h, int op, const int32_t* bins, const float* values, const float* corr, int64_t n,
                       const float* x, const float* rhs, int subset, int nsub, int has_add, float* out,
                       int64_t* invalid) {
  Handle<float>& H = *h->f;
  const auto& g = H.g;
  const float max_quotient = 10000.F;
  double value = 0.0;
  int64_t bad = 0;
  for (int64_t i = 0; i < n; ++i) {
    const float y = values[i];
    if (y == 0.0f) continue;
    Bin<float> b{bins[5 * i], bins[5 * i + 1], bins[5 * i + 2], bins[5 * i + 3], bins[5 * i + 4]};
    if (b.seg < -g.S || b.seg > g.S || b.view < 0 || b.view >= g.num_views || b.tang < g.min_tang ||
        b.tang > g.max_tang || b.tof < g.min_tof || b.tof > g.max_tof || b.ax < 0 || b.ax >= g.nax(b.seg)) {
      ++bad;
      continue;
    }
    if (nsub > 1) {
      Bin<float> basic = b;
      find_op_and_basic(g, basic);
      if (subset != basic.view % nsub) continue;
    }
    const float fwd = H.fwd_bin(b, x) + (has_add ? corr[i] : 0.F);
    const bool cancel = y > max_quotient * fwd;
    if (op == 1) {
      value -= cancel ? y * std::log(static_cast<double>(y / max_quotient)) : y * std::log(static_cast<double>(fwd));
      continue;
    }
    if (op == 0) {
      H.back_bin(b, y / fwd, out);
      continue;
    }
    if (cancel) continue;
    const float c = -y / (fwd * fwd);
    const float r = H.fwd_bin(b, rhs);
    if (r == 0) continue;
    H.back_bin(b, c * r, out);
  }
  if (invalid) *invalid = bad;
  return value;
}

/* ---- Gibbs penalties: GibbsPenalty<float, Potential> (GibbsPenalty.inl) ---------------------------------------
   Potentials as in QuadraticPotential (GibbsQuadraticPenalty.h:50-80) and RelativeDifferencePotential
   (GibbsRelativeDifferencePenalty.h:60-120): each expression is evaluated in the types the reference gives it
   (float operands, double literals 0.5 / 1.0 promote that operation to double, results converted back to
   float where the reference assigns to an elemT).  fabs of a float is taken in float. */
extern "C++" {
struct GibbsQuadraticPotential {
  double value(float c, float n) const {
    const float diff = c - n;
    return static_cast<double>(diff * diff) / 4.0;
  }
  double d10(float c, float n) const { return static_cast<double>(c - n) / 2.0; }
  double d20(float, float) const { return 0.5; }
  double d11(float, float) const { return -0.5; }
};

struct GibbsRDPotential {
  float gamma, epsilon;
  double value(float c, float n) const {
    const float diff = c - n;
    const float add = c + n;
    const float num = static_cast<float>(0.5 * static_cast<double>(diff * diff));
    const float den = static_cast<float>(1.0 / static_cast<double>(add + gamma * std::fabs(diff) + epsilon));
    return static_cast<double>(num * den);
  }
  double d10(float c, float n) const {
    const float diff = c - n;
    const float factor = c + n + gamma * std::fabs(diff) + epsilon;
    const float num = static_cast<float>(0.5 * static_cast<double>(diff) * static_cast<double>(factor + 2 * n + epsilon));
    const float den = static_cast<float>(1.0 / static_cast<double>(factor * factor));
    return static_cast<double>(num * den);
  }
  double d20(float c, float n) const {
    const float num = 2 * n + epsilon;
    const float den = static_cast<float>(1.0 / static_cast<double>(c + n + gamma * std::fabs(c - n) + epsilon));
    return static_cast<double>(num * num * den * den * den);
  }
  double d11(float c, float n) const {
    const float num = -(2 * c + epsilon) * (2 * n + epsilon);
    const float den = static_cast<float>(1.0 / static_cast<double>(c + n + gamma * std::fabs(c - n) + epsilon));
    return static_cast<double>(num * den * den * den);
  }
};

/* weights [wz][wy][wx] with index ranges [-(w/2), w - 1 - w/2] (GibbsPenalty.inl post_processing: an even size
   behaves as if a zero were appended) */
struct GibbsWeights {
  const float* w;
  int wz, wy, wx;
  int lo(int s) const { return -(s / 2); }
  int hi(int s) const { return s - 1 - s / 2; }
  float at(int dz, int dy, int dx) const {
    return w[(static_cast<int64_t>(dz - lo(wz)) * wy + (dy - lo(wy))) * wx + (dx - lo(wx))];
  }
};

template <typename Pot>
double gibbs_run(int op, const Pot& pot, float beta, const GibbsWeights& W, const float* kappa, const float* x,
                 const float* in, int nz, int ny, int nx, int vz, int vy, int vx, float* out) {
  auto at = [&](int z, int y, int xx) { return (static_cast<int64_t>(z) * ny + y) * nx + xx; };
  double total = 0.0;
  if (op == 5) {  // compute_Hessian of one voxel (GibbsPenalty.inl compute_Hessian)
    std::fill(out, out + static_cast<int64_t>(nz) * ny * nx, 0.f);
    if (beta == 0) return 0.0;
    const int z = vz, y = vy, xx = vx;
    const int min_dz = std::max(W.lo(W.wz), -z), max_dz = std::min(W.hi(W.wz), nz - 1 - z);
    const int min_dy = std::max(W.lo(W.wy), -y), max_dy = std::min(W.hi(W.wy), ny - 1 - y);
    const int min_dx = std::max(W.lo(W.wx), -xx), max_dx = std::min(W.hi(W.wx), nx - 1 - xx);
    const int64_t j = at(z, y, xx);
    for (int dz = min_dz; dz <= max_dz; ++dz)
      for (int dy = min_dy; dy <= max_dy; ++dy)
        for (int dx = min_dx; dx <= max_dx; ++dx) {
          float current = 0.0f;
          if (dz == 0 && dy == 0 && dx == 0) {
            for (int ddz = min_dz; ddz <= max_dz; ++ddz)
              for (int ddy = min_dy; ddy <= max_dy; ++ddy)
                for (int ddx = min_dx; ddx <= max_dx; ++ddx) {
                  const int64_t k = at(z + ddz, y + ddy, xx + ddx);
                  float dc = static_cast<float>(W.at(ddz, ddy, ddx) * 2 * pot.d20(x[j], x[k]));
                  if (kappa) dc *= kappa[j] * kappa[k];
                  current += dc;
                }
          } else {
            const int64_t k = at(z + dz, y + dy, xx + dx);
            current = static_cast<float>(W.at(dz, dy, dx) * 2 * pot.d11(x[j], x[k]));
            if (kappa) current *= kappa[j] * kappa[k];
          }
          out[at(z + dz, y + dy, xx + dx)] = current * beta;
        }
    return 0.0;
  }
  if (beta == 0) {
    if (op == 1 || op == 3) std::fill(out, out + static_cast<int64_t>(nz) * ny * nx, 0.f);
    return 0.0;
  }
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int xx = 0; xx < nx; ++xx) {
        const int min_dz = std::max(W.lo(W.wz), -z), max_dz = std::min(W.hi(W.wz), nz - 1 - z);
        const int min_dy = std::max(W.lo(W.wy), -y), max_dy = std::min(W.hi(W.wy), ny - 1 - y);
        const int min_dx = std::max(W.lo(W.wx), -xx), max_dx = std::min(W.hi(W.wx), nx - 1 - xx);
        const int64_t j = at(z, y, xx);
        const float c = x[j];
        if (op == 4) {  // accumulate_Hessian_times_input: float sums, the centre included
          float result = 0;
          for (int dz = min_dz; dz <= max_dz; ++dz)
            for (int dy = min_dy; dy <= max_dy; ++dy)
              for (int dx = min_dx; dx <= max_dx; ++dx) {
                const int64_t k = at(z + dz, y + dy, xx + dx);
                float current = W.at(dz, dy, dx);
                if (dz == 0 && dy == 0 && dx == 0)
                  current = static_cast<float>(current * (pot.d20(c, x[k]) * in[j]));
                else
                  current = static_cast<float>(current * (pot.d20(c, x[k]) * in[j] + pot.d11(c, x[k]) * in[k]));
                if (kappa) current *= kappa[j] * kappa[k];
                result += current;
              }
          out[j] += 2 * result * beta;
          continue;
        }
        double sum = 0.0;
        for (int dz = min_dz; dz <= max_dz; ++dz)
          for (int dy = min_dy; dy <= max_dy; ++dy)
            for (int dx = min_dx; dx <= max_dx; ++dx) {
              if (dz == 0 && dy == 0 && dx == 0) continue;
              const int64_t k = at(z + dz, y + dy, xx + dx);
              const float n = x[k];
              const double f = op == 0 ? pot.value(c, n) : (op == 3 ? pot.d20(c, n) : pot.d10(c, n));
              double current = W.at(dz, dy, dx) * f;
              if (kappa) current *= kappa[j] * kappa[k];
              sum += current;
            }
        if (op == 0)
          total += sum;
        else if (op == 1 || op == 3)
          out[j] = 2 * static_cast<float>(sum * beta);
        else
          total += 2 * sum * in[j];
      }
  return total * beta;
}
}  // extern "C++"

double or_gibbs_f32(int op, int potential, float beta, float gamma, float epsilon, const float* weights, int wz, int wy,
                    int wx, const float* kappa, const float* image, const float* input, int nz, int ny, int nx, int vz,
                    int vy, int vx, float* out) {
  const GibbsWeights W{weights, wz, wy, wx};
  if (potential == 1) return gibbs_run(op, GibbsQuadraticPotential{}, beta, W, kappa, image, input, nz, ny, nx, vz, vy, vx, out);
  return gibbs_run(op, GibbsRDPotential{gamma, epsilon}, beta, W, kappa, image, input, nz, ny, nx, vz, vy, vx, out);
}

/* GibbsPenalty::compute_default_weights (GibbsPenalty.inl): x voxel size / distance over a 3x3x3 neighbourhood
   (1x3x3 with only_2D), centre 0; w holds wz*9 floats, wz returned */
int or_gibbs_default_weights(float vz, float vy, float vx, int only_2D, float* w) {
  const int z0 = only_2D ? 0 : -1, z1 = only_2D ? 0 : 1;
  int i = 0;
  for (int z = z0; z <= z1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        if (z == 0 && y == 0 && x == 0) {
          w[i++] = 0.f;
          continue;
        }
        const float a = x * vx, b = y * vy, c = z * vz;
        w[i++] = vx / std::sqrt(a * a + b * b + c * c);
      }
  return z1 - z0 + 1;
}

int64_t or_ray_trace(const float start[3], const float stop[3], const float vox[3], float norm_const, int32_t* coords,
                     float* values, int64_t cap) {
  Row<float> r;
  ray_trace(r, C3<float>{start[0], start[1], start[2]}, C3<float>{stop[0], stop[1], stop[2]},
            C3<float>{vox[0], vox[1], vox[2]}, norm_const);
  if (static_cast<int64_t>(r.size()) > cap) return -1;
  for (size_t i = 0; i < r.size(); ++i) {
    coords[3 * i] = r[i].z;
    coords[3 * i + 1] = r[i].y;
    coords[3 * i + 2] = r[i].x;
    values[i] = r[i].v;
  }
  return static_cast<int64_t>(r.size());
}

}  // extern "C"
