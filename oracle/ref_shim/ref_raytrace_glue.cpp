/*
 * Glue that links STIR's own RayTraceVoxelsOnCartesianGrid.cxx (compiled from
 * the STIR tree) into oracle/_ref/libref_raytrace.so.  Test infrastructure:
 * it lets the tests compare the oracle's restated Siddon tracer with STIR's
 * compiled one on the same rays.
 *
 * The out-of-line members the tracer reaches are given minimal bodies here:
 * the constructor, reserve/sort of the element vector, and warning().
 */
#include "stir/recon_buildblock/ProjMatrixElemsForOneBin.h"
#include "stir/recon_buildblock/RayTraceVoxelsOnCartesianGrid.h"
#include "stir/CartesianCoordinate3D.h"

#include <algorithm>
#include <cstdarg>
#include <cstdint>
#include <cstdio>

namespace stir {

ProjMatrixElemsForOneBin::ProjMatrixElemsForOneBin(const Bin& b, const int default_capacity) : bin(b) {
  elements.reserve(default_capacity);
}

void ProjMatrixElemsForOneBin::reserve(size_type max_number) { elements.reserve(max_number); }

void ProjMatrixElemsForOneBin::sort() { std::sort(elements.begin(), elements.end(), value_type::coordinates_less); }

void warning(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vfprintf(stderr, fmt, ap);
  va_end(ap);
}

}  // namespace stir

extern "C" int64_t ref_ray_trace(const float start_zyx[3], const float stop_zyx[3], const float vox_zyx[3],
                                 float normalisation_constant, int32_t* coords_zyx, float* values, int64_t capacity) {
  stir::ProjMatrixElemsForOneBin lor;
  const stir::CartesianCoordinate3D<float> start(start_zyx[0], start_zyx[1], start_zyx[2]);
  const stir::CartesianCoordinate3D<float> stop(stop_zyx[0], stop_zyx[1], stop_zyx[2]);
  const stir::CartesianCoordinate3D<float> vox(vox_zyx[0], vox_zyx[1], vox_zyx[2]);
  stir::RayTraceVoxelsOnCartesianGrid(lor, start, stop, vox, normalisation_constant);
  const int64_t n = static_cast<int64_t>(lor.size());
  if (n > capacity) return -1;
  int64_t i = 0;
  for (auto it = lor.begin(); it != lor.end(); ++it, ++i) {
    coords_zyx[3 * i] = it->coord1();
    coords_zyx[3 * i + 1] = it->coord2();
    coords_zyx[3 * i + 2] = it->coord3();
    values[i] = it->get_value();
  }
  return n;
}
