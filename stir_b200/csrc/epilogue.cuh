// What the forward projectors do with one projected bin A x (shared by the per-basic-bin and the
// column-staged kernels).
#pragma once

#include "internal.hpp"

namespace b200 {

// `ax` = A x of the bin at device-layout index `idx`, axial position `a` of a line of segment `seg`,
// view `view`, timing bin index `tofi`, with `nax` axial positions.
template <int EPI>
__device__ __forceinline__ void forward_store(const ProjParams& p, int seg, int view, int tofi, int nax, int64_t idx,
                                              int a, float ax, float* __restrict__ out, const FwdEpilogue& ep, double& ll,
                                              unsigned& ncancel) {
  if (EPI == kEpiNone) {
    out[idx] = ax;
    return;
  }
  // segment 0 end planes zeroed (distributable.cxx:146-158,216-221)
  const bool zend = ep.zero_ends && seg == 0 && (a == 0 || a == nax - 1);
  const float y = zend ? 0.f : __ldg(ep.y + idx);
  const float av = (ep.add && !zend) ? __ldg(ep.add + idx) : 0.f;
  const float sv = ep.small_value[(tofi * (2 * p.S + 1) + seg + p.S) * p.num_views + view];
  if (EPI == kEpiRatio || EPI == kEpiGradient || EPI == kEpiLoglikRatio) {
    // divide_and_truncate (recon_array_functions.cxx:171-266) of y by A x + a
    const float den = ax + av;
    float r;
    if (y <= sv) {
      r = 0.f;
    } else if (y > 10000.F * den) {
      r = 10000.F;
      ++ncancel;
    } else {
      r = y / den;
    }
    if (EPI == kEpiGradient || EPI == kEpiLoglikRatio) r -= zend ? 0.f : (ep.mult ? __ldg(ep.mult + idx) : 1.f);
    out[idx] = r;
  }
  if (EPI == kEpiLoglik || EPI == kEpiLoglikRatio) {
    // accumulate_loglikelihood (recon_array_functions.cxx:335-377) of ybar = (A x + a) * m
    float e = ax + av;
    if (zend)
      e *= 0.f;
    else if (ep.mult)
      e *= __ldg(ep.mult + idx);
    const float ne = fmaxf(e, y / 10000.F);
    ll += (y <= sv) ? -static_cast<double>(ne) : y * log(static_cast<double>(ne)) - static_cast<double>(ne);
    if (EPI == kEpiLoglik && out) out[idx] = e;
  }
}

}  // namespace b200
