// C ABI: the objective function and OSMAPOSL / OSSPS updates, priors, normalisations.
#include "capi.hpp"

using namespace b200;

namespace capi {

// u = A_S^T divide_and_truncate(y, A_S x + a): fused forward projection/ratio, then back projection
void osmaposl_numerator(b200rt_projector& h, const float* x, const float* y, const float* add, int subset, int nsub,
                        int zero_ends, int mode, float* u, cudaStream_t st) {
  const Geometry& g = *h.geo;
  if (!h.ratio.p) {
    h.ratio.alloc(pd_size(h));
    ck(cudaMemsetAsync(h.ratio.p, 0, sizeof(float) * pd_size(h), st), "memset");  // bins outside the subset
  }
  h.small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
  h.cancelled.alloc(1);
  int nv = 0;
  const int* views = subset_views(h, subset, nsub, nv);
  ck(launch_viewgram_small_values(y, h.segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, zero_ends, g.num_tof(),
                                  pd_tof_stride(h), h.small_value.p, st, h.params.view_slot),
     "viewgram thresholds");
  ck(cudaMemsetAsync(h.cancelled.p, 0, sizeof(unsigned int), st), "memset");
  FwdEpilogue ep{};
  ep.mode = kEpiRatio;
  ep.zero_ends = zero_ends;
  ep.y = y;
  ep.add = add;
  ep.small_value = h.small_value.p;
  ep.cancelled = h.cancelled.p;
  forward_subset(h, x, h.ratio.p, subset, nsub, st, &ep);
  back_project_into(h, h.ratio.p, u, subset, nsub, mode, 0, st, 10000.F);
}

// u /= denominator, clamp, x *= u (OSMAPOSLReconstruction.cxx:394-510)
void osmaposl_apply(b200rt_projector& h, float* x, float* u, const float* sens, int nsub, int subiter,
                    const b200rt_prior* prior, float min_rel, float max_rel, cudaStream_t st) {
  const Geometry& g = *h.geo;
  const int64_t ni = g.image_size();
  h.partial_max.alloc(update_num_blocks(ni));
  h.umax.alloc(1);
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  if (has_prior) {
    h.grad.alloc(ni);
    prior_weights(g, prior->only_2D, h.prior_w);
  }
  ck(launch_update(u, x, sens, has_prior ? h.grad.p : nullptr, has_prior ? prior : nullptr, h.prior_w, nsub, subiter,
                   min_rel, max_rel, g.desc().ny, g.desc().nx, g.desc().nz, h.partial_max.p, h.umax.p, st),
     "update");
}

int check_mode_prior(b200rt_projector* h, int mode, const b200rt_prior* prior) {
  if (mode != B200RT_BACKPROJECT_ATOMIC && mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  if (prior && (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE))
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  return B200RT_OK;
}

}  // namespace capi

extern "C" {

int b200rt_osmaposl_subiteration_dev(b200rt_projector* h, float* estimate_dev, const float* y_dev, const float* additive_dev,
                                     const float* sens_dev, int subset_num, int num_subsets, int subiteration_num,
                                     int zero_seg0_end_planes, const b200rt_prior* prior, float min_relative_change,
                                     float max_relative_change, int back_projection_mode, float* update_dev, void* stream) {
  if (!h || !estimate_dev || !y_dev || !sens_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_mode_prior(h, back_projection_mode, prior)) return st;
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!update_dev) h->upd.alloc(h->geo->image_size());
    float* u = update_dev ? update_dev : h->upd.p;
    osmaposl_numerator(*h, estimate_dev, y_dev, additive_dev, subset_num, num_subsets, zero_seg0_end_planes,
                       back_projection_mode, u, st);
    osmaposl_apply(*h, estimate_dev, u, sens_dev, num_subsets, subiteration_num, prior, min_relative_change,
                   max_relative_change, st);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_osmaposl_numerator_dev(b200rt_projector* h, const float* estimate_dev, const float* y_dev,
                                  const float* additive_dev, int subset_num, int num_subsets, int zero_seg0_end_planes,
                                  int back_projection_mode, float* numerator_dev, void* stream) {
  if (!h || !estimate_dev || !y_dev || !numerator_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_mode_prior(h, back_projection_mode, nullptr)) return st;
  try {
    DeviceGuard dg(h->device);
    osmaposl_numerator(*h, estimate_dev, y_dev, additive_dev, subset_num, num_subsets, zero_seg0_end_planes,
                       back_projection_mode, numerator_dev, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_osmaposl_apply_update_dev(b200rt_projector* h, float* estimate_dev, float* numerator_dev, const float* sens_dev,
                                     int num_subsets, int subiteration_num, const b200rt_prior* prior,
                                     float min_relative_change, float max_relative_change, void* stream) {
  if (!h || !estimate_dev || !numerator_dev || !sens_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (num_subsets < 1) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "invalid number of subsets");
  if (int st = check_mode_prior(h, B200RT_BACKPROJECT_ATOMIC, prior)) return st;
  try {
    DeviceGuard dg(h->device);
    osmaposl_apply(*h, estimate_dev, numerator_dev, sens_dev, num_subsets, subiteration_num, prior, min_relative_change,
                   max_relative_change, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_get_device_status(b200rt_projector* h, uint32_t* status, int clear) {
  if (!h || !status) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    unsigned int s = 0;
    if (h->dev_status.p) {
      ck(cudaMemcpy(&s, h->dev_status.p, sizeof(s), cudaMemcpyDeviceToHost), "D2H");
      if (clear && s) ck(cudaMemset(h->dev_status.p, 0, sizeof(s)), "memset");
    }
    *status = s;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_get_num_cancelled(b200rt_projector* h, int64_t* out) {
  if (!h || !out) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    unsigned int c = 0;
    if (h->cancelled.p) ck(cudaMemcpy(&c, h->cancelled.p, sizeof(c), cudaMemcpyDeviceToHost), "D2H");
    *out = c;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_log_likelihood_dev(b200rt_projector* h, const float* image_dev, const float* y_dev, const float* additive_dev,
                              const float* mult_dev, int subset_num, int num_subsets, int zero_seg0_end_planes, double* out,
                              void* stream) {
  if (!h || !image_dev || !y_dev || !out) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int n = 0, nv = 0;
    // one partial sum per CTA: per path item with the column-staged kernel, else per basic bin
    const bool grouped = !h->use_paths && h->params.tof_w;  // one partial per basic bin with all timing bins
    const int* list = h->use_paths ? path_list(*h, subset_num, num_subsets, n)
                      : grouped    ? tof_group_list(*h, subset_num, num_subsets, n)
                                   : subset_list(*h, subset_num, num_subsets, n);
    const int* views = subset_views(*h, subset_num, num_subsets, nv);
    h->small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    if (h->ll_partials.n < static_cast<size_t>(std::max(n, 1))) h->ll_partials.alloc(std::max(n, 1));
    h->ll_sum.alloc(1);
    ck(launch_viewgram_small_values(y_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, zero_seg0_end_planes,
                                    g.num_tof(), pd_tof_stride(*h), h->small_value.p, st, h->params.view_slot),
       "viewgram thresholds");
    FwdEpilogue ep{};
    ep.mode = kEpiLoglik;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.add = additive_dev;
    ep.mult = mult_dev;
    ep.small_value = h->small_value.p;
    ep.partials = h->ll_partials.p;
    if (h->use_paths)
      ck(launch_forward_paths(h->params, h->pparams, list, n, image_dev, nullptr, st, &ep), "log-likelihood");
    else if (grouped)
      ck(launch_forward_tof_grouped(h->params, list, n, image_dev, nullptr, st, &ep), "log-likelihood");
    else
      ck(launch_forward(h->params, list, n, image_dev, nullptr, st, &ep), "log-likelihood");
    ck(launch_reduce_sum(h->ll_partials.p, n, h->ll_sum.p, st), "reduce");
    ck(cudaMemcpyAsync(out, h->ll_sum.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "log-likelihood");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_prior_gradient_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev, float* gradient_dev,
                              void* stream) {
  if (!h || !prior || !image_dev || !gradient_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (prior->type == B200RT_PRIOR_NONE || prior->penalisation_factor == 0) {
      ck(cudaMemsetAsync(gradient_dev, 0, sizeof(float) * g.image_size(), st), "memset");
      return B200RT_OK;
    }
    float w[27];
    prior_weights(g, prior->only_2D, w);
    h->partial_max.alloc(update_num_blocks(g.image_size()));
    ck(launch_prior_gradient(image_dev, gradient_dev, prior, w, g.desc().ny, g.desc().nx, g.desc().nz, h->partial_max.p, st),
       "prior gradient");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_log_likelihood_gradient_dev(b200rt_projector* h, const float* image_dev, const float* y_dev,
                                       const float* additive_dev, const float* mult_dev, int subset_num, int num_subsets,
                                       int zero_seg0_end_planes, int back_projection_mode, float* gradient_dev,
                                       void* stream) {
  if (!h || !image_dev || !y_dev || !gradient_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (back_projection_mode != B200RT_BACKPROJECT_ATOMIC && back_projection_mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!h->ratio.p) {
      h->ratio.alloc(pd_size(*h));
      ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * pd_size(*h), st), "memset");
    }
    h->small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    h->cancelled.alloc(1);
    int nv = 0;
    const int* views = subset_views(*h, subset_num, num_subsets, nv);
    ck(launch_viewgram_small_values(y_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, zero_seg0_end_planes,
                                    g.num_tof(), pd_tof_stride(*h), h->small_value.p, st, h->params.view_slot),
       "viewgram thresholds");
    ck(cudaMemsetAsync(h->cancelled.p, 0, sizeof(unsigned int), st), "memset");
    FwdEpilogue ep{};
    ep.mode = kEpiGradient;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.add = additive_dev;
    ep.mult = mult_dev;
    ep.small_value = h->small_value.p;
    ep.cancelled = h->cancelled.p;
    forward_subset(*h, image_dev, h->ratio.p, subset_num, num_subsets, st, &ep);
    back_project_into(*h, h->ratio.p, gradient_dev, subset_num, num_subsets, back_projection_mode, 0, st);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_attenuation_dev(b200rt_projector* h, const float* mu_dev, float* projdata_dev, int mode, void* stream) {
  if (!h || !mu_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (mode < B200RT_ATTENUATION_FACTORS || mode > B200RT_ATTENUATION_UNDO)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown attenuation mode");
  if (h->geo->num_tof() > 1)
    return fail(h, B200RT_ERR_UNSUPPORTED,
                "BinNormalisationFromAttenuationImage limitation: currently can only handle non_TOF data.");
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Geometry& g = *h->geo;
    if (!h->ratio.p) {
      h->ratio.alloc(pd_size(*h));
      ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * pd_size(*h), st), "memset");
    }
    forward_subset(*h, mu_dev, h->ratio.p, 0, 1, st);
    ck(launch_attenuation(h->ratio.p, projdata_dev, pd_size(*h), mode, st), "attenuation");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_normalisation_dev(b200rt_projector* h, const b200rt_norm_term* terms, int num_terms, int mode,
                             float* projdata_dev, void* stream) {
  if (!h || !projdata_dev || (num_terms > 0 && !terms) || num_terms < 0)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (mode < B200RT_NORM_FACTORS || mode > B200RT_NORM_UNDO)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown normalisation mode");
  const Geometry& g = *h->geo;
  for (int t = 0; t < num_terms; ++t) {
    if (!terms[t].data_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null normalisation data");
    if (terms[t].kind == B200RT_NORM_ATTENUATION) {
      if (g.num_tof() > 1)
        return fail(h, B200RT_ERR_UNSUPPORTED,
                    "BinNormalisationFromAttenuationImage limitation: currently can only handle non_TOF data.");
    } else if (terms[t].kind != B200RT_NORM_PROJDATA) {
      return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown normalisation kind");
    }
  }
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = pd_size(*h);
    int step = mode;
    if (mode == B200RT_NORM_FACTORS) {
      ck(launch_fill(projdata_dev, n, 1.f, st), "fill");
      step = B200RT_NORM_UNDO;
    }
    for (int t = 0; t < num_terms; ++t) {
      if (terms[t].kind == B200RT_NORM_PROJDATA) {
        const int64_t fstride = (terms[t].non_tof && g.num_tof() > 1) ? g.tof_stride() : 0;
        ck(launch_norm_projdata(terms[t].data_dev, projdata_dev, n, fstride, step, st), "normalisation");
      } else {
        if (!h->ratio.p) {
          h->ratio.alloc(n);
          ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * n, st), "memset");
        }
        forward_subset(*h, terms[t].data_dev, h->ratio.p, 0, 1, st);
        ck(launch_attenuation(h->ratio.p, projdata_dev, n,
                              step == B200RT_NORM_APPLY ? B200RT_ATTENUATION_APPLY : B200RT_ATTENUATION_UNDO, st),
           "attenuation");
      }
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_ossps_denominator_dev(b200rt_projector* h, const float* y_dev, const float* norm_dev, float* denominator_dev,
                                 int back_projection_mode, void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_ossps_denominator_dev");
  if (!h || !y_dev || !denominator_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_mode_prior(h, back_projection_mode, nullptr)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!h->ratio.p) {
      h->ratio.alloc(pd_size(*h));
      ck(cudaMemsetAsync(h->ratio.p, 0, sizeof(float) * pd_size(*h), st), "memset");
    }
    if (!h->ones.p) {
      h->ones.alloc(g.image_size());
      ck(launch_fill(h->ones.p, g.image_size(), 1.F, st), "fill");
    }
    h->small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    forward_subset(*h, h->ones.p, h->ratio.p, 0, 1, st);
    int nv = 0;
    const int* views = subset_views(*h, 0, 1, nv);
    // divide_and_truncate's small value from the forward projection of ones
    ck(launch_viewgram_small_values(h->ratio.p, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, 0, g.num_tof(),
                                    g.tof_stride(), h->small_value.p, st),
       "viewgram thresholds");
    ck(launch_hessian_ratio(h->ratio.p, y_dev, norm_dev, h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv,
                            g.num_tof(), g.tof_stride(), h->small_value.p, st),
       "Hessian data term");
    back_project_into(*h, h->ratio.p, denominator_dev, 0, 1, back_projection_mode, 0, st);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_ossps_subiteration_dev(b200rt_projector* h, float* estimate_dev, float* denominator_dev, const float* y_dev,
                                  const float* additive_dev, const float* mult_dev, const float* sens_dev,
                                  int subset_num, int num_subsets, int subiteration_num, int start_subiteration_num,
                                  int zero_seg0_end_planes, const b200rt_prior* prior, float relaxation_parameter,
                                  float relaxation_gamma, float upper_bound, int back_projection_mode, void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_ossps_subiteration_dev");
  if (!h || !estimate_dev || !denominator_dev || !y_dev || !sens_dev)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_mode_prior(h, back_projection_mode, prior)) return st;
  const bool has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
  if (has_prior && prior->type != B200RT_PRIOR_QUADRATIC)
    return fail(h, B200RT_ERR_UNSUPPORTED, "OSSPS needs a prior with a parabolic surrogate (QuadraticPrior)");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t ni = g.image_size();
    h->ossps_g.alloc(ni);
    if (has_prior) h->ossps_pg.alloc(ni);
    h->ossps_partial.alloc(update_num_blocks(ni));
    h->ossps_minpos.alloc(1);
    const bool first = subiteration_num == start_subiteration_num;
    // fill_nonidentifiable_target_parameters at the first sub-iteration (OSSPSReconstruction.cxx:287-291)
    if (first) ck(launch_zero_unidentifiable(estimate_dev, sens_dev, ni, st), "unidentifiable voxels");
    if (int rc = b200rt_log_likelihood_gradient_dev(h, estimate_dev, y_dev, additive_dev, mult_dev, subset_num,
                                                    num_subsets, zero_seg0_end_planes, back_projection_mode,
                                                    h->ossps_g.p, stream))
      return rc;
    // relaxation_parameter / (1 + relaxation_gamma * (subiteration_num / num_subsets)), integer division
    // (OSSPSReconstruction.cxx:370-372)
    const float relax = relaxation_parameter / (1 + relaxation_gamma * (subiteration_num / num_subsets));
    if (has_prior) prior_weights(g, prior->only_2D, h->prior_w);
    ck(launch_ossps_update(estimate_dev, denominator_dev, h->ossps_g.p, has_prior ? h->ossps_pg.p : nullptr, sens_dev,
                           has_prior ? prior : nullptr, h->prior_w, g.desc().ny, g.desc().nx, g.desc().nz, num_subsets,
                           first ? 1 : 0, relax, upper_bound, h->ossps_partial.p, h->ossps_minpos.p, st),
       "OSSPS update");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_prior_hessian_times_input_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev,
                                         const float* input_dev, float* output_dev, void* stream) {
  if (!h || !prior || !image_dev || !input_dev || !output_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_mode_prior(h, B200RT_BACKPROJECT_ATOMIC, prior)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    float w[27];
    prior_weights(g, prior->only_2D, w);
    ck(launch_prior_hessian_times_input(output_dev, image_dev, input_dev, prior, w, g.desc().ny, g.desc().nx,
                                        g.desc().nz, static_cast<cudaStream_t>(stream)),
       "prior Hessian");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_prior_value_dev(b200rt_projector* h, const b200rt_prior* prior, const float* image_dev, double* out,
                           void* stream) {
  if (!h || !prior || !image_dev || !out) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (prior->type == B200RT_PRIOR_NONE || prior->penalisation_factor == 0) {
      *out = 0.0;
      return B200RT_OK;
    }
    float w[27];
    prior_weights(g, prior->only_2D, w);
    const int np = update_num_blocks(g.image_size());
    h->ll_partials.alloc(std::max<size_t>(h->ll_partials.n, static_cast<size_t>(np)));
    h->ll_sum.alloc(1);
    ck(launch_prior_value(image_dev, prior, w, g.desc().ny, g.desc().nx, g.desc().nz, h->ll_partials.p, np, h->ll_sum.p, st),
       "prior value");
    double v = 0.0;
    ck(cudaMemcpyAsync(&v, h->ll_sum.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "prior value");
    *out = v * prior->penalisation_factor;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"
