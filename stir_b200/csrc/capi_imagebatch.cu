// C ABI: a batch of images through one projector (torch.autograd batches, noise realisations), one launch over
// (path item, image) where the column-staged kernels apply, else image by image.
#include "capi.hpp"

using namespace b200;

namespace {

int check_batch(b200rt_projector* h, int batch, int64_t image_stride, int64_t pd_stride) {
  if (batch < 1 || batch > 65535) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "batch must be 1..65535");
  const Geometry& g = *h->geo;
  if (batch > 1 && (image_stride < g.image_size() || pd_stride < pd_size(*h)))
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "batch strides smaller than an image / the projection data");
  return B200RT_OK;
}

// thresholds of every image's data (y of image b at y + b y_stride; one set when y_stride is 0)
float* batch_thresholds(b200rt_projector& h, const float* y, int64_t y_stride, int batch, int subset, int nsub,
                        int zero_ends, cudaStream_t st, int64_t& sv_stride) {
  const Geometry& g = *h.geo;
  const int64_t nsv = static_cast<int64_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views();
  const int nsets = y_stride ? batch : 1;
  if (h.small_value.n < static_cast<size_t>(nsv * nsets)) h.small_value.alloc(nsv * nsets);
  int nv = 0;
  const int* views = subset_views(h, subset, nsub, nv);
  for (int b = 0; b < nsets; ++b)
    ck(launch_viewgram_small_values(y + b * y_stride, h.segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, zero_ends,
                                    g.num_tof(), pd_tof_stride(h), h.small_value.p + b * nsv, st, h.params.view_slot),
       "viewgram thresholds");
  sv_stride = y_stride ? nsv : 0;
  return h.small_value.p;
}

}  // namespace

extern "C" {

int b200rt_forward_project_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                     float* projdata_dev, int64_t projdata_stride, int batch, int subset_num,
                                     int num_subsets, void* stream) {
  if (!h || !images_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_batch(h, batch, image_stride, projdata_stride)) return st;
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (h->use_paths) {
      int n = 0;
      const int* list = path_list(*h, subset_num, num_subsets, n);
      ck(launch_forward_paths_batch(h->params, h->pparams, list, n, images_dev, image_stride, projdata_dev,
                                    projdata_stride, batch, st, nullptr),
         "forward projection");
    } else {
      for (int b = 0; b < batch; ++b)
        forward_subset(*h, images_dev + b * image_stride, projdata_dev + b * projdata_stride, subset_num, num_subsets, st);
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_back_project_batch_dev(b200rt_projector* h, const float* projdata_dev, int64_t projdata_stride,
                                  float* images_dev, int64_t image_stride, int batch, int subset_num, int num_subsets,
                                  int back_projection_mode, void* stream) {
  if (!h || !images_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_batch(h, batch, image_stride, projdata_stride)) return st;
  if (back_projection_mode != B200RT_BACKPROJECT_ATOMIC && back_projection_mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t ni = h->geo->image_size();
    if (h->use_paths && back_projection_mode == B200RT_BACKPROJECT_ATOMIC) {
      int n = 0;
      const int* list = path_list(*h, subset_num, num_subsets, n);
      for (int b = 0; b < batch; ++b) ck(cudaMemsetAsync(images_dev + b * image_stride, 0, sizeof(float) * ni, st), "memset");
      ck(launch_back_paths_atomic_batch(h->params, h->pparams, list, n, projdata_dev, projdata_stride, images_dev,
                                        image_stride, batch, st, 0),
         "back projection");
    } else {
      for (int b = 0; b < batch; ++b)
        back_project_into(*h, projdata_dev + b * projdata_stride, images_dev + b * image_stride, subset_num, num_subsets,
                          back_projection_mode, 0, st);
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_log_likelihood_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                    const float* y_dev, int64_t y_stride, const float* additive_dev,
                                    int64_t additive_stride, const float* mult_dev, int64_t mult_stride, int batch,
                                    int subset_num, int num_subsets, int zero_seg0_end_planes, double* values,
                                    void* stream) {
  if (!h || !images_dev || !y_dev || !values) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_batch(h, batch, image_stride, pd_size(*h))) return st;
  if (!h->use_paths) {  // the per-basic-bin and TOF-grouped kernels take one image at a time
    for (int b = 0; b < batch; ++b)
      if (int st = b200rt_log_likelihood_dev(h, images_dev + b * image_stride, y_dev + b * y_stride,
                                             additive_dev ? additive_dev + b * additive_stride : nullptr,
                                             mult_dev ? mult_dev + b * mult_stride : nullptr, subset_num, num_subsets,
                                             zero_seg0_end_planes, values + b, stream))
        return st;
    return B200RT_OK;
  }
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int n = 0;
    const int* list = path_list(*h, subset_num, num_subsets, n);
    FwdEpilogue ep{};
    ep.mode = kEpiLoglik;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.y_stride = y_stride;
    ep.add = additive_dev;
    ep.add_stride = additive_stride;
    ep.mult = mult_dev;
    ep.mult_stride = mult_stride;
    ep.small_value = batch_thresholds(*h, y_dev, y_stride, batch, subset_num, num_subsets, zero_seg0_end_planes, st,
                                      ep.sv_stride);
    const size_t np = static_cast<size_t>(std::max(n, 1)) * batch;
    if (h->ll_partials.n < np) h->ll_partials.alloc(np);
    if (h->ll_sum.n < static_cast<size_t>(batch)) h->ll_sum.alloc(batch);
    ep.partials = h->ll_partials.p;
    ck(launch_forward_paths_batch(h->params, h->pparams, list, n, images_dev, image_stride, nullptr, 0, batch, st, &ep),
       "log-likelihood");
    for (int b = 0; b < batch; ++b)
      ck(launch_reduce_sum(h->ll_partials.p + static_cast<int64_t>(b) * n, n, h->ll_sum.p + b, st), "reduce");
    ck(cudaMemcpyAsync(values, h->ll_sum.p, sizeof(double) * batch, cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "log-likelihood");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_log_likelihood_and_ratio_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                               const float* y_dev, int64_t y_stride, const float* additive_dev,
                                               int64_t additive_stride, const float* mult_dev, int64_t mult_stride,
                                               int batch, int subset_num, int num_subsets, int zero_seg0_end_planes,
                                               double* values, float* ratio_dev, int64_t ratio_stride, void* stream) {
  if (!h || !images_dev || !y_dev || !values || !ratio_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_batch(h, batch, image_stride, ratio_stride)) return st;
  if (!h->use_paths)
    return fail(h, B200RT_ERR_UNSUPPORTED,
                "b200rt_log_likelihood_and_ratio_batch_dev needs the column-staged kernels (non-TOF projector)");
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int n = 0;
    const int* list = path_list(*h, subset_num, num_subsets, n);
    h->cancelled.alloc(1);
    ck(cudaMemsetAsync(h->cancelled.p, 0, sizeof(unsigned int), st), "memset");
    FwdEpilogue ep{};
    ep.mode = kEpiLoglikRatio;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.y_stride = y_stride;
    ep.add = additive_dev;
    ep.add_stride = additive_stride;
    ep.mult = mult_dev;
    ep.mult_stride = mult_stride;
    ep.cancelled = h->cancelled.p;
    ep.small_value = batch_thresholds(*h, y_dev, y_stride, batch, subset_num, num_subsets, zero_seg0_end_planes, st,
                                      ep.sv_stride);
    const size_t np = static_cast<size_t>(std::max(n, 1)) * batch;
    if (h->ll_partials.n < np) h->ll_partials.alloc(np);
    if (h->ll_sum.n < static_cast<size_t>(batch)) h->ll_sum.alloc(batch);
    ep.partials = h->ll_partials.p;
    ck(launch_forward_paths_batch(h->params, h->pparams, list, n, images_dev, image_stride, ratio_dev, ratio_stride,
                                  batch, st, &ep),
       "log-likelihood");
    for (int b = 0; b < batch; ++b)
      ck(launch_reduce_sum(h->ll_partials.p + static_cast<int64_t>(b) * n, n, h->ll_sum.p + b, st), "reduce");
    ck(cudaMemcpyAsync(values, h->ll_sum.p, sizeof(double) * batch, cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "log-likelihood");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_log_likelihood_gradient_batch_dev(b200rt_projector* h, const float* images_dev, int64_t image_stride,
                                             const float* y_dev, int64_t y_stride, const float* additive_dev,
                                             int64_t additive_stride, const float* mult_dev, int64_t mult_stride,
                                             int batch, int subset_num, int num_subsets, int zero_seg0_end_planes,
                                             int back_projection_mode, float* gradients_dev, int64_t gradient_stride,
                                             void* stream) {
  if (!h || !images_dev || !y_dev || !gradients_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (int st = check_batch(h, batch, std::min(image_stride, gradient_stride), pd_size(*h))) return st;
  if (back_projection_mode != B200RT_BACKPROJECT_ATOMIC && back_projection_mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  if (!h->use_paths || back_projection_mode != B200RT_BACKPROJECT_ATOMIC) {
    for (int b = 0; b < batch; ++b)
      if (int st = b200rt_log_likelihood_gradient_dev(h, images_dev + b * image_stride, y_dev + b * y_stride,
                                                      additive_dev ? additive_dev + b * additive_stride : nullptr,
                                                      mult_dev ? mult_dev + b * mult_stride : nullptr, subset_num,
                                                      num_subsets, zero_seg0_end_planes, back_projection_mode,
                                                      gradients_dev + b * gradient_stride, stream))
        return st;
    return B200RT_OK;
  }
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int n = 0;
    const int* list = path_list(*h, subset_num, num_subsets, n);
    // the gradient ratios of every image: projection data outside the subset stay zero (never written)
    const size_t need = static_cast<size_t>(pd_size(*h)) * batch;
    if (h->ratio_batch.n < need) {
      h->ratio_batch.alloc(need);
      ck(cudaMemsetAsync(h->ratio_batch.p, 0, sizeof(float) * need, st), "memset");
    }
    h->cancelled.alloc(1);
    ck(cudaMemsetAsync(h->cancelled.p, 0, sizeof(unsigned int), st), "memset");
    FwdEpilogue ep{};
    ep.mode = kEpiGradient;
    ep.zero_ends = zero_seg0_end_planes;
    ep.y = y_dev;
    ep.y_stride = y_stride;
    ep.add = additive_dev;
    ep.add_stride = additive_stride;
    ep.mult = mult_dev;
    ep.mult_stride = mult_stride;
    ep.cancelled = h->cancelled.p;
    ep.small_value = batch_thresholds(*h, y_dev, y_stride, batch, subset_num, num_subsets, zero_seg0_end_planes, st,
                                      ep.sv_stride);
    ck(launch_forward_paths_batch(h->params, h->pparams, list, n, images_dev, image_stride, h->ratio_batch.p,
                                  pd_size(*h), batch, st, &ep),
       "forward projection");
    for (int b = 0; b < batch; ++b)
      ck(cudaMemsetAsync(gradients_dev + b * gradient_stride, 0, sizeof(float) * g.image_size(), st), "memset");
    ck(launch_back_paths_atomic_batch(h->params, h->pparams, list, n, h->ratio_batch.p, pd_size(*h),
                                      gradients_dev, gradient_stride, batch, st, 0),
       "back projection");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"
