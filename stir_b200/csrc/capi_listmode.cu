// C ABI: the list-mode objective.
#include "capi.hpp"

using namespace b200;

namespace {

void ensure_lm_table(b200rt_projector& h) {
  if (h.lm_table.p) return;
  const Geometry& g = *h.geo;
  const int nseg = 2 * g.S() + 1, nv = g.num_views(), nt = g.num_tang(), ntof = g.num_tof();
  std::vector<int4> table(static_cast<size_t>(ntof) * nseg * nv * nt, make_int4(-1, -1, -1, 0));
  for (int b = 0; b < static_cast<int>(h.h_bins.size()); ++b) {
    const ProjBinDev& pb = h.h_bins[b];
    for (int l = 0; l < pb.num_lines; ++l) {
      const LineDev& L = h.h_lines[pb.first_line + l];
      const int tang = L.tang_sign * pb.tang;
      if (tang < g.min_tang() || tang > g.max_tang()) continue;
      const size_t k = ((static_cast<size_t>(pb.tof - g.min_tof()) * nseg + (L.seg + g.S())) * nv + L.view) * nt +
                       (tang - g.min_tang());
      table[k] = make_int4(b, l, h.h_bin_view[b], 0);
    }
  }
  h.lm_table.upload(table, h.stream);
  h.lm_invalid.alloc(1);
  ck(cudaMemsetAsync(h.lm_invalid.p, 0, sizeof(unsigned), h.stream), "memset");
  ck(cudaStreamSynchronize(h.stream), "list-mode table");
}

int lm_check(b200rt_projector* h, const b200rt_lm_event* ev, int64_t n, const float* x, int subset, int nsub) {
  if (!h || (!ev && n > 0) || !x || n < 0) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  return check_subset(h, subset, nsub);
}

// binned (projection kernels over the subset) or per event (one row walk per event): automatically binned once
// the events number at least 1/16 of the bins, where two whole-subset projections cost less than the events'
// rows (on the clinical geometry a forward plus a back projection take ~0.4 ns per bin, a row walk ~5 ns per
// event)
bool lm_binned(const b200rt_projector& h, int64_t n) {
  if (h.lm_method == B200RT_LISTMODE_PER_EVENT) return false;
  if (h.lm_method == B200RT_LISTMODE_BINNED) return n > 0;
  return n > 0 && n * 16 >= h.geo->projdata_size();
}

// A x of the subset into buf (device layout).  The buffer is zeroed when allocated: a bin no line reaches is
// never written and reads as 0, as its empty row would give.
const float* lm_forward(b200rt_projector& h, DevBuf<float>& buf, const float* x, int subset, int nsub,
                        cudaStream_t st) {
  const size_t np = static_cast<size_t>(h.geo->projdata_size());
  if (buf.n != np) {
    buf.alloc(np);
    ck(cudaMemsetAsync(buf.p, 0, sizeof(float) * np, st), "memset");
  }
  forward_subset(h, x, buf.p, subset, nsub, st);
  return buf.p;
}

float* lm_zeroed_hist(b200rt_projector& h, cudaStream_t st) {
  const size_t np = static_cast<size_t>(h.geo->projdata_size());
  h.lm_hist.alloc(np);
  ck(cudaMemsetAsync(h.lm_hist.p, 0, sizeof(float) * np, st), "memset");
  return h.lm_hist.p;
}

// out = A^T hist over the subset, or out += it
void lm_back(b200rt_projector& h, int subset, int nsub, int accumulate, float* out, cudaStream_t st) {
  if (!accumulate) {
    back_project_into(h, h.lm_hist.p, out, subset, nsub, B200RT_BACKPROJECT_ATOMIC, 0, st);
    return;
  }
  const int64_t ni = h.geo->image_size();
  h.lm_img.alloc(ni);
  back_project_into(h, h.lm_hist.p, h.lm_img.p, subset, nsub, B200RT_BACKPROJECT_ATOMIC, 0, st);
  ck(launch_add(out, h.lm_img.p, ni, st), "add");
}

}  // namespace

static_assert(sizeof(b200rt_lm_event) == sizeof(LmEventDev), "list-mode event layouts agree");

extern "C" {

int b200rt_listmode_gradient_dev(b200rt_projector* h, const b200rt_lm_event* events_dev, int64_t num_events,
                                 const float* image_dev, int subset_num, int num_subsets, int has_add,
                                 const float* subset_sensitivity_dev, int accumulate, float* gradient_dev,
                                 void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_listmode_gradient_dev");
  if (int st = lm_check(h, events_dev, num_events, image_dev, subset_num, num_subsets)) return st;
  if (!gradient_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t ni = h->geo->image_size();
    const auto* ev = reinterpret_cast<const LmEventDev*>(events_dev);
    if (lm_binned(*h, num_events)) {
      const float* fwd = lm_forward(*h, h->lm_fwd, image_dev, subset_num, num_subsets, st);
      ck(launch_listmode_binned(h->params, h->lm_table.p, ev, num_events, 0, fwd, nullptr, subset_num, num_subsets,
                                has_add, lm_zeroed_hist(*h, st), nullptr, h->lm_invalid.p, st),
         "list-mode gradient");
      lm_back(*h, subset_num, num_subsets, accumulate, gradient_dev, st);
    } else {
      if (!accumulate) ck(cudaMemsetAsync(gradient_dev, 0, sizeof(float) * ni, st), "memset");
      if (num_events > 0)
        ck(launch_listmode(h->params, h->lm_table.p, ev, num_events, 0, image_dev, nullptr, subset_num, num_subsets,
                           has_add, gradient_dev, nullptr, h->lm_invalid.p, st),
           "list-mode gradient");
    }
    if (subset_sensitivity_dev) ck(launch_subtract(gradient_dev, subset_sensitivity_dev, ni, st), "subtract");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_listmode_value_dev(b200rt_projector* h, const b200rt_lm_event* events_dev, int64_t num_events,
                              const float* image_dev, int subset_num, int num_subsets, int has_add, double* value,
                              void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_listmode_value_dev");
  if (int st = lm_check(h, events_dev, num_events, image_dev, subset_num, num_subsets)) return st;
  if (!value) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const auto* ev = reinterpret_cast<const LmEventDev*>(events_dev);
    const bool binned = lm_binned(*h, num_events);
    const int nb = binned ? listmode_binned_num_blocks(num_events) : listmode_num_blocks(num_events);
    h->lm_partial.alloc(std::max<size_t>(h->lm_partial.n, static_cast<size_t>(nb)));
    h->lm_sum.alloc(1);
    if (binned) {
      const float* fwd = lm_forward(*h, h->lm_fwd, image_dev, subset_num, num_subsets, st);
      ck(launch_listmode_binned(h->params, h->lm_table.p, ev, num_events, 1, fwd, nullptr, subset_num, num_subsets,
                                has_add, nullptr, h->lm_partial.p, h->lm_invalid.p, st),
         "list-mode value");
    } else {
      ck(launch_listmode(h->params, h->lm_table.p, ev, num_events, 1, image_dev, nullptr, subset_num, num_subsets,
                         has_add, nullptr, h->lm_partial.p, h->lm_invalid.p, st),
         "list-mode value");
    }
    ck(launch_reduce_sum(h->lm_partial.p, nb, h->lm_sum.p, st), "list-mode value");
    ck(cudaMemcpyAsync(value, h->lm_sum.p, sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "list-mode value");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_listmode_hessian_times_input_dev(b200rt_projector* h, const b200rt_lm_event* events_dev,
                                            int64_t num_events, const float* image_dev, const float* rhs_dev,
                                            int subset_num, int num_subsets, int has_add, float* output_dev,
                                            void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_listmode_hessian_times_input_dev");
  if (int st = lm_check(h, events_dev, num_events, image_dev, subset_num, num_subsets)) return st;
  if (!rhs_dev || !output_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const auto* ev = reinterpret_cast<const LmEventDev*>(events_dev);
    if (lm_binned(*h, num_events)) {
      const float* fwd = lm_forward(*h, h->lm_fwd, image_dev, subset_num, num_subsets, st);
      const float* fwd_rhs = lm_forward(*h, h->lm_fwd_rhs, rhs_dev, subset_num, num_subsets, st);
      ck(launch_listmode_binned(h->params, h->lm_table.p, ev, num_events, 2, fwd, fwd_rhs, subset_num, num_subsets,
                                has_add, lm_zeroed_hist(*h, st), nullptr, h->lm_invalid.p, st),
         "list-mode Hessian");
      lm_back(*h, subset_num, num_subsets, 1, output_dev, st);
    } else if (num_events > 0) {
      ck(launch_listmode(h->params, h->lm_table.p, ev, num_events, 2, image_dev, rhs_dev, subset_num, num_subsets,
                         has_add, output_dev, nullptr, h->lm_invalid.p, st),
         "list-mode Hessian");
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_listmode_set_method(b200rt_projector* h, int method) {
  if (!h) return B200RT_ERR_INVALID_ARGUMENT;
  if (method != B200RT_LISTMODE_AUTO && method != B200RT_LISTMODE_PER_EVENT && method != B200RT_LISTMODE_BINNED)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown list-mode method");
  h->lm_method = method;
  return B200RT_OK;
}

int b200rt_listmode_num_invalid(b200rt_projector* h, int64_t* count) {
  if (!h || !count) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    DeviceGuard dg(h->device);
    ensure_lm_table(*h);
    unsigned v = 0;
    ck(cudaMemcpy(&v, h->lm_invalid.p, sizeof(unsigned), cudaMemcpyDeviceToHost), "D2H");
    ck(cudaMemset(h->lm_invalid.p, 0, sizeof(unsigned)), "memset");
    *count = v;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"
