// C ABI: viewgram access and the subset forward / back projections (device and host buffers).
#include "capi.hpp"

using namespace b200;

namespace {

// the device-layout block of viewgram (segment, view, timing position): [tangential][axial], contiguous
const char* viewgram_block(const b200rt_projector& h, int seg, int view, int tof, int64_t& off, int& nax) {
  const Geometry& g = *h.geo;
  if (seg < -g.S() || seg > g.S()) return "segment out of range";
  if (view < 0 || view >= g.num_views()) return "view out of range";
  if (tof < g.min_tof() || tof >= g.min_tof() + g.num_tof()) return "timing position out of range";
  nax = g.nax(seg);
  off = static_cast<int64_t>(tof - g.min_tof()) * g.tof_stride() + g.dev_segment_offset(seg) +
        static_cast<int64_t>(view) * g.num_tang() * nax;
  return nullptr;
}

bool is_device_pointer(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" {

int b200rt_get_viewgram(b200rt_projector* h, const float* projdata_dev, int segment_num, int view_num,
                        int timing_pos_num, float* viewgram, void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_get_viewgram");
  if (!h || !projdata_dev || !viewgram) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  int64_t off = 0;
  int nax = 0;
  if (const char* why = viewgram_block(*h, segment_num, view_num, timing_pos_num, off, nax))
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, why);
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nt = h->geo->num_tang();
    const size_t n = static_cast<size_t>(nt) * nax;
    const bool dev_out = is_device_pointer(viewgram);
    float* dst = viewgram;
    if (!dev_out) {
      h->vg_scratch.alloc(std::max(h->vg_scratch.n, 2 * n));
      dst = h->vg_scratch.p;
    }
    ck(launch_transpose(projdata_dev + off, dst, nt, nax, nax, nt, st), "viewgram");
    if (!dev_out) {
      ck(cudaMemcpyAsync(viewgram, dst, sizeof(float) * n, cudaMemcpyDeviceToHost, st), "D2H");
      ck(cudaStreamSynchronize(st), "viewgram");
    }
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_set_viewgram(b200rt_projector* h, float* projdata_dev, int segment_num, int view_num, int timing_pos_num,
                        const float* viewgram, int accumulate, void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_set_viewgram");
  if (!h || !projdata_dev || !viewgram) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  int64_t off = 0;
  int nax = 0;
  if (const char* why = viewgram_block(*h, segment_num, view_num, timing_pos_num, off, nax))
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, why);
  try {
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nt = h->geo->num_tang();
    const size_t n = static_cast<size_t>(nt) * nax;
    h->vg_scratch.alloc(std::max(h->vg_scratch.n, 2 * n));
    const float* src = viewgram;
    if (!is_device_pointer(viewgram)) {
      ck(cudaMemcpyAsync(h->vg_scratch.p, viewgram, sizeof(float) * n, cudaMemcpyHostToDevice, st), "H2D");
      src = h->vg_scratch.p;
    }
    // [axial][tangential] -> [tangential][axial]
    if (accumulate) {
      ck(launch_transpose(src, h->vg_scratch.p + n, nax, nt, nt, nax, st), "viewgram");
      ck(launch_add(projdata_dev + off, h->vg_scratch.p + n, static_cast<int64_t>(n), st), "viewgram");
    } else {
      ck(launch_transpose(src, projdata_dev + off, nax, nt, nt, nax, st), "viewgram");
    }
    // the host source may be reused by the caller as soon as this returns
    if (src != viewgram) ck(cudaStreamSynchronize(st), "viewgram");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_forward_project_dev(b200rt_projector* h, const float* image_dev, float* projdata_dev, int subset_num,
                               int num_subsets, void* stream) {
  if (!h || !image_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    forward_subset(*h, image_dev, projdata_dev, subset_num, num_subsets, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_back_project_dev(b200rt_projector* h, const float* projdata_dev, float* image_dev, int subset_num,
                            int num_subsets, int mode, void* stream) {
  if (!h || !image_dev || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (mode != B200RT_BACKPROJECT_ATOMIC && mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    back_project_into(*h, projdata_dev, image_dev, subset_num, num_subsets, mode, 0, static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_forward_project(b200rt_projector* h, const float* image_host, float* projdata_host, int subset_num,
                           int num_subsets) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_forward_project");
  if (!h || !image_host || !projdata_host) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = h->stream;
    h->st_img_a.alloc(g.image_size());
    h->st_img_b.alloc(g.image_size());
    h->st_pd_a.alloc(g.projdata_size());
    h->st_pd_b.alloc(g.projdata_size());
    ck(cudaMemcpyAsync(h->st_img_a.p, image_host, sizeof(float) * g.image_size(), cudaMemcpyHostToDevice, st), "H2D");
    ck(launch_image_to_dev(h->st_img_a.p, h->st_img_b.p, g.desc().nz, g.desc().ny, g.desc().nx, st), "layout");
    ck(cudaMemsetAsync(h->st_pd_b.p, 0, sizeof(float) * g.projdata_size(), st), "memset");
    if (h->use_paths && h->paths_view_split) {
      // group by group of views: projection, layout change, then the group's copy to the host on the copy
      // stream while the next group is projected
      const b200rt_projector::ViewGroups& vg = view_groups(*h, subset_num, num_subsets);
      ensure_copy_stream(*h);
      for (size_t gi = 0; gi + 1 < vg.v0.size(); ++gi) {
        const int n = vg.off[gi + 1] - vg.off[gi];
        if (n > 0)
          ck(launch_forward_paths(h->params, h->pparams, vg.list->p + vg.off[gi], n, h->st_img_b.p, h->st_pd_b.p, st,
                                  nullptr),
             "forward projection");
        ck(projdata_layout_views(*h, h->st_pd_b.p, h->st_pd_a.p, false, vg.v0[gi], vg.v0[gi + 1], st), "layout");
        ck(cudaEventRecord(h->copy_events[gi], st), "cudaEventRecord");
        ck(cudaStreamWaitEvent(h->copy_stream, h->copy_events[gi], 0), "cudaStreamWaitEvent");
        ck(copy_views(g, projdata_host, h->st_pd_a.p, vg.v0[gi], vg.v0[gi + 1], cudaMemcpyDeviceToHost, h->copy_stream),
           "D2H");
      }
      ck(cudaStreamSynchronize(h->copy_stream), "forward projection");
      ck(cudaStreamSynchronize(st), "forward projection");
      return B200RT_OK;
    }
    forward_subset(*h, h->st_img_b.p, h->st_pd_b.p, subset_num, num_subsets, st);
    ck(projdata_layout(*h, h->st_pd_b.p, h->st_pd_a.p, false, st), "layout");
    ck(cudaMemcpyAsync(projdata_host, h->st_pd_a.p, sizeof(float) * g.projdata_size(), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "forward projection");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_back_project(b200rt_projector* h, const float* projdata_host, float* image_host, int subset_num,
                        int num_subsets, int mode) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_back_project");
  if (!h || !image_host || !projdata_host) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (mode != B200RT_BACKPROJECT_ATOMIC && mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    const Geometry& g = *h->geo;
    const cudaStream_t st = h->stream;
    h->st_img_a.alloc(g.image_size());
    h->st_img_b.alloc(g.image_size());
    h->st_pd_a.alloc(g.projdata_size());
    h->st_pd_b.alloc(g.projdata_size());
    if (h->use_paths && h->paths_view_split && mode == B200RT_BACKPROJECT_ATOMIC) {
      // group by group of views: the copy stream brings the groups' data in order, the projection stream
      // changes each group's layout and back-projects its items as soon as its data are in
      const b200rt_projector::ViewGroups& vg = view_groups(*h, subset_num, num_subsets);
      ensure_copy_stream(*h);
      const size_t G = vg.v0.size() - 1;
      ck(cudaEventRecord(h->copy_events[G], st), "cudaEventRecord");  // staging buffers free
      ck(cudaStreamWaitEvent(h->copy_stream, h->copy_events[G], 0), "cudaStreamWaitEvent");
      for (size_t gi = 0; gi < G; ++gi) {
        ck(copy_views(g, h->st_pd_a.p, projdata_host, vg.v0[gi], vg.v0[gi + 1], cudaMemcpyHostToDevice, h->copy_stream),
           "H2D");
        ck(cudaEventRecord(h->copy_events[gi], h->copy_stream), "cudaEventRecord");
      }
      ck(cudaMemsetAsync(h->st_img_b.p, 0, sizeof(float) * g.image_size(), st), "memset");
      for (size_t gi = 0; gi < G; ++gi) {
        ck(cudaStreamWaitEvent(st, h->copy_events[gi], 0), "cudaStreamWaitEvent");
        ck(projdata_layout_views(*h, h->st_pd_a.p, h->st_pd_b.p, true, vg.v0[gi], vg.v0[gi + 1], st), "layout");
        const int n = vg.off[gi + 1] - vg.off[gi];
        if (n > 0)
          ck(launch_back_paths_atomic(h->params, h->pparams, vg.list->p + vg.off[gi], n, h->st_pd_b.p, h->st_img_b.p,
                                      st, 0),
             "back projection");
      }
    } else {
      ck(cudaMemcpyAsync(h->st_pd_a.p, projdata_host, sizeof(float) * g.projdata_size(), cudaMemcpyHostToDevice, st),
         "H2D");
      ck(projdata_layout(*h, h->st_pd_a.p, h->st_pd_b.p, true, st), "layout");
      back_project_into(*h, h->st_pd_b.p, h->st_img_b.p, subset_num, num_subsets, mode, 0, st);
    }
    ck(launch_image_from_dev(h->st_img_b.p, h->st_img_a.p, g.desc().nz, g.desc().ny, g.desc().nx, st), "layout");
    ck(cudaMemcpyAsync(image_host, h->st_img_a.p, sizeof(float) * g.image_size(), cudaMemcpyDeviceToHost, st), "D2H");
    ck(cudaStreamSynchronize(st), "back projection");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_sensitivity_dev(b200rt_projector* h, const float* mult_dev, float* sens_dev, int subset_num, int num_subsets,
                           int zero_seg0_end_planes, int back_projection_mode, void* stream) {
  if (!h || !sens_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (int st = check_subset(h, subset_num, num_subsets)) return st;
  if (back_projection_mode != B200RT_BACKPROJECT_ATOMIC && back_projection_mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return fail(h, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  try {
    DeviceGuard dg(h->device);
    back_project_into(*h, mult_dev, sens_dev, subset_num, num_subsets, back_projection_mode, zero_seg0_end_planes,
                      static_cast<cudaStream_t>(stream));
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"
