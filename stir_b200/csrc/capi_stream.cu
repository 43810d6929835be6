// C ABI: projection data as Interfile byte streams on the device.
#include "capi.hpp"

using namespace b200;

namespace {

// the stream's segment groups for the projector's segments and timing positions; throws on a mismatch
std::vector<StreamSegment> stream_plan(const Geometry& g, const b200rt_stream_format& f, int64_t& total_elems) {
  if (f.storage_order != B200RT_STORAGE_SEGMENT_VIEW_AXIAL_TANG && f.storage_order != B200RT_STORAGE_SEGMENT_AXIAL_VIEW_TANG)
    throw std::invalid_argument("unsupported storage order");
  if (numeric_type_size(f.number_type) == 0) throw std::invalid_argument("unknown number type");
  if (f.num_segments < 1 || !f.segment_sequence || !f.num_axial_poss)
    throw std::invalid_argument("the stream needs its segment sequence and axial sizes");
  if (f.num_timing_poss != g.num_tof())
    throw std::invalid_argument("the stream's number of timing positions differs from the projector's");
  const int64_t nvt = static_cast<int64_t>(g.num_views()) * g.num_tang();
  int64_t size3d = 0;
  for (int i = 0; i < f.num_segments; ++i) {
    if (f.num_axial_poss[i] < 0) throw std::invalid_argument("negative axial size");
    size3d += f.num_axial_poss[i] * nvt;
  }
  total_elems = size3d * f.num_timing_poss;
  std::vector<StreamSegment> plan;
  for (int k = 0; k < g.num_tof(); ++k) {
    int ti = k;  // the stream's index of timing position min_tof + k
    if (f.timing_poss_sequence) {
      ti = -1;
      for (int i = 0; i < f.num_timing_poss; ++i)
        if (f.timing_poss_sequence[i] == g.min_tof() + k) ti = i;
      if (ti < 0) throw std::invalid_argument("a timing position of the projector is missing from the stream");
    }
    for (int s = -g.S(); s <= g.S(); ++s) {
      int64_t off = 0;
      int idx = -1;
      for (int i = 0; i < f.num_segments && idx < 0; ++i) {
        if (f.segment_sequence[i] == s)
          idx = i;
        else
          off += f.num_axial_poss[i] * nvt;
      }
      if (idx < 0) throw std::invalid_argument("segment " + std::to_string(s) + " is missing from the stream");
      if (f.num_axial_poss[idx] != g.nax(s))
        throw std::invalid_argument("segment " + std::to_string(s) + " has another number of axial positions");
      StreamSegment ss{};
      ss.order = f.storage_order == B200RT_STORAGE_SEGMENT_AXIAL_VIEW_TANG ? kStorageSegmentAxialViewTang
                                                                           : kStorageSegmentViewAxialTang;
      ss.type = f.number_type;
      ss.swap = f.swap_bytes ? 1 : 0;
      ss.scale = f.scale_factor;
      ss.nax = g.nax(s);
      ss.nv = g.num_views();
      ss.nt = g.num_tang();
      ss.stream_elem = ti * size3d + off;
      ss.dev_off = k * g.tof_stride() + g.dev_segment_offset(s);
      plan.push_back(ss);
    }
  }
  return plan;
}

}  // namespace

extern "C" {

int b200rt_stream_bytes(b200rt_projector* h, const b200rt_stream_format* fmt, int64_t* bytes) {
  if (!h || !fmt || !bytes) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    int64_t n = 0;
    stream_plan(*h->geo, *fmt, n);
    *bytes = n * numeric_type_size(fmt->number_type);
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_projdata_from_stream_dev(b200rt_projector* h, const void* stream_dev, int64_t stream_bytes,
                                    const b200rt_stream_format* fmt, float* projdata_dev, void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_projdata_from_stream_dev");
  if (!h || !stream_dev || !fmt || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  try {
    int64_t n = 0;
    const std::vector<StreamSegment> plan = stream_plan(*h->geo, *fmt, n);
    if (stream_bytes < n * numeric_type_size(fmt->number_type))
      return fail(h, B200RT_ERR_INVALID_ARGUMENT, "the stream is shorter than its format says");
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (const StreamSegment& ss : plan) ck(launch_stream_segment(ss, true, stream_dev, projdata_dev, st), "stream read");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

int b200rt_projdata_to_stream_dev(b200rt_projector* h, const float* projdata_dev, const b200rt_stream_format* fmt,
                                  void* stream_dev, int64_t stream_bytes, void* stream) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_projdata_to_stream_dev");
  if (!h || !stream_dev || !fmt || !projdata_dev) return fail(h, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (fmt->number_type != B200RT_NUMBER_FLOAT && fmt->number_type != B200RT_NUMBER_DOUBLE)
    return fail(h, B200RT_ERR_UNSUPPORTED, "streams are written as float or double");
  if (fmt->scale_factor != 1.f) return fail(h, B200RT_ERR_UNSUPPORTED, "streams are written with scale factor 1");
  try {
    int64_t n = 0;
    const std::vector<StreamSegment> plan = stream_plan(*h->geo, *fmt, n);
    if (stream_bytes < n * numeric_type_size(fmt->number_type))
      return fail(h, B200RT_ERR_INVALID_ARGUMENT, "the stream is shorter than its format says");
    DeviceGuard dg(h->device);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (const StreamSegment& ss : plan) ck(launch_stream_segment(ss, false, projdata_dev, stream_dev, st), "stream write");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return fail(h, status_of(e), e.what());
  }
}

}  // extern "C"
