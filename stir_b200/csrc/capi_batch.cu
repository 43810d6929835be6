// C ABI: batched OSMAPOSL reconstructions (several frames per sub-iteration).
#include "capi.hpp"

using namespace b200;

// ---- batched OSMAPOSL ---------------------------------------------------------------------------
// Frames of a batch advance together.  Each batched sub-iteration is, on one stream:
//   per frame: viewgram thresholds of its subset, zero the cancelled count and the numerator
//   one persistent forward launch over the (frame, basic bin) items of every frame's subset, writing
//     divide_and_truncate(y, A x + a) into the frame's ratio buffer
//   one persistent back projection of those ratios into the frames' numerators
//   per frame: the update (division by the sensitivity or the MAP-OSL denominator, clamp, x *= u).
// Items are frame-major, so the CTAs share one or two frames' images in L2 at a time.  Everything the
// sequence touches is allocated and uploaded before it runs, so that it can be captured in a CUDA graph.

struct b200rt_batch {
  struct Frame {
    b200rt_projector* h = nullptr;
    int geom = 0;
    float* x = nullptr;
    const float* y = nullptr;
    const float* add = nullptr;
    std::vector<const float*> sens;
    int nsub = 1, start_subset = 0, num_subiters = 0, zero_ends = 0;
    bool has_prior = false;
    b200rt_prior prior{};
    float prior_w[27] = {0};
    float min_rel = 0.f, max_rel = 0.f;
    DevBuf<float> ratio, u, grad, small_value, partial_max, umax;
    DevBuf<unsigned int> cancelled;
    // B200RT_BACKPROJECT_DETERMINISTIC: fixed-point numerator, its scale (from the ratio's bound 1e4 and the
    // projector's largest column sum, as the frame's own back projection), the bound and a reduction scratch
    int mode = B200RT_BACKPROJECT_ATOMIC;
    DevBuf<unsigned long long> acc64;
    DevBuf<double> fixed_scale;
    DevBuf<float> bound, det_partial;
  };
  int device = 0;
  std::string err;
  std::vector<std::unique_ptr<Frame>> frames;
  std::vector<b200rt_projector*> geoms;
  DevBuf<b200::ProjParams> d_geoms;
  DevBuf<b200::PathParams> d_pgeoms;
  // kernel families (index B200RT_BATCH_KERNELS_*) the frames allow, the one in use, and each one's most
  // persistent CTAs per SM (forward, back)
  bool avail[5] = {false, false, false, false, false};
  int family = B200RT_BATCH_KERNELS_PATHS;
  int max_f[5] = {0, 0, 0, 0, 0}, max_b[5] = {0, 0, 0, 0, 0};
  int num_tof = 1;
  int smem_f = 0, smem_b = 0;
  DevBuf<b200::BatchFrameDev> d_frames;
  DevBuf<unsigned int> counters;  // work-queue heads of the forward and back launches
  bool ready = false;
  int npa = 0;
  size_t smem = 0;
  int num_sms = 0, max_fwd = 0, max_back = 0;
  b200rt_batch_config cfg{0, 0, 0, B200RT_BATCH_KERNELS_AUTO};
  // item lists by (order, subset of each frame or -1)
  std::map<std::vector<int>, std::unique_ptr<DevBuf<b200::BatchItem>>> items;
  std::map<std::vector<int>, int> item_counts;
  std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
  // per batched sub-iteration: the update arguments of its frames (device table), their count, the most blocks
  std::map<int, std::unique_ptr<DevBuf<b200::BatchUpdateDev>>> updates;
  std::map<int, std::pair<int, int>> update_counts;
  cudaStream_t capture_stream = nullptr;
};

namespace {


int bfail(b200rt_batch* b, int code, const std::string& msg) {
  if (b) b->err = msg;
  return code;
}

void drop_graphs(b200rt_batch& b) {
  for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
  b.graphs.clear();
}

int frame_subset(const b200rt_batch::Frame& f, int k) { return (f.start_subset + k - 1) % f.nsub; }

// makes `kernels` (B200RT_BATCH_KERNELS_*; AUTO: the first the frames allow) the family in use
void use_family(b200rt_batch& b, int kernels) {
  int f = kernels;
  if (f == B200RT_BATCH_KERNELS_AUTO)
    for (int c : {B200RT_BATCH_KERNELS_PATHS, B200RT_BATCH_KERNELS_TOF_GROUPED, B200RT_BATCH_KERNELS_PACKED,
                  B200RT_BATCH_KERNELS_BASIC_BINS})
      if (b.avail[c]) {
        f = c;
        break;
      }
  if (f < B200RT_BATCH_KERNELS_PATHS || f > B200RT_BATCH_KERNELS_BASIC_BINS || !b.avail[f])
    throw std::invalid_argument("the batch's frames do not allow that kernel family");
  if (b.max_f[f] < 1 || b.max_b[f] < 1) throw std::runtime_error("batched projector does not fit on an SM");
  b.family = f;
  b.max_fwd = b.max_f[f];
  b.max_back = b.max_b[f];
}

// device tables and per-frame scratch; done once after the last add_frame
void batch_finalize(b200rt_batch& b) {
  if (b.ready) return;
  std::vector<b200::ProjParams> gp;
  int npa = -1, max_row = 1;
  for (auto* h : b.geoms) {
    gp.push_back(h->params);
    npa = npa < 0 ? h->params.uniform_npa : (npa == h->params.uniform_npa ? npa : 0);
    max_row = std::max(max_row, h->params.max_row_len);
  }
  b.npa = npa < 0 ? 0 : npa;
  b.smem = b200::proj_smem_bytes(max_row);
  cudaStream_t st = b.capture_stream;
  b.d_geoms.upload(gp, st);
  bool paths = true, tof_grouped = true, packed = true, deterministic = false;
  b.num_tof = b.geoms.empty() ? 1 : b.geoms[0]->params.num_tof;
  for (auto* h : b.geoms) {
    paths = paths && h->use_paths;
    // one timing-bin count for the whole batch (the kernels' group size)
    tof_grouped = tof_grouped && h->params.tof_w != nullptr && h->params.num_tof == b.num_tof;
    packed = packed && h->params.max_nax <= b200::kPackedMaxNax;
  }
  for (auto& fp : b.frames) deterministic = deterministic || fp->mode == B200RT_BACKPROJECT_DETERMINISTIC;
  if (deterministic && !paths) throw std::invalid_argument("deterministic batched frames need the column-staged kernels");
  // the fixed-point numerators exist in the column-staged kernels only
  b.avail[B200RT_BATCH_KERNELS_PATHS] = paths;
  b.avail[B200RT_BATCH_KERNELS_TOF_GROUPED] = tof_grouped && !deterministic;
  b.avail[B200RT_BATCH_KERNELS_PACKED] = packed && !deterministic;
  b.avail[B200RT_BATCH_KERNELS_BASIC_BINS] = !deterministic;
  if (paths) {
    std::vector<b200::PathParams> pg;
    b.smem_f = b.smem_b = 0;
    for (auto* h : b.geoms) {
      const b200::PathParams& pp = h->pparams;
      pg.push_back(pp);
      b.smem_f = std::max(b.smem_f, b200::path_smem_fwd(pp.K, h->params.nz, pp.zpad, pp.max_lines, pp.max_acc,
                                                          pp.npa_max).total);
      b.smem_b = std::max(b.smem_b, b200::path_smem_back(h->params.nz, pp.max_lines, pp.max_members, pp.nax_max,
                                                          pp.npa_max).total);
    }
    b.d_pgeoms.upload(pg, st);
  }
  std::vector<BatchFrameDev> fd;
  for (auto& fp : b.frames) {
    auto& f = *fp;
    const b200::Geometry& g = *f.h->geo;
    f.ratio.alloc(g.projdata_size());
    f.u.alloc(g.image_size());
    if (f.has_prior) f.grad.alloc(g.image_size());
    f.small_value.alloc(static_cast<size_t>(g.num_tof()) * (2 * g.S() + 1) * g.num_views());
    f.partial_max.alloc(b200::update_num_blocks(g.image_size()));
    f.umax.alloc(1);
    f.cancelled.alloc(1);
    for (int s = 0; s < f.nsub; ++s) {
      int nv = 0;
      subset_views(*f.h, s, f.nsub, nv);  // cached device view lists, uploaded now
    }
    {
      int nv = 0;
      subset_views(*f.h, 0, 1, nv);  // all views, for the thresholds
    }
    if (f.mode == B200RT_BACKPROJECT_DETERMINISTIC) {
      f.acc64.alloc(g.image_size());
      f.fixed_scale.alloc(1);
      f.det_partial.alloc(1);
      const float bound = 10000.F;  // the ratio's clip (divide_and_truncate): the scale does not depend on data
      f.bound.upload(std::vector<float>{bound}, st);
      ensure_colmax(*f.h, f.u.p, st);
      ck(launch_fixed_scale(f.bound.p, 1, f.h->colmax.p, f.det_partial.p, f.fixed_scale.p, st), "scale");
    }
    BatchFrameDev d{};
    d.geom = f.geom;
    d.x = f.x;
    d.ratio = f.ratio.p;
    d.u = f.u.p;
    d.acc64 = f.mode == B200RT_BACKPROJECT_DETERMINISTIC ? f.acc64.p : nullptr;
    d.fixed_scale = f.mode == B200RT_BACKPROJECT_DETERMINISTIC ? f.fixed_scale.p : nullptr;
    d.ep.mode = b200::kEpiRatio;
    d.ep.zero_ends = f.zero_ends;
    d.ep.y = f.y;
    d.ep.add = f.add;
    d.ep.small_value = f.small_value.p;
    d.ep.cancelled = f.cancelled.p;
    fd.push_back(d);
  }
  b.d_frames.upload(fd, st);
  b.counters.alloc(2);
  ck(cudaDeviceGetAttribute(&b.num_sms, cudaDevAttrMultiProcessorCount, b.device), "device attribute");
  if (b.avail[B200RT_BATCH_KERNELS_PATHS]) {
    b.max_f[B200RT_BATCH_KERNELS_PATHS] = b200::batch_paths_max_ctas_per_sm(b.npa, b.smem_f, true);
    b.max_b[B200RT_BATCH_KERNELS_PATHS] = b200::batch_paths_max_ctas_per_sm(b.npa, b.smem_b, false);
  }
  if (b.avail[B200RT_BATCH_KERNELS_TOF_GROUPED]) {
    b.max_f[B200RT_BATCH_KERNELS_TOF_GROUPED] = b200::batch_tof_max_ctas_per_sm(b.num_tof, true);
    b.max_b[B200RT_BATCH_KERNELS_TOF_GROUPED] = b200::batch_tof_max_ctas_per_sm(b.num_tof, false);
  }
  if (b.avail[B200RT_BATCH_KERNELS_PACKED]) {
    b.max_f[B200RT_BATCH_KERNELS_PACKED] = b200::batch_packed_max_ctas_per_sm(true);
    b.max_b[B200RT_BATCH_KERNELS_PACKED] = b200::batch_packed_max_ctas_per_sm(false);
  }
  if (b.avail[B200RT_BATCH_KERNELS_BASIC_BINS]) {
    b.max_f[B200RT_BATCH_KERNELS_BASIC_BINS] = b200::batch_max_ctas_per_sm(b.npa, b.smem, true);
    b.max_b[B200RT_BATCH_KERNELS_BASIC_BINS] = b200::batch_max_ctas_per_sm(b.npa, b.smem, false);
  }
  for (int f = B200RT_BATCH_KERNELS_PATHS; f <= B200RT_BATCH_KERNELS_BASIC_BINS; ++f)  // a family that does not fit
    if (b.avail[f] && (b.max_f[f] < 1 || b.max_b[f] < 1)) b.avail[f] = false;      // an SM is not offered
  use_family(b, b.cfg.kernels);
  ck(cudaStreamSynchronize(st), "batch set-up");
  b.ready = true;
}

// the (frame, basic bin) work of batched sub-iteration k, uploaded on first use
const BatchItem* batch_items(b200rt_batch& b, int k, int order, int& count) {
  std::vector<int> key{order, b.family};
  for (auto& f : b.frames) key.push_back(k <= f->num_subiters ? frame_subset(*f, k) : -1);
  auto it = b.items.find(key);
  if (it != b.items.end()) {
    count = b.item_counts[key];
    return it->second->p;
  }
  std::vector<BatchItem> list;
  std::vector<std::vector<int>> per_frame(b.frames.size());
  for (size_t fi = 0; fi < b.frames.size(); ++fi) {
    if (key[fi + 2] < 0) continue;
    const auto& f = *b.frames[fi];
    const b200rt_projector& h = *f.h;
    std::vector<int> bins;  // basic bins, or path items with the column-staged kernels
    if (b.family == B200RT_BATCH_KERNELS_PATHS) {
      for (int i = 0; i < static_cast<int>(h.h_item_view.size()); ++i)
        if (h.h_item_view[i] % f.nsub == key[fi + 2]) bins.push_back(i);
      if (order == 1) {
        std::stable_sort(bins.begin(), bins.end(), [&](int a, int c) {
          const auto& pa = h.h_path_items[a];
          const auto& pc = h.h_path_items[c];
          return static_cast<int64_t>(pa.ncols) * pa.num_lines > static_cast<int64_t>(pc.ncols) * pc.num_lines;
        });
      }
    } else if (b.family == B200RT_BATCH_KERNELS_TOF_GROUPED) {
      for (int bin = 0; bin < static_cast<int>(h.h_tof_basic_view.size()); ++bin)
        if (h.h_tof_basic_view[bin] % f.nsub == key[fi + 2]) bins.push_back(bin);
    } else {
      for (int bin = 0; bin < static_cast<int>(h.h_bins.size()); ++bin)
        if (h.h_bin_view[bin] % f.nsub == key[fi + 2]) bins.push_back(bin);
      if (order == 1) {
        std::stable_sort(bins.begin(), bins.end(), [&](int a, int c) {
          const auto& pa = h.h_bins[a];
          const auto& pc = h.h_bins[c];
          return static_cast<int64_t>(pa.row_len) * pa.num_lines > static_cast<int64_t>(pc.row_len) * pc.num_lines;
        });
      }
    }
    per_frame[fi] = std::move(bins);
  }
  if (order == 2) {
    // item-major: frames of one geometry in the same subset take each work item in turn, so that its row is read
    // from HBM once for all of them
    std::vector<bool> done(b.frames.size(), false);
    for (size_t fi = 0; fi < b.frames.size(); ++fi) {
      if (done[fi] || key[fi + 2] < 0) continue;
      std::vector<size_t> group;
      for (size_t fj = fi; fj < b.frames.size(); ++fj)
        if (!done[fj] && key[fj + 2] == key[fi + 2] && b.frames[fj]->geom == b.frames[fi]->geom &&
            b.frames[fj]->nsub == b.frames[fi]->nsub) {
          group.push_back(fj);
          done[fj] = true;
        }
      for (size_t i = 0; i < per_frame[fi].size(); ++i)
        for (size_t fj : group) list.push_back(BatchItem{static_cast<int>(fj), per_frame[fj][i]});
    }
  } else {
    for (size_t fi = 0; fi < b.frames.size(); ++fi)
      for (int bin : per_frame[fi]) list.push_back(BatchItem{static_cast<int>(fi), bin});
  }
  auto buf = std::make_unique<DevBuf<BatchItem>>();
  buf->upload(list, b.capture_stream);
  ck(cudaStreamSynchronize(b.capture_stream), "batch items");
  count = static_cast<int>(list.size());
  b.item_counts[key] = count;
  const BatchItem* p = buf->p;
  b.items[key] = std::move(buf);
  return p;
}

int grid_of(const b200rt_batch& b, int per_sm, int max_per_sm) {
  const int c = per_sm > 0 ? std::min(per_sm, max_per_sm) : max_per_sm;
  return c * b.num_sms;
}

// divide_and_truncate's threshold of every viewgram of every frame taking part in sub-iterations first.. (it
// depends on the data only, so once per run covers all the run's subsets)
void batch_thresholds(b200rt_batch& b, int first, cudaStream_t st) {
  for (auto& fp : b.frames) {
    auto& f = *fp;
    if (first > f.num_subiters) continue;
    const b200::Geometry& g = *f.h->geo;
    int nv = 0;
    const int* views = subset_views(*f.h, 0, 1, nv);
    ck(launch_viewgram_small_values(f.y, f.h->segs.p, g.S(), g.num_views(), g.num_tang(), views, nv, f.zero_ends,
                                    g.num_tof(), g.tof_stride(), f.small_value.p, st),
       "viewgram thresholds");
  }
}

// zero the numerators and cancelled counts of the frames taking part in sub-iteration k
void batch_zero(b200rt_batch& b, int k, cudaStream_t st) {
  for (auto& fp : b.frames) {
    auto& f = *fp;
    if (k > f.num_subiters) continue;
    ck(cudaMemsetAsync(f.cancelled.p, 0, sizeof(unsigned int), st), "memset");
    if (f.mode == B200RT_BACKPROJECT_DETERMINISTIC)
      ck(cudaMemsetAsync(f.acc64.p, 0, sizeof(unsigned long long) * f.h->geo->image_size(), st), "memset");
    else
      ck(cudaMemsetAsync(f.u.p, 0, sizeof(float) * f.h->geo->image_size(), st), "memset");
  }
}

// one batched launch of one direction (0 forward with the ratio epilogue, 1 back projection of the ratios)
cudaError_t batch_launch(b200rt_batch& b, int dir, const BatchItem* items, int n, int grid, cudaStream_t st) {
  if (b.family == B200RT_BATCH_KERNELS_PATHS)
    return dir == 0 ? b200::launch_forward_batch_paths(b.d_geoms.p, b.d_pgeoms.p, b.npa, b.smem_f, b.d_frames.p, items,
                                                       n, b.counters.p, grid, st)
                    : b200::launch_back_batch_paths(b.d_geoms.p, b.d_pgeoms.p, b.smem_b, b.d_frames.p, items, n,
                                                    b.counters.p + 1, grid, st);
  if (b.family == B200RT_BATCH_KERNELS_TOF_GROUPED)
    return dir == 0 ? b200::launch_forward_batch_tof(b.d_geoms.p, b.num_tof, b.d_frames.p, items, n, b.counters.p, grid,
                                                     st)
                    : b200::launch_back_batch_tof(b.d_geoms.p, b.num_tof, b.d_frames.p, items, n, b.counters.p + 1,
                                                  grid, st);
  if (b.family == B200RT_BATCH_KERNELS_PACKED)
    return dir == 0 ? b200::launch_forward_batch_packed(b.d_geoms.p, b.d_frames.p, items, n, b.counters.p, grid, st)
                    : b200::launch_back_batch_packed(b.d_geoms.p, b.d_frames.p, items, n, b.counters.p + 1, grid, st);
  return dir == 0 ? b200::launch_forward_batch(b.d_geoms.p, b.npa, b.smem, b.d_frames.p, items, n, b.counters.p, grid, st)
                  : b200::launch_back_batch(b.d_geoms.p, b.npa, b.smem, b.d_frames.p, items, n, b.counters.p + 1, grid,
                                            st);
}

void batch_projections(b200rt_batch& b, int k, cudaStream_t st) {
  int n = 0;
  const BatchItem* items = batch_items(b, k, b.cfg.order, n);
  ck(cudaMemsetAsync(b.counters.p, 0, 2 * sizeof(unsigned int), st), "memset");
  ck(batch_launch(b, 0, items, n, grid_of(b, b.cfg.ctas_per_sm_forward, b.max_fwd), st), "batched forward projection");
  ck(batch_launch(b, 1, items, n, grid_of(b, b.cfg.ctas_per_sm_back, b.max_back), st), "batched back projection");
}

// the update arguments of the frames taking part in sub-iteration k, uploaded on first use
const b200::BatchUpdateDev* batch_updates(b200rt_batch& b, int k, int& count, int& max_blocks) {
  auto it = b.updates.find(k);
  if (it != b.updates.end()) {
    count = b.update_counts[k].first;
    max_blocks = b.update_counts[k].second;
    return it->second->p;
  }
  std::vector<b200::BatchUpdateDev> v;
  max_blocks = 1;
  for (auto& fp : b.frames) {
    auto& f = *fp;
    if (k > f.num_subiters) continue;
    const b200::Geometry& g = *f.h->geo;
    b200::BatchUpdateDev d;
    b200::fill_batch_update(d, f.u.p, f.x, f.sens[frame_subset(f, k)], f.has_prior ? f.grad.p : nullptr,
                            f.has_prior ? &f.prior : nullptr, f.prior_w, f.nsub, k, f.min_rel, f.max_rel, g.desc().ny,
                            g.desc().nx, g.desc().nz, f.partial_max.p, f.umax.p);
    max_blocks = std::max(max_blocks, d.nblocks);
    v.push_back(d);
  }
  auto buf = std::make_unique<DevBuf<b200::BatchUpdateDev>>();
  buf->upload(v, b.capture_stream);
  ck(cudaStreamSynchronize(b.capture_stream), "batch updates");
  count = static_cast<int>(v.size());
  b.update_counts[k] = {count, max_blocks};
  const b200::BatchUpdateDev* p = buf->p;
  b.updates[k] = std::move(buf);
  return p;
}

void batch_subiteration(b200rt_batch& b, int k, cudaStream_t st) {
  batch_zero(b, k, st);
  batch_projections(b, k, st);
  for (auto& fp : b.frames)  // deterministic frames: their fixed-point numerators to float
    if (k <= fp->num_subiters && fp->mode == B200RT_BACKPROJECT_DETERMINISTIC)
      ck(launch_fixed_to_float(fp->acc64.p, fp->fixed_scale.p, fp->u.p, fp->h->geo->image_size(), st), "numerator");
  // every frame's update (OSMAPOSLReconstruction.cxx:394-510) in three launches
  int n = 0, max_blocks = 1;
  const b200::BatchUpdateDev* upd = batch_updates(b, k, n, max_blocks);
  bool any_prior = false;
  for (auto& fp : b.frames) any_prior = any_prior || (k <= fp->num_subiters && fp->has_prior);
  ck(b200::launch_batch_update(upd, n, max_blocks, any_prior, st), "update");
}

}  // namespace

extern "C" {

int b200rt_batch_create(int device, b200rt_batch** out) {
  if (!out) return B200RT_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return B200RT_ERR_INVALID_ARGUMENT;
  auto b = std::make_unique<b200rt_batch>();
  b->device = device;
  try {
    DeviceGuard dg(device);
    ck(cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking), "cudaStreamCreate");
  } catch (const std::exception&) {
    return B200RT_ERR_CUDA;
  }
  *out = b.release();
  return B200RT_OK;
}

void b200rt_batch_destroy(b200rt_batch* b) {
  if (!b) return;
  {
    DeviceGuard dg(b->device);
    if (b->capture_stream) cudaStreamSynchronize(b->capture_stream);
    cudaDeviceSynchronize();  // graphs may still run on a caller's stream
    drop_graphs(*b);
    b->items.clear();
    b->updates.clear();
    b->update_counts.clear();
    b->frames.clear();
    b->d_geoms.release();
    b->d_pgeoms.release();
    b->d_frames.release();
    b->counters.release();
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
  }
  delete b;
}

const char* b200rt_batch_last_error(const b200rt_batch* b) { return b ? b->err.c_str() : "null batch"; }

int b200rt_batch_num_frames(const b200rt_batch* b) { return b ? static_cast<int>(b->frames.size()) : 0; }

int b200rt_batch_set_frame_mode(b200rt_batch* b, int frame, int back_projection_mode) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (frame < 0 || frame >= static_cast<int>(b->frames.size())) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "no such frame");
  if (back_projection_mode != B200RT_BACKPROJECT_ATOMIC && back_projection_mode != B200RT_BACKPROJECT_DETERMINISTIC)
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "unknown back-projection mode");
  if (back_projection_mode == B200RT_BACKPROJECT_DETERMINISTIC && !b->frames[frame]->h->use_paths)
    return bfail(b, B200RT_ERR_UNSUPPORTED, "deterministic batched frames need the column-staged kernels (non-TOF)");
  b->frames[frame]->mode = back_projection_mode;
  drop_graphs(*b);
  b->ready = false;
  return B200RT_OK;
}

int b200rt_batch_add_frame(b200rt_batch* b, b200rt_projector* h, float* estimate_dev, const float* y_dev,
                           const float* additive_dev, const float* const* sensitivity_devs, int num_subsets,
                           int start_subset, int num_subiterations, int zero_seg0_end_planes, const b200rt_prior* prior,
                           float min_relative_change, float max_relative_change, int* frame) {
  if (h && sharded(*h)) return refuse_shard(h, "b200rt_batch_add_frame");
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (!h || !estimate_dev || !y_dev || !sensitivity_devs) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "null argument");
  if (h->device != b->device) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "projector is on another device");
  if (num_subsets < 1 || start_subset < 0 || start_subset >= num_subsets)
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid subset number");
  if (num_subiterations < 1) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid number of sub-iterations");
  for (int s = 0; s < num_subsets; ++s)
    if (!sensitivity_devs[s]) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "null sensitivity");
  if (prior && (prior->type < B200RT_PRIOR_NONE || prior->type > B200RT_PRIOR_RELATIVE_DIFFERENCE))
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "unknown prior type");
  try {
    DeviceGuard dg(b->device);
    auto f = std::make_unique<b200rt_batch::Frame>();
    f->h = h;
    auto git = std::find(b->geoms.begin(), b->geoms.end(), h);
    f->geom = static_cast<int>(git - b->geoms.begin());
    if (git == b->geoms.end()) b->geoms.push_back(h);
    f->x = estimate_dev;
    f->y = y_dev;
    f->add = additive_dev;
    f->sens.assign(sensitivity_devs, sensitivity_devs + num_subsets);
    f->nsub = num_subsets;
    f->start_subset = start_subset;
    f->num_subiters = num_subiterations;
    f->zero_ends = zero_seg0_end_planes;
    f->has_prior = prior && prior->type != B200RT_PRIOR_NONE && prior->penalisation_factor != 0;
    if (f->has_prior) {
      f->prior = *prior;
      prior_weights(*h->geo, prior->only_2D, f->prior_w);
    }
    f->min_rel = min_relative_change;
    f->max_rel = max_relative_change;
    drop_graphs(*b);
    b->items.clear();
    b->updates.clear();
    b->update_counts.clear();
    b->item_counts.clear();
    b->ready = false;
    b->frames.push_back(std::move(f));
    if (frame) *frame = static_cast<int>(b->frames.size()) - 1;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return bfail(b, status_of(e), e.what());
  }
}

int b200rt_batch_run(b200rt_batch* b, int first_subiteration, int count, int use_graph, void* stream) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (first_subiteration < 1 || count < 0) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid sub-iteration range");
  if (b->frames.empty() || count == 0) return B200RT_OK;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  try {
    DeviceGuard dg(b->device);
    batch_finalize(*b);
    for (int k = first_subiteration; k < first_subiteration + count; ++k) {
      int n = 0;
      batch_items(*b, k, b->cfg.order, n);  // uploads happen here, never inside a capture
      int nu = 0, mb = 0;
      batch_updates(*b, k, nu, mb);
    }
    if (!use_graph) {
      batch_thresholds(*b, first_subiteration, st);
      for (int k = first_subiteration; k < first_subiteration + count; ++k) batch_subiteration(*b, k, st);
      return B200RT_OK;
    }
    const auto key = std::make_pair(first_subiteration, count);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
      cudaStream_t cs = b->capture_stream;
      ck(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
      try {
        batch_thresholds(*b, first_subiteration, cs);
        for (int k = first_subiteration; k < first_subiteration + count; ++k) batch_subiteration(*b, k, cs);
      } catch (...) {
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(cs, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      cudaGraph_t graph = nullptr;
      ck(cudaStreamEndCapture(cs, &graph), "cudaStreamEndCapture");
      cudaGraphExec_t exec = nullptr;
      const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
      cudaGraphDestroy(graph);
      ck(e, "cudaGraphInstantiate");
      it = b->graphs.emplace(key, exec).first;
    }
    ck(cudaGraphLaunch(it->second, st), "cudaGraphLaunch");
    return B200RT_OK;
  } catch (const std::exception& e) {
    return bfail(b, status_of(e), e.what());
  }
}

int b200rt_batch_autotune(b200rt_batch* b, int subiteration, b200rt_batch_config* out) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (subiteration < 1) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid sub-iteration");
  if (b->frames.empty()) return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "empty batch");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  try {
    DeviceGuard dg(b->device);
    batch_finalize(*b);
    const cudaStream_t st = b->capture_stream;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    batch_thresholds(*b, subiteration, st);  // the forward epilogue reads them
    batch_zero(*b, subiteration, st);        // numerators are scratch
    // time one launch of one direction: the best of two after a warm-up
    auto time_launch = [&](int dir, const BatchItem* items, int n, int grid) {
      float t = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        ck(cudaMemsetAsync(b->counters.p, 0, 2 * sizeof(unsigned int), st), "memset");
        ck(cudaEventRecord(e0, st), "cudaEventRecord");
        ck(batch_launch(*b, dir, items, n, grid, st), dir == 0 ? "batched forward projection" : "batched back projection");
        ck(cudaEventRecord(e1, st), "cudaEventRecord");
        ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        if (rep > 0) t = std::min(t, ms);
      }
      return t;
    };
    float best_total = 1e30f;
    b200rt_batch_config best = b->cfg;
    for (int fam = B200RT_BATCH_KERNELS_PATHS; fam <= B200RT_BATCH_KERNELS_BASIC_BINS; ++fam) {
      if (!b->avail[fam]) continue;
      use_family(*b, fam);
      for (int order = 0; order <= 2; ++order) {
        if (order == 1 && fam == B200RT_BATCH_KERNELS_TOF_GROUPED) continue;  // TOF-grouped items: no length sort
        int n = 0;
        const BatchItem* items = batch_items(*b, subiteration, order, n);
        float tdir[2] = {1e30f, 1e30f};
        int cdir[2] = {1, 1};
        for (int dir = 0; dir < 2; ++dir)
          for (int c = 1; c <= (dir == 0 ? b->max_fwd : b->max_back); ++c) {
            const float t = time_launch(dir, items, n, c * b->num_sms);
            if (t < tdir[dir]) {
              tdir[dir] = t;
              cdir[dir] = c;
            }
          }
        if (tdir[0] + tdir[1] < best_total) {
          best_total = tdir[0] + tdir[1];
          best = b200rt_batch_config{cdir[0], cdir[1], order, fam};
        }
      }
    }
    use_family(*b, best.kernels);
    b->cfg = best;
    if (out) *out = best;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    drop_graphs(*b);
    return B200RT_OK;
  } catch (const std::exception& e) {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    return bfail(b, status_of(e), e.what());
  }
}

int b200rt_batch_set_config(b200rt_batch* b, const b200rt_batch_config* config) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (!config || config->ctas_per_sm_forward < 0 || config->ctas_per_sm_back < 0 || config->order < 0 ||
      config->order > 2 || config->kernels < B200RT_BATCH_KERNELS_AUTO || config->kernels > B200RT_BATCH_KERNELS_BASIC_BINS)
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid batch configuration");
  if (b->ready) {  // otherwise checked when the batch is set up
    try {
      use_family(*b, config->kernels);
    } catch (const std::exception& e) {
      use_family(*b, b->cfg.kernels);
      return bfail(b, B200RT_ERR_UNSUPPORTED, e.what());
    }
  }
  b->cfg = *config;
  drop_graphs(*b);
  return B200RT_OK;
}

int b200rt_batch_get_config(const b200rt_batch* b, b200rt_batch_config* out) {
  if (!b || !out) return B200RT_ERR_INVALID_ARGUMENT;
  *out = b->cfg;
  return B200RT_OK;
}

int b200rt_batch_get_num_cancelled(b200rt_batch* b, int frame, int64_t* out) {
  if (!b) return B200RT_ERR_INVALID_ARGUMENT;
  if (!out || frame < 0 || frame >= static_cast<int>(b->frames.size()))
    return bfail(b, B200RT_ERR_INVALID_ARGUMENT, "invalid frame");
  *out = 0;
  auto& f = *b->frames[frame];
  if (!f.cancelled.p) return B200RT_OK;
  try {
    DeviceGuard dg(b->device);
    unsigned int c = 0;
    ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    ck(cudaMemcpy(&c, f.cancelled.p, sizeof(c), cudaMemcpyDeviceToHost), "D2H");
    *out = c;
    return B200RT_OK;
  } catch (const std::exception& e) {
    return bfail(b, status_of(e), e.what());
  }
}

}  // extern "C"
